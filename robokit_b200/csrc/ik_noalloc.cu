// ik_noalloc.cu — a persistent LM solve that allocates no device memory.
//
// Who needs it: a caller that may not allocate once it is running — a
// real-time control loop that forbids allocation after start-up (an
// allocation can block on the driver for milliseconds), or a plug-in whose
// host framework owns every device buffer and hands out only the arrays it
// manages.  ik_problem_create would cudaMalloc the table blob and the work
// queue counter; this entry point keeps both in one file-scope device array
// instead, so each call only copies and launches.
//
// The scratch array is shared by every call on a device: calls that overlap
// in time (two host threads, or two streams whose work overlaps) race on it.
// Serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "b200ik.h"
#include "ik_host.h"
#include "ik_lm.cuh"

using namespace b200ik;
using namespace b200ik::host;

namespace {

// [0, 256): the work-queue counter (must be zero when the kernel starts);
// [256, 256 + IK_NOALLOC_MAX_TABLE_BYTES): the problem's table blob.
constexpr int kQueueBytes = 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kQueueBytes + IK_NOALLOC_MAX_TABLE_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device.  The lookup is the first-call set-up: it may load the module,
// so the first call on a device must come before any stream capture.
int scratch_address(unsigned char** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(IK_E_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(IK_E_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(IK_E_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        if (!p) return fail(IK_E_CUDA, "cudaGetSymbolAddress returned NULL");
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
    return IK_OK;
}

#define IK_NA_CK(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return fail(IK_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

template <int G>
int launch(const ProblemTables& t, unsigned char* scratch, int batch, float* d_q, float* d_base,
           const IkLmParams& prm, float* d_cost, float* d_lambda, int32_t* d_iters, int32_t* d_status,
           cudaStream_t stream) {
    auto kfn = lm_persistent_kernel<G>;
    const int smem = smem_bytes(t.blob_bytes, t.ws_bytes, G);
    int rc = prepare_kernel(kfn, smem);
    if (rc) return rc;
    int grid = 0;
    rc = grid_for(kfn, smem, batch, G, 0, grid, kBlockThreads);
    if (rc) return rc;
    int* queue = reinterpret_cast<int*>(scratch);
    char* blob = reinterpret_cast<char*>(scratch + kQueueBytes);
    IK_NA_CK(cudaMemsetAsync(queue, 0, sizeof(int), stream));
    // Pageable source: the call returns once the bytes are staged, so the
    // host vector may go out of scope afterwards.
    IK_NA_CK(cudaMemcpyAsync(blob, t.blob.data(), t.blob.size(), cudaMemcpyHostToDevice, stream));
    kfn<<<grid, kBlockThreads, smem, stream>>>(blob, batch, d_q, d_base, prm, queue, d_cost, d_lambda, d_iters,
                                               d_status);
    return check_launch();
}

}  // namespace

extern "C" int ik_solve_persistent_noalloc(const IkRobotDesc* robot, int32_t floating_base, const IkTermDesc* terms,
                                           int32_t num_terms, const float* active_dof_mask, int32_t batch,
                                           float* d_q, float* d_base, const IkLmParams* params, float* d_cost,
                                           float* d_lambda, int32_t* d_iters, int32_t* d_status, void* stream) {
    if (batch < 0) return fail(IK_E_INVALID, "batch %d < 0", batch);
    int rc = check_params(params);
    if (rc) return rc;
    if (params->stop_rules & IK_STOP_ALL_COST)
        return fail(IK_E_INVALID, "the all-problems cost rule needs the plain form");
    RobotHost r;
    rc = fill_robot(robot, r);
    if (rc) return rc;
    const int floating = floating_base ? 1 : 0;
    const int D = (floating ? 6 : 0) + r.na;
    if (D > kMaxDim) return fail(IK_E_UNSUPPORTED, "tangent dimension %d exceeds %d", D, kMaxDim);
    if (D < 1) return fail(IK_E_INVALID, "tangent dimension is 0");
    std::vector<TermHost> th;
    int R = 0;
    rc = fill_terms(r, floating, terms, num_terms, th, R);
    if (rc) return rc;
    std::vector<float> mask;
    if (active_dof_mask) mask.assign(active_dof_mask, active_dof_mask + D);
    ProblemTables t;
    rc = build_tables(r, floating, th, mask, R, t);
    if (rc) return rc;
    if (t.blob_bytes > IK_NOALLOC_MAX_TABLE_BYTES || (int)t.blob.size() > IK_NOALLOC_MAX_TABLE_BYTES)
        return fail(IK_E_UNSUPPORTED, "tables need %d B; the allocation-free solve holds at most %d B", t.blob_bytes,
                    IK_NOALLOC_MAX_TABLE_BYTES);
    if (!d_q && r.na > 0) return fail(IK_E_INVALID, "q is NULL");
    if (floating && !d_base) return fail(IK_E_INVALID, "floating base problem needs a base array");
    const int G = choose_group(t.D, t.blob_bytes, t.ws_bytes, 0);
    if (smem_bytes(t.blob_bytes, t.ws_bytes, G) > max_smem_optin())
        return fail(IK_E_UNSUPPORTED, "problem needs %d B of shared memory per block",
                    smem_bytes(t.blob_bytes, t.ws_bytes, G));
    unsigned char* scratch = nullptr;
    rc = scratch_address(&scratch);
    if (rc) return rc;
    if (batch == 0) return IK_OK;
    const IkLmParams prm = *params;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    switch (G) {
        case 8: return launch<8>(t, scratch, batch, d_q, d_base, prm, d_cost, d_lambda, d_iters, d_status, s);
        case 16: return launch<16>(t, scratch, batch, d_q, d_base, prm, d_cost, d_lambda, d_iters, d_status, s);
        case 32: return launch<32>(t, scratch, batch, d_q, d_base, prm, d_cost, d_lambda, d_iters, d_status, s);
        default: return fail(IK_E_INVALID, "group width %d not in {8,16,32}", G);
    }
}
