// ik_api.cu — host side of libb200ik.so: validation, table lowering, launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "b200ik.h"
#include "ik_host.h"
#include "ik_kernels.cuh"
#include "ik_thread.cuh"

using namespace b200ik;
using host::ProblemTables;
using host::RobotHost;
using host::TermHost;

namespace {

// whether automatic schedules pick one lane per problem where it applies
constexpr bool kThreadByDefault = false;

thread_local std::string g_last_error;
thread_local int g_capture_kernels = -1;  // >= 0 while this thread captures a graph
std::atomic<long long> g_launches{0};

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return fail(IK_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

struct BlobBuilder {
    std::vector<char> buf;
    BlobBuilder() { buf.resize((sizeof(TabHeader) + 15) & ~size_t(15), 0); }
    int add(const void* p, size_t bytes) {
        const size_t off = buf.size();
        const size_t padded = (bytes + 15) & ~size_t(15);
        buf.resize(off + (padded ? padded : 16), 0);
        if (bytes) std::memcpy(buf.data() + off, p, bytes);
        return (int)off;
    }
    template <typename T>
    int addv(const std::vector<T>& v) { return add(v.data(), v.size() * sizeof(T)); }
    TabHeader* hdr() { return reinterpret_cast<TabHeader*>(buf.data()); }
};

}  // namespace

namespace b200ik {
namespace host {
int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

}  // namespace host
}  // namespace b200ik
using host::fail;

struct IkProblem {
    IkRobot* robot = nullptr;
    int capacity = 0, floating = 0, D = 0, R = 0, E = 0;
    std::vector<TermHost> terms;
    std::vector<float> mask;
    int mask_any = 0;
    std::vector<char> blob;
    char* d_blob = nullptr;
    int blob_bytes = 0, ws_bytes = 0;
    float* d_rec = nullptr;
    int* d_counters = nullptr;
    int* d_queue = nullptr;
    int group = 0;          // 0 = automatic
    int blocks_per_sm = 0;  // 0 = automatic
};

namespace b200ik {
namespace host {

int num_sms() {
    static int sms = -1;
    if (sms < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

int max_smem_optin() {
    static int v = -1;
    if (v < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (v <= 0) v = 227 * 1024;
    }
    return v;
}

inline int al16(int x) { return (x + 15) & ~15; }

// Workspace layout of one group.  Returns bytes.
int layout_workspace(TabHeader* h, int npose, int ncoll_slots_bytes, bool need_sph, bool need_lbw) {
    int off = 0;
    auto take = [&](int bytes) {
        const int o = off;
        off += al16(std::max(bytes, 16));
        return o;
    };
    const int nj = h->nj, nl = h->nl, na = h->na, ns = h->ns, D = h->D;
    h->w_T0 = take(nj * 8 * 4);
    h->w_T1 = take(nj * 8 * 4);
    h->w_anc = take(2 * nj * 4);
    h->w_sph = take(need_sph ? ns * 16 : 0);
    h->w_lbw = take(need_lbw ? nl * 16 : 0);
    h->w_tgt = take(npose * 8 * 4);
    h->w_rpose = take(std::max(h->pose_rows, 3 * npose) * 4);
    h->w_fM = take(h->nframe * 18 * 4);
    h->w_jref = take(h->njref * na * 4);
    h->w_bref = take(h->nbref * 8 * 4);
    h->w_rlim = take(na * 4);
    // The Jacobian chunk and its row records live only inside a linearisation and
    // the FP64 factor only inside a solve: they share one region.
    const int chunk_bytes = al16(kChunkRows * h->Dp * 4) + al16(kChunkRows * 2 * 4);
    const int factor_bytes = D > kSmallD ? h->T * 8 : 0;  // small systems are factorised in registers
    h->w_Jc = take(std::max(chunk_bytes, factor_bytes));
    h->w_rowmeta = h->w_Jc + al16(kChunkRows * h->Dp * 4);
    h->w_L = h->w_Jc;
    h->w_rc = take(0);
    h->w_Hs = take(h->E * 4);
    h->w_Hc = take(h->E * 4);
    h->w_tmp = take(0);
    h->w_y = take(0);
    h->w_q = take(na * 4);
    h->w_qp = take(na * 4);
    h->w_base = take(h->base_off ? 32 : 0);
    h->w_basep = take(h->base_off ? 32 : 0);
    h->w_d32 = take(D * 4);
    h->w_misc = take((8 + h->ncoll + h->nscene) * 4);  // [8 + ci]: filled slots of collision term ci, then
                                                       // the scene index of each scene term
    const int slots_off = take(ncoll_slots_bytes);
    h->ws_bytes = off;
    return slots_off;
}

void add_robot_tables(BlobBuilder& b, const RobotHost& r) {
    TabHeader* h = b.hdr();
    h->nj = r.nj;
    h->nl = r.nl;
    h->na = r.na;
    h->ns = r.ns;
    h->fk_rounds = r.fk_rounds;
    int o;
    o = b.addv(r.jtype); b.hdr()->o_jtype = o;
    o = b.addv(r.jparent); b.hdr()->o_jparent = o;
    o = b.addv(r.jact); b.hdr()->o_jact = o;
    o = b.addv(r.jmimic); b.hdr()->o_jmimic = o;
    o = b.addv(r.jmul); b.hdr()->o_jmul = o;
    o = b.addv(r.joff); b.hdr()->o_joff = o;
    o = b.addv(r.jaxis); b.hdr()->o_jaxis = o;
    o = b.addv(r.jpt); b.hdr()->o_jpt = o;
    o = b.addv(r.lpj); b.hdr()->o_lpj = o;
    o = b.addv(r.lanc); b.hdr()->o_lanc = o;
    o = b.addv(r.lbound); b.hdr()->o_lbound = o;
    o = b.addv(r.sph); b.hdr()->o_sph = o;
    o = b.addv(r.sphlink); b.hdr()->o_sphlink = o;
    o = b.addv(r.lim); b.hdr()->o_lim = o;
    o = b.addv(r.colstart); b.hdr()->o_colstart = o;
    o = b.addv(r.coljoint); b.hdr()->o_coljoint = o;
    o = b.addv(r.colmul); b.hdr()->o_colmul = o;
    o = b.addv(r.jorder); b.hdr()->o_jorder = o;
}

std::vector<uint16_t> ab_table(int D) {
    std::vector<uint16_t> ab;
    for (int a = 0; a < D; ++a)
        for (int c = 0; c <= a; ++c) ab.push_back((uint16_t)((a << 8) | c));
    return ab;
}

// A blob with robot tables, no terms; used by FK / Jacobian / metrics kernels.
void build_robot_blob(const RobotHost& r, int floating, std::vector<char>& out, int& ws_bytes) {
    BlobBuilder b;
    add_robot_tables(b, r);
    TabHeader* h = b.hdr();
    h->D = (floating ? 6 : 0) + r.na;
    h->base_off = floating ? 6 : 0;
    h->T = h->D * (h->D + 1) / 2;
    h->E = h->T + h->D;
    h->Dp = (h->D + 4) & ~3;  // chunk row: D Jacobian columns + the residual, 16-byte rows
    std::vector<float> mask(h->D, 1.f);
    int o = b.addv(mask);
    b.hdr()->o_mask = o;
    std::vector<uint16_t> ab = ab_table(b.hdr()->D);
    o = b.addv(ab);
    b.hdr()->o_ab = o;
    h = b.hdr();
    h->o_pose = h->o_coll = h->o_limw = h->o_mask;
    layout_workspace(h, 0, 0, r.ns > 0, r.nl > 0);
    h->bytes = (int)b.buf.size();
    ws_bytes = h->ws_bytes;
    out = b.buf;
}

int smem_bytes(int blob_bytes, int ws_bytes, int G) { return blob_bytes + (kBlockThreads / G) * ws_stride(ws_bytes, G); }

int choose_group(int D, int blob_bytes, int ws_bytes, int requested) {
    if (requested) return requested;
    int G = D <= 8 ? 8 : (D <= 16 ? 16 : 32);
    while (G < 32 && smem_bytes(blob_bytes, ws_bytes, G) > max_smem_optin()) G *= 2;
    return G;
}

int check_launch() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(IK_E_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    // launches recorded into a graph under capture count when the graph runs
    if (g_capture_kernels >= 0)
        ++g_capture_kernels;
    else
        g_launches.fetch_add(1);
    return IK_OK;
}

// The persistent kernel without the frame and joint-reference paths.
template <int G>
constexpr auto lm_persistent_core = lm_persistent_kernel<G, false>;

// Dispatch a templated kernel on the group width.
#define IK_DISPATCH(G, KERNEL, ...)                                   \
    do {                                                              \
        switch (G) {                                                  \
            case 8: { auto kfn = KERNEL<8>; __VA_ARGS__; break; }     \
            case 16: { auto kfn = KERNEL<16>; __VA_ARGS__; break; }   \
            case 32: { auto kfn = KERNEL<32>; __VA_ARGS__; break; }   \
            default: return fail(IK_E_INVALID, "group width %d not in {8,16,32}", G); \
        }                                                             \
    } while (0)

int validate_robot(const IkRobotDesc* d) {
    if (!d) return fail(IK_E_INVALID, "robot descriptor is NULL");
    if (d->num_joints < 0 || d->num_joints > kMaxJoints)
        return fail(IK_E_UNSUPPORTED, "num_joints %d outside [0, %d]", d->num_joints, kMaxJoints);
    if (d->num_links < 1 || d->num_links > kMaxLinks)
        return fail(IK_E_UNSUPPORTED, "num_links %d outside [1, %d]", d->num_links, kMaxLinks);
    if (d->num_actuated < 0 || d->num_actuated + 6 > kMaxDim + 6 || d->num_actuated > kMaxDim)
        return fail(IK_E_UNSUPPORTED, "num_actuated %d outside [0, %d]", d->num_actuated, kMaxDim);
    if (d->num_spheres < 0 || d->num_spheres > kMaxSpheres)
        return fail(IK_E_UNSUPPORTED, "num_spheres %d outside [0, %d]", d->num_spheres, kMaxSpheres);
    const int nj = d->num_joints, nl = d->num_links, na = d->num_actuated, ns = d->num_spheres;
    if (nj > 0 && (!d->joint_types || !d->joint_axes || !d->parent_transforms || !d->parent_joints ||
                   !d->actuated_indices || !d->mimic_indices || !d->mimic_multipliers || !d->mimic_offsets))
        return fail(IK_E_INVALID, "joint tables must be non-NULL");
    if (!d->link_parent_joints) return fail(IK_E_INVALID, "link_parent_joints is NULL");
    if (na > 0 && !d->actuated_limits) return fail(IK_E_INVALID, "actuated_limits is NULL");
    if (ns > 0 && (!d->sphere_centers || !d->sphere_radii || !d->sphere_links))
        return fail(IK_E_INVALID, "sphere tables must be non-NULL");
    for (int j = 0; j < nj; ++j) {
        const int ty = d->joint_types[j];
        if (ty < 0 || ty > 2) return fail(IK_E_INVALID, "joint %d has type %d", j, ty);
        const int p = d->parent_joints[j];
        if (p < -1 || p >= nj) return fail(IK_E_INVALID, "joint %d parent %d out of range", j, p);
        const int a = d->actuated_indices[j], m = d->mimic_indices[j];
        if (a < -1 || a >= na) return fail(IK_E_INVALID, "joint %d actuated index %d out of range", j, a);
        if (m < -1 || m >= na) return fail(IK_E_INVALID, "joint %d mimic index %d out of range", j, m);
        for (int k = 0; k < 7; ++k)
            if (!std::isfinite(d->parent_transforms[7 * j + k]))
                return fail(IK_E_INVALID, "joint %d parent transform is not finite", j);
        if (ty != 0) {
            const float* ax = d->joint_axes + 3 * j;
            const float n = std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
            if (!(n > 0.f) || !std::isfinite(n)) return fail(IK_E_INVALID, "joint %d has a zero-length axis", j);
        }
    }
    // the parent relation must be a forest: walking up from every joint ends
    for (int j = 0; j < nj; ++j) {
        int cur = j, steps = 0;
        while (cur != -1) {
            cur = d->parent_joints[cur];
            if (++steps > nj) return fail(IK_E_INVALID, "joint parent table has a cycle through joint %d", j);
        }
    }
    for (int l = 0; l < nl; ++l) {
        const int pj = d->link_parent_joints[l];
        if (pj < -1 || pj >= nj) return fail(IK_E_INVALID, "link %d parent joint %d out of range", l, pj);
    }
    for (int s = 0; s < ns; ++s) {
        const int l = d->sphere_links[s];
        if (l < 0 || l >= nl) return fail(IK_E_INVALID, "sphere %d link %d out of range", s, l);
    }
    return IK_OK;
}

}  // namespace host
}  // namespace b200ik
using namespace b200ik::host;

// =============================================================================
int b200ik::host::fill_robot(const IkRobotDesc* d, RobotHost& r) {
    int rc = validate_robot(d);
    if (rc) return rc;
    r.nj = d->num_joints;
    r.nl = d->num_links;
    r.na = d->num_actuated;
    r.ns = d->num_spheres;
    const int nj = r.nj, nl = r.nl, na = r.na, ns = r.ns;
    r.jtype.assign(d->joint_types, d->joint_types + nj);
    r.jparent.assign(d->parent_joints, d->parent_joints + nj);
    r.jact.assign(d->actuated_indices, d->actuated_indices + nj);
    r.jmimic.assign(d->mimic_indices, d->mimic_indices + nj);
    r.jmul.assign(d->mimic_multipliers, d->mimic_multipliers + nj);
    r.joff.assign(d->mimic_offsets, d->mimic_offsets + nj);
    r.jaxis.assign(4 * nj, 0.f);
    r.jpt.assign(8 * nj, 0.f);
    for (int j = 0; j < nj; ++j) {
        for (int k = 0; k < 3; ++k) r.jaxis[4 * j + k] = d->joint_axes[3 * j + k];
        for (int k = 0; k < 7; ++k) r.jpt[8 * j + k] = d->parent_transforms[7 * j + k];
    }
    r.lpj.assign(d->link_parent_joints, d->link_parent_joints + nl);
    r.lim.assign(2 * na, 0.f);
    for (int i = 0; i < 2 * na; ++i) r.lim[i] = d->actuated_limits[i];
    r.sph.assign(4 * std::max(ns, 0), 0.f);
    r.sphlink.assign(ns, 0);
    for (int s = 0; s < ns; ++s) {
        for (int k = 0; k < 3; ++k) r.sph[4 * s + k] = d->sphere_centers[3 * s + k];
        r.sph[4 * s + 3] = d->sphere_radii[s];
        r.sphlink[s] = d->sphere_links[s];
    }
    r.lbound.assign(4 * nl, 0.f);
    if (d->link_bound_centers && d->link_bound_radii)
        for (int l = 0; l < nl; ++l) {
            for (int k = 0; k < 3; ++k) r.lbound[4 * l + k] = d->link_bound_centers[3 * l + k];
            r.lbound[4 * l + 3] = d->link_bound_radii[l];
        }
    // ancestors of each link (robot_spec.py:1133-1142)
    r.lanc.assign(nl, 0ull);
    for (int l = 0; l < nl; ++l) {
        int j = r.lpj[l];
        while (j != -1) {
            r.lanc[l] |= 1ull << j;
            j = r.jparent[j];
        }
    }
    // tangent column -> contributing joints (robot_spec.py:1119-1131)
    r.colstart.assign(na + 1, 0);
    for (int a = 0; a < na; ++a) {
        r.colstart[a] = (int)r.coljoint.size();
        for (int j = 0; j < nj; ++j) {
            if (r.jact[j] == a) {
                r.coljoint.push_back(j);
                r.colmul.push_back(1.f);
            } else if (r.jact[j] < 0 && r.jmimic[j] == a) {
                r.coljoint.push_back(j);
                r.colmul.push_back(r.jmul[j]);
            }
        }
    }
    r.colstart[na] = (int)r.coljoint.size();
    if (r.coljoint.empty()) {
        r.coljoint.push_back(0);
        r.colmul.push_back(0.f);
    }
    // pointer-jumping rounds
    int maxd = 0;
    for (int j = 0; j < nj; ++j) {
        int dpt = 0, cur = j;
        while (cur != -1) {
            ++dpt;
            cur = r.jparent[cur];
        }
        maxd = std::max(maxd, dpt);
    }
    int rounds = 0;
    while ((1 << rounds) < maxd) ++rounds;
    r.fk_rounds = rounds;
    // topological order: by depth, ties in index order
    std::vector<int> depth(nj, 0);
    for (int j = 0; j < nj; ++j)
        for (int cur = r.jparent[j]; cur != -1; cur = r.jparent[cur]) ++depth[j];
    r.jorder.resize(nj);
    for (int j = 0; j < nj; ++j) r.jorder[j] = j;
    std::stable_sort(r.jorder.begin(), r.jorder.end(), [&](int a, int b) { return depth[a] < depth[b]; });
    return IK_OK;
}

extern "C" {

const char* ik_last_error(void) { return g_last_error.c_str(); }
int ik_version(void) { return 10000; }

int ik_device_count(int* out) {
    if (!out) return fail(IK_E_INVALID, "out is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *out = 0;
        return fail(IK_E_NO_DEVICE, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    }
    *out = n;
    return IK_OK;
}

int ik_set_device(int device) {
    CK(cudaSetDevice(device));
    return IK_OK;
}

// ---- CUDA graphs of library calls --------------------------------------------
struct IkGraph {
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
};

int ik_graph_begin(void* stream) {
    if (!stream) return fail(IK_E_INVALID, "capture needs a created stream, not the legacy default stream");
    if (g_capture_kernels >= 0) return fail(IK_E_INVALID, "a capture is already open on this thread");
    CK(cudaStreamBeginCapture(S(stream), cudaStreamCaptureModeThreadLocal));
    g_capture_kernels = 0;
    return IK_OK;
}

int ik_graph_end(void* stream, void** graph) {
    if (!stream || !graph) return fail(IK_E_INVALID, "stream or out is NULL");
    *graph = nullptr;
    const int kernels = g_capture_kernels;
    g_capture_kernels = -1;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(S(stream), &g);
    if (e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return fail(IK_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    }
    IkGraph* G = new IkGraph();
    e = cudaGraphInstantiate(&G->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        delete G;
        return fail(IK_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    G->kernels = kernels < 0 ? 0 : kernels;
    *graph = G;
    return IK_OK;
}

int ik_graph_launch(void* graph, void* stream) {
    if (!graph) return fail(IK_E_INVALID, "graph is NULL");
    IkGraph* G = static_cast<IkGraph*>(graph);
    CK(cudaGraphLaunch(G->exec, S(stream)));
    g_launches.fetch_add(G->kernels);
    return IK_OK;
}

int ik_graph_destroy(void* graph) {
    if (!graph) return IK_OK;
    IkGraph* G = static_cast<IkGraph*>(graph);
    if (G->exec) cudaGraphExecDestroy(G->exec);
    delete G;
    return IK_OK;
}

int ik_launch_count(int64_t* out) {
    if (!out) return fail(IK_E_INVALID, "out is NULL");
    *out = g_launches.load();
    return IK_OK;
}

int ik_robot_create(const IkRobotDesc* d, IkRobot** out) {
    if (!out) return fail(IK_E_INVALID, "out is NULL");
    *out = nullptr;
    IkRobot* R = new IkRobot();
    const int rc = fill_robot(d, R->h);
    if (rc) {
        delete R;
        return rc;
    }
    RobotHost& r = R->h;
    for (int f = 0; f < 2; ++f) {
        std::vector<char> blob;
        int ws = 0;
        build_robot_blob(r, f, blob, ws);
        R->blob_bytes[f] = (int)blob.size();
        R->ws_bytes[f] = ws;
        cudaError_t e = cudaMalloc(&R->d_blob[f], blob.size());
        if (e != cudaSuccess) {
            ik_robot_destroy(R);
            return fail(IK_E_OOM, "cudaMalloc robot tables: %s", cudaGetErrorString(e));
        }
        e = cudaMemcpy(R->d_blob[f], blob.data(), blob.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            ik_robot_destroy(R);
            return fail(IK_E_CUDA, "copy robot tables: %s", cudaGetErrorString(e));
        }
    }
    *out = R;
    return IK_OK;
}

int ik_robot_destroy(IkRobot* robot) {
    if (!robot) return IK_OK;
    for (int f = 0; f < 2; ++f)
        if (robot->d_blob[f]) cudaFree(robot->d_blob[f]);
    delete robot;
    return IK_OK;
}

}  // extern "C"

namespace {

}  // namespace

int b200ik::host::build_tables(const RobotHost& r, int floating, const std::vector<TermHost>& terms,
                               const std::vector<float>& mask_in, int R, ProblemTables& out) {
    BlobBuilder b;
    add_robot_tables(b, r);
    TabHeader* h = b.hdr();
    const int boff = floating ? 6 : 0;
    h->D = boff + r.na;
    h->base_off = boff;
    h->T = h->D * (h->D + 1) / 2;
    h->E = h->T + h->D;
    h->Dp = (h->D + 4) & ~3;  // chunk row: D Jacobian columns + the residual, 16-byte rows
    int mask_any = 0;
    for (float m : mask_in)
        if (m != 1.f) mask_any = 1;
    h->mask_any = mask_any;
    h->R_ref = R;
    // pose entries
    std::vector<PoseEntry> pose;
    std::vector<CollEntry> coll;
    std::vector<float> limw(std::max(r.na, 1), 0.f);
    int has_limit = 0, limit_row = 0, pose_rows = 0, nframe = 0;
    for (size_t ti = 0; ti < terms.size(); ++ti) {
        const TermHost& th = terms[ti];
        const int kind = th.d.kind;
        if (kind == IK_TERM_POSITION || kind == IK_TERM_ROTATION || kind == IK_TERM_FRAME) {
            const bool frame = kind == IK_TERM_FRAME;
            for (int f = 0; f < th.d.num_frames; ++f) {
                PoseEntry e;
                std::memset(&e, 0, sizeof(e));
                e.link = th.frame_links[f];
                e.kind = frame ? kPoseFrame : (kind == IK_TERM_POSITION ? kPosePosition : kPoseRotation);
                e.term = (int)ti;
                e.frame = f;
                e.num_frames = th.d.num_frames;
                e.out_row = th.row + (frame ? 6 : 3) * f;
                e.target_rows = th.d.target_rows;
                e.r0 = pose_rows;
                e.fm = frame ? nframe++ : -1;
                if (frame) {
                    e.w[0] = th.weights[2 * f];
                    e.w[1] = th.weights[2 * f + 1];
                } else {
                    for (int k = 0; k < 3; ++k) e.w[k] = th.weights[3 * f + k];
                }
                e.targets = th.d.d_targets;
                pose_rows += frame ? 6 : 3;
                pose.push_back(e);
            }
        } else if (kind == IK_TERM_POSITION_LIMIT) {
            has_limit = 1;
            limit_row = th.row;
            for (int a = 0; a < r.na; ++a) limw[a] = th.weights[a];
        }
    }
    // joint-reference terms: weights into the blob, entries after
    std::vector<JointRefEntry> jref;
    for (size_t ti = 0; ti < terms.size(); ++ti) {
        const TermHost& th = terms[ti];
        if (th.d.kind != IK_TERM_JOINT_REF && th.d.kind != IK_TERM_VELOCITY_LIMIT) continue;
        JointRefEntry e;
        std::memset(&e, 0, sizeof(e));
        e.out_row = th.row;
        e.target_rows = th.d.target_rows;
        e.o_w = b.addv(th.weights);
        e.ws_ref = 0;  // set with the workspace layout
        e.ref = th.d.d_targets;
        if (th.d.kind == IK_TERM_VELOCITY_LIMIT) {
            e.o_vlim = b.addv(th.vlim);
            e.dt = th.d.dt;
        }
        jref.push_back(e);
    }
    // base-reference blocks
    std::vector<BaseRefEntry> bref;
    for (size_t ti = 0; ti < terms.size(); ++ti) {
        const TermHost& th = terms[ti];
        if (th.d.kind != IK_TERM_BASE_REF) continue;
        BaseRefEntry e;
        std::memset(&e, 0, sizeof(e));
        e.out_row = th.row;
        e.target_rows = th.d.target_rows;
        for (int k = 0; k < 6; ++k) e.w[k] = th.weights[k];
        e.ref = th.d.d_targets;
        bref.push_back(e);
    }
    // scene-collision terms
    std::vector<SceneEntry> scene;
    for (size_t ti = 0; ti < terms.size(); ++ti) {
        const TermHost& th = terms[ti];
        if (th.d.kind != IK_TERM_SCENE_COLLISION) continue;
        SceneEntry e;
        std::memset(&e, 0, sizeof(e));
        e.out_row = th.row;
        e.nq = (int)th.qsph.size();
        e.o_q = b.addv(th.qsph);
        e.o_w = b.addv(th.weights);
        e.o_elem = b.addv(th.selem);
        e.o_off = b.addv(th.soff);
        e.nscenes = th.d.num_scenes;
        e.penalty = th.d.penalty;
        e.use_sqrt = th.d.residual_sqrt ? 1 : 0;
        e.margin = th.d.margin;
        e.eps = th.d.residual_eps;
        e.scene_rows = th.d.d_scene_indices ? th.d.scene_rows : 0;
        e.scene_idx = th.d.d_scene_indices;
        scene.push_back(e);
    }
    h = b.hdr();
    h->npose = (int)pose.size();
    h->pose_rows = pose_rows;
    h->nframe = nframe;
    h->njref = (int)jref.size();
    h->has_limit = has_limit;
    h->limit_row = limit_row;
    // collision arrays
    int slot_bytes = 0;
    std::vector<int> coll_slot_rel;
    for (size_t ti = 0; ti < terms.size(); ++ti) {
        const TermHost& th = terms[ti];
        if (th.d.kind != IK_TERM_SELF_COLLISION) continue;
        CollEntry c;
        std::memset(&c, 0, sizeof(c));
        c.mode = th.d.pair_mode;
        c.K = th.d.max_active_pairs;
        c.nlp = th.d.num_link_pairs;
        c.nsp = th.d.num_sphere_pairs;
        c.out_row = th.row;
        c.rows = th.rows;
        c.margin = th.d.margin;
        c.weight = th.weights[0];
        c.o_lp = b.addv(th.lp);
        c.o_lpoff = b.addv(th.lpoff);
        c.o_sp = b.addv(th.sp);
        coll_slot_rel.push_back(slot_bytes);
        if (c.mode == IK_PAIRS_SLOTS)
            slot_bytes += al16(std::min(c.K, std::max(c.nlp, 1)) * (int)sizeof(Slot));
        else  // candidate link pairs (pruned scan) or one activity mask per lane (flat scan)
            slot_bytes += al16(std::max(std::max(c.nlp, 1) * (int)sizeof(int), 32 * (int)sizeof(unsigned long long)));
        coll.push_back(c);
    }
    int max_slots = 0;
    for (auto& c : coll)
        if (c.mode == IK_PAIRS_SLOTS) max_slots += std::min(c.K, c.nlp);
    int o = b.add(pose.data(), pose.size() * sizeof(PoseEntry));
    b.hdr()->o_pose = o;
    const int o_coll = b.add(coll.data(), coll.size() * sizeof(CollEntry));
    b.hdr()->o_coll = o_coll;
    const int o_jref = b.add(jref.data(), jref.size() * sizeof(JointRefEntry));
    if (scene.size() > IK_SCENE_MAX_TERMS) return fail(IK_E_UNSUPPORTED, "more than %d scene-collision terms", IK_SCENE_MAX_TERMS);
    const int o_scene = b.add(scene.data(), scene.size() * sizeof(SceneEntry));
    b.hdr()->o_scene = o_scene;
    b.hdr()->nscene = (int)scene.size();
    const int o_bref = b.add(bref.data(), bref.size() * sizeof(BaseRefEntry));
    b.hdr()->o_bref = o_bref;
    b.hdr()->nbref = (int)bref.size();
    b.hdr()->o_jref = o_jref;
    o = b.addv(limw);
    b.hdr()->o_limw = o;
    std::vector<float> mask = mask_in;
    if (mask.empty()) mask.assign(b.hdr()->D, 1.f);
    o = b.addv(mask);
    b.hdr()->o_mask = o;
    std::vector<uint16_t> ab = ab_table(b.hdr()->D);
    o = b.addv(ab);
    b.hdr()->o_ab = o;
    h = b.hdr();
    h->ncoll = (int)coll.size();
    h->max_slots = max_slots;
    const int slots_off = layout_workspace(h, h->npose, slot_bytes, h->ncoll > 0 || h->nscene > 0, h->ncoll > 0);
    CollEntry* ce = reinterpret_cast<CollEntry*>(b.buf.data() + o_coll);
    for (size_t i = 0; i < coll.size(); ++i) ce[i].ws_slots = slots_off + coll_slot_rel[i];
    JointRefEntry* je = reinterpret_cast<JointRefEntry*>(b.buf.data() + o_jref);
    for (size_t i = 0; i < jref.size(); ++i) je[i].ws_ref = h->w_jref / 4 + (int)i * h->na;
    BaseRefEntry* be = reinterpret_cast<BaseRefEntry*>(b.buf.data() + o_bref);
    for (size_t i = 0; i < bref.size(); ++i) be[i].ws_ref = h->w_bref / 4 + 8 * (int)i;
    SceneEntry* se = reinterpret_cast<SceneEntry*>(b.buf.data() + o_scene);
    for (size_t i = 0; i < scene.size(); ++i) se[i].misc = 8 + h->ncoll + (int)i;
    // lane-per-problem layout: small systems with all-pairs collision terms only
    {
        int off = 0;
        auto take = [&](int n) {
            const int o2 = off;
            off += n;
            return o2;
        };
        h->t_Tj = take(7 * h->nj);
        h->t_S = take(6 * h->nj);
        h->t_sph = take(h->ncoll > 0 ? 3 * h->ns : 0);
        h->t_tgt = take(7 * h->npose);
        h->t_Hs = take(h->E);
        h->t_Hc = take(h->E);
        h->t_q = take(std::max(h->na, 1));
        h->t_qp = take(std::max(h->na, 1));
        h->t_base = take(h->base_off ? 7 : 0);
        h->t_basep = take(h->base_off ? 7 : 0);
        bool ok = h->D <= kSmallD && h->nframe == 0 && h->njref == 0 && h->nscene == 0 && h->nbref == 0;
        for (size_t i = 0; i < coll.size(); ++i) {
            if (ce[i].mode != IK_PAIRS_ALL) ok = false;
            ce[i].t_mask = take((ce[i].nsp + 31) / 32);
        }
        h->t_floats = off;
        h->thread_ok = ok ? 1 : 0;
    }
    h->bytes = (int)b.buf.size();
    out.blob = b.buf;
    out.blob_bytes = h->bytes;
    out.ws_bytes = h->ws_bytes;
    out.D = h->D;
    out.R = R;
    out.E = h->E;
    return IK_OK;
}

// Check a scene-collision term and turn its primitives into device records:
// inverse pose rows [R^T | -R^T t], parameters, (type, scale), stably sorted by
// scene so that each scene's primitives keep their query order.
static int scene_records(const RobotHost& r, const IkTermDesc& d, int i, TermHost& th) {
    if (r.ns < 1) return fail(IK_E_INVALID, "term %d: robot has no collision spheres", i);
    if (d.num_query_spheres < 1 || !d.query_spheres || !d.weights)
        return fail(IK_E_INVALID, "term %d: scene collision needs query spheres and weights", i);
    if (d.num_scenes < 1) return fail(IK_E_INVALID, "term %d: num_scenes %d < 1", i, d.num_scenes);
    if (d.num_geoms < 0 || (d.num_geoms > 0 && !d.geoms)) return fail(IK_E_INVALID, "term %d: geoms are NULL", i);
    if (d.penalty < IK_PENALTY_SMOOTH || d.penalty > IK_PENALTY_SURFACE_DISTANCE)
        return fail(IK_E_INVALID, "Unsupported penalty: %d", d.penalty);
    if (d.scene_rows < 0 || (d.scene_rows > 0 && !d.d_scene_indices))
        return fail(IK_E_INVALID, "term %d: scene indices are NULL", i);
    th.qsph.assign(d.query_spheres, d.query_spheres + d.num_query_spheres);
    for (int s : th.qsph)
        if (s < 0 || s >= r.ns) return fail(IK_E_INVALID, "sphere_indices contains out-of-range indices.");
    std::vector<int> order(d.num_geoms);
    for (int k = 0; k < d.num_geoms; ++k) {
        const float* g = d.geoms + (size_t)k * IK_GEOM_FLOATS;
        const int type = (int)g[0], scene = (int)g[1];
        if (g[0] != (float)type || type < IK_GEOM_BOX || type > IK_GEOM_CAPSULE)
            return fail(IK_E_INVALID, "term %d: geom %d has type %g", i, k, g[0]);
        if (g[1] != (float)scene || scene < 0 || scene >= d.num_scenes)
            return fail(IK_E_INVALID, "term %d: geom %d in scene %g of %d", i, k, g[1], d.num_scenes);
        if (!(g[2] > 0.f)) return fail(IK_E_INVALID, "term %d: geom %d scale %g", i, k, g[2]);
        order[k] = k;
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return d.geoms[(size_t)a * IK_GEOM_FLOATS + 1] < d.geoms[(size_t)b * IK_GEOM_FLOATS + 1]; });
    th.soff.assign(d.num_scenes + 1, 0);
    th.selem.clear();
    for (int k : order) {
        const float* g = d.geoms + (size_t)k * IK_GEOM_FLOATS;
        th.soff[(int)g[1] + 1] += 1;
        double qw = g[11], qx = g[12], qy = g[13], qz = g[14];
        const double n = std::sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
        if (!(n > 0.0)) return fail(IK_E_INVALID, "term %d: geom %d has a zero quaternion", i, k);
        qw /= n, qx /= n, qy /= n, qz /= n;
        const double R[3][3] = {{1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy)},
                                {2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx)},
                                {2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)}};
        const double t[3] = {g[8], g[9], g[10]};
        for (int row = 0; row < 3; ++row) {  // row `row` of R^T is column `row` of R
            const double c0 = R[0][row], c1 = R[1][row], c2 = R[2][row];
            th.selem.push_back((float)c0);
            th.selem.push_back((float)c1);
            th.selem.push_back((float)c2);
            th.selem.push_back((float)-(c0 * t[0] + c1 * t[1] + c2 * t[2]));
        }
        for (int k2 = 0; k2 < 4; ++k2) th.selem.push_back(g[4 + k2]);
        th.selem.push_back(g[0]);
        th.selem.push_back(g[2]);
        th.selem.push_back(0.f);
        th.selem.push_back(0.f);
    }
    for (int s = 0; s < d.num_scenes; ++s) th.soff[s + 1] += th.soff[s];
    return IK_OK;
}

int b200ik::host::fill_terms(const RobotHost& r, int floating, const IkTermDesc* terms, int num_terms,
                              std::vector<TermHost>& out, int& R) {
    (void)floating;
    out.clear();
    if (num_terms < 0 || (num_terms > 0 && !terms)) return fail(IK_E_INVALID, "terms array is NULL");
    int row = 0, nlimit = 0;
    for (int i = 0; i < num_terms; ++i) {
        const IkTermDesc& d = terms[i];
        TermHost th;
        th.d = d;
        th.row = row;
        if (d.kind == IK_TERM_POSITION || d.kind == IK_TERM_ROTATION || d.kind == IK_TERM_FRAME) {
            if (d.num_frames < 1 || !d.frame_links || !d.weights) {
                return fail(IK_E_INVALID, "term %d: pose term needs frames and weights", i);
            }
            if (!d.d_targets) {
                return fail(IK_E_INVALID, "term %d: pose term needs a target array", i);
            }
            th.frame_links.assign(d.frame_links, d.frame_links + d.num_frames);
            for (int f : th.frame_links)
                if (f < 0 || f >= r.nl) {
                        return fail(IK_E_INVALID, "term %d: frame link %d out of range", i, f);
                }
            const int per = d.kind == IK_TERM_FRAME ? 2 : 3;
            th.weights.assign(d.weights, d.weights + per * d.num_frames);
            th.rows = (d.kind == IK_TERM_FRAME ? 6 : 3) * d.num_frames;
        } else if (d.kind == IK_TERM_BASE_REF) {
            if (!floating) return fail(IK_E_INVALID, "term %d: base residuals need a floating base", i);
            if (!d.weights) return fail(IK_E_INVALID, "term %d: base weights are NULL", i);
            if (!d.d_targets) return fail(IK_E_INVALID, "term %d: base-reference term needs reference poses", i);
            if (d.target_rows < 1) return fail(IK_E_INVALID, "term %d: target_rows %d", i, d.target_rows);
            th.weights.assign(d.weights, d.weights + 6);
            th.rows = 6;
        } else if (d.kind == IK_TERM_SCENE_COLLISION) {
            int rc = scene_records(r, d, i, th);
            if (rc) return rc;
            th.weights.assign(d.weights, d.weights + d.num_query_spheres);
            th.rows = d.num_query_spheres;
        } else if (d.kind == IK_TERM_JOINT_REF || d.kind == IK_TERM_VELOCITY_LIMIT) {
            if (!d.weights && r.na > 0) return fail(IK_E_INVALID, "term %d: joint weights are NULL", i);
            if (!d.d_targets) return fail(IK_E_INVALID, "term %d: joint-reference term needs a reference array", i);
            if (d.target_rows < 1) return fail(IK_E_INVALID, "term %d: target_rows %d", i, d.target_rows);
            th.weights.assign(d.weights, d.weights + r.na);
            if (d.kind == IK_TERM_VELOCITY_LIMIT) {
                if (!(d.dt > 0.f)) return fail(IK_E_INVALID, "dt must be positive");
                if (!d.velocity_limits && r.na > 0) return fail(IK_E_INVALID, "term %d: velocity limits are NULL", i);
                th.vlim.assign(d.velocity_limits, d.velocity_limits + r.na);
            }
            th.rows = r.na;
        } else if (d.kind == IK_TERM_POSITION_LIMIT) {
            if (++nlimit > 1) {
                return fail(IK_E_UNSUPPORTED, "more than one PositionLimit term");
            }
            if (!d.weights && r.na > 0) {
                return fail(IK_E_INVALID, "term %d: limit weights are NULL", i);
            }
            th.weights.assign(d.weights, d.weights + r.na);
            th.rows = r.na;
        } else if (d.kind == IK_TERM_SELF_COLLISION) {
            if (r.ns < 2) {
                return fail(IK_E_INVALID, "term %d: robot has no collision spheres", i);
            }
            if (d.pair_mode != IK_PAIRS_SLOTS && d.pair_mode != IK_PAIRS_ALL) {
                return fail(IK_E_INVALID, "term %d: pair_mode %d", i, d.pair_mode);
            }
            if (d.pair_mode == IK_PAIRS_SLOTS && d.max_active_pairs < 1) {
                return fail(IK_E_INVALID, "max_active_pairs must be >= 1.");
            }
            if (!d.weights) {
                return fail(IK_E_INVALID, "term %d: weight is NULL", i);
            }
            th.weights.assign(d.weights, d.weights + 1);
            if (d.num_link_pairs < 0 || d.num_sphere_pairs < 0 ||
                (d.num_link_pairs > 0 && (!d.link_pairs || !d.link_pair_offsets || !d.sphere_pairs))) {
                return fail(IK_E_INVALID, "term %d: pair tables are inconsistent", i);
            }
            th.lp.assign(d.link_pairs, d.link_pairs + 2 * d.num_link_pairs);
            th.lpoff.assign(d.link_pair_offsets, d.link_pair_offsets + d.num_link_pairs + 1);
            if (d.num_link_pairs == 0) th.lpoff.assign(1, 0);
            if (th.lpoff.front() != 0 || th.lpoff.back() != d.num_sphere_pairs) {
                return fail(IK_E_INVALID, "term %d: link pair offsets do not cover the sphere pairs", i);
            }
            for (int k = 0; k < d.num_link_pairs; ++k) {
                if (th.lpoff[k + 1] < th.lpoff[k]) {
                        return fail(IK_E_INVALID, "term %d: link pair offsets decrease", i);
                }
                for (int s = 0; s < 2; ++s)
                    if (th.lp[2 * k + s] < 0 || th.lp[2 * k + s] >= r.nl) {
                                return fail(IK_E_INVALID, "term %d: link pair %d out of range", i, k);
                    }
            }
            th.sp.resize(d.num_sphere_pairs);
            for (int k = 0; k < d.num_sphere_pairs; ++k) {
                const int a = d.sphere_pairs[2 * k], b = d.sphere_pairs[2 * k + 1];
                if (a < 0 || a >= r.ns || b < 0 || b >= r.ns) {
                        return fail(IK_E_INVALID, "term %d: sphere pair %d out of range", i, k);
                }
                th.sp[k] = a | (b << 16);
            }
            th.rows = d.pair_mode == IK_PAIRS_SLOTS ? d.max_active_pairs : d.num_sphere_pairs;
        } else {
            return fail(IK_E_INVALID, "term %d: unknown kind %d", i, d.kind);
        }
        row += th.rows;
        out.push_back(th);
    }
    R = row;
    return IK_OK;
}

namespace {

int build_problem_blob(IkProblem* P) {
    ProblemTables t;
    const int rc = build_tables(P->robot->h, P->floating, P->terms, P->mask, P->R, t);
    if (rc) return rc;
    P->blob = std::move(t.blob);
    P->blob_bytes = t.blob_bytes;
    P->ws_bytes = t.ws_bytes;
    P->E = t.E;
    return IK_OK;
}

int upload_blob(IkProblem* P, void* stream) {
    if (!P->d_blob) {
        cudaError_t e = cudaMalloc(&P->d_blob, P->blob.size());
        if (e != cudaSuccess) return fail(IK_E_OOM, "cudaMalloc tables: %s", cudaGetErrorString(e));
    }
    if (stream)
        CK(cudaMemcpyAsync(P->d_blob, P->blob.data(), P->blob.size(), cudaMemcpyHostToDevice, S(stream)));
    else
        CK(cudaMemcpy(P->d_blob, P->blob.data(), P->blob.size(), cudaMemcpyHostToDevice));
    return IK_OK;
}

// lane-group width of the stage kernels (the lane-per-problem schedule only exists for solves)
int problem_group(const IkProblem* P) {
    return choose_group(P->D, P->blob_bytes, P->ws_bytes, P->group == 1 ? 0 : P->group);
}

int thread_smem(const IkProblem* P) {
    const TabHeader* h = reinterpret_cast<const TabHeader*>(P->blob.data());
    return P->blob_bytes + kThreadBlock * h->t_floats * (int)sizeof(float);
}

bool thread_ok(const IkProblem* P) {
    const TabHeader* h = reinterpret_cast<const TabHeader*>(P->blob.data());
    return h->thread_ok && thread_smem(P) <= max_smem_optin();
}

// schedule of the whole-solve kernels: 1 = one lane per problem, else the group width
int solve_lanes(const IkProblem* P) {
    if ((P->group == 1 || (P->group == 0 && kThreadByDefault)) && thread_ok(P)) return 1;
    return problem_group(P);
}

int check_batch(const IkProblem* P, int batch) {
    if (!P) return fail(IK_E_INVALID, "problem is NULL");
    if (batch < 0) return fail(IK_E_INVALID, "batch %d < 0", batch);
    if (batch > P->capacity)
        return fail(IK_E_CAPACITY, "batch size %d exceeds the %d this optimizer was built for", batch, P->capacity);
    return IK_OK;
}

}  // namespace
int b200ik::host::check_params(const IkLmParams* p) {
    if (!p) return fail(IK_E_INVALID, "params is NULL");
    if (!(p->lambda_factor > 0.f) || !(p->lambda_min >= 0.f) || !(p->lambda_max >= p->lambda_min))
        return fail(IK_E_INVALID, "damping parameters are inconsistent");
    if (p->max_iter < 0) return fail(IK_E_INVALID, "max_iter < 0");
    return IK_OK;
}

namespace {
}  // namespace

extern "C" {

int ik_problem_create(IkRobot* robot, int32_t capacity, int32_t floating_base, const IkTermDesc* terms,
                      int32_t num_terms, const float* active_dof_mask, IkProblem** out) {
    if (!out) return fail(IK_E_INVALID, "out is NULL");
    *out = nullptr;
    if (!robot) return fail(IK_E_INVALID, "robot is NULL");
    if (capacity < 1) return fail(IK_E_INVALID, "capacity %d < 1", capacity);
    if (num_terms < 0 || (num_terms > 0 && !terms)) return fail(IK_E_INVALID, "terms array is NULL");
    const RobotHost& r = robot->h;
    const int D = (floating_base ? 6 : 0) + r.na;
    if (D > kMaxDim) return fail(IK_E_UNSUPPORTED, "tangent dimension %d exceeds %d", D, kMaxDim);
    if (D < 1) return fail(IK_E_INVALID, "tangent dimension is 0");
    IkProblem* P = new IkProblem();
    P->robot = robot;
    P->capacity = capacity;
    P->floating = floating_base ? 1 : 0;
    P->D = D;
    int rc = fill_terms(r, P->floating, terms, num_terms, P->terms, P->R);
    if (rc) {
        delete P;
        return rc;
    }
    if (active_dof_mask) {
        P->mask.assign(active_dof_mask, active_dof_mask + D);
        for (float m : P->mask)
            if (m != 1.f) P->mask_any = 1;
    }
    rc = build_problem_blob(P);
    if (!rc) rc = upload_blob(P, nullptr);
    if (!rc) {
        const int rs = rec_stride(P->E);
        cudaError_t e = cudaMalloc(&P->d_rec, (size_t)capacity * rs * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&P->d_counters, 8 * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&P->d_queue, sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(P->d_counters, 0, 8 * sizeof(int));
        if (e != cudaSuccess) rc = fail(IK_E_OOM, "problem buffers: %s", cudaGetErrorString(e));
    }
    if (!rc) {
        const int G = problem_group(P);
        if (smem_bytes(P->blob_bytes, P->ws_bytes, G) > max_smem_optin())
            rc = fail(IK_E_UNSUPPORTED, "problem needs %d B of shared memory per block",
                      smem_bytes(P->blob_bytes, P->ws_bytes, G));
    }
    if (rc) {
        ik_problem_destroy(P);
        return rc;
    }
    *out = P;
    return IK_OK;
}

int ik_problem_destroy(IkProblem* P) {
    if (!P) return IK_OK;
    if (P->d_blob) cudaFree(P->d_blob);
    if (P->d_rec) cudaFree(P->d_rec);
    if (P->d_counters) cudaFree(P->d_counters);
    if (P->d_queue) cudaFree(P->d_queue);
    delete P;
    return IK_OK;
}

int ik_problem_info(const IkProblem* P, int32_t* tangent_dim, int32_t* residual_dim, int32_t* capacity) {
    if (!P) return fail(IK_E_INVALID, "problem is NULL");
    if (tangent_dim) *tangent_dim = P->D;
    if (residual_dim) *residual_dim = P->R;
    if (capacity) *capacity = P->capacity;
    return IK_OK;
}

int ik_problem_set_targets(IkProblem* P, int32_t term_index, const float* d_targets, int32_t target_rows) {
    if (!P) return fail(IK_E_INVALID, "problem is NULL");
    if (term_index < 0 || term_index >= (int)P->terms.size()) return fail(IK_E_INVALID, "term %d out of range", term_index);
    TermHost& th = P->terms[term_index];
    if (th.d.kind != IK_TERM_POSITION && th.d.kind != IK_TERM_ROTATION && th.d.kind != IK_TERM_FRAME &&
        th.d.kind != IK_TERM_JOINT_REF && th.d.kind != IK_TERM_VELOCITY_LIMIT && th.d.kind != IK_TERM_BASE_REF)
        return fail(IK_E_INVALID, "term %d has no pose targets", term_index);
    if (!d_targets) return fail(IK_E_INVALID, "targets are NULL");
    th.d.d_targets = d_targets;
    th.d.target_rows = target_rows;
    int rc = build_problem_blob(P);
    if (rc) return rc;
    return upload_blob(P, nullptr);
}

int ik_problem_set_schedule(IkProblem* P, int32_t group_lanes, int32_t blocks_per_sm) {
    if (!P) return fail(IK_E_INVALID, "problem is NULL");
    if (group_lanes != 0 && group_lanes != 1 && group_lanes != 8 && group_lanes != 16 && group_lanes != 32)
        return fail(IK_E_INVALID, "group_lanes %d not in {0, 1, 8, 16, 32}", group_lanes);
    if (blocks_per_sm < 0) return fail(IK_E_INVALID, "blocks_per_sm < 0");
    if (group_lanes == 1 && !thread_ok(P))
        return fail(IK_E_UNSUPPORTED, "one lane per problem needs D <= %d, all-pairs collision terms and %d B of "
                    "shared memory", kSmallD, thread_smem(P));
    if (group_lanes > 1 && smem_bytes(P->blob_bytes, P->ws_bytes, group_lanes) > max_smem_optin())
        return fail(IK_E_UNSUPPORTED, "group width %d needs too much shared memory", group_lanes);
    P->group = group_lanes;
    P->blocks_per_sm = blocks_per_sm;
    return IK_OK;
}

int ik_problem_get_schedule(const IkProblem* P, int32_t* group_lanes, int32_t* blocks_per_sm) {
    if (!P) return fail(IK_E_INVALID, "problem is NULL");
    if (group_lanes) *group_lanes = solve_lanes(P);
    if (blocks_per_sm) *blocks_per_sm = P->blocks_per_sm;
    return IK_OK;
}

int ik_solve_plain(IkProblem* P, int32_t batch, float* d_q, float* d_base, const IkLmParams* params, float* d_cost,
                   float* d_lambda, int32_t* d_iters, int32_t* d_status, void* stream) {
    int rc = check_batch(P, batch);
    if (rc) return rc;
    rc = check_params(params);
    if (rc) return rc;
    if (!d_q && P->robot->h.na > 0) return fail(IK_E_INVALID, "q is NULL");
    if (P->floating && !d_base) return fail(IK_E_INVALID, "floating base problem needs a base array");
    if (batch == 0) return IK_OK;
    const IkLmParams prm = *params;
    if (solve_lanes(P) == 1) {
        const int smem = thread_smem(P);
        rc = prepare_kernel(lm_thread_plain_kernel, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(lm_thread_plain_kernel, smem, batch, 1, P->blocks_per_sm, grid, kThreadBlock);
        if (rc) return rc;
        for (int k = -1; k < prm.max_iter; ++k) {
            lm_thread_plain_kernel<<<grid, kThreadBlock, smem, S(stream)>>>(
                P->d_blob, batch, d_q, d_base, P->d_rec, prm, k < 0 ? 0 : 1, k < 0 ? 0 : k, P->d_counters, d_cost,
                d_lambda, d_iters, d_status);
            rc = check_launch();
            if (rc) return rc;
        }
        return IK_OK;
    }
    const int G = problem_group(P);
    const int smem = smem_bytes(P->blob_bytes, P->ws_bytes, G);
    IK_DISPATCH(G, lm_plain_kernel, {
        rc = prepare_kernel(kfn, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(kfn, smem, batch, G, P->blocks_per_sm, grid, kBlockThreads);
        if (rc) return rc;
        for (int k = -1; k < prm.max_iter; ++k) {
            kfn<<<grid, kBlockThreads, smem, S(stream)>>>(P->d_blob, batch, d_q, d_base, P->d_rec, prm,
                                                          k < 0 ? 0 : 1, k < 0 ? 0 : k, P->d_counters, d_cost,
                                                          d_lambda, d_iters, d_status);
            rc = check_launch();
            if (rc) return rc;
        }
    });
    return IK_OK;
}

int ik_solve_persistent(IkProblem* P, int32_t batch, float* d_q, float* d_base, const IkLmParams* params,
                        float* d_cost, float* d_lambda, int32_t* d_iters, int32_t* d_status, void* stream) {
    int rc = check_batch(P, batch);
    if (rc) return rc;
    rc = check_params(params);
    if (rc) return rc;
    if (params->stop_rules & IK_STOP_ALL_COST)
        return fail(IK_E_INVALID, "the all-problems cost rule needs the plain form");
    if (!d_q && P->robot->h.na > 0) return fail(IK_E_INVALID, "q is NULL");
    if (P->floating && !d_base) return fail(IK_E_INVALID, "floating base problem needs a base array");
    if (batch == 0) return IK_OK;
    const IkLmParams prm = *params;
    CK(cudaMemsetAsync(P->d_queue, 0, sizeof(int), S(stream)));
    if (solve_lanes(P) == 1) {
        const int smem = thread_smem(P);
        rc = prepare_kernel(lm_thread_persistent_kernel, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(lm_thread_persistent_kernel, smem, batch, 1, P->blocks_per_sm, grid, kThreadBlock);
        if (rc) return rc;
        lm_thread_persistent_kernel<<<grid, kThreadBlock, smem, S(stream)>>>(P->d_blob, batch, d_q, d_base, prm,
                                                                          P->d_queue, d_cost, d_lambda, d_iters,
                                                                          d_status);
        return check_launch();
    }
    const int G = problem_group(P);
    const int smem = smem_bytes(P->blob_bytes, P->ws_bytes, G);
    const TabHeader* th = reinterpret_cast<const TabHeader*>(P->blob.data());
    if (th->nframe == 0 && th->njref == 0 && th->nscene == 0 && th->nbref == 0) {
        // no frame, joint-reference, base-reference or scene entries: the kernel without those paths
        // (a smaller instruction footprint)
        IK_DISPATCH(G, lm_persistent_core, {
            rc = prepare_kernel(kfn, smem);
            if (rc) return rc;
            int grid = 0;
            rc = grid_for(kfn, smem, batch, G, P->blocks_per_sm, grid, kBlockThreads);
            if (rc) return rc;
            kfn<<<grid, kBlockThreads, smem, S(stream)>>>(P->d_blob, batch, d_q, d_base, prm, P->d_queue, d_cost,
                                                          d_lambda, d_iters, d_status);
            rc = check_launch();
            if (rc) return rc;
        });
        return IK_OK;
    }
    IK_DISPATCH(G, lm_persistent_kernel, {
        rc = prepare_kernel(kfn, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(kfn, smem, batch, G, P->blocks_per_sm, grid, kBlockThreads);
        if (rc) return rc;
        kfn<<<grid, kBlockThreads, smem, S(stream)>>>(P->d_blob, batch, d_q, d_base, prm, P->d_queue, d_cost,
                                                      d_lambda, d_iters, d_status);
        rc = check_launch();
        if (rc) return rc;
    });
    return IK_OK;
}

int ik_fk(IkRobot* R, int32_t batch, const float* d_q, const float* d_base, float* d_T_joint, float* d_T_link,
          float* d_S_world, float* d_spheres, float* d_link_bounds, void* stream) {
    if (!R) return fail(IK_E_INVALID, "robot is NULL");
    if (batch < 0) return fail(IK_E_INVALID, "batch < 0");
    if (batch == 0) return IK_OK;
    if (!d_q && R->h.na > 0) return fail(IK_E_INVALID, "q is NULL");
    const int f = d_base ? 1 : 0;
    const int D = (f ? 6 : 0) + R->h.na;
    const int G = choose_group(D, R->blob_bytes[f], R->ws_bytes[f], 0);
    const int smem = smem_bytes(R->blob_bytes[f], R->ws_bytes[f], G);
    int rc = 0;
    IK_DISPATCH(G, fk_kernel, {
        rc = prepare_kernel(kfn, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(kfn, smem, batch, G, 0, grid, kBlockThreads);
        if (rc) return rc;
        kfn<<<grid, kBlockThreads, smem, S(stream)>>>(R->d_blob[f], batch, d_q, d_base, d_T_joint, d_T_link,
                                                      d_S_world, d_spheres, d_link_bounds);
        rc = check_launch();
        if (rc) return rc;
    });
    return IK_OK;
}

int ik_link_jacobian(IkRobot* R, int32_t batch, const float* d_q, const float* d_base, int32_t link,
                     int32_t body_frame, float* d_J, void* stream) {
    if (!R) return fail(IK_E_INVALID, "robot is NULL");
    if (batch < 0) return fail(IK_E_INVALID, "batch < 0");
    if (link < 0 || link >= R->h.nl) return fail(IK_E_INVALID, "link %d out of range", link);
    if (!d_J) return fail(IK_E_INVALID, "output is NULL");
    if (batch == 0) return IK_OK;
    const int f = d_base ? 1 : 0;
    const int D = (f ? 6 : 0) + R->h.na;
    const int G = choose_group(D, R->blob_bytes[f], R->ws_bytes[f], 0);
    const int smem = smem_bytes(R->blob_bytes[f], R->ws_bytes[f], G);
    int rc = 0;
    IK_DISPATCH(G, link_jacobian_kernel, {
        rc = prepare_kernel(kfn, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(kfn, smem, batch, G, 0, grid, kBlockThreads);
        if (rc) return rc;
        kfn<<<grid, kBlockThreads, smem, S(stream)>>>(R->d_blob[f], batch, d_q, d_base, link, body_frame ? 1 : 0,
                                                      d_J);
        rc = check_launch();
        if (rc) return rc;
    });
    return IK_OK;
}

int ik_residual_jacobian(IkProblem* P, int32_t batch, const float* d_q, const float* d_base, float* d_r, float* d_J,
                         void* stream) {
    int rc = check_batch(P, batch);
    if (rc) return rc;
    if (P->floating && !d_base) return fail(IK_E_INVALID, "floating base problem needs a base array");
    if (batch == 0) return IK_OK;
    if (d_r) CK(cudaMemsetAsync(d_r, 0, (size_t)batch * P->R * sizeof(float), S(stream)));
    if (d_J) CK(cudaMemsetAsync(d_J, 0, (size_t)batch * P->R * P->D * sizeof(float), S(stream)));
    const int G = problem_group(P);
    const int smem = smem_bytes(P->blob_bytes, P->ws_bytes, G);
    IK_DISPATCH(G, resjac_kernel, {
        rc = prepare_kernel(kfn, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(kfn, smem, batch, G, 0, grid, kBlockThreads);
        if (rc) return rc;
        kfn<<<grid, kBlockThreads, smem, S(stream)>>>(P->d_blob, batch, d_q, d_base, d_r, d_J);
        rc = check_launch();
        if (rc) return rc;
    });
    return IK_OK;
}

int ik_normal_equations(IkProblem* P, int32_t batch, const float* d_q, const float* d_base, float* d_H, float* d_g,
                        float* d_cost, void* stream) {
    int rc = check_batch(P, batch);
    if (rc) return rc;
    if (P->floating && !d_base) return fail(IK_E_INVALID, "floating base problem needs a base array");
    if (batch == 0) return IK_OK;
    const int G = problem_group(P);
    const int smem = smem_bytes(P->blob_bytes, P->ws_bytes, G);
    IK_DISPATCH(G, normal_kernel, {
        rc = prepare_kernel(kfn, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(kfn, smem, batch, G, 0, grid, kBlockThreads);
        if (rc) return rc;
        kfn<<<grid, kBlockThreads, smem, S(stream)>>>(P->d_blob, batch, d_q, d_base, d_H, d_g, d_cost);
        rc = check_launch();
        if (rc) return rc;
    });
    return IK_OK;
}

int ik_damped_solve(int32_t batch, int32_t dim, const float* d_H, const float* d_g, const float* d_lambda,
                    float* d_delta, float* d_pred, int32_t* d_spd, void* stream) {
    if (batch < 0) return fail(IK_E_INVALID, "batch < 0");
    if (dim < 1 || dim > kMaxDim) return fail(IK_E_UNSUPPORTED, "dimension %d outside [1, %d]", dim, kMaxDim);
    if (!d_H || !d_g || !d_lambda || !d_delta || !d_pred) return fail(IK_E_INVALID, "NULL array");
    if (batch == 0) return IK_OK;
    // a table blob that carries only the dimension and its entry table
    static thread_local std::vector<char*> cache(kMaxDim + 1, nullptr);
    static thread_local std::vector<int> cache_bytes(kMaxDim + 1, 0), cache_ws(kMaxDim + 1, 0);
    if (!cache[dim]) {
        RobotHost r;
        r.na = dim;
        r.nj = 0;
        r.nl = 1;
        r.lpj.assign(1, -1);
        r.lanc.assign(1, 0ull);
        r.lbound.assign(4, 0.f);
        r.lim.assign(2 * dim, 0.f);
        r.colstart.assign(dim + 1, 0);
        r.coljoint.assign(1, 0);
        r.colmul.assign(1, 0.f);
        std::vector<char> blob;
        int ws = 0;
        build_robot_blob(r, 0, blob, ws);
        char* d = nullptr;
        CK(cudaMalloc(&d, blob.size()));
        CK(cudaMemcpy(d, blob.data(), blob.size(), cudaMemcpyHostToDevice));
        cache[dim] = d;
        cache_bytes[dim] = (int)blob.size();
        cache_ws[dim] = ws;
    }
    const int G = choose_group(dim, cache_bytes[dim], cache_ws[dim], 0);
    const int smem = smem_bytes(cache_bytes[dim], cache_ws[dim], G);
    int rc = 0;
    IK_DISPATCH(G, damped_solve_kernel, {
        rc = prepare_kernel(kfn, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(kfn, smem, batch, G, 0, grid, kBlockThreads);
        if (rc) return rc;
        kfn<<<grid, kBlockThreads, smem, S(stream)>>>(cache[dim], batch, d_H, d_g, d_lambda, d_delta, d_pred, d_spd);
        rc = check_launch();
        if (rc) return rc;
    });
    return IK_OK;
}

int ik_step(IkProblem* P, int32_t batch, float* d_q, float* d_base, float* d_lambda, const IkLmParams* params,
            float* d_cost, float* d_delta, float* d_pred, float* d_cost_new, int32_t* d_accept, void* stream) {
    int rc = check_batch(P, batch);
    if (rc) return rc;
    rc = check_params(params);
    if (rc) return rc;
    if (!d_lambda) return fail(IK_E_INVALID, "lambda is NULL");
    if (P->floating && !d_base) return fail(IK_E_INVALID, "floating base problem needs a base array");
    if (batch == 0) return IK_OK;
    const int G = problem_group(P);
    const int smem = smem_bytes(P->blob_bytes, P->ws_bytes, G);
    const IkLmParams prm = *params;
    IK_DISPATCH(G, step_kernel, {
        rc = prepare_kernel(kfn, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(kfn, smem, batch, G, 0, grid, kBlockThreads);
        if (rc) return rc;
        kfn<<<grid, kBlockThreads, smem, S(stream)>>>(P->d_blob, batch, d_q, d_base, d_lambda, prm, d_cost, d_delta,
                                                      d_pred, d_cost_new, d_accept);
        rc = check_launch();
        if (rc) return rc;
    });
    return IK_OK;
}

int ik_accept_reject(int32_t batch, float* d_cost, const float* d_cost_new, const float* d_pred, float* d_lambda,
                     int32_t* d_accept, const IkLmParams* params, void* stream) {
    if (batch < 0) return fail(IK_E_INVALID, "batch < 0");
    int rc = check_params(params);
    if (rc) return rc;
    if (!d_cost || !d_cost_new || !d_pred || !d_lambda || !d_accept) return fail(IK_E_INVALID, "NULL array");
    if (batch == 0) return IK_OK;
    accept_kernel<<<(batch + 127) / 128, 128, 0, S(stream)>>>(batch, d_cost, d_cost_new, d_pred, d_lambda, d_accept,
                                                              *params);
    return check_launch();
}

int ik_metrics(IkRobot* R, int32_t batch, const float* d_q, const float* d_base, int32_t num_targets,
               const int32_t* d_target_links, const float* d_targets, float pos_threshold, float rot_threshold,
               float* d_pos_err, float* d_rot_err, int32_t* d_success, void* stream) {
    if (!R) return fail(IK_E_INVALID, "robot is NULL");
    if (batch < 0 || num_targets < 1) return fail(IK_E_INVALID, "batch < 0 or no targets");
    if (!d_target_links || !d_targets || !d_pos_err || !d_rot_err || !d_success)
        return fail(IK_E_INVALID, "NULL array");
    if (batch == 0) return IK_OK;
    const int f = d_base ? 1 : 0;
    const int D = (f ? 6 : 0) + R->h.na;
    const int G = choose_group(D, R->blob_bytes[f], R->ws_bytes[f], 0);
    const int smem = smem_bytes(R->blob_bytes[f], R->ws_bytes[f], G);
    int rc = 0;
    IK_DISPATCH(G, metrics_kernel, {
        rc = prepare_kernel(kfn, smem);
        if (rc) return rc;
        int grid = 0;
        rc = grid_for(kfn, smem, batch, G, 0, grid, kBlockThreads);
        if (rc) return rc;
        kfn<<<grid, kBlockThreads, smem, S(stream)>>>(R->d_blob[f], batch, d_q, d_base, num_targets, d_target_links,
                                                      d_targets, pos_threshold, rot_threshold, d_pos_err, d_rot_err,
                                                      d_success);
        rc = check_launch();
        if (rc) return rc;
    });
    return IK_OK;
}

int ik_integrate(int32_t batch, int32_t num_actuated, int32_t floating_base, const float* d_q, const float* d_base,
                 const float* d_delta, const float* d_mask, float* d_q_out, float* d_base_out, void* stream) {
    if (batch < 0 || num_actuated < 0) return fail(IK_E_INVALID, "negative size");
    if (!d_q || !d_delta || !d_q_out) return fail(IK_E_INVALID, "NULL array");
    if (floating_base && (!d_base || !d_base_out)) return fail(IK_E_INVALID, "base arrays are NULL");
    if (batch == 0) return IK_OK;
    integrate_kernel<<<(batch + 127) / 128, 128, 0, S(stream)>>>(batch, num_actuated, floating_base ? 1 : 0, d_q,
                                                                 d_base, d_delta, d_mask, d_q_out, d_base_out);
    return check_launch();
}

int ik_measure_fma_peak(int32_t fp64, float* tflops) {
    if (!tflops) return fail(IK_E_INVALID, "out is NULL");
    const int blocks = num_sms() * 8, threads = 256;
    const int iters = fp64 ? 2048 : 4096;
    void* out = nullptr;
    CK(cudaMalloc(&out, blocks * sizeof(double)));
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        CK(cudaEventRecord(a, 0));
        if (fp64)
            fma_peak_kernel<double><<<blocks, threads>>>((double*)out, iters);
        else
            fma_peak_kernel<float><<<blocks, threads>>>((float*)out, iters);
        CK(cudaEventRecord(b, 0));
        CK(cudaEventSynchronize(b));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, a, b));
        if (rep > 0) best = std::min(best, ms);  // first launch is warm-up
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    const double flops = 2.0 * 32.0 * iters * (double)blocks * threads;
    *tflops = (float)(flops / (best * 1e-3) / 1e12);
    return IK_OK;
}

static int elementwise_grid(long long n) {
    long long g = (n + 255) / 256;
    if (g < 1) g = 1;
    if (g > 65535) g = 65535;
    return (int)g;
}

int ik_copy_rows(int32_t rows, int32_t width, const float* d_src, int64_t src_stride, float* d_dst, int64_t dst_stride,
                 void* stream) {
    if (rows < 0 || width < 0) return fail(IK_E_INVALID, "negative size");
    if (rows == 0 || width == 0) return IK_OK;
    if (!d_src || !d_dst) return fail(IK_E_INVALID, "NULL array");
    copy_rows_kernel<<<elementwise_grid((long long)rows * width), 256, 0, S(stream)>>>(rows, width, d_src, src_stride,
                                                                                        d_dst, dst_stride);
    return check_launch();
}

int ik_gather_rows(int32_t rows, int32_t width, const int32_t* d_index, int32_t src_rows, const float* d_src,
                   float* d_dst, int32_t* d_bad, void* stream) {
    if (rows < 0 || width < 0 || src_rows < 0) return fail(IK_E_INVALID, "negative size");
    if (rows == 0 || width == 0) return IK_OK;
    if (!d_index || !d_src || !d_dst) return fail(IK_E_INVALID, "NULL array");
    gather_rows_kernel<<<elementwise_grid((long long)rows * width), 256, 0, S(stream)>>>(rows, width, d_index,
                                                                                         src_rows, d_src, d_dst, d_bad);
    return check_launch();
}

int ik_masked_copy_rows(int32_t rows, int32_t width, const int32_t* d_mask, const float* d_src, float* d_dst,
                        void* stream) {
    if (rows < 0 || width < 0) return fail(IK_E_INVALID, "negative size");
    if (rows == 0 || width == 0) return IK_OK;
    if (!d_mask || !d_src || !d_dst) return fail(IK_E_INVALID, "NULL array");
    masked_copy_rows_kernel<<<elementwise_grid((long long)rows * width), 256, 0, S(stream)>>>(rows, width, d_mask,
                                                                                               d_src, d_dst);
    return check_launch();
}

int ik_row_sumsq(int32_t rows, int32_t width, const float* d_x, int64_t stride, float* d_out, int32_t accumulate,
                 void* stream) {
    if (rows < 0 || width < 0) return fail(IK_E_INVALID, "negative size");
    if (stride < width) return fail(IK_E_INVALID, "stride < width");
    if (rows == 0) return IK_OK;
    if (!d_out || (width > 0 && !d_x)) return fail(IK_E_INVALID, "NULL array");
    row_sumsq_kernel<<<elementwise_grid(rows), 256, 0, S(stream)>>>(rows, width, d_x, stride, d_out, accumulate ? 1 : 0);
    return check_launch();
}

int ik_pose_from_matrix(int32_t n, const float* d_mats, float* d_poses, void* stream) {
    if (n < 0) return fail(IK_E_INVALID, "negative size");
    if (n == 0) return IK_OK;
    if (!d_mats || !d_poses) return fail(IK_E_INVALID, "NULL array");
    pose_from_matrix_kernel<<<elementwise_grid(n), 256, 0, S(stream)>>>(n, d_mats, d_poses);
    return check_launch();
}

int ik_matrix_from_pose(int32_t n, const float* d_poses, float* d_mats, void* stream) {
    if (n < 0) return fail(IK_E_INVALID, "negative size");
    if (n == 0) return IK_OK;
    if (!d_mats || !d_poses) return fail(IK_E_INVALID, "NULL array");
    matrix_from_pose_kernel<<<elementwise_grid(n), 256, 0, S(stream)>>>(n, d_poses, d_mats);
    return check_launch();
}

int ik_select_best(int32_t batch, int32_t num_candidates, int32_t keep, const float* d_cost, const float* d_q,
                   const float* d_base, int32_t num_actuated, float* d_q_out, float* d_base_out, float* d_cost_out,
                   int32_t* d_index_out, void* stream) {
    if (batch < 0) return fail(IK_E_INVALID, "batch < 0");
    if (num_candidates < 1 || keep < 1 || keep > num_candidates)
        return fail(IK_E_INVALID, "keep %d of %d candidates", keep, num_candidates);
    if (num_actuated < 0 || num_actuated > kMaxDim) return fail(IK_E_INVALID, "num_actuated %d", num_actuated);
    if (!d_cost || (num_actuated > 0 && (!d_q || !d_q_out)) || (d_base && !d_base_out))
        return fail(IK_E_INVALID, "NULL array");
    if (batch == 0) return IK_OK;
    const int threads = 128;
    const int blocks = (int)(((size_t)batch * 32 + threads - 1) / threads);
    select_best_kernel<<<blocks, threads, 0, S(stream)>>>(batch, num_candidates, keep, d_cost, d_q, d_base, num_actuated,
                                                        d_q_out, d_base_out, d_cost_out, d_index_out);
    return check_launch();
}

int ik_keep_previous(int32_t batch, int32_t num_actuated, const float* d_prev_cost, const float* d_cost,
                     const float* d_prev_q, const float* d_prev_base, float* d_q, float* d_base, void* stream) {
    if (batch < 0 || num_actuated < 0) return fail(IK_E_INVALID, "negative size");
    if (!d_prev_base != !d_base) return fail(IK_E_INVALID, "give both base arrays or neither");
    const int w = num_actuated + (d_base ? 7 : 0);
    if (batch == 0 || w == 0) return IK_OK;
    if (!d_prev_cost || !d_cost || (num_actuated > 0 && (!d_prev_q || !d_q))) return fail(IK_E_INVALID, "NULL array");
    keep_previous_kernel<<<elementwise_grid((long long)batch * w), 256, 0, S(stream)>>>(
        batch, num_actuated, d_prev_cost, d_cost, d_prev_q, d_base ? d_prev_base : nullptr, d_q, d_base);
    return check_launch();
}

int ik_clamp_q(int32_t batch, int32_t num_actuated, float* d_q, const float* d_limits, const float* d_mask,
               void* stream) {
    if (batch < 0 || num_actuated < 0) return fail(IK_E_INVALID, "negative size");
    if (batch == 0 || num_actuated == 0) return IK_OK;
    if (!d_q || !d_limits) return fail(IK_E_INVALID, "NULL array");
    clamp_q_kernel<<<elementwise_grid((long long)batch * num_actuated), 256, 0, S(stream)>>>(batch, num_actuated, d_q,
                                                                                             d_limits, d_mask);
    return check_launch();
}

// ---- memory / streams / events -------------------------------------------------
int ik_malloc(void** p, size_t bytes) {
    if (!p) return fail(IK_E_INVALID, "out is NULL");
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) return fail(IK_E_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    return IK_OK;
}
int ik_free(void* p) {
    if (p) CK(cudaFree(p));
    return IK_OK;
}
int ik_malloc_host(void** p, size_t bytes) {
    if (!p) return fail(IK_E_INVALID, "out is NULL");
    cudaError_t e = cudaMallocHost(p, bytes ? bytes : 16);
    if (e != cudaSuccess) return fail(IK_E_OOM, "cudaMallocHost(%zu): %s", bytes, cudaGetErrorString(e));
    return IK_OK;
}
int ik_free_host(void* p) {
    if (p) CK(cudaFreeHost(p));
    return IK_OK;
}
int ik_memcpy_htod(void* d, const void* h, size_t bytes, void* stream) {
    if (bytes == 0) return IK_OK;
    CK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, S(stream)));
    return IK_OK;
}
int ik_memcpy_dtoh(void* h, const void* d, size_t bytes, void* stream) {
    if (bytes == 0) return IK_OK;
    CK(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, S(stream)));
    return IK_OK;
}
int ik_memcpy_dtod(void* d, const void* s, size_t bytes, void* stream) {
    if (bytes == 0) return IK_OK;
    CK(cudaMemcpyAsync(d, s, bytes, cudaMemcpyDeviceToDevice, S(stream)));
    return IK_OK;
}
int ik_memset(void* d, int value, size_t bytes, void* stream) {
    if (bytes == 0) return IK_OK;
    CK(cudaMemsetAsync(d, value, bytes, S(stream)));
    return IK_OK;
}
int ik_stream_create(void** stream) {
    if (!stream) return fail(IK_E_INVALID, "out is NULL");
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream = s;
    return IK_OK;
}
int ik_stream_destroy(void* stream) {
    if (stream) CK(cudaStreamDestroy(S(stream)));
    return IK_OK;
}
int ik_stream_synchronize(void* stream) {
    CK(cudaStreamSynchronize(S(stream)));
    return IK_OK;
}
int ik_device_synchronize(void) {
    CK(cudaDeviceSynchronize());
    return IK_OK;
}
int ik_event_create(void** ev) {
    if (!ev) return fail(IK_E_INVALID, "out is NULL");
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    *ev = e;
    return IK_OK;
}
int ik_event_destroy(void* ev) {
    if (ev) CK(cudaEventDestroy(reinterpret_cast<cudaEvent_t>(ev)));
    return IK_OK;
}
int ik_event_record(void* ev, void* stream) {
    CK(cudaEventRecord(reinterpret_cast<cudaEvent_t>(ev), S(stream)));
    return IK_OK;
}
int ik_event_elapsed_ms(void* a, void* b, float* ms) {
    if (!ms) return fail(IK_E_INVALID, "out is NULL");
    CK(cudaEventElapsedTime(ms, reinterpret_cast<cudaEvent_t>(a), reinterpret_cast<cudaEvent_t>(b)));
    return IK_OK;
}

}  // extern "C"
