// ik_server.cu — continuous batching of IK requests on one GPU.
//
// A server keeps the tables of each registered problem type (robot + terms +
// LM parameters) resident and runs, per type, a persistent kernel on its own
// stream.  Requests of any batch size are admitted into free problem slots as
// they arrive; their problems go into a ring of tickets that the running
// kernel's lane groups claim whenever a problem of theirs stops, so new work
// overlaps with problems already in flight and converged problems retire and
// are replaced mid-launch.
//
// Host <-> device traffic goes through mapped pinned host memory, with no
// CUDA call on the submit or poll path:
//   host  -> device: request inputs (start point, targets), the ring entries,
//                    then the ring tail (release store; the kernel reads it
//                    with an acquire load at system scope);
//   device -> host: solutions and scalars, then a per-request done flag
//                    (system-scope fence before the flag store).
// The only device-memory state is the claim counter of each ring and the
// per-request completion counters.  A kernel exits after a bounded idle time
// with no work; poll() relaunches it when published work is left unclaimed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <map>
#include <unordered_map>
#include <vector>

#include "b200ik.h"
#include "ik_host.h"
#include "ik_lm.cuh"

using namespace b200ik;
using namespace b200ik::host;

namespace b200ik {

// Device-side view of one problem type's queue and buffers (kernel argument).
struct ServerCtrl {
    int* head;              // device: next ring ticket to claim
    int* mirror;            // device: last host tail seen by any warp
    unsigned long long* last_poll;  // device: time of the last read of the host tail
    const int* tail;        // mapped: tickets published by the host
    const int2* ring;       // mapped [cap]: (slot, request) per ticket
    int cap;                // ring capacity = slots
    const float* q_in;      // mapped [slots, na]
    const float* base_in;   // mapped [slots, 7] or null
    float* q_out;           // mapped [slots, na]
    float* base_out;        // mapped [slots, 7] or null
    float* cost;            // mapped [slots]
    float* lambda;          // mapped [slots]
    int* iters;             // mapped [slots]
    int* status;            // mapped [slots]
    const int* req_size;    // mapped [slots]: problems of each request
    int* req_count;         // device [slots]: problems finished so far
    unsigned long long* req_ns;   // device [slots]: summed lane-group time of the request's problems
    unsigned long long* req_ns_out;  // mapped [slots]: the same, published with the done flag
    int* req_flag;          // mapped [slots]: 1 when the request is complete
    const int* stop;        // mapped: 1 asks idle warps to exit
    int* quit_gen;          // device: highest launch generation that stopped claiming
    int* host_quit;         // mapped: the same, for the host
    int* host_head;         // mapped: the head as last claimed, for the host
    int gen;                // generation of this launch
    long long idle_ns;      // idle time after which the launch stops claiming
    long long slice_ns;     // running time after which the launch stops claiming (the host relaunches
                            // with rebalanced shares); 0 = no limit
};

__device__ __forceinline__ int ld_acquire_sys(const int* p) {
    int v;
    asm volatile("ld.acquire.sys.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ long long global_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Host memory is read over the bus: warps read the device mirror of the tail
// and at most one warp per kPollNs refreshes it from the host copy (always
// when `force`, which an idle warp does once before it exits).
constexpr long long kPollNs = 4000;

__device__ __forceinline__ int refresh_tail(const ServerCtrl& c, bool force) {
    const unsigned long long now = (unsigned long long)global_ns();
    const unsigned long long last = *reinterpret_cast<volatile unsigned long long*>(c.last_poll);
    if (!force && (now < last + kPollNs || atomicCAS(c.last_poll, last, now) != last))
        return *reinterpret_cast<volatile int*>(c.mirror);
    const int ht = ld_acquire_sys(c.tail);
    const int old = atomicMax(c.mirror, ht);
    __threadfence();
    return max(old, ht);
}

// Inputs live in host memory that the host rewrites between requests: read
// them with cache-volatile loads so no stale cached line is used.
template <int G>
__device__ __forceinline__ void load_request_point(const Group<G>& g, const Tabs& t, Ws& w, int slot,
                                                   const ServerCtrl& c) {
    const TabHeader* h = t.h;
    for (int a = g.lane; a < h->na; a += G) w.q[a] = __ldcv(c.q_in + (size_t)slot * h->na + a);
    if (h->base_off && g.lane < 7) w.base[g.lane] = __ldcv(c.base_in + (size_t)slot * 7 + g.lane);
    const int items = h->npose * 7;
    for (int it = g.lane; it < items; it += G) {
        const int e = it / 7, k = it - 7 * e;
        const PoseEntry& pe = t.pose()[e];
        w.tgt()[8 * e + k] = __ldcv(pe.targets + ((size_t)slot * pe.num_frames + pe.frame) * 7 + k);
    }
    // the type's shared references: one row per joint or base reference, one scene (checked at registration)
    load_refs<G>(g, t, w, 0, 1);
}

template <int G>
__device__ __forceinline__ void finish_request_problem(const Group<G>& g, const Tabs& t, const Ws& w,
                                                       const LmState& st, int slot, int req, const ServerCtrl& c,
                                                       long long busy_ns) {
    store_solution<G>(g, t, w, st, slot, c.q_out, c.base_out, c.cost, c.lambda, c.iters, c.status);
    __threadfence_system();
    g.sync();
    if (g.lane == 0) {
        atomicAdd(c.req_ns + req, (unsigned long long)(busy_ns > 0 ? busy_ns : 0));
        __threadfence();
        const int done = atomicAdd(c.req_count + req, 1) + 1;
        if (done == __ldcv(c.req_size + req)) {
            // the last problem of the request: no further increments on these counters
            __threadfence();
            c.req_ns_out[req] = atomicExch(c.req_ns + req, 0ull);
            c.req_count[req] = 0;
            __threadfence_system();
            *reinterpret_cast<volatile int*>(c.req_flag + req) = 1;
        }
    }
}

// This generation stops claiming: later tickets go to a new launch.
__device__ __forceinline__ void stop_generation(const ServerCtrl& c) {
    atomicMax(c.quit_gen, c.gen);
    __threadfence();
    *reinterpret_cast<volatile int*>(c.host_head) = *reinterpret_cast<volatile int*>(c.head);
    __threadfence_system();
    *reinterpret_cast<volatile int*>(c.host_quit) = c.gen;
}

// The serving form of the persistent kernel: lane groups own one problem at a
// time and take the next published ticket when their problem stops.
template <int G>
__global__ void __launch_bounds__(kBlockThreads, 4) lm_server_kernel(const char* __restrict__ blob, ServerCtrl c,
                                                                 IkLmParams P) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int wg = lane / G;
    int slot = -1, req = -1;
    bool fresh = false;
    LmState st;
    long long idle_since = __shfl_sync(full, global_ns(), 0);
    const long long t_launch = idle_since;
    long long t_problem = 0;
    while (true) {
        const unsigned need = __ballot_sync(full, slot < 0 && g.lane == 0);
        int got = 0;
        if (need) {
            int hd = 0, k = 0;
            bool may_claim = false;
            if (lane == 0) {
                may_claim = *reinterpret_cast<volatile int*>(c.quit_gen) < c.gen &&
                            *reinterpret_cast<const volatile int*>(c.stop) == 0;
                if (may_claim && c.slice_ns > 0 && global_ns() - t_launch > c.slice_ns) {
                    stop_generation(c);
                    may_claim = false;
                }
            }
            if (lane == 0 && may_claim) {
                const int want = __popc(need);
                hd = *reinterpret_cast<volatile int*>(c.head);
                int tl = *reinterpret_cast<volatile int*>(c.mirror);
                if (tl - hd < want) tl = max(tl, refresh_tail(c, false));
                k = max(0, min(want, tl - hd));
            }
            hd = __shfl_sync(full, hd, 0);
            k = __shfl_sync(full, k, 0);
            if (k > 0) {
                // read the entries before the claim: once the head moves past a
                // ticket, the host may reuse its ring position
                int2 e = make_int2(-1, -1);
                if (lane < k) {
                    const int* ep = reinterpret_cast<const int*>(c.ring + (hd + lane) % c.cap);
                    e.x = __ldcv(ep);
                    e.y = __ldcv(ep + 1);
                }
                int ok = 0;
                if (lane == 0) {
                    ok = atomicCAS(c.head, hd, hd + k) == hd;
                    if (ok) *reinterpret_cast<volatile int*>(c.host_head) = hd + k;
                }
                ok = __shfl_sync(full, ok, 0);
                const int rank = __popc(need & ((1u << (wg * G)) - 1u));
                const int es = __shfl_sync(full, e.x, rank);
                const int er = __shfl_sync(full, e.y, rank);
                if (ok) {
                    got = k;
                    if (slot < 0 && rank < k) {
                        slot = es;
                        req = er;
                        fresh = true;
                        t_problem = global_ns();
                        load_request_point<G>(g, t, w, slot, c);
                        g.sync();
                    }
                }
            }
        }
        if (!__any_sync(full, slot >= 0)) {
            if (got > 0) {
                idle_since = __shfl_sync(full, global_ns(), 0);
                continue;
            }
            // With nothing to run: leave once this generation stopped claiming.
            // A warp idle for idle_ns stops the whole generation (after a last
            // look at the host tail); the host launches a new one for later work,
            // so a launch never shrinks to a few warps that serve a large request.
            int quit = 0;
            if (lane == 0) {
                quit = *reinterpret_cast<volatile int*>(c.quit_gen) >= c.gen ||
                       *reinterpret_cast<const volatile int*>(c.stop) != 0;
                if (!quit && global_ns() - idle_since > c.idle_ns &&
                    refresh_tail(c, true) <= *reinterpret_cast<volatile int*>(c.head)) {
                    stop_generation(c);
                    quit = 1;
                }
            }
            if (__shfl_sync(full, quit, 0)) break;
            __nanosleep(5000);
            continue;
        }
        idle_since = __shfl_sync(full, global_ns(), 0);
        if (slot >= 0) {
            bool stop = group_step<G>(g, t, w, st, P, fresh);
            if (fresh) stop = start_stops<G>(st, P);
            fresh = false;
            if (stop) {
                finish_request_problem<G>(g, t, w, st, slot, req, c, global_ns() - t_problem);
                g.sync();
                w.bind(group_ws<G>(wsbase, h, gib), h);
                slot = -1;
            }
        }
    }
}

}  // namespace b200ik

namespace {

constexpr int kStateHeader = 8;  // ints of d_state before the request counters
constexpr int kHostQuit = 16;    // int offsets in the mapped tail block (separate 64-byte lines)
constexpr int kHostHead = 32;
constexpr int kStreams = 4;

#define IK_SV_CK(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return fail(IK_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// Mapped pinned host allocation with its device alias.
struct Mapped {
    void* host = nullptr;
    void* dev = nullptr;
    size_t bytes = 0;
    int alloc(size_t n) {
        bytes = n ? n : 16;
        cudaError_t e = cudaHostAlloc(&host, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
        if (e != cudaSuccess) {
            host = nullptr;
            return fail(IK_E_OOM, "cudaHostAlloc %zu B: %s", bytes, cudaGetErrorString(e));
        }
        std::memset(host, 0, bytes);
        e = cudaHostGetDevicePointer(&dev, host, 0);
        if (e != cudaSuccess) return fail(IK_E_CUDA, "cudaHostGetDevicePointer: %s", cudaGetErrorString(e));
        return IK_OK;
    }
    void release() {
        if (host) cudaFreeHost(host);
        host = dev = nullptr;
    }
    template <typename T>
    T* h() const { return static_cast<T*>(host); }
    template <typename T>
    T* d() const { return static_cast<T*>(dev); }
};

struct Request {
    int64_t id = 0;
    int type = 0, batch = 0, slot0 = -1, req = -1;
    bool done = false;
    // inputs held on the host while the request waits for slots
    std::vector<float> q0, base0;
    std::vector<std::vector<float>> targets;
};

struct ServerType {
    ProblemTables tab;
    int na = 0, floating = 0, slots = 0, G = 8, smem = 0, per_sm = 0;
    std::vector<int> pose_terms;     // term index of each pose term
    std::vector<int> pose_frames;    // frames of each pose term
    IkLmParams params{};
    char* d_blob = nullptr;
    int* d_state = nullptr;          // [0] head, [1] tail mirror, [2..3] last poll time, [4] quit generation,
                                     // [8..] request counters
    unsigned long long* d_req_ns = nullptr;  // [slots] summed problem times of running requests
    Mapped req_ns_out;
    double ns_per_problem = 0.0;     // running estimate of one problem's lane-group time (0 = none yet)
    Mapped q_in, base_in, q_out, base_out, cost, lambda, iters, status, ring, req_size, req_flag, tail;
    std::vector<Mapped> targets;     // one slab per pose term
    // generations rotate over kStreams streams, so a new launch can start
    // while earlier ones finish the problems they already claimed
    cudaStream_t stream[kStreams] = {};
    cudaEvent_t done_ev[kStreams] = {};
    int gen = 0;                     // generation of the latest launch (0 = none yet)
    int tail_host = 0;               // tickets published so far
    std::map<int, int> free_ranges;  // slot start -> length
    std::vector<int> free_req;
    std::deque<int64_t> pending;     // admitted in order when slots free up
    std::vector<int64_t> inflight;   // admitted, not yet reported done
    int64_t launches = 0;
    int64_t bytes = 0;

    int alloc_slots(int n) {
        for (auto it = free_ranges.begin(); it != free_ranges.end(); ++it) {
            if (it->second >= n) {
                const int s = it->first, len = it->second;
                free_ranges.erase(it);
                if (len > n) free_ranges[s + n] = len - n;
                return s;
            }
        }
        return -1;
    }
    void free_slots(int s, int n) {
        auto it = free_ranges.emplace(s, n).first;
        auto nx = std::next(it);
        if (nx != free_ranges.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_ranges.erase(nx);
        }
        if (it != free_ranges.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_ranges.erase(it);
            }
        }
    }
};

}  // namespace

struct IkServer {
    int64_t budget = 0, used = 0;
    long long idle_ns = 200000;
    long long slice_ns = 4000000;  // generations rebalance the GPU share at least this often under load
    int stop_flag_set = 0;
    Mapped stop;
    std::vector<ServerType*> types;
    std::unordered_map<int64_t, Request> requests;
    int64_t next_id = 1;
};

namespace {

int launch_type(IkServer* S, ServerType& T) {
    ServerCtrl c;
    c.head = T.d_state;
    c.mirror = T.d_state + 1;
    c.last_poll = reinterpret_cast<unsigned long long*>(T.d_state + 2);
    c.tail = T.tail.d<int>();
    c.ring = T.ring.d<int2>();
    c.cap = T.slots;
    c.q_in = T.q_in.d<float>();
    c.base_in = T.floating ? T.base_in.d<float>() : nullptr;
    c.q_out = T.q_out.d<float>();
    c.base_out = T.floating ? T.base_out.d<float>() : nullptr;
    c.cost = T.cost.d<float>();
    c.lambda = T.lambda.d<float>();
    c.iters = T.iters.d<int>();
    c.status = T.status.d<int>();
    c.req_size = T.req_size.d<int>();
    c.req_count = T.d_state + kStateHeader;
    c.req_ns = T.d_req_ns;
    c.req_ns_out = T.req_ns_out.d<unsigned long long>();
    c.slice_ns = S->slice_ns;
    c.req_flag = T.req_flag.d<int>();
    c.stop = S->stop.d<int>();
    c.quit_gen = T.d_state + 4;
    c.host_quit = T.tail.d<int>() + kHostQuit;
    c.host_head = T.tail.d<int>() + kHostHead;
    c.gen = T.gen + 1;
    const int sidx = c.gen % kStreams;
    c.idle_ns = S->idle_ns;
    // Share the GPU between the kernels of the types with work, so that all of them stay resident: by
    // their waiting work in block-time (waiting problems x measured time per problem / groups per block)
    // once every such type has a measurement, else evenly.
    double total = 0.0, mine = 0.0;
    int ntypes = 0;
    bool measured = true;
    for (ServerType* o : S->types) {
        if (o != &T && o->inflight.empty()) continue;
        ++ntypes;
        const int waiting = std::max(1, o->tail_host - __atomic_load_n(o->tail.h<int>() + kHostHead, __ATOMIC_ACQUIRE));
        const double d = waiting * o->ns_per_problem / (kBlockThreads / o->G);
        if (o->ns_per_problem <= 0.0) measured = false;
        total += d;
        if (o == &T) mine = d;
    }
    ntypes = std::max(ntypes, 1);
    const double share = (measured && total > 0.0) ? std::max(mine / total, 0.02) : 1.0 / ntypes;
    const int gpb = kBlockThreads / T.G;
    const int need = (T.slots + gpb - 1) / gpb;
    int grid = std::max(1, (int)(T.per_sm * num_sms() * share + 0.5));
    grid = std::min(grid, need);
    // types of the same group width share a kernel: set its shared-memory limit for this type
    int rc = IK_OK;
    switch (T.G) {
        case 8:
            rc = prepare_kernel(lm_server_kernel<8>, T.smem);
            if (!rc) lm_server_kernel<8><<<grid, kBlockThreads, T.smem, T.stream[sidx]>>>(T.d_blob, c, T.params);
            break;
        case 16:
            rc = prepare_kernel(lm_server_kernel<16>, T.smem);
            if (!rc) lm_server_kernel<16><<<grid, kBlockThreads, T.smem, T.stream[sidx]>>>(T.d_blob, c, T.params);
            break;
        case 32:
            rc = prepare_kernel(lm_server_kernel<32>, T.smem);
            if (!rc) lm_server_kernel<32><<<grid, kBlockThreads, T.smem, T.stream[sidx]>>>(T.d_blob, c, T.params);
            break;
        default: return fail(IK_E_INVALID, "group width %d", T.G);
    }
    if (rc) return rc;
    rc = check_launch();
    if (rc) return rc;
    IK_SV_CK(cudaEventRecord(T.done_ev[sidx], T.stream[sidx]));
    T.gen = c.gen;
    T.launches += 1;
    return IK_OK;
}

// Launch a new generation when published tickets are unclaimed and the latest
// launch has exited or stopped claiming.
int ensure_running(IkServer* S, ServerType& T) {
    if (T.inflight.empty()) return IK_OK;
    const int* hm = T.tail.h<int>();
    if (T.gen > 0) {
        if (T.tail_host - __atomic_load_n(hm + kHostHead, __ATOMIC_ACQUIRE) <= 0) return IK_OK;
        const cudaError_t e = cudaEventQuery(T.done_ev[T.gen % kStreams]);
        if (e != cudaSuccess && e != cudaErrorNotReady)
            return fail(IK_E_CUDA, "server kernel: %s", cudaGetErrorString(e));
        if (e == cudaErrorNotReady && __atomic_load_n(hm + kHostQuit, __ATOMIC_ACQUIRE) < T.gen) return IK_OK;
    }
    return launch_type(S, T);
}

// Copy a request's inputs into its slots and publish its tickets.
void publish(ServerType& T, Request& R, const float* q0, const float* base0, const float* const* targets) {
    const int na = T.na, s0 = R.slot0, n = R.batch;
    if (na) std::memcpy(T.q_in.h<float>() + (size_t)s0 * na, q0, sizeof(float) * (size_t)n * na);
    if (T.floating) std::memcpy(T.base_in.h<float>() + (size_t)s0 * 7, base0, sizeof(float) * (size_t)n * 7);
    for (size_t k = 0; k < T.pose_terms.size(); ++k) {
        const size_t per = (size_t)T.pose_frames[k] * 7;
        std::memcpy(T.targets[k].h<float>() + (size_t)s0 * per, targets[k], sizeof(float) * n * per);
    }
    T.req_size.h<int>()[R.req] = n;
    T.req_flag.h<int>()[R.req] = 0;
    int2* ring = T.ring.h<int2>();
    for (int i = 0; i < n; ++i) ring[(T.tail_host + i) % T.slots] = make_int2(s0 + i, R.req);
    T.tail_host += n;
    // every store above becomes visible before the new tail
    __atomic_store_n(T.tail.h<int>(), T.tail_host, __ATOMIC_RELEASE);
    T.inflight.push_back(R.id);
}

bool try_admit(ServerType& T, Request& R) {
    if (T.free_req.empty()) return false;
    const int s0 = T.alloc_slots(R.batch);
    if (s0 < 0) return false;
    R.slot0 = s0;
    R.req = T.free_req.back();
    T.free_req.pop_back();
    return true;
}

void release_type(ServerType* T) {
    if (!T) return;
    for (int k = 0; k < kStreams; ++k)
        if (T->stream[k]) cudaStreamSynchronize(T->stream[k]);
    for (Mapped* m : {&T->q_in, &T->base_in, &T->q_out, &T->base_out, &T->cost, &T->lambda, &T->iters, &T->status,
                      &T->ring, &T->req_size, &T->req_flag, &T->tail, &T->req_ns_out})
        m->release();
    if (T->d_req_ns) cudaFree(T->d_req_ns);
    for (auto& m : T->targets) m.release();
    if (T->d_blob) cudaFree(T->d_blob);
    if (T->d_state) cudaFree(T->d_state);
    for (int k = 0; k < kStreams; ++k) {
        if (T->done_ev[k]) cudaEventDestroy(T->done_ev[k]);
        if (T->stream[k]) cudaStreamDestroy(T->stream[k]);
    }
    delete T;
}

}  // namespace

extern "C" {

int ik_server_create(int64_t budget_bytes, int32_t idle_us, IkServer** out) {
    if (!out) return fail(IK_E_INVALID, "out is NULL");
    *out = nullptr;
    if (budget_bytes <= 0) return fail(IK_E_INVALID, "budget_bytes must be > 0");
    if (idle_us < 0) return fail(IK_E_INVALID, "idle_us < 0");
    int dev = 0;
    IK_SV_CK(cudaGetDevice(&dev));
    IkServer* S = new IkServer();
    S->budget = budget_bytes;
    S->idle_ns = (long long)(idle_us ? idle_us : 200) * 1000;
    int rc = S->stop.alloc(64);
    if (rc) {
        delete S;
        return rc;
    }
    *out = S;
    return IK_OK;
}

int ik_server_destroy(IkServer* S) {
    if (!S) return IK_OK;
    if (S->stop.host) __atomic_store_n(S->stop.h<int>(), 1, __ATOMIC_RELEASE);
    for (ServerType* T : S->types) release_type(T);
    S->stop.release();
    delete S;
    return IK_OK;
}

int ik_server_add_type(IkServer* S, IkRobot* robot, int32_t floating_base, const IkTermDesc* terms,
                       int32_t num_terms, const float* active_dof_mask, const IkLmParams* params, int32_t slots,
                       int32_t* type_id) {
    if (!S || !robot) return fail(IK_E_INVALID, "server or robot is NULL");
    if (slots < 1) return fail(IK_E_INVALID, "slots %d < 1", slots);
    int rc = check_params(params);
    if (rc) return rc;
    if (params->stop_rules & IK_STOP_ALL_COST)
        return fail(IK_E_INVALID, "the all-problems cost rule needs the plain form");
    const RobotHost& r = robot->h;
    const int floating = floating_base ? 1 : 0;
    const int D = (floating ? 6 : 0) + r.na;
    if (D < 1 || D > kMaxDim) return fail(IK_E_UNSUPPORTED, "tangent dimension %d not in [1, %d]", D, kMaxDim);
    // pose targets come from each request: point the terms at the type's slabs
    std::vector<IkTermDesc> descs(terms, terms + (num_terms > 0 ? num_terms : 0));
    ServerType* T = new ServerType();
    T->na = r.na;
    T->floating = floating;
    T->slots = slots;
    T->params = *params;
    for (int i = 0; i < num_terms; ++i)
        if ((descs[i].kind == IK_TERM_JOINT_REF || descs[i].kind == IK_TERM_VELOCITY_LIMIT ||
             descs[i].kind == IK_TERM_BASE_REF) && descs[i].target_rows != 1) {
            delete T;
            return fail(IK_E_UNSUPPORTED, "term %d: a served reference term needs one shared reference row, not %d "
                        "(requests carry no references)", i, descs[i].target_rows);
        } else if (descs[i].kind == IK_TERM_SCENE_COLLISION && descs[i].scene_rows > 1) {
            delete T;
            return fail(IK_E_UNSUPPORTED, "term %d: a served scene term needs one scene for every problem, not %d "
                        "scene rows (requests carry no scene indices)", i, descs[i].scene_rows);
        } else if (descs[i].kind == IK_TERM_POSITION || descs[i].kind == IK_TERM_ROTATION || descs[i].kind == IK_TERM_FRAME) {
            if (descs[i].num_frames < 1) {
                delete T;
                return fail(IK_E_INVALID, "term %d: pose term needs frames", i);
            }
            T->pose_terms.push_back(i);
            T->pose_frames.push_back(descs[i].num_frames);
        }
    int64_t bytes = 0;
    auto take = [&](Mapped& m, size_t n) {
        bytes += (int64_t)n;
        return m.alloc(n);
    };
    const size_t ns = (size_t)slots;
    rc = take(T->q_in, ns * std::max(r.na, 1) * 4);
    if (!rc) rc = take(T->q_out, ns * std::max(r.na, 1) * 4);
    if (!rc && floating) rc = take(T->base_in, ns * 7 * 4);
    if (!rc && floating) rc = take(T->base_out, ns * 7 * 4);
    if (!rc) rc = take(T->cost, ns * 4);
    if (!rc) rc = take(T->lambda, ns * 4);
    if (!rc) rc = take(T->iters, ns * 4);
    if (!rc) rc = take(T->status, ns * 4);
    if (!rc) rc = take(T->ring, ns * 8);
    if (!rc) rc = take(T->req_size, ns * 4);
    if (!rc) rc = take(T->req_flag, ns * 4);
    if (!rc) rc = take(T->tail, 256);
    if (!rc) rc = take(T->req_ns_out, ns * 8);
    T->targets.resize(T->pose_terms.size());
    for (size_t k = 0; k < T->pose_terms.size() && !rc; ++k) {
        rc = take(T->targets[k], ns * T->pose_frames[k] * 7 * 4);
        if (!rc) {
            descs[T->pose_terms[k]].d_targets = T->targets[k].d<float>();
            descs[T->pose_terms[k]].target_rows = slots;
        }
    }
    if (!rc && S->used + bytes > S->budget)
        rc = fail(IK_E_OOM, "type needs %lld B; %lld B of the server budget are left", (long long)bytes,
                  (long long)(S->budget - S->used));
    std::vector<TermHost> th;
    int R = 0;
    if (!rc) rc = fill_terms(r, floating, descs.data(), num_terms, th, R);
    std::vector<float> mask;
    if (active_dof_mask) mask.assign(active_dof_mask, active_dof_mask + D);
    if (!rc) rc = build_tables(r, floating, th, mask, R, T->tab);
    if (!rc) {
        T->G = choose_group(T->tab.D, T->tab.blob_bytes, T->tab.ws_bytes, 0);
        T->smem = smem_bytes(T->tab.blob_bytes, T->tab.ws_bytes, T->G);
        if (T->smem > max_smem_optin())
            rc = fail(IK_E_UNSUPPORTED, "problem needs %d B of shared memory per block", T->smem);
    }
    if (!rc) {
        cudaError_t e = cudaMalloc(&T->d_blob, T->tab.blob.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(T->d_blob, T->tab.blob.data(), T->tab.blob.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&T->d_state, (ns + kStateHeader) * sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(T->d_state, 0, (ns + kStateHeader) * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&T->d_req_ns, ns * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemset(T->d_req_ns, 0, ns * sizeof(unsigned long long));
        for (int k = 0; k < kStreams; ++k) {
            if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&T->stream[k], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&T->done_ev[k], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) rc = fail(IK_E_OOM, "server type buffers: %s", cudaGetErrorString(e));
        bytes += (int64_t)T->tab.blob.size() + (int64_t)(ns + kStateHeader) * 4 + (int64_t)ns * 8;
    }
    if (!rc) {
        int per_sm = 0;
        switch (T->G) {
            case 8: rc = prepare_kernel(lm_server_kernel<8>, T->smem);
                if (!rc) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lm_server_kernel<8>, kBlockThreads, T->smem);
                break;
            case 16: rc = prepare_kernel(lm_server_kernel<16>, T->smem);
                if (!rc) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lm_server_kernel<16>, kBlockThreads, T->smem);
                break;
            default: rc = prepare_kernel(lm_server_kernel<32>, T->smem);
                if (!rc) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lm_server_kernel<32>, kBlockThreads, T->smem);
                break;
        }
        if (!rc && per_sm < 1) rc = fail(IK_E_UNSUPPORTED, "server kernel does not fit on an SM");
        T->per_sm = per_sm;
    }
    if (rc) {
        release_type(T);
        return rc;
    }
    T->bytes = bytes;
    S->used += bytes;
    T->free_ranges[0] = slots;
    T->free_req.reserve(slots);
    for (int i = slots - 1; i >= 0; --i) T->free_req.push_back(i);
    S->types.push_back(T);
    if (type_id) *type_id = (int32_t)S->types.size() - 1;
    return IK_OK;
}

int ik_server_submit(IkServer* S, int32_t type, int32_t batch, const float* h_q0, const float* h_base0,
                     const float* const* h_targets, int64_t* request_id) {
    if (!S) return fail(IK_E_INVALID, "server is NULL");
    if (type < 0 || type >= (int)S->types.size()) return fail(IK_E_INVALID, "type %d not registered", type);
    ServerType& T = *S->types[type];
    if (batch < 1) return fail(IK_E_INVALID, "batch %d < 1", batch);
    if (batch > T.slots)
        return fail(IK_E_CAPACITY, "batch size %d exceeds the %d slots of this problem type", batch, T.slots);
    if (T.na && !h_q0) return fail(IK_E_INVALID, "q0 is NULL");
    if (T.floating && !h_base0) return fail(IK_E_INVALID, "floating base problem needs a base array");
    if (!T.pose_terms.empty() && !h_targets) return fail(IK_E_INVALID, "targets are NULL");
    for (size_t k = 0; k < T.pose_terms.size(); ++k)
        if (!h_targets[k]) return fail(IK_E_INVALID, "targets of pose term %zu are NULL", k);
    Request R;
    R.id = S->next_id++;
    R.type = type;
    R.batch = batch;
    if (T.pending.empty() && try_admit(T, R)) {
        publish(T, R, h_q0, h_base0, h_targets);
    } else {
        // wait on the host for free slots, in arrival order
        if (T.na) R.q0.assign(h_q0, h_q0 + (size_t)batch * T.na);
        if (T.floating) R.base0.assign(h_base0, h_base0 + (size_t)batch * 7);
        for (size_t k = 0; k < T.pose_terms.size(); ++k)
            R.targets.emplace_back(h_targets[k], h_targets[k] + (size_t)batch * T.pose_frames[k] * 7);
        T.pending.push_back(R.id);
    }
    const int64_t id = R.id;
    S->requests.emplace(id, std::move(R));
    if (request_id) *request_id = id;
    return ensure_running(S, T);
}

int ik_server_poll(IkServer* S, int64_t* done_ids, int32_t max_done, int32_t* num_done) {
    if (!S) return fail(IK_E_INVALID, "server is NULL");
    int n = 0;
    for (ServerType* Tp : S->types) {
        ServerType& T = *Tp;
        for (size_t i = 0; i < T.inflight.size();) {
            Request& R = S->requests[T.inflight[i]];
            if (__atomic_load_n(T.req_flag.h<int>() + R.req, __ATOMIC_ACQUIRE) == 1 &&
                (done_ids == nullptr || n < max_done)) {
                R.done = true;
                const double per = (double)T.req_ns_out.h<unsigned long long>()[R.req] / R.batch;
                T.ns_per_problem = T.ns_per_problem > 0.0 ? 0.8 * T.ns_per_problem + 0.2 * per : per;
                if (done_ids) done_ids[n] = R.id;
                ++n;
                T.inflight[i] = T.inflight.back();
                T.inflight.pop_back();
            } else {
                ++i;
            }
        }
        int rc = ensure_running(S, T);
        if (rc) return rc;
    }
    if (num_done) *num_done = n;
    return IK_OK;
}

int ik_server_fetch(IkServer* S, int64_t request_id, float* h_q, float* h_base, float* h_cost, int32_t* h_iters,
                    int32_t* h_status) {
    if (!S) return fail(IK_E_INVALID, "server is NULL");
    auto it = S->requests.find(request_id);
    if (it == S->requests.end()) return fail(IK_E_INVALID, "request %lld is unknown", (long long)request_id);
    Request& R = it->second;
    if (!R.done) return fail(IK_E_INVALID, "request %lld is not finished", (long long)request_id);
    ServerType& T = *S->types[R.type];
    const int s0 = R.slot0, n = R.batch;
    if (h_q && T.na) std::memcpy(h_q, T.q_out.h<float>() + (size_t)s0 * T.na, sizeof(float) * (size_t)n * T.na);
    if (h_base && T.floating) std::memcpy(h_base, T.base_out.h<float>() + (size_t)s0 * 7, sizeof(float) * (size_t)n * 7);
    if (h_cost) std::memcpy(h_cost, T.cost.h<float>() + s0, sizeof(float) * n);
    if (h_iters) std::memcpy(h_iters, T.iters.h<int>() + s0, sizeof(int) * n);
    if (h_status) std::memcpy(h_status, T.status.h<int>() + s0, sizeof(int) * n);
    T.req_flag.h<int>()[R.req] = 0;
    T.free_slots(s0, n);
    T.free_req.push_back(R.req);
    S->requests.erase(it);
    // admit waiting requests into the freed slots, in arrival order
    while (!T.pending.empty()) {
        Request& P = S->requests[T.pending.front()];
        if (!try_admit(T, P)) break;
        std::vector<const float*> tp;
        for (auto& v : P.targets) tp.push_back(v.data());
        publish(T, P, P.q0.data(), P.base0.data(), tp.data());
        P.q0.clear();
        P.q0.shrink_to_fit();
        P.base0.clear();
        P.base0.shrink_to_fit();
        P.targets.clear();
        T.pending.pop_front();
    }
    return ensure_running(S, T);
}

int ik_server_info(IkServer* S, int32_t type, int32_t* free_slots, int32_t* pending, int32_t* inflight,
                   int64_t* launches) {
    if (!S) return fail(IK_E_INVALID, "server is NULL");
    if (type < 0 || type >= (int)S->types.size()) return fail(IK_E_INVALID, "type %d not registered", type);
    ServerType& T = *S->types[type];
    int fs = 0;
    for (auto& kv : T.free_ranges) fs += kv.second;
    if (free_slots) *free_slots = fs;
    if (pending) *pending = (int32_t)T.pending.size();
    if (inflight) *inflight = (int32_t)T.inflight.size();
    if (launches) *launches = T.launches;
    return IK_OK;
}

}  // extern "C"
