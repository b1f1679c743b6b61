// ik_lm.cuh — the LM loop of one lane group and the two whole-solve kernels
// (plain: one launch per iteration; persistent: one launch per solve).
// Only templates and inline functions, so several translation units may include it.
#pragma once
#include "b200ik.h"
#include "ik_device.cuh"

namespace b200ik {

constexpr int kBlockThreads = 128;

// Per-problem record the plain form keeps in HBM between its per-iteration
// launches: cached normal equations of the current point plus scalars.
struct RecScalars {
    float cost, lambda, pos_err, rot_err;
    int status, iters, pad0, pad1;
};
__host__ __device__ inline int rec_stride(int E) { return ((E + 8) + 3) & ~3; }

// per-problem solver state kept in registers (identical in every lane of the group)
struct LmState {
    float cost, lambda, pos_err, rot_err;
    int status, iters, accepts;
};

// Stage the table blob into shared memory; returns the start of group workspaces.
__device__ __forceinline__ char* stage_tables(const char* __restrict__ blob, char* smem) {
    const TabHeader* gh = reinterpret_cast<const TabHeader*>(blob);
    const int n16 = gh->bytes >> 4;
    const int4* src = reinterpret_cast<const int4*>(blob);
    int4* dst = reinterpret_cast<int4*>(smem);
    for (int i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    return smem + gh->bytes;
}

template <int G>
__device__ __forceinline__ void load_point(const Group<G>& g, const Tabs& t, Ws& w, int p, const float* q,
                                           const float* base) {
    const TabHeader* h = t.h;
    for (int a = g.lane; a < h->na; a += G) w.q[a] = q[(size_t)p * h->na + a];
    if (h->base_off && g.lane < 7) w.base[g.lane] = base[(size_t)p * 7 + g.lane];
}

// The references of problem p other than its pose targets: base reference poses, scene indices and joint
// references, each read at the broadcast row of p (row p / (batch / rows)).
template <int G>
__device__ __forceinline__ void load_refs(const Group<G>& g, const Tabs& t, Ws& w, int p, int batch) {
    const TabHeader* h = t.h;
    for (int it = g.lane; it < h->nbref * 7; it += G) {
        const BaseRefEntry& be = t.bref()[it / 7];
        const int c = it % 7;
        int rep = batch / be.target_rows;
        if (rep < 1) rep = 1;
        const int row = min(p / rep, be.target_rows - 1);
        reinterpret_cast<float*>(w.raw)[be.ws_ref + c] = be.ref[(size_t)row * 7 + c];
    }
    // the problem's scene per scene term (scene_collision_task.py:486-500: row b / (batch / rows)),
    // clamped to the scenes that exist
    for (int k = g.lane; k < h->nscene; k += G) {
        const SceneEntry& se = t.scene()[k];
        int sid = 0;
        if (se.scene_rows > 0) {
            int rep = batch / se.scene_rows;
            if (rep < 1) rep = 1;
            sid = se.scene_idx[min(p / rep, se.scene_rows - 1)];
        }
        reinterpret_cast<int*>(w.misc())[se.misc] = min(max(sid, 0), se.nscenes - 1);
    }
    for (int je = 0; je < h->njref; ++je) {
        const JointRefEntry& jr = t.jref()[je];
        const int rows = jr.target_rows > 0 ? jr.target_rows : batch;
        int rep = batch / rows;
        if (rep < 1) rep = 1;
        const int row = min(p / rep, rows - 1);
        float* dst = reinterpret_cast<float*>(w.raw) + jr.ws_ref;
        for (int a = g.lane; a < h->na; a += G) dst[a] = jr.ref[(size_t)row * h->na + a];
    }
}

template <int G>
__device__ __forceinline__ void load_targets(const Group<G>& g, const Tabs& t, Ws& w, int p, int batch) {
    const TabHeader* h = t.h;
    load_refs<G>(g, t, w, p, batch);
    const int items = h->npose * 7;
    for (int it = g.lane; it < items; it += G) {
        const int e = it / 7, c = it - 7 * e;
        const PoseEntry& pe = t.pose()[e];
        const int rows = pe.target_rows > 0 ? pe.target_rows : batch;
        int rep = batch / rows;
        if (rep < 1) rep = 1;
        const int row = min(p / rep, rows - 1);
        w.tgt()[8 * e + c] = pe.targets[((size_t)row * pe.num_frames + pe.frame) * 7 + c];
    }
}

template <int G>
__device__ __forceinline__ const float* cur_base(const Tabs& t, const Ws& w) {
    return t.h->base_off ? w.base : nullptr;
}

template <int G>
__device__ __forceinline__ bool check_stop(LmState& st, const IkLmParams& P) {
    bool stop = false;
    if ((P.stop_rules & IK_STOP_POSE) && st.pos_err <= P.pose_pos_tol && st.rot_err <= P.pose_rot_tol) stop = true;
    if ((P.stop_rules & IK_STOP_COST) && st.cost <= P.cost_tol) stop = true;
    if (stop) st.status |= IK_ST_CONVERGED;
    return stop;
}

struct StepTrace {  // optional per-step outputs (ik_step)
    float cost_before, cost_new, pred;
    int accepted;
};

// One step of a problem's LM loop with a single call site for each heavy
// phase (kernels that run both the start and the iterations keep one copy of
// the evaluation and linearisation code, which keeps them in the instruction
// cache).
//  fresh: start at the loaded point — evaluate, set the damping, linearise;
//         returns false (the caller applies its start rules).
//  else:  one LM iteration from the cached linearisation (LMOptimizer._step_body,
//         lm_optimizer.py:834-1005); returns true when the problem stops.
// F = false compiles out the frame and joint-reference paths (for problems with
// neither).
template <int G, bool F = true>
__device__ __forceinline__ bool group_step(const Group<G>& g, const Tabs& t, Ws& w, LmState& st, const IkLmParams& P,
                                           bool fresh, StepTrace* trace = nullptr) {
    const bool floating = t.h->base_off != 0;
    double pred = 0.0, dnorm = 0.0;
    if (!fresh) {
        const bool ok = group_damped_solve<G>(g, t, w, w.Hs(), st.lambda, pred, dnorm);
        if (!ok) st.status |= IK_ST_NOT_SPD;
        if ((P.stop_rules & IK_STOP_STEP) && ok && dnorm < (double)P.step_tol && trace == nullptr) {
            st.status |= IK_ST_CONVERGED;
            return true;
        }
        group_integrate<G>(g, t, w, w.q, w.base, w.qp, w.basep);
    }
    const EvalOut ev = group_eval<G, F>(g, t, w, fresh ? w.q : w.qp, floating ? (fresh ? w.base : w.basep) : nullptr);
    bool acc = true;
    if (!fresh) {
        // gain ratio in FP64 (lm_optimizer.py:319-329)
        acc = pred > 0.0;
        if (acc) {
            const double rho = ((double)st.cost - (double)ev.cost) / (pred + (double)P.gain_ratio_epsilon);
            acc = rho >= (double)P.rho_min;
        }
        if (trace) {
            trace->cost_before = st.cost;
            trace->cost_new = ev.cost;
            trace->pred = (float)pred;
            trace->accepted = acc ? 1 : 0;
        }
    }
    if (acc) {
        if (fresh) {
            st.lambda = P.lambda_init;
            st.status = isfinite(ev.cost) ? IK_ST_RUNNING : IK_ST_NONFINITE;
            st.iters = 0;
            st.accepts = 0;
        } else {
            float* tq = w.q;
            w.q = w.qp;
            w.qp = tq;
            float* tb = w.base;
            w.base = w.basep;
            w.basep = tb;
            st.lambda = fmaxf(st.lambda / P.lambda_factor, P.lambda_min);
            st.accepts += 1;
        }
        st.cost = ev.cost;
        st.pos_err = ev.max_pos;
        st.rot_err = ev.max_rot;
        group_linearize<G, F>(g, t, w, ev, floating ? w.base : nullptr);
    } else {
        st.lambda = fminf(fmaxf(st.lambda * P.lambda_factor, P.lambda_min), P.lambda_max);
    }
    if (fresh) return false;
    st.iters += 1;
    bool stop = check_stop<G>(st, P);
    if (!stop && st.iters >= P.max_iter) {
        st.status |= IK_ST_MAX_ITER;
        stop = true;
    }
    return stop;
}

// Start a solve at the loaded point: evaluate, linearise, set damping.
template <int G>
__device__ __forceinline__ void group_start(const Group<G>& g, const Tabs& t, Ws& w, LmState& st, const IkLmParams& P) {
    group_step<G>(g, t, w, st, P, true);
}

// One LM iteration from the cached linearisation.  Returns true when the problem stops.
template <int G>
__device__ __forceinline__ bool group_iterate(const Group<G>& g, const Tabs& t, Ws& w, LmState& st, const IkLmParams& P,
                                              StepTrace* trace = nullptr) {
    return group_step<G>(g, t, w, st, P, false, trace);
}

// A problem that stops at its start point: apply the start rules, returns true to stop.
template <int G>
__device__ __forceinline__ bool start_stops(LmState& st, const IkLmParams& P) {
    const bool stop = (st.status & IK_ST_NONFINITE) != 0 || check_stop<G>(st, P) || P.max_iter <= 0;
    if (stop && st.iters >= P.max_iter && !(st.status & IK_ST_CONVERGED)) st.status |= IK_ST_MAX_ITER;
    return stop;
}

// Workspace of lane group `gib`: groups are staggered across shared-memory banks.
template <int G>
__device__ __forceinline__ char* group_ws(char* wsbase, const TabHeader* h, int gib) {
    return wsbase + (size_t)gib * ws_stride(h->ws_bytes, G);
}

template <int G>
__device__ __forceinline__ void store_solution(const Group<G>& g, const Tabs& t, const Ws& w, const LmState& st, int p, float* q,
                               float* base, float* cost, float* lambda, int* iters, int* status) {
    const TabHeader* h = t.h;
    for (int a = g.lane; a < h->na; a += G) q[(size_t)p * h->na + a] = w.q[a];
    if (h->base_off && g.lane < 7) base[(size_t)p * 7 + g.lane] = w.base[g.lane];
    if (g.lane == 0) {
        if (cost) cost[p] = st.cost;
        if (lambda) lambda[p] = st.lambda;
        if (iters) iters[p] = st.iters;
        if (status) status[p] = (st.status & IK_ST_FLAGS) | (st.accepts << 8);
    }
}

// ---------------------------------------------------------------------------
// plain form: mode 0 = start (evaluate + linearise), mode 1 = one iteration.
// Static grid-stride over problems; state round-trips through `rec`.
// counters[0..2]: per-iteration "cost above tolerance" counts, counters[3]:
// sticky stop flag of the all-problems cost rule (opt/optimizer.py:237-239).
// ---------------------------------------------------------------------------
template <int G>
__global__ void __launch_bounds__(kBlockThreads, 4) lm_plain_kernel(const char* __restrict__ blob, int batch, float* q,
                                                                float* base, float* rec, IkLmParams P, int mode,
                                                                int k, int* counters, float* out_cost,
                                                                float* out_lambda, int* out_iters, int* out_status) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    const bool all_rule = (P.stop_rules & IK_STOP_ALL_COST) != 0;
    if (mode == 1 && all_rule) {
        if (counters[3] != 0) return;
        const int interval = P.check_interval > 0 ? P.check_interval : 1;
        if (k >= 1 && (k % interval) == 0 && counters[(k - 1) % 3] == 0) {
            if (threadIdx.x == 0) counters[3] = 1;
            return;
        }
    }
    if (mode == 0 && blockIdx.x == 0 && threadIdx.x < 4) counters[threadIdx.x] = 0;
    if (mode == 1 && blockIdx.x == 0 && threadIdx.x == 0) counters[(k + 1) % 3] = 0;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    const int ngroups = gridDim.x * (kBlockThreads / G);
    const int rs = rec_stride(h->E);
    for (int p = blockIdx.x * (kBlockThreads / G) + gib; p < batch; p += ngroups) {
        float* r = rec + (size_t)p * rs;
        RecScalars* rsc = reinterpret_cast<RecScalars*>(r + h->E);
        LmState st;
        bool touched = true;
        load_point<G>(g, t, w, p, q, base);
        load_targets<G>(g, t, w, p, batch);
        if (mode == 1) {
            const RecScalars s = *rsc;
            st.cost = s.cost;
            st.lambda = s.lambda;
            st.pos_err = s.pos_err;
            st.rot_err = s.rot_err;
            st.status = s.status;
            st.iters = s.iters;
            st.accepts = s.pad0;
            const bool done = (st.status & (IK_ST_CONVERGED | IK_ST_MAX_ITER | IK_ST_NONFINITE)) != 0;
            touched = !done;
            if (!done)
                for (int e = g.lane; e < h->E; e += G) w.Hs()[e] = r[e];
        }
        if (touched) {
            g.sync();
            group_step<G>(g, t, w, st, P, mode == 0);
        }
        if (mode == 0) {
            check_stop<G>(st, P);
            if (P.max_iter <= 0) st.status |= IK_ST_MAX_ITER;
        }
        if (all_rule && g.lane == 0 && mode == 1 && !(st.cost <= P.cost_tol)) atomicAdd(&counters[k % 3], 1);
        g.sync();
        if (touched)
            for (int e = g.lane; e < h->E; e += G) r[e] = w.Hs()[e];
        if (g.lane == 0) {
            RecScalars s;
            s.cost = st.cost;
            s.lambda = st.lambda;
            s.pos_err = st.pos_err;
            s.rot_err = st.rot_err;
            s.status = st.status;
            s.iters = st.iters;
            s.pad0 = st.accepts;
            s.pad1 = 0;
            *rsc = s;
        }
        store_solution<G>(g, t, w, st, p, q, base, out_cost, out_lambda, out_iters, out_status);
        g.sync();
    }
}

// ---------------------------------------------------------------------------
// persistent form: groups pull problems from a device work queue and iterate
// each to its own stop rule inside the launch.
// ---------------------------------------------------------------------------
template <int G, bool F = true>
__global__ void __launch_bounds__(kBlockThreads, 4) lm_persistent_kernel(const char* __restrict__ blob, int batch,
                                                                     float* q, float* base, IkLmParams P,
                                                                     int* queue, float* out_cost, float* out_lambda,
                                                                     int* out_iters, int* out_status) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    // Each group owns one problem at a time.  A group whose problem stops
    // stores it and takes the next one from the queue at the top of the next
    // round (the warp claims for all such groups with one atomic), so a warp
    // never idles behind its slowest group while the queue still has work.
    const unsigned full = 0xffffffffu;
    const int wg = (threadIdx.x & 31) / G;
    int p = -1;
    bool exhausted = false, fresh = false;
    LmState st;
    while (true) {
        const unsigned need = __ballot_sync(full, p < 0 && g.lane == 0);
        if (need && !exhausted) {
            int first = 0;
            if ((threadIdx.x & 31) == 0) first = atomicAdd(queue, __popc(need));
            first = __shfl_sync(full, first, 0);
            if (first + __popc(need) >= batch) exhausted = true;
            if (p < 0) {
                const int np = first + __popc(need & ((1u << (wg * G)) - 1u));
                if (np < batch) {
                    p = np;
                    fresh = true;
                    load_point<G>(g, t, w, p, q, base);
                    load_targets<G>(g, t, w, p, batch);
                    g.sync();
                }
            }
        }
        if (!__any_sync(full, p >= 0)) {
            if (exhausted) break;
            continue;
        }
        if (p >= 0) {
            bool stop = group_step<G, F>(g, t, w, st, P, fresh);
            if (fresh) stop = start_stops<G>(st, P);
            fresh = false;
            if (stop) {
                store_solution<G>(g, t, w, st, p, q, base, out_cost, out_lambda, out_iters, out_status);
                g.sync();
                // restore the canonical buffer order (the accept path swaps q/qp and base/basep)
                w.bind(group_ws<G>(wsbase, h, gib), h);
                p = -1;
            }
        }
    }
}
}  // namespace b200ik
