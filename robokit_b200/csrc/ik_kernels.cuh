// ik_kernels.cuh — solver and single-stage kernels built from ik_device.cuh.
#pragma once
#include "ik_lm.cuh"

namespace b200ik {

// ---------------------------------------------------------------------------
// single-stage kernels
// ---------------------------------------------------------------------------
template <int G>
__global__ void __launch_bounds__(kBlockThreads) fk_kernel(const char* __restrict__ blob, int batch, const float* q,
                                                          const float* base, float* T_joint, float* T_link,
                                                          float* S_world, float* spheres, float* link_bounds) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    const int ngroups = gridDim.x * (kBlockThreads / G);
    const int nj = h->nj, nl = h->nl, ns = h->ns;
    for (int p = blockIdx.x * (kBlockThreads / G) + gib; p < batch; p += ngroups) {
        load_point<G>(g, t, w, p, q, base);
        g.sync();
        const float* b = cur_base<G>(t, w);
        float* Tj = group_fk<G>(g, t, w, w.q, b);
        if (T_joint)
            for (int it = g.lane; it < nj * 7; it += G) {
                const int j = it / 7, c = it - 7 * j;
                T_joint[((size_t)p * nj + j) * 7 + c] = Tj[8 * j + c];
            }
        if (T_link)
            for (int it = g.lane; it < nl * 7; it += G) {
                const int l = it / 7, c = it - 7 * l;
                const int j = t.lpj()[l];
                float v;
                if (j >= 0)
                    v = Tj[8 * j + c];
                else
                    v = b ? b[c] : (c == 3 ? 1.f : 0.f);
                T_link[((size_t)p * nl + l) * 7 + c] = v;
            }
        if (S_world)
            for (int j = g.lane; j < nj; j += G) {
                V3 v, om;
                joint_subspace(t, Tj, j, v, om);
                float* s = S_world + (size_t)p * 6 * nj;
                s[0 * nj + j] = v.x;
                s[1 * nj + j] = v.y;
                s[2 * nj + j] = v.z;
                s[3 * nj + j] = om.x;
                s[4 * nj + j] = om.y;
                s[5 * nj + j] = om.z;
            }
        if (spheres)
            for (int s = g.lane; s < ns; s += G) {
                const Pose P = link_pose(t, Tj, b, t.sphlink()[s]);
                const float* c = t.sph() + 4 * s;
                const V3 wc = pose_apply(P, V3{c[0], c[1], c[2]});
                float* o = spheres + ((size_t)p * ns + s) * 3;
                o[0] = wc.x;
                o[1] = wc.y;
                o[2] = wc.z;
            }
        if (link_bounds)
            for (int l = g.lane; l < nl; l += G) {
                const Pose P = link_pose(t, Tj, b, l);
                const float* c = t.lbound() + 4 * l;
                const V3 wc = pose_apply(P, V3{c[0], c[1], c[2]});
                float* o = link_bounds + ((size_t)p * nl + l) * 3;
                o[0] = wc.x;
                o[1] = wc.y;
                o[2] = wc.z;
            }
        g.sync();
    }
}

// link Jacobian, robo/robot_kernels.py:668-737 (frame 0 spatial, 1 body)
template <int G>
__global__ void __launch_bounds__(kBlockThreads) link_jacobian_kernel(const char* __restrict__ blob, int batch,
                                                                     const float* q, const float* base, int link,
                                                                     int body, float* J) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    const int ngroups = gridDim.x * (kBlockThreads / G);
    const int D = h->D, boff = h->base_off;
    for (int p = blockIdx.x * (kBlockThreads / G) + gib; p < batch; p += ngroups) {
        load_point<G>(g, t, w, p, q, base);
        g.sync();
        const float* b = cur_base<G>(t, w);
        float* Tj = group_fk<G>(g, t, w, w.q, b);
        float* S = (Tj == w.T0()) ? w.T1() : w.T0();
        for (int j = g.lane; j < h->nj; j += G) {
            V3 v, om;
            joint_subspace(t, Tj, j, v, om);
            float* s = S + 8 * j;
            s[0] = v.x;
            s[1] = v.y;
            s[2] = v.z;
            s[3] = om.x;
            s[4] = om.y;
            s[5] = om.z;
        }
        g.sync();
        const Pose F = link_pose(t, Tj, b, link);
        for (int c = g.lane; c < D; c += G) {
            V3 v, om;
            if (c < boff) {
                const Pose B = pose_load(b);
                if (body) {
                    // Ad(T_frame_base) e_c with T_frame_base = T_frame_world o T_world_base
                    const Pose Fi{0.f, 0.f, 0.f, F.w, -F.i, -F.j, -F.k};
                    const V3 ti = qrot(Fi.w, Fi.i, Fi.j, Fi.k, V3{F.x, F.y, F.z});
                    const Pose Finv{-ti.x, -ti.y, -ti.z, F.w, -F.i, -F.j, -F.k};
                    const Pose FB = compose(Finv, B);
                    if (c < 3) {
                        const V3 e{c == 0 ? 1.f : 0.f, c == 1 ? 1.f : 0.f, c == 2 ? 1.f : 0.f};
                        v = qrot(FB.w, FB.i, FB.j, FB.k, e);
                        om = V3{0.f, 0.f, 0.f};
                    } else {
                        const V3 e{c == 3 ? 1.f : 0.f, c == 4 ? 1.f : 0.f, c == 5 ? 1.f : 0.f};
                        om = qrot(FB.w, FB.i, FB.j, FB.k, e);
                        v = cross(V3{FB.x, FB.y, FB.z}, om);
                    }
                } else {
                    column_twist(t, S, b, c, link, v, om);
                }
            } else {
                column_twist(t, S, b, c, link, v, om);
                if (body) {
                    // Ad(T_frame_world) [v; w] = [R^T (v - t x w); R^T w]
                    const V3 tf{F.x, F.y, F.z};
                    const V3 vv = v - cross(tf, om);
                    v = qrot(F.w, -F.i, -F.j, -F.k, vv);
                    om = qrot(F.w, -F.i, -F.j, -F.k, om);
                }
            }
            float* o = J + (size_t)p * 6 * D;
            o[0 * D + c] = v.x;
            o[1 * D + c] = v.y;
            o[2 * D + c] = v.z;
            o[3 * D + c] = om.x;
            o[4 * D + c] = om.y;
            o[5 * D + c] = om.z;
        }
        g.sync();
    }
}

// residuals + Jacobian rows in the reference row layout (outputs pre-zeroed)
template <int G>
__global__ void __launch_bounds__(kBlockThreads) resjac_kernel(const char* __restrict__ blob, int batch,
                                                              const float* q, const float* base, float* rout,
                                                              float* Jout) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    const int ngroups = gridDim.x * (kBlockThreads / G);
    const int D = h->D, Dp = h->Dp, R = h->R_ref, boff = h->base_off;
    for (int p = blockIdx.x * (kBlockThreads / G) + gib; p < batch; p += ngroups) {
        load_point<G>(g, t, w, p, q, base);
        load_targets<G>(g, t, w, p, batch);
        g.sync();
        const float* b = cur_base<G>(t, w);
        const EvalOut ev = group_eval<G>(g, t, w, w.q, b);
        float* ro = rout ? rout + (size_t)p * R : nullptr;
        float* Jo = Jout ? Jout + (size_t)p * R * D : nullptr;
        // residuals
        if (ro) {
            for (int e = g.lane; e < h->npose; e += G) {
                const PoseEntry& pe = t.pose()[e];
                for (int k = 0; k < pose_entry_rows(pe); ++k) ro[pe.out_row + k] = w.rpose()[pe.r0 + k];
            }
            if (h->has_limit)
                for (int a = g.lane; a < h->na; a += G) ro[h->limit_row + a] = w.rlim()[a];
            for (int je = 0; je < h->njref; ++je) {
                const JointRefEntry& jr = t.jref()[je];
                for (int a = g.lane; a < h->na; a += G) ro[jr.out_row + a] = jref_row(t, w, jr, w.q[a], a).r;
            }
            for (int k = 0; k < h->nscene; ++k) {
                const SceneEntry& se = t.scene()[k];
                for (int i = g.lane; i < se.nq; i += G) ro[se.out_row + i] = scene_row(t, w, se, scene_of(w, se), i).r;
            }
            for (int k = 0; b && k < h->nbref; ++k) {
                float r6[6];
                base_ref_rows(t.bref()[k], w, pose_load(b), r6, nullptr);
                if (g.lane < 6) ro[t.bref()[k].out_row + g.lane] = r6[g.lane];
            }
        }
        float* S = ev.S;
        for (int j = g.lane; j < h->nj; j += G) {
            V3 v, om;
            joint_subspace(t, ev.Tj, j, v, om);
            float* s = S + 8 * j;
            s[0] = v.x;
            s[1] = v.y;
            s[2] = v.z;
            s[3] = om.x;
            s[4] = om.y;
            s[5] = om.z;
        }
        g.sync();
        if (Jo) {
            group_frame_factors<G>(g, t, w, ev.Tj, b);
            for (int e0 = 0; e0 < h->npose;) {
                const int e1 = pose_chunk_end(t, e0);
                group_pose_rows<G>(g, t, w, ev.Tj, S, b, e0, e1);
                const int rbase = t.pose()[e0].r0;
                const int nr = (e1 < h->npose ? t.pose()[e1].r0 : h->pose_rows) - rbase;
                for (int it = g.lane; it < nr * D; it += G) {
                    const int rr = it / D, c = it - rr * D;
                    int el = e0;
                    while (t.pose()[el].r0 + pose_entry_rows(t.pose()[el]) <= rbase + rr) ++el;
                    const int row = t.pose()[el].out_row + (rbase + rr - t.pose()[el].r0);
                    Jo[(size_t)row * D + c] = w.Jc()[rr * Dp + c];
                }
                g.sync();
                e0 = e1;
            }
            if (h->has_limit)
                for (int a = g.lane; a < h->na; a += G) {
                    const float qv = w.q[a];
                    const float lo = t.lim()[2 * a], hi = t.lim()[2 * a + 1];
                    const float sg = qv > hi ? 1.f : (qv < lo ? -1.f : 0.f);
                    Jo[(size_t)(h->limit_row + a) * D + boff + a] = t.limw()[a] * sg;
                }
            for (int je = 0; je < h->njref; ++je) {
                const JointRefEntry& jr = t.jref()[je];
                for (int a = g.lane; a < h->na; a += G)
                    Jo[(size_t)(jr.out_row + a) * D + boff + a] = jref_row(t, w, jr, w.q[a], a).js;
            }
            for (int k = 0; b && k < h->nbref; ++k) {
                if (g.lane < 6) {
                    float r6[6], J6[36];
                    base_ref_rows(t.bref()[k], w, pose_load(b), r6, J6);
                    for (int c = 0; c < D; ++c)
                        Jo[(size_t)(t.bref()[k].out_row + g.lane) * D + c] = c < 6 ? J6[6 * g.lane + c] : 0.f;
                }
            }
            for (int k = 0; k < h->nscene; ++k) {
                const SceneEntry& se = t.scene()[k];
                for (int i = g.lane; i < se.nq; i += G) {
                    const SceneRow sr = scene_row(t, w, se, scene_of(w, se), i);
                    for (int c = 0; c < D; ++c)
                        Jo[(size_t)(se.out_row + i) * D + c] =
                            sr.act ? sr.scale * dot(sr.n, point_column(t, S, b, c, sr.link, sr.p)) : 0.f;
                }
            }
        }
        for (int ci = 0; ci < h->ncoll; ++ci) {
            const CollEntry& ce = t.coll()[ci];
            const int* spk = t.at<int>(ce.o_sp);
            if (ce.mode == 0) {
                const Slot* slots = reinterpret_cast<const Slot*>(w.raw + ce.ws_slots);
                const int nsl = reinterpret_cast<const int*>(w.misc())[8 + ci];
                if (ro)
                    for (int k = g.lane; k < nsl; k += G) ro[ce.out_row + k] = slots[k].r;
                for (int k0 = 0; Jo && k0 < nsl; k0 += kChunkRows) {
                    const int nr = min(kChunkRows, nsl - k0);
                    for (int r = g.lane; r < nr; r += G) {
                        rowmeta_put(w, r, slots[k0 + r].i, slots[k0 + r].j, slots[k0 + r].r);
                    }
                    g.sync();
                    group_collision_rows<G>(g, t, w, S, b, ce, nr);
                    for (int it = g.lane; it < nr * D; it += G) {
                        const int rr = it / D, c = it - rr * D;
                        Jo[(size_t)(ce.out_row + k0 + rr) * D + c] = w.Jc()[rr * Dp + c];
                    }
                    g.sync();
                }
            } else {
                for (int p0 = 0; p0 < ce.nsp; p0 += kChunkRows) {
                    const int nr = min(kChunkRows, ce.nsp - p0);
                    for (int r = g.lane; r < nr; r += G) {
                        const int pk = spk[p0 + r];
                        const float4 a = *reinterpret_cast<const float4*>(w.sph() + 4 * (pk & 0xffff));
                        const float4 bb = *reinterpret_cast<const float4*>(w.sph() + 4 * (pk >> 16));
                        const float d = norm3(V3{a.x - bb.x, a.y - bb.y, a.z - bb.z});
                        const float pen = ce.margin - (d - a.w - bb.w);
                        const float res = ce.weight * fmaxf(0.f, pen);
                        rowmeta_put(w, r, pk & 0xffff, pk >> 16, res);
                        if (ro) ro[ce.out_row + p0 + r] = res;
                    }
                    g.sync();
                    if (Jo) {
                        group_collision_rows<G>(g, t, w, S, b, ce, nr);
                        for (int it = g.lane; it < nr * D; it += G) {
                            const int rr = it / D, c = it - rr * D;
                            Jo[(size_t)(ce.out_row + p0 + rr) * D + c] = w.Jc()[rr * Dp + c];
                        }
                    }
                    g.sync();
                }
            }
        }
        g.sync();
    }
}

// normal equations as the fused solver forms them
template <int G>
__global__ void __launch_bounds__(kBlockThreads) normal_kernel(const char* __restrict__ blob, int batch,
                                                              const float* q, const float* base, float* H, float* gv,
                                                              float* cost) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    const int ngroups = gridDim.x * (kBlockThreads / G);
    const int D = h->D, T = h->T;
    for (int p = blockIdx.x * (kBlockThreads / G) + gib; p < batch; p += ngroups) {
        load_point<G>(g, t, w, p, q, base);
        load_targets<G>(g, t, w, p, batch);
        g.sync();
        const float* b = cur_base<G>(t, w);
        const EvalOut ev = group_eval<G>(g, t, w, w.q, b);
        group_linearize<G>(g, t, w, ev, b);
        if (H)
            for (int e = g.lane; e < T; e += G) {
                const unsigned ab = t.ab()[e];
                const int a = ab >> 8, c = ab & 0xff;
                H[(size_t)p * D * D + a * D + c] = w.Hs()[e];
                H[(size_t)p * D * D + c * D + a] = w.Hs()[e];
            }
        if (gv)
            for (int i = g.lane; i < D; i += G) gv[(size_t)p * D + i] = w.Hs()[T + i];
        if (cost && g.lane == 0) cost[p] = ev.cost;
        g.sync();
    }
}

// damped solve on given H (full D x D), g, lambda
template <int G>
__global__ void __launch_bounds__(kBlockThreads) damped_solve_kernel(const char* __restrict__ blob, int batch,
                                                                    const float* H, const float* gv,
                                                                    const float* lambda, float* delta, float* pred,
                                                                    int* spd) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    const int ngroups = gridDim.x * (kBlockThreads / G);
    const int D = h->D, T = h->T;
    for (int p = blockIdx.x * (kBlockThreads / G) + gib; p < batch; p += ngroups) {
        for (int e = g.lane; e < T; e += G) {
            const unsigned ab = t.ab()[e];
            w.Hs()[e] = H[(size_t)p * D * D + (ab >> 8) * D + (ab & 0xff)];
        }
        for (int i = g.lane; i < D; i += G) w.Hs()[T + i] = gv[(size_t)p * D + i];
        g.sync();
        double pr = 0.0, dn = 0.0;
        const bool ok = group_damped_solve<G>(g, t, w, w.Hs(), lambda[p], pr, dn);
        for (int i = g.lane; i < D; i += G) delta[(size_t)p * D + i] = w.d32()[i];
        if (g.lane == 0) {
            pred[p] = (float)pr;
            if (spd) spd[p] = ok ? 1 : 0;
        }
        g.sync();
    }
}

// one LM iteration with the reference's per-step buffers
template <int G>
__global__ void __launch_bounds__(kBlockThreads) step_kernel(const char* __restrict__ blob, int batch, float* q,
                                                            float* base, float* lambda, IkLmParams P, float* cost,
                                                            float* delta, float* pred, float* cost_new, int* accept) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    const int ngroups = gridDim.x * (kBlockThreads / G);
    const int D = h->D;
    for (int p = blockIdx.x * (kBlockThreads / G) + gib; p < batch; p += ngroups) {
        load_point<G>(g, t, w, p, q, base);
        load_targets<G>(g, t, w, p, batch);
        g.sync();
        LmState st;
        group_start<G>(g, t, w, st, P);
        st.lambda = lambda[p];
        IkLmParams P1 = P;
        P1.stop_rules = 0;
        P1.max_iter = 1 << 30;
        StepTrace tr;
        group_iterate<G>(g, t, w, st, P1, &tr);
        if (delta)
            for (int i = g.lane; i < D; i += G) delta[(size_t)p * D + i] = w.d32()[i];
        if (g.lane == 0) {
            lambda[p] = st.lambda;
            if (cost) cost[p] = tr.accepted ? tr.cost_new : tr.cost_before;
            if (pred) pred[p] = tr.pred;
            if (cost_new) cost_new[p] = tr.cost_new;
            if (accept) accept[p] = tr.accepted;
        }
        store_solution<G>(g, t, w, st, p, q, base, nullptr, nullptr, nullptr, nullptr);
        g.sync();
        w.bind(group_ws<G>(wsbase, h, gib), h);
    }
}

// IK metrics, helpers/ik/ik.py:60-82
template <int G>
__global__ void __launch_bounds__(kBlockThreads) metrics_kernel(const char* __restrict__ blob, int batch,
                                                               const float* q, const float* base, int nt,
                                                               const int* links, const float* targets, float pth,
                                                               float rth, float* perr, float* rerr, int* success) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    Group<G> g;
    Ws w;
    const int gib = threadIdx.x / G;
    w.bind(group_ws<G>(wsbase, h, gib), h);
    const int ngroups = gridDim.x * (kBlockThreads / G);
    for (int p = blockIdx.x * (kBlockThreads / G) + gib; p < batch; p += ngroups) {
        load_point<G>(g, t, w, p, q, base);
        g.sync();
        const float* b = cur_base<G>(t, w);
        float* Tj = group_fk<G>(g, t, w, w.q, b);
        int ok = 1;
        for (int i = g.lane; i < nt; i += G) {
            const Pose L = link_pose(t, Tj, b, links[i]);
            const Pose Tg = pose_load7(targets + ((size_t)p * nt + i) * 7);
            // err = L^-1 o T (se3_inverse_func :70-78, se3_compose_func)
            const V3 ti = qrot(L.w, -L.i, -L.j, -L.k, V3{L.x, L.y, L.z});
            const Pose Li{-ti.x, -ti.y, -ti.z, L.w, -L.i, -L.j, -L.k};
            const Pose E = compose(Li, Tg);
            const float pe = sqrtf(E.x * E.x + E.y * E.y + E.z * E.z);
            const float ae = 2.0f * asinf(fminf(sqrtf(E.i * E.i + E.j * E.j + E.k * E.k), 1.0f));
            perr[(size_t)p * nt + i] = pe;
            rerr[(size_t)p * nt + i] = ae;
            if (pe >= pth || ae >= rth) ok = 0;
        }
        const unsigned bad = g.ballot(ok == 0);
        if (g.lane == 0) success[p] = bad ? 0 : 1;
        g.sync();
    }
}

// integrate a tangent step, robo/robot_kernels.py:563-644 (one thread per problem)
__global__ void integrate_kernel(int batch, int na, int floating, const float* q, const float* base,
                                 const float* delta, const float* mask, float* qo, float* baseo) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= batch) return;
    const int boff = floating ? 6 : 0;
    const int D = boff + na;
    const float* d = delta + (size_t)p * D;
    for (int a = 0; a < na; ++a) {
        const float m = mask ? mask[boff + a] : 1.f;
        qo[(size_t)p * na + a] = q[(size_t)p * na + a] + m * d[boff + a];
    }
    if (floating) {
        float xi[6];
        for (int k = 0; k < 6; ++k) xi[k] = d[k];
        if (mask)
            for (int k = 3; k < 6; ++k) xi[k] *= mask[k];
        const Pose B = pose_load7(base + (size_t)p * 7);
        Pose N = compose(B, se3_exp(xi, 1e-4f));
        if (mask) {
            if (mask[0] == 0.f) N.x = B.x;
            if (mask[1] == 0.f) N.y = B.y;
            if (mask[2] == 0.f) N.z = B.z;
        }
        float* o = baseo + (size_t)p * 7;
        o[0] = N.x;
        o[1] = N.y;
        o[2] = N.z;
        o[3] = N.w;
        o[4] = N.i;
        o[5] = N.j;
        o[6] = N.k;
    }
}

// Independent FMA chains per thread: the CUDA-core FP32 / FP64 throughput the
// roofline of the (non-tensor) IK kernels is stated against.
template <typename T>
__global__ void fma_peak_kernel(T* out, int iters) {
    T a[8];
    const T b = (T)0.9999999, c = (T)1e-7;
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = (T)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
        }
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == (T)-1) out[blockIdx.x] = s;  // keeps the chains live
}

__global__ void copy_rows_kernel(int rows, int width, const float* src, long long ss, float* dst, long long ds) {
    const long long n = (long long)rows * width;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / width, c = i - r * width;
        dst[r * ds + c] = src[r * ss + c];
    }
}

// Row gather: dst[r, :] = src[index[r], :].  An index outside [0, src_rows) leaves its row untouched and is
// counted in *bad (robo/robot_state.py gather, robot_kernels.py gather kernels).
__global__ void gather_rows_kernel(int rows, int width, const int* index, int src_rows, const float* src, float* dst,
                                   int* bad) {
    const long long n = (long long)rows * width;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / width, c = i - r * width;
        const int s = index[r];
        if (s < 0 || s >= src_rows) {
            if (c == 0 && bad) atomicAdd(bad, 1);
            continue;
        }
        dst[i] = src[(long long)s * width + c];
    }
}

__global__ void masked_copy_rows_kernel(int rows, int width, const int* mask, const float* src, float* dst) {
    const long long n = (long long)rows * width;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / width;
        if (mask[r] == 1) dst[i] = src[i];
    }
}

// Row cost: out[r] = (acc ? out[r] : 0) + sum_i x[r, i]^2, summed in column order in FP32 with one fused
// multiply-add per element, one thread per row (opt/optimizer.py:21-33).
__global__ void row_sumsq_kernel(int rows, int width, const float* x, long long stride, float* out, int acc) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows; r += (long long)gridDim.x * blockDim.x) {
        const float* row = x + r * stride;
        float c = acc ? out[r] : 0.f;
        float s = 0.f;
        for (int i = 0; i < width; ++i) s = fmaf(row[i], row[i], s);
        out[r] = c + s;
    }
}

// Homogeneous 4x4 row-major matrices <-> poses [x, y, z, qw, qx, qy, qz] (xform se3_from_matrix /
// se3_to_matrix, used by IKSolver.solve_torch, helpers/ik/ik.py:306-347).  The quaternion follows
// Shepperd's method (J. Guidance and Control 1(3), 1978): the largest of 1 + trace and 1 + 2 R_ii - trace
// picks the component computed from a square root, the others come from off-diagonal sums and
// differences; the result is normalised with qw >= 0.
__global__ void pose_from_matrix_kernel(int n, const float* mats, float* poses) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float* m = mats + i * 16;
        const float r00 = m[0], r01 = m[1], r02 = m[2], r10 = m[4], r11 = m[5], r12 = m[6];
        const float r20 = m[8], r21 = m[9], r22 = m[10];
        const float tr = r00 + r11 + r22;
        float q[4];  // w, x, y, z
        if (tr >= r00 && tr >= r11 && tr >= r22) {
            const float s = 2.f * sqrtf(fmaxf(1.f + tr, 0.f));
            q[0] = 0.25f * s;
            q[1] = (r21 - r12) / s;
            q[2] = (r02 - r20) / s;
            q[3] = (r10 - r01) / s;
        } else if (r00 >= r11 && r00 >= r22) {
            const float s = 2.f * sqrtf(fmaxf(1.f + r00 - r11 - r22, 0.f));
            q[0] = (r21 - r12) / s;
            q[1] = 0.25f * s;
            q[2] = (r01 + r10) / s;
            q[3] = (r02 + r20) / s;
        } else if (r11 >= r22) {
            const float s = 2.f * sqrtf(fmaxf(1.f + r11 - r00 - r22, 0.f));
            q[0] = (r02 - r20) / s;
            q[1] = (r01 + r10) / s;
            q[2] = 0.25f * s;
            q[3] = (r12 + r21) / s;
        } else {
            const float s = 2.f * sqrtf(fmaxf(1.f + r22 - r00 - r11, 0.f));
            q[0] = (r10 - r01) / s;
            q[1] = (r02 + r20) / s;
            q[2] = (r12 + r21) / s;
            q[3] = 0.25f * s;
        }
        float nrm = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if (q[0] < 0.f) nrm = -nrm;
        float* p = poses + i * 7;
        p[0] = m[3];
        p[1] = m[7];
        p[2] = m[11];
        for (int k = 0; k < 4; ++k) p[3 + k] = q[k] / nrm;
    }
}

__global__ void matrix_from_pose_kernel(int n, const float* poses, float* mats) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float* p = poses + i * 7;
        float w = p[3], x = p[4], y = p[5], z = p[6];
        const float inv = 1.f / sqrtf(w * w + x * x + y * y + z * z);
        w *= inv, x *= inv, y *= inv, z *= inv;
        float* m = mats + i * 16;
        m[0] = 1.f - 2.f * (y * y + z * z), m[1] = 2.f * (x * y - w * z), m[2] = 2.f * (x * z + w * y), m[3] = p[0];
        m[4] = 2.f * (x * y + w * z), m[5] = 1.f - 2.f * (x * x + z * z), m[6] = 2.f * (y * z - w * x), m[7] = p[1];
        m[8] = 2.f * (x * z - w * y), m[9] = 2.f * (y * z + w * x), m[10] = 1.f - 2.f * (x * x + y * y), m[11] = p[2];
        m[12] = 0.f, m[13] = 0.f, m[14] = 0.f, m[15] = 1.f;
    }
}

__global__ void keep_previous_kernel(int batch, int na, const float* prev_cost, const float* cost, const float* prev_q,
                                     const float* prev_base, float* q, float* base) {
    const int w = na + (base ? 7 : 0);
    const long long n = (long long)batch * w;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long b = i / w;
        const int c = (int)(i - b * w);
        if (!(prev_cost[b] <= cost[b])) continue;
        if (c < na)
            q[b * na + c] = prev_q[b * na + c];
        else
            base[b * 7 + (c - na)] = prev_base[b * 7 + (c - na)];
    }
}

__global__ void clamp_q_kernel(int batch, int na, float* q, const float* lim, const float* mask) {
    const long long n = (long long)batch * na;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(i % na);
        if (mask && mask[a] == 0.f) continue;
        q[i] = fminf(fmaxf(q[i], lim[2 * a]), lim[2 * a + 1]);
    }
}

// gain-ratio accept/reject on scalars, lm_optimizer.py:338-362 (FP64 ratio)
__global__ void accept_kernel(int batch, float* cost, const float* cost_new, const float* pred, float* lambda,
                              int* accept, IkLmParams P) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= batch) return;
    bool acc = pred[p] > 0.f;
    if (acc) {
        const double rho = ((double)cost[p] - (double)cost_new[p]) / ((double)pred[p] + (double)P.gain_ratio_epsilon);
        acc = rho >= (double)P.rho_min;
    }
    if (acc) {
        accept[p] = 1;
        lambda[p] = fmaxf(lambda[p] / P.lambda_factor, P.lambda_min);
        cost[p] = cost_new[p];
    } else {
        accept[p] = 0;
        lambda[p] = fminf(fmaxf(lambda[p] * P.lambda_factor, P.lambda_min), P.lambda_max);
    }
}

}  // namespace b200ik

namespace b200ik {

// Best `keep` of the `nc` candidates of every instance by cost, ascending,
// equal costs in candidate order and NaN costs last (the select of
// opt/population_solver.py:490-528).  One warp per instance: `keep` passes of
// a warp arg-min over the candidates that come after the last pick in
// (cost, index) order; the picks' points are gathered instance-major.
__global__ void select_best_kernel(int batch, int nc, int keep, const float* __restrict__ cost,
                                   const float* __restrict__ q, const float* __restrict__ base, int na,
                                   float* __restrict__ q_out, float* __restrict__ base_out, float* __restrict__ cost_out,
                                   int* __restrict__ idx_out) {
    const int inst = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (inst >= batch) return;  // uniform per warp
    const float* c = cost + (size_t)inst * nc;
    float last_c = -INFINITY;
    int last_i = -1;
    for (int j = 0; j < keep; ++j) {
        float bc = INFINITY;
        int bi = 0x7fffffff;
        for (int k = lane; k < nc; k += 32) {
            float v = c[k];
            if (!(v == v)) v = INFINITY;
            const bool after = v > last_c || (v == last_c && k > last_i);
            if (after && (v < bc || (v == bc && k < bi))) {
                bc = v;
                bi = k;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float oc = __shfl_xor_sync(0xffffffffu, bc, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (oc < bc || (oc == bc && oi < bi)) {
                bc = oc;
                bi = oi;
            }
        }
        last_c = bc;
        last_i = bi;
        const size_t src = (size_t)inst * nc + bi, dst = (size_t)inst * keep + j;
        for (int a = lane; a < na; a += 32) q_out[dst * na + a] = q[src * na + a];
        if (base && base_out && lane < 7) base_out[dst * 7 + lane] = base[src * 7 + lane];
        if (lane == 0) {
            if (cost_out) cost_out[dst] = c[bi];
            if (idx_out) idx_out[dst] = bi;
        }
    }
}

}  // namespace b200ik
