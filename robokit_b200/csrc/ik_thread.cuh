// ik_thread.cuh — one lane per problem: the LM solve of small systems.
//
// For tangent dimension D <= kSmallD a single lane owns a whole problem:
// forward kinematics in topological joint order, residuals, Jacobian rows
// built one at a time and folded into J^T J / J^T r in registers, and the FP64
// factorisation in registers.  Nothing on a problem's path shuffles or waits
// for other lanes, and a warp carries 32 problems.  Per-problem arrays live in
// shared memory interleaved by lane (float k of lane t at [k * blockDim + t]),
// so the lanes of a warp that touch the same k hit 32 distinct banks.
//
// The arithmetic is that of the lane-group kernels (ik_device.cuh): the same
// residual, Jacobian and accept formulas, FP32 rows with compensated
// accumulation across 32-row chunks, FP64 factorisation and gain ratio.
#pragma once
#include "ik_lm.cuh"

namespace b200ik {

constexpr int kThreadBlock = 64;

// this lane's slice of the interleaved workspace
struct TWs {
    float* p;
    int n;
    __device__ __forceinline__ float& operator[](int k) const { return p[k * n]; }
};

__device__ __forceinline__ Pose tload(const TWs& w, int o) {
    return Pose{w[o], w[o + 1], w[o + 2], w[o + 3], w[o + 4], w[o + 5], w[o + 6]};
}
__device__ __forceinline__ void tstore(const TWs& w, int o, const Pose& P) {
    w[o] = P.x;
    w[o + 1] = P.y;
    w[o + 2] = P.z;
    w[o + 3] = P.w;
    w[o + 4] = P.i;
    w[o + 5] = P.j;
    w[o + 6] = P.k;
}

// where the current point lives: q / base workspace offsets (base < 0: fixed base)
struct TPoint {
    int q, base;
};

// forward kinematics, robo/robot_kernels.py:265-297,390-478: T_world_joint of
// every joint in topological order (base applied last, as the group kernels do)
__device__ __forceinline__ void thread_fk(const Tabs& t, const TWs& w, TPoint x) {
    const TabHeader* h = t.h;
    const int nj = h->nj, oT = h->t_Tj;
    for (int idx = 0; idx < nj; ++idx) {
        const int j = t.jorder()[idx];
        float pos = 0.f;
        const int mim = t.jmimic()[j];
        const int act = t.jact()[j];
        if (mim >= 0)
            pos = w[x.q + mim] * t.jmul()[j] + t.joff()[j];
        else if (act >= 0)
            pos = w[x.q + act];
        const Pose P = pose_load(t.jpt() + 8 * j);
        const int ty = t.jtype()[j];
        const float ax = t.jaxis()[4 * j], ay = t.jaxis()[4 * j + 1], az = t.jaxis()[4 * j + 2];
        Pose X;
        if (ty == 2) {
            float s, c;
            sincosf(pos * 0.5f, &s, &c);
            X = compose(P, Pose{0.f, 0.f, 0.f, c, ax * s, ay * s, az * s});
        } else if (ty == 1) {
            X = compose(P, Pose{ax * pos, ay * pos, az * pos, 1.f, 0.f, 0.f, 0.f});
        } else {
            X = P;
        }
        const int par = t.jparent()[j];
        if (par >= 0) X = compose(tload(w, oT + 7 * par), X);
        tstore(w, oT + 7 * j, X);
    }
    if (x.base >= 0) {
        const Pose B = tload(w, x.base);
        for (int j = 0; j < nj; ++j) tstore(w, oT + 7 * j, compose(B, tload(w, oT + 7 * j)));
    }
}

__device__ __forceinline__ Pose tlink_pose(const Tabs& t, const TWs& w, TPoint x, int link) {
    const int j = t.lpj()[link];
    if (j >= 0) return tload(w, t.h->t_Tj + 7 * j);
    return x.base >= 0 ? tload(w, x.base) : pose_identity();
}

__device__ __forceinline__ V3 tsphere(const TWs& w, int osph, int s) {
    return V3{w[osph + 3 * s], w[osph + 3 * s + 1], w[osph + 3 * s + 2]};
}

// residual of one pose entry (position_task.py:189-212, rotation_task.py:324-349)
__device__ __forceinline__ V3 tpose_residual(const Tabs& t, const TWs& w, const PoseEntry& pe, int e, const Pose& P,
                                             float& err) {
    const int o = t.h->t_tgt + 7 * e;
    if (pe.kind == kPosePosition) {
        const V3 d{w[o] - P.x, w[o + 1] - P.y, w[o + 2] - P.z};
        err = norm3(d);
        return V3{pe.w[0] * d.x, pe.w[1] * d.y, pe.w[2] * d.z};
    }
    float qw, qi, qj, qk;
    qmul_std(P.w, P.i, P.j, P.k, w[o + 3], -w[o + 4], -w[o + 5], -w[o + 6], qw, qi, qj, qk);
    const V3 aa = quat_to_axis_angle(qw, qi, qj, qk, err);
    return V3{pe.w[0] * aa.x, pe.w[1] * aa.y, pe.w[2] * aa.z};
}

// margin - surface distance of sphere pair pk, or <= 0 when clearly apart
__device__ __forceinline__ float tpair_penetration(const Tabs& t, const TWs& w, int osph, int pk, float margin) {
    const int si = pk & 0xffff, sj = pk >> 16;
    const V3 a = tsphere(w, osph, si), b = tsphere(w, osph, sj);
    const float ra = t.sph()[4 * si + 3], rb = t.sph()[4 * sj + 3];
    const V3 d{a.x - b.x, a.y - b.y, a.z - b.z};
    const float thr = margin + ra + rb;
    const float d2 = dot(d, d);
    if (!(thr > 0.f) || d2 >= thr * thr * 1.0001f) return -1.f;
    return margin - (sqrtf(d2) - ra - rb);
}

// every residual at point x: FK, spheres, pose / limit / collision residuals,
// cost 0.5 |r|^2 (compensated) and the largest pose errors; all-pairs
// collision terms record which pairs are active (one bit per pair)
__device__ __forceinline__ EvalOut thread_eval(const Tabs& t, const TWs& w, TPoint x) {
    const TabHeader* h = t.h;
    thread_fk(t, w, x);
    const int osph = h->t_sph;
    if (h->ncoll > 0) {
        for (int s = 0; s < h->ns; ++s) {
            const Pose P = tlink_pose(t, w, x, t.sphlink()[s]);
            const float* c = t.sph() + 4 * s;
            const V3 wc = pose_apply(P, V3{c[0], c[1], c[2]});
            w[osph + 3 * s] = wc.x;
            w[osph + 3 * s + 1] = wc.y;
            w[osph + 3 * s + 2] = wc.z;
        }
    }
    float ks = 0.f, kc = 0.f, max_pos = 0.f, max_rot = 0.f;
    for (int e = 0; e < h->npose; ++e) {
        const PoseEntry& pe = t.pose()[e];
        const Pose P = tlink_pose(t, w, x, pe.link);
        float err;
        const V3 r = tpose_residual(t, w, pe, e, P, err);
        if (pe.kind == kPosePosition)
            max_pos = fmaxf(max_pos, err);
        else
            max_rot = fmaxf(max_rot, err);
        kadd(ks, kc, r.x * r.x);
        kadd(ks, kc, r.y * r.y);
        kadd(ks, kc, r.z * r.z);
    }
    if (h->has_limit) {
        for (int a = 0; a < h->na; ++a) {
            const float v = w[x.q + a];
            const float lo = t.lim()[2 * a], hi = t.lim()[2 * a + 1];
            const float r = t.limw()[a] * (fmaxf(0.f, v - hi) + fmaxf(0.f, lo - v));
            kadd(ks, kc, r * r);
        }
    }
    for (int ci = 0; ci < h->ncoll; ++ci) {
        const CollEntry& ce = t.coll()[ci];
        const int* spk = t.at<int>(ce.o_sp);
        unsigned word = 0u;
        for (int p = 0; p < ce.nsp; ++p) {
            const float pen = tpair_penetration(t, w, osph, spk[p], ce.margin);
            if (pen > 0.f) {
                const float r = ce.weight * pen;
                kadd(ks, kc, r * r);
                word |= 1u << (p & 31);
            }
            if ((p & 31) == 31 || p == ce.nsp - 1) {
                w[ce.t_mask + (p >> 5)] = __uint_as_float(word);
                word = 0u;
            }
        }
    }
    EvalOut o;
    o.cost = 0.5f * (ks + kc);
    o.max_pos = max_pos;
    o.max_rot = max_rot;
    o.Tj = nullptr;
    o.S = nullptr;
    o.nslots = 0;
    return o;
}

// spatial column of tangent column c over the ancestors of `link`
// (position_task.py:242-249,261-272)
__device__ __forceinline__ void tcolumn_twist(const Tabs& t, const TWs& w, TPoint x, int c, int link, V3& v, V3& om) {
    const int boff = t.h->base_off;
    if (c < boff) {
        const Pose B = tload(w, x.base);
        if (c < 3) {
            const V3 e{c == 0 ? 1.f : 0.f, c == 1 ? 1.f : 0.f, c == 2 ? 1.f : 0.f};
            v = qrot(B.w, B.i, B.j, B.k, e);
            om = V3{0.f, 0.f, 0.f};
        } else {
            const V3 e{c == 3 ? 1.f : 0.f, c == 4 ? 1.f : 0.f, c == 5 ? 1.f : 0.f};
            om = qrot(B.w, B.i, B.j, B.k, e);
            v = cross(V3{B.x, B.y, B.z}, om);
        }
        return;
    }
    const int a = c - boff, oS = t.h->t_S;
    v = V3{0.f, 0.f, 0.f};
    om = V3{0.f, 0.f, 0.f};
    const unsigned long long anc = t.lanc()[link];
    for (int idx = t.colstart()[a]; idx < t.colstart()[a + 1]; ++idx) {
        const int j = t.coljoint()[idx];
        if ((anc >> j) & 1ull) {
            const float m = t.colmul()[idx];
            v = v + m * V3{w[oS + 6 * j], w[oS + 6 * j + 1], w[oS + 6 * j + 2]};
            om = om + m * V3{w[oS + 6 * j + 3], w[oS + 6 * j + 4], w[oS + 6 * j + 5]};
        }
    }
}

// d(centre distance)/d(column c) (self_collision_task.py:260-321)
__device__ __forceinline__ float tcollision_column(const Tabs& t, const TWs& w, TPoint x, int c, int li, int lj, V3 ci,
                                                   V3 cj, V3 n) {
    const int boff = t.h->base_off;
    if (c < boff) {
        if (c < 3) return 0.f;
        const Pose B = tload(w, x.base);
        const V3 e{c == 3 ? 1.f : 0.f, c == 4 ? 1.f : 0.f, c == 5 ? 1.f : 0.f};
        const V3 om = qrot(B.w, B.i, B.j, B.k, e);
        return dot(n, cross(om, ci - cj));
    }
    const int a = c - boff, oS = t.h->t_S;
    const unsigned long long ai = t.lanc()[li], aj = t.lanc()[lj];
    float val = 0.f;
    for (int idx = t.colstart()[a]; idx < t.colstart()[a + 1]; ++idx) {
        const int j = t.coljoint()[idx];
        const bool bi = (ai >> j) & 1ull, bj = (aj >> j) & 1ull;
        if (!bi && !bj) continue;
        const V3 v{w[oS + 6 * j], w[oS + 6 * j + 1], w[oS + 6 * j + 2]};
        const V3 om{w[oS + 6 * j + 3], w[oS + 6 * j + 4], w[oS + 6 * j + 5]};
        V3 col_i{0.f, 0.f, 0.f}, col_j{0.f, 0.f, 0.f};
        if (bi) col_i = v + cross(om, ci);
        if (bj) col_j = v + cross(om, cj);
        val += t.colmul()[idx] * dot(n, col_i - col_j);
    }
    return val;
}

// J^T J / J^T r accumulator of one 32-row chunk, in registers
constexpr int kTE = ctri(kSmallD, 0) + kSmallD;

struct TAcc {
    float a[kTE];
    int rows;
    __device__ __forceinline__ void zero() {
        sfor<kTE>([&](auto E) { a[decltype(E)::value] = 0.f; });
        rows = 0;
    }
    // one row: Jacobian entries j (zero past D) and residual r
    __device__ __forceinline__ void row(const float (&j)[kSmallD], float r) {
        sfor<kSmallD>([&](auto I) {
            constexpr int i = decltype(I)::value;
            sfor<i + 1>([&](auto J) {
                constexpr int c = decltype(J)::value;
                a[ctri(i, c)] = fmaf(j[i], j[c], a[ctri(i, c)]);
            });
            a[ctri(kSmallD, 0) + i] = fmaf(r, j[i], a[ctri(kSmallD, 0) + i]);
        });
        rows += 1;
    }
};

// fold the chunk into the compensated sums of the workspace
__device__ __forceinline__ void tacc_flush(const Tabs& t, const TWs& w, TAcc& acc) {
    const int D = t.h->D, T = t.h->T, oH = t.h->t_Hs, oC = t.h->t_Hc;
    sfor<kSmallD>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if (i < D) {
            sfor<i + 1>([&](auto J) {
                constexpr int c = decltype(J)::value;
                float hs = w[oH + ctri(i, c)], hc = w[oC + ctri(i, c)];
                kadd(hs, hc, acc.a[ctri(i, c)]);
                w[oH + ctri(i, c)] = hs;
                w[oC + ctri(i, c)] = hc;
            });
            float hs = w[oH + T + i], hc = w[oC + T + i];
            kadd(hs, hc, acc.a[ctri(kSmallD, 0) + i]);
            w[oH + T + i] = hs;
            w[oC + T + i] = hc;
        }
    });
    acc.zero();
}

__device__ __forceinline__ void tacc_row(const Tabs& t, const TWs& w, TAcc& acc, const float (&j)[kSmallD], float r) {
    acc.row(j, r);
    if (acc.rows == kChunkRows) tacc_flush(t, w, acc);
}

// linearisation at the last evaluated point x (see group_linearize): H and g in
// the workspace at t_Hs (packed lower J^T J, then J^T r)
__device__ __forceinline__ void thread_linearize(const Tabs& t, const TWs& w, TPoint x) {
    const TabHeader* h = t.h;
    const int D = h->D, T = h->T, E = h->E, oS = h->t_S, oT = h->t_Tj, osph = h->t_sph;
    for (int j = 0; j < h->nj; ++j) {
        V3 v{0.f, 0.f, 0.f}, om{0.f, 0.f, 0.f};
        const int ty = t.jtype()[j];
        if (ty != 0) {
            const Pose P = tload(w, oT + 7 * j);
            const V3 a{t.jaxis()[4 * j], t.jaxis()[4 * j + 1], t.jaxis()[4 * j + 2]};
            const V3 Ra = qrot(P.w, P.i, P.j, P.k, a);
            if (ty == 2) {
                om = Ra;
                v = cross(V3{P.x, P.y, P.z}, Ra);
            } else {
                v = Ra;
            }
        }
        w[oS + 6 * j] = v.x;
        w[oS + 6 * j + 1] = v.y;
        w[oS + 6 * j + 2] = v.z;
        w[oS + 6 * j + 3] = om.x;
        w[oS + 6 * j + 4] = om.y;
        w[oS + 6 * j + 5] = om.z;
    }
    for (int e = 0; e < E; ++e) {
        w[h->t_Hs + e] = 0.f;
        w[h->t_Hc + e] = 0.f;
    }
    TAcc acc;
    acc.zero();
    // pose rows (position_task.py:216-272, rotation_task.py:353-401)
    for (int e = 0; e < h->npose; ++e) {
        const PoseEntry& pe = t.pose()[e];
        const Pose P = tlink_pose(t, w, x, pe.link);
        float err;
        const V3 r = tpose_residual(t, w, pe, e, P, err);
        float j0[kSmallD], j1[kSmallD], j2[kSmallD];
        sfor<kSmallD>([&](auto C) {
            constexpr int c = decltype(C)::value;
            j0[c] = j1[c] = j2[c] = 0.f;
            if (c < D) {
                V3 v, om;
                tcolumn_twist(t, w, x, c, pe.link, v, om);
                if (pe.kind == kPosePosition) {
                    const V3 pv = v + cross(om, V3{P.x, P.y, P.z});
                    j0[c] = -pe.w[0] * pv.x;
                    j1[c] = -pe.w[1] * pv.y;
                    j2[c] = -pe.w[2] * pv.z;
                } else {
                    j0[c] = pe.w[0] * om.x;
                    j1[c] = pe.w[1] * om.y;
                    j2[c] = pe.w[2] * om.z;
                }
            }
        });
        tacc_row(t, w, acc, j0, r.x);
        tacc_row(t, w, acc, j1, r.y);
        tacc_row(t, w, acc, j2, r.z);
    }
    // active collision rows, from the evaluation's activity bits
    for (int ci = 0; ci < h->ncoll; ++ci) {
        const CollEntry& ce = t.coll()[ci];
        const int* spk = t.at<int>(ce.o_sp);
        const int nw = (ce.nsp + 31) / 32;
        for (int wi = 0; wi < nw; ++wi) {
            unsigned bits = __float_as_uint(w[ce.t_mask + wi]);
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1u;
                const int pk = spk[32 * wi + b];
                const int si = pk & 0xffff, sj = pk >> 16;
                const V3 cI = tsphere(w, osph, si), cJ = tsphere(w, osph, sj);
                const float ra = t.sph()[4 * si + 3], rb = t.sph()[4 * sj + 3];
                const V3 diff = cI - cJ;
                const float dist = norm3(diff);
                const float pen = ce.margin - (dist - ra - rb);
                const float res = ce.weight * tpair_penetration(t, w, osph, pk, ce.margin);
                float jr[kSmallD];
                sfor<kSmallD>([&](auto C) {
                    constexpr int c = decltype(C)::value;
                    jr[c] = 0.f;
                    if (c < D && pen > 0.f) {
                        const float den = fmaxf(1e-8f, dist);
                        const V3 n{diff.x / den, diff.y / den, diff.z / den};
                        jr[c] = -ce.weight * tcollision_column(t, w, x, c, t.sphlink()[si], t.sphlink()[sj], cI, cJ, n);
                    }
                });
                tacc_row(t, w, acc, jr, res);
            }
        }
    }
    if (acc.rows > 0) tacc_flush(t, w, acc);
    // fold the compensation, joint-limit diagonal (position_limit.py:538-573), DOF mask
    const int boff = h->base_off;
    for (int e = 0; e < E; ++e) {
        float v = w[h->t_Hs + e] + w[h->t_Hc + e];
        int a, b;
        if (e < T) {
            const unsigned ab = t.ab()[e];
            a = ab >> 8;
            b = ab & 0xff;
            if (h->has_limit && a == b && a >= boff) {
                const int k = a - boff;
                const float qv = w[x.q + k];
                const float lo = t.lim()[2 * k], hi = t.lim()[2 * k + 1];
                const float sg = qv > hi ? 1.f : (qv < lo ? -1.f : 0.f);
                const float js = t.limw()[k] * sg;
                v += js * js;
            }
        } else {
            a = e - T;
            b = a;
            if (h->has_limit && a >= boff) {
                const int k = a - boff;
                const float qv = w[x.q + k];
                const float lo = t.lim()[2 * k], hi = t.lim()[2 * k + 1];
                const float sg = qv > hi ? 1.f : (qv < lo ? -1.f : 0.f);
                const float rl = t.limw()[k] * (fmaxf(0.f, qv - hi) + fmaxf(0.f, lo - qv));
                v += t.limw()[k] * sg * rl;
            }
        }
        if (h->mask_any) v *= (e < T) ? t.mask()[a] * t.mask()[b] : t.mask()[a];
        w[h->t_Hs + e] = v;
    }
}

// damped FP64 solve in registers (as group_small_solve); step into d[]
__device__ __forceinline__ bool thread_solve(const Tabs& t, const TWs& w, float lambda_f, double& pred, double& dnorm,
                                             float (&d)[kSmallD]) {
    const int D = t.h->D, T = t.h->T, oH = t.h->t_Hs;
    const double lam = (double)lambda_f;
    double a[ctri(kSmallD, 0)];
    double y[kSmallD];
    sfor<kSmallD>([&](auto I) {
        constexpr int i = decltype(I)::value;
        sfor<i + 1>([&](auto J) {
            constexpr int j = decltype(J)::value;
            double v = (i == j) ? 1.0 : 0.0;
            if (i < D) v = (double)w[oH + ctri(i, j)] + ((i == j) ? lam : 0.0);
            a[ctri(i, j)] = v;
        });
        y[i] = (i < D) ? -(double)w[oH + T + i] : 0.0;
    });
    bool ok = true;
    sfor<kSmallD>([&](auto K) {
        constexpr int k = decltype(K)::value;
        double s = a[ctri(k, k)];
        sfor<k>([&](auto M) { constexpr int m = decltype(M)::value; s -= a[ctri(k, m)] * a[ctri(k, m)]; });
        ok = ok && (s > 0.0);
        const double inv = rsqrt(s);
        a[ctri(k, k)] = inv;
        sfor<kSmallD - k - 1>([&](auto I0) {
            constexpr int i = k + 1 + decltype(I0)::value;
            double v = a[ctri(i, k)];
            sfor<k>([&](auto M) { constexpr int m = decltype(M)::value; v -= a[ctri(i, m)] * a[ctri(k, m)]; });
            a[ctri(i, k)] = v * inv;
        });
    });
    if (!ok) {
        sfor<kSmallD>([&](auto I) { d[decltype(I)::value] = 0.f; });
        pred = 0.0;
        dnorm = 0.0;
        return false;
    }
    sfor<kSmallD>([&](auto I) {
        constexpr int i = decltype(I)::value;
        double v = y[i];
        sfor<i>([&](auto M) { constexpr int m = decltype(M)::value; v -= a[ctri(i, m)] * y[m]; });
        y[i] = v * a[ctri(i, i)];
    });
    sfor<kSmallD>([&](auto I0) {
        constexpr int i = kSmallD - 1 - decltype(I0)::value;
        double v = y[i];
        sfor<kSmallD - 1 - i>([&](auto M0) {
            constexpr int m = i + 1 + decltype(M0)::value;
            v -= a[ctri(m, i)] * y[m];
        });
        y[i] = v * a[ctri(i, i)];
    });
    double pp = 0.0, nn = 0.0;
    sfor<kSmallD>([&](auto I) {
        constexpr int i = decltype(I)::value;
        d[i] = 0.f;
        if (i < D) {
            pp += y[i] * (lam * y[i] - (double)w[oH + T + i]);
            nn += y[i] * y[i];
            d[i] = (float)y[i];
        }
    });
    pred = 0.5 * pp;
    dnorm = sqrt(nn);
    return true;
}

// q' = q + mask * delta, base' = base * exp(delta_base) (robo/robot_kernels.py:563-644)
__device__ __forceinline__ void thread_integrate(const Tabs& t, const TWs& w, TPoint x, TPoint xo,
                                                 const float (&d)[kSmallD]) {
    const TabHeader* h = t.h;
    const int boff = h->base_off;
    sfor<kSmallD>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if (i >= boff && i - boff < h->na) {
            const int a = i - boff;
            const float m = h->mask_any ? t.mask()[i] : 1.f;
            w[xo.q + a] = w[x.q + a] + m * d[i];
        }
    });
    if (boff) {
        float xi[6];
        sfor<6>([&](auto K) { xi[decltype(K)::value] = d[decltype(K)::value]; });
        if (h->mask_any)
            for (int k = 3; k < 6; ++k) xi[k] *= t.mask()[k];
        const Pose B = tload(w, x.base);
        Pose N = compose(B, se3_exp(xi, 1e-4f));
        if (h->mask_any) {
            if (t.mask()[0] == 0.f) N.x = B.x;
            if (t.mask()[1] == 0.f) N.y = B.y;
            if (t.mask()[2] == 0.f) N.z = B.z;
        }
        tstore(w, xo.base, N);
    }
}

__device__ __forceinline__ void thread_start(const Tabs& t, const TWs& w, TPoint x, LmState& st, const IkLmParams& P) {
    const EvalOut ev = thread_eval(t, w, x);
    st.cost = ev.cost;
    st.pos_err = ev.max_pos;
    st.rot_err = ev.max_rot;
    st.lambda = P.lambda_init;
    st.status = isfinite(ev.cost) ? IK_ST_RUNNING : IK_ST_NONFINITE;
    st.iters = 0;
    st.accepts = 0;
    thread_linearize(t, w, x);
}

// one LM iteration from the cached linearisation (as group_iterate); x and xp
// swap when the step is accepted.  Returns true when the problem stops.
__device__ __forceinline__ bool thread_iterate(const Tabs& t, const TWs& w, TPoint& x, TPoint& xp, LmState& st,
                                               const IkLmParams& P) {
    double pred = 0.0, dnorm = 0.0;
    float d[kSmallD];
    const bool ok = thread_solve(t, w, st.lambda, pred, dnorm, d);
    if (!ok) st.status |= IK_ST_NOT_SPD;
    if ((P.stop_rules & IK_STOP_STEP) && ok && dnorm < (double)P.step_tol) {
        st.status |= IK_ST_CONVERGED;
        return true;
    }
    thread_integrate(t, w, x, xp, d);
    const EvalOut ev = thread_eval(t, w, xp);
    bool acc = pred > 0.0;
    if (acc) {
        const double rho = ((double)st.cost - (double)ev.cost) / (pred + (double)P.gain_ratio_epsilon);
        acc = rho >= (double)P.rho_min;
    }
    if (acc) {
        const TPoint tmp = x;
        x = xp;
        xp = tmp;
        st.cost = ev.cost;
        st.pos_err = ev.max_pos;
        st.rot_err = ev.max_rot;
        st.lambda = fmaxf(st.lambda / P.lambda_factor, P.lambda_min);
        st.accepts += 1;
        thread_linearize(t, w, x);
    } else {
        st.lambda = fminf(fmaxf(st.lambda * P.lambda_factor, P.lambda_min), P.lambda_max);
    }
    st.iters += 1;
    bool stop = check_stop<1>(st, P);
    if (!stop && st.iters >= P.max_iter) {
        st.status |= IK_ST_MAX_ITER;
        stop = true;
    }
    return stop;
}

__device__ __forceinline__ TPoint tpoint0(const TabHeader* h) { return TPoint{h->t_q, h->base_off ? h->t_base : -1}; }
__device__ __forceinline__ TPoint tpoint1(const TabHeader* h) { return TPoint{h->t_qp, h->base_off ? h->t_basep : -1}; }

__device__ __forceinline__ void thread_load(const Tabs& t, const TWs& w, TPoint x, int p, int batch, const float* q,
                                            const float* base) {
    const TabHeader* h = t.h;
    for (int a = 0; a < h->na; ++a) w[x.q + a] = q[(size_t)p * h->na + a];
    if (x.base >= 0)
        for (int k = 0; k < 7; ++k) w[x.base + k] = base[(size_t)p * 7 + k];
    for (int e = 0; e < h->npose; ++e) {
        const PoseEntry& pe = t.pose()[e];
        const int rows = pe.target_rows > 0 ? pe.target_rows : batch;
        int rep = batch / rows;
        if (rep < 1) rep = 1;
        const int row = min(p / rep, rows - 1);
        const float* src = pe.targets + ((size_t)row * pe.num_frames + pe.frame) * 7;
        for (int c = 0; c < 7; ++c) w[h->t_tgt + 7 * e + c] = src[c];
    }
}

__device__ __forceinline__ void thread_store(const Tabs& t, const TWs& w, TPoint x, const LmState& st, int p, float* q,
                                             float* base, float* cost, float* lambda, int* iters, int* status) {
    const TabHeader* h = t.h;
    for (int a = 0; a < h->na; ++a) q[(size_t)p * h->na + a] = w[x.q + a];
    if (x.base >= 0)
        for (int k = 0; k < 7; ++k) base[(size_t)p * 7 + k] = w[x.base + k];
    if (cost) cost[p] = st.cost;
    if (lambda) lambda[p] = st.lambda;
    if (iters) iters[p] = st.iters;
    if (status) status[p] = (st.status & IK_ST_FLAGS) | (st.accepts << 8);
}

// ---------------------------------------------------------------------------
// persistent form, one lane per problem: a lane whose problem stops stores it
// and takes the next one (the warp claims for all such lanes with one atomic)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreadBlock, 6) lm_thread_persistent_kernel(const char* __restrict__ blob, int batch,
                                                                            float* q, float* base, IkLmParams P,
                                                                            int* queue, float* out_cost,
                                                                            float* out_lambda, int* out_iters,
                                                                            int* out_status) {
    extern __shared__ __align__(16) char smem[];
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    const TWs w{reinterpret_cast<float*>(wsbase) + threadIdx.x, (int)blockDim.x};
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int p = -1;
    bool exhausted = false;
    LmState st;
    TPoint x = tpoint0(h), xp = tpoint1(h);
    while (true) {
        const unsigned need = __ballot_sync(full, p < 0);
        if (need && !exhausted) {
            int first = 0;
            if (lane == 0) first = atomicAdd(queue, __popc(need));
            first = __shfl_sync(full, first, 0);
            if (first + __popc(need) >= batch) exhausted = true;
            if (p < 0) {
                const int np = first + __popc(need & ((1u << lane) - 1u));
                if (np < batch) {
                    p = np;
                    x = tpoint0(h);
                    xp = tpoint1(h);
                    thread_load(t, w, x, p, batch, q, base);
                    thread_start(t, w, x, st, P);
                    if ((st.status & IK_ST_NONFINITE) != 0 || check_stop<1>(st, P) || P.max_iter <= 0) {
                        if (st.iters >= P.max_iter && !(st.status & IK_ST_CONVERGED)) st.status |= IK_ST_MAX_ITER;
                        thread_store(t, w, x, st, p, q, base, out_cost, out_lambda, out_iters, out_status);
                        p = -1;
                    }
                }
            }
        }
        if (!__any_sync(full, p >= 0)) {
            if (exhausted) break;
            continue;
        }
        if (p >= 0 && thread_iterate(t, w, x, xp, st, P)) {
            thread_store(t, w, x, st, p, q, base, out_cost, out_lambda, out_iters, out_status);
            p = -1;
        }
    }
}

// ---------------------------------------------------------------------------
// plain form, one lane per problem (as lm_plain_kernel): mode 0 = start,
// mode 1 = one iteration; state round-trips through `rec`
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreadBlock, 6) lm_thread_plain_kernel(const char* __restrict__ blob, int batch,
                                                                       float* q, float* base, float* rec,
                                                                       IkLmParams P, int mode, int k, int* counters,
                                                                       float* out_cost, float* out_lambda,
                                                                       int* out_iters, int* out_status) {
    extern __shared__ __align__(16) char smem[];
    const bool all_rule = (P.stop_rules & IK_STOP_ALL_COST) != 0;
    if (mode == 1 && all_rule) {
        if (counters[3] != 0) return;
        const int interval = P.check_interval > 0 ? P.check_interval : 1;
        if (k >= 1 && (k % interval) == 0 && counters[(k - 1) % 3] == 0) {
            if (threadIdx.x == 0) counters[3] = 1;
            return;
        }
    }
    char* wsbase = stage_tables(blob, smem);
    Tabs t;
    t.bind(smem);
    const TabHeader* h = t.h;
    if (mode == 0 && blockIdx.x == 0 && threadIdx.x < 4) counters[threadIdx.x] = 0;
    if (mode == 1 && blockIdx.x == 0 && threadIdx.x == 0) counters[(k + 1) % 3] = 0;
    const TWs w{reinterpret_cast<float*>(wsbase) + threadIdx.x, (int)blockDim.x};
    const int rs = rec_stride(h->E);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < batch; p += gridDim.x * blockDim.x) {
        float* r = rec + (size_t)p * rs;
        RecScalars* rsc = reinterpret_cast<RecScalars*>(r + h->E);
        LmState st;
        bool touched = true;
        TPoint x = tpoint0(h), xp = tpoint1(h);
        thread_load(t, w, x, p, batch, q, base);
        if (mode == 0) {
            thread_start(t, w, x, st, P);
            check_stop<1>(st, P);
            if (P.max_iter <= 0) st.status |= IK_ST_MAX_ITER;
        } else {
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
            if (!done) {
                for (int e = 0; e < h->E; ++e) w[h->t_Hs + e] = r[e];
                thread_iterate(t, w, x, xp, st, P);
            }
        }
        if (all_rule && mode == 1 && !(st.cost <= P.cost_tol)) atomicAdd(&counters[k % 3], 1);
        if (touched)
            for (int e = 0; e < h->E; ++e) r[e] = w[h->t_Hs + e];
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
        thread_store(t, w, x, st, p, q, base, out_cost, out_lambda, out_iters, out_status);
    }
}

}  // namespace b200ik
