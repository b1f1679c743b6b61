/*
 * ik_oracle.c — FP64 CPU restatement of robokit's batched Levenberg–Marquardt
 * inverse kinematics (the path of opt/lm_optimizer.py).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline; never part of the product.  Each routine cites the reference code
 * it restates.  Parity pinning: tests/test_oracle.py checks this code against
 * the reference's FK and Jacobian golden files (tests/robo/fk_ground_truth.json,
 * tests/robo/jacobian_ground_truth.json, panda entries) committed under
 * tests/golden/, and against the reference's accept/reject and LM-step tests.
 *
 * Deliberate choices where the reference leaves freedom:
 *  - self-collision slots take the first K penetrating link pairs in link-pair
 *    order; the reference's set is the atomic-claim subset when more than K
 *    link pairs penetrate (self_collision_task.py:110-122) and its slot order
 *    is a hash order (:104-159).  Cost, J^T J and J^T r do not depend on slot
 *    order.
 */
#include "ik_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define MAXJ 64
#define MAXL 128
#define MAXD 64

typedef struct {
    double t[3];
    double q[4]; /* w x y z */
} P7;

static P7 p7_identity(void) {
    P7 p = {{0, 0, 0}, {1, 0, 0, 0}};
    return p;
}

static void cross3(const double* a, const double* b, double* o) {
    const double x = a[1] * b[2] - a[2] * b[1];
    const double y = a[2] * b[0] - a[0] * b[2];
    const double z = a[0] * b[1] - a[1] * b[0];
    o[0] = x;
    o[1] = y;
    o[2] = z;
}
static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* quaternion_apply_func, xform/warp/rotation_conversions.py:192-200 */
static void qrot(const double* q, const double* v, double* o) {
    double uv[3], uuv[3];
    cross3(q + 1, v, uv);
    cross3(q + 1, uv, uuv);
    for (int k = 0; k < 3; ++k) o[k] = v[k] + 2.0 * (q[0] * uv[k] + uuv[k]);
}

/* quaternion_multiply_func with standardisation, rotation_conversions.py:268-279 */
static void qmul(const double* a, const double* b, double* o) {
    double w = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    double x = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
    double y = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
    double z = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
    if (w < 0) {
        w = -w;
        x = -x;
        y = -y;
        z = -z;
    }
    o[0] = w;
    o[1] = x;
    o[2] = y;
    o[3] = z;
}

/* se3_compose_func, lie/se3_kernels.py:88-109 */
static P7 compose(const P7* A, const P7* B) {
    P7 o;
    double rt[3];
    qmul(A->q, B->q, o.q);
    qrot(A->q, B->t, rt);
    for (int k = 0; k < 3; ++k) o.t[k] = A->t[k] + rt[k];
    return o;
}

/* se3_inverse_func, lie/se3_kernels.py:70-78 */
static P7 inverse(const P7* A) {
    P7 o;
    o.q[0] = A->q[0];
    o.q[1] = -A->q[1];
    o.q[2] = -A->q[2];
    o.q[3] = -A->q[3];
    double t[3];
    qrot(o.q, A->t, t);
    for (int k = 0; k < 3; ++k) o.t[k] = -t[k];
    return o;
}

static P7 p7_from_f(const float* p) {
    P7 o;
    for (int k = 0; k < 3; ++k) o.t[k] = p[k];
    for (int k = 0; k < 4; ++k) o.q[k] = p[3 + k];
    return o;
}
static void p7_to_d(const P7* p, double* o) {
    for (int k = 0; k < 3; ++k) o[k] = p->t[k];
    for (int k = 0; k < 4; ++k) o[3 + k] = p->q[k];
}

/* se3_exp_map_func with regularised angle, lie/se3_kernels.py:126-167 */
static P7 se3_exp(const double* xi, double eps) {
    const double* tl = xi;
    const double* rl = xi + 3;
    const double asq = dot3(rl, rl);
    const double asr = asq + eps * eps;
    const double ar = sqrt(asr);
    const double k = sin(0.5 * ar) / ar;
    double q[4] = {cos(0.5 * ar), k * rl[0], k * rl[1], k * rl[2]};
    const double qn = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int i = 0; i < 4; ++i) q[i] /= qn;
    const double A = sin(ar) / ar;
    const double c1 = (1.0 - cos(ar)) / asr;
    const double c2 = (1.0 - A) / asr;
    double kt[3], kkt[3];
    cross3(rl, tl, kt);
    cross3(rl, kt, kkt);
    P7 o;
    for (int i = 0; i < 3; ++i) o.t[i] = tl[i] + c1 * kt[i] + c2 * kkt[i];
    for (int i = 0; i < 4; ++i) o.q[i] = q[i];
    return o;
}

/* quaternion_to_axis_angle_func, rotation_conversions.py:228-247 */
static void quat_axis_angle(const double* q, double* o) {
    const double n = sqrt(q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const double half = atan2(n, q[0]);
    const double angle = 2.0 * half;
    double s;
    if (fabs(angle) < 1e-6)
        s = 0.5 - angle * angle / 48.0;
    else
        s = sin(half) / angle;
    for (int k = 0; k < 3; ++k) o[k] = q[1 + k] / s;
}

/* 3x3 helpers, row-major */
static void m3_hat(const double* a, double* H) {
    H[0] = 0.0; H[1] = -a[2]; H[2] = a[1];
    H[3] = a[2]; H[4] = 0.0; H[5] = -a[0];
    H[6] = -a[1]; H[7] = a[0]; H[8] = 0.0;
}
static void m3_mul(const double* A, const double* B, double* C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
static void m3_quat(const double* q, double* R) {
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z); R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z); R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y); R[7] = 2 * (y * z + w * x); R[8] = 1 - 2 * (x * x + y * y);
}

/* SE(3) logarithm [V^-1(w) t; w], V^-1 = I - W/2 + c2 W^2 (se3_log_map_func and
 * se3_V_matrix_inverse_func, lie/se3_kernels.py:230-311; eps 1e-4 as frame_task.py:523) */
static void se3_log6(const P7* E, double* out) {
    double w[3];
    quat_axis_angle(E->q, w);
    const double th = sqrt(dot3(w, w));
    double c2 = 1.0 / 12.0;
    if (!(th < 1e-4)) {
        const double omc = 1.0 - cos(th);
        if (!(fabs(omc) < 1e-4)) c2 = (1.0 / (th * th)) * (1.0 - (th * sin(th)) / (2.0 * omc));
    }
    double wt[3], wwt[3];
    cross3(w, E->t, wt);
    cross3(w, wt, wwt);
    for (int k = 0; k < 3; ++k) {
        out[k] = E->t[k] - 0.5 * wt[k] + c2 * wwt[k];
        out[3 + k] = w[k];
    }
}

/* 6x6 SE(3) jlog (se3_jlog_func, lie/se3_kernels.py:359-428, with so3_jac_left_inv_func,
 * lie/so3_kernels.py:14-40): [[A, B], [0, A]], A = Jl^-1(w)^T; eps 1e-4 on |w|^2 */
static void se3_jlog6(const P7* F, double* M) {
    double w[3], W[9], W2[9], A[9], B[9], Hp[9];
    quat_axis_angle(F->q, w);
    const double th2 = dot3(w, w);
    const int taylor = th2 < 1e-4;
    m3_hat(w, W);
    m3_mul(W, W, W2);
    double coeff = 1.0 / 12.0, th = 1.0;
    if (!taylor) {
        th = sqrt(th2);
        coeff = (1.0 - th * cos(0.5 * th) / (2.0 * sin(0.5 * th))) / th2;
    }
    for (int k = 0; k < 9; ++k) A[k] = ((k % 4) == 0 ? 1.0 : 0.0) + 0.5 * W[k] + coeff * W2[k];
    m3_hat(F->t, Hp);
    if (taylor) {
        for (int k = 0; k < 9; ++k) B[k] = 0.5 * Hp[k];
    } else {
        const double st = sin(th), ct = cos(th), inv = 1.0 / th, inv2 = inv * inv;
        const double i22 = 1.0 / (2.0 * (1.0 - ct));
        const double beta = inv2 - st * inv * i22;
        const double bdot = -2.0 * inv2 * inv2 + (1.0 + st * inv) * inv2 * i22;
        const double wtp = dot3(w, F->t);
        double C[9];
        for (int i = 0; i < 3; ++i) {
            const double v3 = bdot * wtp * w[i] - (th2 * bdot + 2.0 * beta) * F->t[i];
            for (int j = 0; j < 3; ++j)
                C[3 * i + j] = v3 * w[j] + beta * w[i] * F->t[j] + (i == j ? wtp * beta : 0.0) + 0.5 * Hp[3 * i + j];
        }
        m3_mul(C, A, B);
    }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double v = 0.0;
            if (i < 3 && j < 3) v = A[3 * i + j];
            else if (i < 3) v = B[3 * i + j - 3];
            else if (j >= 3) v = A[3 * (i - 3) + j - 3];
            M[6 * i + j] = v;
        }
}

/* 6x6 adjoint [[R, hat(t) R], [0, R]] (se3_adjoint_func, lie/se3_kernels.py:314-346) */
static void se3_adjoint6(const P7* T, double* M) {
    double R[9], H[9], HR[9];
    m3_quat(T->q, R);
    m3_hat(T->t, H);
    m3_mul(H, R, HR);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double v = 0.0;
            if (i < 3 && j < 3) v = R[3 * i + j];
            else if (i < 3) v = HR[3 * i + j - 3];
            else if (j >= 3) v = R[3 * (i - 3) + j - 3];
            M[6 * i + j] = v;
        }
}

/* ------------------------------------------------------------------------ */
/* per-problem kinematic state                                               */
/* ------------------------------------------------------------------------ */
typedef struct {
    P7 Tj[MAXJ];
    double S[MAXJ][6];
    P7 base;
    int floating;
} Kin;

static unsigned long long link_ancestors(const OrRobot* r, int link) {
    unsigned long long m = 0ull;
    int j = r->link_parent_joints[link];
    while (j != -1) {
        m |= 1ull << j;
        j = r->parent_joints[j];
    }
    return m;
}

/* FK, robo/robot_kernels.py:265-297 (local transform) and the ancestor
 * composition of compute_forward_kinematics_accum_kernel :328-377; motion
 * subspace Ad(T_world_joint) twist, :651-664. */
static void fk_one(const OrRobot* r, const double* q, const P7* base, Kin* K) {
    P7 local[MAXJ];
    for (int j = 0; j < r->nj; ++j) {
        double pos = 0.0;
        const int mim = r->mimic_indices[j], act = r->actuated_indices[j];
        if (mim >= 0)
            pos = q[mim] * (double)r->mimic_multipliers[j] + (double)r->mimic_offsets[j];
        else if (act >= 0)
            pos = q[act];
        const P7 P = p7_from_f(r->parent_transforms + 7 * j);
        const float* ax = r->joint_axes + 3 * j;
        P7 X = p7_identity();
        if (r->joint_types[j] == 2) {
            const double s = sin(0.5 * pos), c = cos(0.5 * pos);
            X.q[0] = c;
            X.q[1] = ax[0] * s;
            X.q[2] = ax[1] * s;
            X.q[3] = ax[2] * s;
        } else if (r->joint_types[j] == 1) {
            X.t[0] = ax[0] * pos;
            X.t[1] = ax[1] * pos;
            X.t[2] = ax[2] * pos;
        }
        local[j] = compose(&P, &X);
    }
    for (int j = 0; j < r->nj; ++j) {
        P7 Xw = local[j];
        int p = r->parent_joints[j];
        while (p != -1) {
            Xw = compose(&local[p], &Xw);
            p = r->parent_joints[p];
        }
        K->Tj[j] = compose(base, &Xw);
        /* S = Ad(T) twist; revolute twist [0; a], prismatic [a; 0] */
        const float* ax = r->joint_axes + 3 * j;
        const double a[3] = {ax[0], ax[1], ax[2]};
        double Ra[3];
        qrot(K->Tj[j].q, a, Ra);
        for (int k = 0; k < 6; ++k) K->S[j][k] = 0.0;
        if (r->joint_types[j] == 2) {
            double v[3];
            cross3(K->Tj[j].t, Ra, v);
            for (int k = 0; k < 3; ++k) {
                K->S[j][k] = v[k];
                K->S[j][3 + k] = Ra[k];
            }
        } else if (r->joint_types[j] == 1) {
            for (int k = 0; k < 3; ++k) K->S[j][k] = Ra[k];
        }
    }
    K->base = *base;
}

static P7 link_pose(const OrRobot* r, const Kin* K, int link) {
    const int j = r->link_parent_joints[link];
    return j >= 0 ? K->Tj[j] : K->base;
}

/* spatial column of tangent column c restricted to the ancestors of `link`
 * (position_task.py:242-249, 261-272; robot_kernels.py:668-737) */
static void column_twist(const OrRobot* r, const Kin* K, int floating, int c, int link, double* v, double* w) {
    const int boff = floating ? 6 : 0;
    for (int k = 0; k < 3; ++k) v[k] = w[k] = 0.0;
    if (c < boff) {
        double e[3] = {0, 0, 0};
        e[c % 3] = 1.0;
        double Re[3];
        qrot(K->base.q, e, Re);
        if (c < 3) {
            for (int k = 0; k < 3; ++k) v[k] = Re[k];
        } else {
            for (int k = 0; k < 3; ++k) w[k] = Re[k];
            cross3(K->base.t, Re, v);
        }
        return;
    }
    const int a = c - boff;
    const unsigned long long anc = link_ancestors(r, link);
    for (int j = 0; j < r->nj; ++j) {
        if (!((anc >> j) & 1ull)) continue;
        double m = 0.0;
        if (r->actuated_indices[j] == a)
            m = 1.0;
        else if (r->actuated_indices[j] < 0 && r->mimic_indices[j] == a)
            m = r->mimic_multipliers[j];
        if (m == 0.0) continue;
        for (int k = 0; k < 3; ++k) {
            v[k] += K->S[j][k] * m;
            w[k] += K->S[j][3 + k] * m;
        }
    }
}

/* world sphere centres (robo/robot.py:428; robot_kernels.py:469-478) */
static void world_spheres(const OrRobot* r, const Kin* K, double* c /*[ns*3]*/) {
    for (int s = 0; s < r->ns; ++s) {
        const P7 P = link_pose(r, K, r->sphere_links[s]);
        const double lc[3] = {r->sphere_centers[3 * s], r->sphere_centers[3 * s + 1], r->sphere_centers[3 * s + 2]};
        double w[3];
        qrot(P.q, lc, w);
        for (int k = 0; k < 3; ++k) c[3 * s + k] = w[k] + P.t[k];
    }
}

static double sph_dist(const double* C, int i, int j) {
    const double d[3] = {C[3 * i] - C[3 * j], C[3 * i + 1] - C[3 * j + 1], C[3 * i + 2] - C[3 * j + 2]};
    return sqrt(dot3(d, d));
}

/* row of d(distance)/d(tangent) for a sphere pair, self_collision_task.py:260-321 */
static void collision_row(const OrRobot* r, const Kin* K, int floating, const double* C, int si, int sj, double* row,
                          int D) {
    const int boff = floating ? 6 : 0;
    const double* ci = C + 3 * si;
    const double* cj = C + 3 * sj;
    double diff[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
    const double dist = sqrt(dot3(diff, diff));
    const double den = dist > 1e-8 ? dist : 1e-8;
    const double n[3] = {diff[0] / den, diff[1] / den, diff[2] / den};
    for (int c = 0; c < D; ++c) row[c] = 0.0;
    if (floating) {
        for (int c = 3; c < 6; ++c) {
            double e[3] = {0, 0, 0}, om[3], rc[3];
            e[c - 3] = 1.0;
            qrot(K->base.q, e, om);
            cross3(om, diff, rc);
            row[c] = dot3(n, rc);
        }
    }
    const unsigned long long ai = link_ancestors(r, r->sphere_links[si]);
    const unsigned long long aj = link_ancestors(r, r->sphere_links[sj]);
    for (int j = 0; j < r->nj; ++j) {
        const int bi = (ai >> j) & 1ull, bj = (aj >> j) & 1ull;
        if (!bi && !bj) continue;
        int col;
        double m;
        if (r->actuated_indices[j] >= 0) {
            col = r->actuated_indices[j];
            m = 1.0;
        } else if (r->mimic_indices[j] >= 0) {
            col = r->mimic_indices[j];
            m = r->mimic_multipliers[j];
        } else
            continue;
        const double* v = K->S[j];
        const double* om = K->S[j] + 3;
        double coli[3] = {0, 0, 0}, colj[3] = {0, 0, 0}, t[3];
        if (bi) {
            cross3(om, ci, t);
            for (int k = 0; k < 3; ++k) coli[k] = v[k] + t[k];
        }
        if (bj) {
            cross3(om, cj, t);
            for (int k = 0; k < 3; ++k) colj[k] = v[k] + t[k];
        }
        const double dd[3] = {coli[0] - colj[0], coli[1] - colj[1], coli[2] - colj[2]};
        row[boff + col] += m * dot3(n, dd);
    }
}

/* Scene SDF at world point p over the primitives of scene `sid` in query order:
 * the first of strictly least signed distance and its world normal
 * (geom/sdf_kernels.py:223-344); 1e6 and a zero normal for an empty scene. */
static double scene_sdf(const OrTerm* t, int sid, const double* p, double* n_out) {
    double best = 1.0e6;
    n_out[0] = n_out[1] = n_out[2] = 0.0;
    for (int e = 0; e < t->num_geoms; ++e) {
        const float* g = t->geoms + (size_t)e * 16;
        if ((int)g[1] != sid) continue;
        const int type = (int)g[0];
        const double s = g[2];
        P7 P;
        P.t[0] = g[8], P.t[1] = g[9], P.t[2] = g[10];
        double qn = sqrt((double)g[11] * g[11] + (double)g[12] * g[12] + (double)g[13] * g[13] + (double)g[14] * g[14]);
        P.q[0] = g[11] / qn, P.q[1] = g[12] / qn, P.q[2] = g[13] / qn, P.q[3] = g[14] / qn;
        const P7 Pi = inverse(&P);
        double ql[3];
        qrot(Pi.q, p, ql);
        for (int k = 0; k < 3; ++k) ql[k] = (ql[k] + Pi.t[k]) / s;
        double un = 0.0, nl[3] = {0.0, 0.0, 1.0};
        if (type == 0) { /* box */
            const double he[3] = {g[4], g[5], g[6]};
            double qv[3], qp[3];
            for (int k = 0; k < 3; ++k) {
                qv[k] = fabs(ql[k]) - he[k];
                qp[k] = qv[k] > 0 ? qv[k] : 0.0;
            }
            const double qmax = fmax(fmax(qv[0], qv[1]), qv[2]);
            un = sqrt(dot3(qp, qp)) + (qmax < 0 ? qmax : 0.0);
            if (qmax < 0) {
                int ax = (qv[0] >= qv[1] && qv[0] >= qv[2]) ? 0 : (qv[1] >= qv[2] ? 1 : 2);
                nl[0] = nl[1] = nl[2] = 0.0;
                nl[ax] = ql[ax] < 0 ? -1.0 : 1.0;
            } else {
                double d[3];
                for (int k = 0; k < 3; ++k) d[k] = ql[k] - fmin(fmax(ql[k], -he[k]), he[k]);
                const double dl = sqrt(dot3(d, d));
                if (dl > 1e-10)
                    for (int k = 0; k < 3; ++k) nl[k] = d[k] / dl;
            }
        } else if (type == 1) { /* sphere */
            const double l = sqrt(dot3(ql, ql));
            un = l - g[4];
            if (l > 1e-10)
                for (int k = 0; k < 3; ++k) nl[k] = ql[k] / l;
            else
                nl[0] = 1.0, nl[1] = nl[2] = 0.0;
        } else if (type == 2) { /* plane: local z */
            un = ql[2];
        } else { /* capsule along local z */
            const double tz = fmin(fmax(ql[2], -(double)g[5]), (double)g[5]);
            const double d[3] = {ql[0], ql[1], ql[2] - tz};
            const double l = sqrt(dot3(d, d));
            un = l - g[4];
            if (l > 1e-10)
                for (int k = 0; k < 3; ++k) nl[k] = d[k] / l;
            else
                nl[0] = 1.0, nl[1] = nl[2] = 0.0;
        }
        const double dist = un * s;
        if (dist < best) {
            best = dist;
            qrot(P.q, nl, n_out);
        }
    }
    return best;
}

/* penalty and its derivative, terms/sphere_collision_kernels.py:17-41 */
static void scene_penalty(double sd, double margin, int mode, double* pen, double* dpen) {
    *pen = *dpen = 0.0;
    if (mode == 2) {
        *pen = fabs(sd);
        *dpen = sd > 0 ? 1.0 : (sd < 0 ? -1.0 : 0.0);
    } else if (mode == 1) {
        if (sd < margin) *pen = margin - sd, *dpen = -1.0;
    } else if (sd < 0) {
        *pen = 0.5 * margin - sd, *dpen = -1.0;
    } else if (sd <= margin) {
        const double inv = 1.0 / (margin + 1e-6);
        *pen = 0.5 * inv * (sd - margin) * (sd - margin);
        *dpen = inv * (sd - margin);
    }
}

int or_residual_dim(const OrRobot* r, const OrTerm* terms, int32_t nterms) {
    int R = 0;
    for (int i = 0; i < nterms; ++i) {
        const OrTerm* t = terms + i;
        if (t->kind == 1 || t->kind == 2)
            R += 3 * t->num_frames;
        else if (t->kind == 5)
            R += 6 * t->num_frames;
        else if (t->kind == 3 || t->kind == 6 || t->kind == 7)
            R += r->na;
        else if (t->kind == 8)
            R += t->num_query_spheres;
        else if (t->kind == 9)
            R += 6;
        else if (t->kind == 4)
            R += t->pair_mode == 0 ? t->max_active_pairs : t->num_sphere_pairs;
    }
    return R;
}

static const float* term_target(const OrTerm* t, int b, int B, int f) {
    const int rows = t->target_rows > 0 ? t->target_rows : B;
    int rep = B / rows;
    if (rep < 1) rep = 1;
    int row = b / rep;
    if (row > rows - 1) row = rows - 1;
    return t->targets + ((size_t)row * t->num_frames + f) * 7;
}

/* Residuals and Jacobian of every term in the reference row layout
 * (LMOptimizer._default_offsets, lm_optimizer.py:594-602).  J may be NULL.
 * Also reports the pose errors of the current point. */
static void eval_terms(const OrRobot* r, const OrTerm* terms, int nterms, int floating, const Kin* K, const double* q,
                       int b, int B, double* res, double* J, double* max_pos, double* max_rot) {
    const int D = (floating ? 6 : 0) + r->na;
    const int boff = floating ? 6 : 0;
    double C[3 * 1024];
    int have_C = 0;
    int row = 0;
    double mp = 0.0, mr = 0.0;
    for (int ti = 0; ti < nterms; ++ti) {
        const OrTerm* t = terms + ti;
        if (t->kind == 1 || t->kind == 2) {
            for (int f = 0; f < t->num_frames; ++f) {
                const P7 P = link_pose(r, K, t->frame_links[f]);
                const float* tg = term_target(t, b, B, f);
                const float* w = t->weights + 3 * f;
                double rr[3];
                if (t->kind == 1) {
                    /* position_task.py:189-212 */
                    const double e[3] = {tg[0] - P.t[0], tg[1] - P.t[1], tg[2] - P.t[2]};
                    const double pe = sqrt(dot3(e, e));
                    if (pe > mp) mp = pe;
                    for (int k = 0; k < 3; ++k) rr[k] = w[k] * e[k];
                } else {
                    /* rotation_task.py:324-349 */
                    const double qt[4] = {tg[3], -tg[4], -tg[5], -tg[6]};
                    double qe[4], aa[3];
                    qmul(P.q, qt, qe);
                    quat_axis_angle(qe, aa);
                    double sn = sqrt(qe[1] * qe[1] + qe[2] * qe[2] + qe[3] * qe[3]);
                    if (sn > 1.0) sn = 1.0;
                    const double ang = 2.0 * asin(sn);
                    if (ang > mr) mr = ang;
                    for (int k = 0; k < 3; ++k) rr[k] = w[k] * aa[k];
                }
                for (int k = 0; k < 3; ++k) res[row + 3 * f + k] = rr[k];
                if (J) {
                    for (int c = 0; c < D; ++c) {
                        double v[3], om[3];
                        column_twist(r, K, floating, c, t->frame_links[f], v, om);
                        if (t->kind == 1) {
                            /* position_task.py:251-272 */
                            double wp[3];
                            cross3(om, P.t, wp);
                            for (int k = 0; k < 3; ++k) J[(size_t)(row + 3 * f + k) * D + c] = -w[k] * (v[k] + wp[k]);
                        } else {
                            /* rotation_task.py:386-401 */
                            for (int k = 0; k < 3; ++k) J[(size_t)(row + 3 * f + k) * D + c] = w[k] * om[k];
                        }
                    }
                }
            }
            row += 3 * t->num_frames;
        } else if (t->kind == 5) {
            /* frame_task.py:391-527 ("log"): r = w (.) log(T_frame^-1 T_target);
             * J column = -w (.) jlog(T_target^-1 T_frame) Ad(T_frame^-1) [v; om] */
            for (int f = 0; f < t->num_frames; ++f) {
                const P7 P = link_pose(r, K, t->frame_links[f]);
                const P7 T = p7_from_f(term_target(t, b, B, f));
                const double wp = t->weights[2 * f], wr = t->weights[2 * f + 1];
                const P7 Pi = inverse(&P);
                const P7 E = compose(&Pi, &T);
                double lg[6];
                se3_log6(&E, lg);
                const double pe = sqrt(dot3(E.t, E.t));
                if (pe > mp) mp = pe;
                double sn = sqrt(E.q[1] * E.q[1] + E.q[2] * E.q[2] + E.q[3] * E.q[3]);
                if (sn > 1.0) sn = 1.0;
                const double ang = 2.0 * asin(sn);
                if (ang > mr) mr = ang;
                for (int k = 0; k < 6; ++k) res[row + 6 * f + k] = (k < 3 ? wp : wr) * lg[k];
                if (J) {
                    const P7 Ti = inverse(&T);
                    const P7 F = compose(&Ti, &P);
                    double M1[36], M2[36], M[36];
                    se3_jlog6(&F, M1);
                    se3_adjoint6(&Pi, M2);
                    for (int i = 0; i < 6; ++i)
                        for (int j = 0; j < 6; ++j) {
                            double v = 0.0;
                            for (int k = 0; k < 6; ++k) v += M1[6 * i + k] * M2[6 * k + j];
                            M[6 * i + j] = v;
                        }
                    for (int c = 0; c < D; ++c) {
                        double v[3], om[3], s6[6];
                        column_twist(r, K, floating, c, t->frame_links[f], v, om);
                        for (int k = 0; k < 3; ++k) {
                            s6[k] = v[k];
                            s6[3 + k] = om[k];
                        }
                        for (int i = 0; i < 6; ++i) {
                            double col = 0.0;
                            for (int k = 0; k < 6; ++k) col += M[6 * i + k] * s6[k];
                            J[(size_t)(row + 6 * f + i) * D + c] = -(i < 3 ? wp : wr) * col;
                        }
                    }
                }
            }
            row += 6 * t->num_frames;
        } else if (t->kind == 3) {
            /* position_limit.py:509-573 ("abs") */
            for (int a = 0; a < r->na; ++a) {
                const double lo = r->actuated_limits[2 * a], hi = r->actuated_limits[2 * a + 1];
                const double v = q[a];
                const double e = (v - hi > 0 ? v - hi : 0) + (lo - v > 0 ? lo - v : 0);
                res[row + a] = t->weights[a] * e;
                if (J) {
                    for (int c = 0; c < D; ++c) J[(size_t)(row + a) * D + c] = 0.0;
                    const double sg = v > hi ? 1.0 : (v < lo ? -1.0 : 0.0);
                    J[(size_t)(row + a) * D + boff + a] = t->weights[a] * sg;
                }
            }
            row += r->na;
        } else if (t->kind == 6 || t->kind == 7) {
            /* kind 6 — smoothness_task.py:350-366, configuration_task.py:322-334:
             *   r_a = w_a (q_a - ref_a);
             * kind 7 — velocity_limit_task.py:188-232: qd = (q_a - prev_a) / dt,
             *   r_a = w_a max(0, |qd| - vmax_a), J = w_a sign(qd) / dt where |qd| > vmax_a;
             * the reference row repeated over batch / rows problems */
            const int rows = t->target_rows > 0 ? t->target_rows : B;
            int rep = B / rows;
            if (rep < 1) rep = 1;
            int rr = b / rep;
            if (rr > rows - 1) rr = rows - 1;
            const float* ref = t->targets + (size_t)rr * r->na;
            for (int a = 0; a < r->na; ++a) {
                const double d = q[a] - (double)ref[a];
                double rv = t->weights[a] * d, jv = t->weights[a];
                if (t->kind == 7) {
                    const double qd = d / (double)t->dt, vmax = t->velocity_limits[a];
                    const int act = fabs(qd) > vmax;
                    rv = act ? t->weights[a] * (fabs(qd) - vmax) : 0.0;
                    jv = act ? t->weights[a] * (qd > 0 ? 1.0 : -1.0) / (double)t->dt : 0.0;
                }
                res[row + a] = rv;
                if (J) {
                    for (int c = 0; c < D; ++c) J[(size_t)(row + a) * D + c] = 0.0;
                    J[(size_t)(row + a) * D + boff + a] = jv;
                }
            }
            row += r->na;
        } else if (t->kind == 9) {
            /* smoothness_task.py:369-460, configuration_task.py:337-384: r = w (.) log(T_base T_ref^-1),
             * base columns w (.) jlog(E) Ad(T_ref), joint columns 0 */
            const int rows = t->target_rows > 0 ? t->target_rows : B;
            int rep = B / rows;
            if (rep < 1) rep = 1;
            int rr = b / rep;
            if (rr > rows - 1) rr = rows - 1;
            const P7 Tr = p7_from_f(t->targets + (size_t)rr * 7);
            const P7 Tri = inverse(&Tr);
            const P7 E = compose(&K->base, &Tri);
            double lg[6];
            se3_log6(&E, lg);
            for (int k = 0; k < 6; ++k) res[row + k] = t->weights[k] * lg[k];
            if (J) {
                double M1[36], M2[36];
                se3_jlog6(&E, M1);
                se3_adjoint6(&Tr, M2);
                for (int i = 0; i < 6; ++i)
                    for (int c = 0; c < D; ++c) {
                        double v = 0.0;
                        if (c < 6 && floating)
                            for (int k = 0; k < 6; ++k) v += M1[6 * i + k] * M2[6 * k + c];
                        J[(size_t)(row + i) * D + c] = t->weights[i] * v;
                    }
            }
            row += 6;
        } else if (t->kind == 8) {
            /* scene_collision_task.py:34-82, 550-647 with primitive geometry */
            if (!have_C) {
                world_spheres(r, K, C);
                have_C = 1;
            }
            int sid = 0;
            if (t->scene_rows > 0 && t->scene_indices) {
                int rep = B / t->scene_rows;
                if (rep < 1) rep = 1;
                int rr = b / rep;
                if (rr > t->scene_rows - 1) rr = t->scene_rows - 1;
                sid = t->scene_indices[rr];
            }
            if (sid < 0) sid = 0;
            if (sid > t->num_scenes - 1) sid = t->num_scenes - 1;
            for (int k = 0; k < t->num_query_spheres; ++k) {
                const int s = t->query_spheres[k];
                const double* c = C + 3 * s;
                double n[3];
                const double sd = scene_sdf(t, sid, c, n) - r->sphere_radii[s];
                double pen, dpen;
                scene_penalty(sd, t->margin, t->penalty, &pen, &dpen);
                double rv = pen, sc = dpen;
                if (t->residual_sqrt) {
                    if (pen > 0) sc *= 0.5 / sqrt(pen + t->residual_eps);
                    rv = sqrt(pen + t->residual_eps);
                }
                res[row + k] = t->weights[k] * rv;
                if (J) {
                    double* jr = J + (size_t)(row + k) * D;
                    const int act = t->penalty == 2 || sd <= t->margin;
                    for (int col = 0; col < D; ++col) {
                        jr[col] = 0.0;
                        if (!act) continue;
                        double v[3], w[3], x[3];
                        column_twist(r, K, floating, col, r->sphere_links[s], v, w);
                        cross3(w, c, x);
                        const double pc[3] = {v[0] + x[0], v[1] + x[1], v[2] + x[2]};
                        jr[col] = t->weights[k] * sc * dot3(n, pc);
                    }
                }
            }
            row += t->num_query_spheres;
        } else if (t->kind == 4) {
            if (!have_C) {
                world_spheres(r, K, C);
                have_C = 1;
            }
            const double wgt = t->weights[0];
            const int* sp = t->sphere_pairs;
            if (t->pair_mode == 1) {
                for (int p = 0; p < t->num_sphere_pairs; ++p) {
                    const int si = sp[2 * p], sj = sp[2 * p + 1];
                    const double surf = sph_dist(C, si, sj) - r->sphere_radii[si] - r->sphere_radii[sj];
                    const double pen = t->margin - surf;
                    res[row + p] = wgt * (pen > 0 ? pen : 0.0);
                    if (J) {
                        double* jr = J + (size_t)(row + p) * D;
                        if (pen > 0) {
                            collision_row(r, K, floating, C, si, sj, jr, D);
                            for (int c = 0; c < D; ++c) jr[c] *= -wgt;
                        } else
                            for (int c = 0; c < D; ++c) jr[c] = 0.0;
                    }
                }
                row += t->num_sphere_pairs;
            } else {
                /* broad phase over link bounding spheres (self_collision_task.py:73-87), first K
                 * penetrating link pairs in order, most penetrating sphere pair each (:166-217) */
                double L[3 * MAXL];
                for (int l = 0; l < r->nl; ++l) {
                    const P7 P = link_pose(r, K, l);
                    const double lc[3] = {r->link_bound_centers[3 * l], r->link_bound_centers[3 * l + 1],
                                          r->link_bound_centers[3 * l + 2]};
                    double wc[3];
                    qrot(P.q, lc, wc);
                    for (int k = 0; k < 3; ++k) L[3 * l + k] = wc[k] + P.t[k];
                }
                int nsl = 0;
                for (int lp = 0; lp < t->num_link_pairs && nsl < t->max_active_pairs; ++lp) {
                    const int la = t->link_pairs[2 * lp], lb = t->link_pairs[2 * lp + 1];
                    const double pen = r->link_bound_radii[la] + r->link_bound_radii[lb] + t->margin -
                                       sph_dist(L, la, lb);
                    if (!(pen > 0)) continue;
                    double best = 1.0e10;
                    int bp = t->link_pair_offsets[lp];
                    for (int p = t->link_pair_offsets[lp]; p < t->link_pair_offsets[lp + 1]; ++p) {
                        const int si = sp[2 * p], sj = sp[2 * p + 1];
                        const double s = sph_dist(C, si, sj) - r->sphere_radii[si] - r->sphere_radii[sj];
                        if (s < best) {
                            best = s;
                            bp = p;
                        }
                    }
                    const int si = sp[2 * bp], sj = sp[2 * bp + 1];
                    const double surf = sph_dist(C, si, sj) - r->sphere_radii[si] - r->sphere_radii[sj];
                    const double pn = t->margin - surf;
                    res[row + nsl] = wgt * (pn > 0 ? pn : 0.0);
                    if (J) {
                        double* jr = J + (size_t)(row + nsl) * D;
                        if (pn > 0) {
                            collision_row(r, K, floating, C, si, sj, jr, D);
                            for (int c = 0; c < D; ++c) jr[c] *= -wgt;
                        } else
                            for (int c = 0; c < D; ++c) jr[c] = 0.0;
                    }
                    ++nsl;
                }
                for (int k = nsl; k < t->max_active_pairs; ++k) {
                    res[row + k] = 0.0;
                    if (J)
                        for (int c = 0; c < D; ++c) J[(size_t)(row + k) * D + c] = 0.0;
                }
                row += t->max_active_pairs;
            }
        }
    }
    if (max_pos) *max_pos = mp;
    if (max_rot) *max_rot = mr;
}

static P7 base_of(const float* base, int b) {
    if (!base) return p7_identity();
    return p7_from_f(base + (size_t)7 * b);
}

int or_fk(const OrRobot* r, int32_t B, const float* q, const float* base, double* T_joint, double* T_link,
          double* S_world, double* spheres, double* bounds) {
    Kin K;
    double qq[MAXD];
    for (int b = 0; b < B; ++b) {
        for (int a = 0; a < r->na; ++a) qq[a] = q[(size_t)b * r->na + a];
        const P7 bp = base_of(base, b);
        fk_one(r, qq, &bp, &K);
        if (T_joint)
            for (int j = 0; j < r->nj; ++j) p7_to_d(&K.Tj[j], T_joint + ((size_t)b * r->nj + j) * 7);
        if (T_link)
            for (int l = 0; l < r->nl; ++l) {
                const P7 P = link_pose(r, &K, l);
                p7_to_d(&P, T_link + ((size_t)b * r->nl + l) * 7);
            }
        if (S_world)
            for (int j = 0; j < r->nj; ++j)
                for (int k = 0; k < 6; ++k) S_world[(size_t)b * 6 * r->nj + k * r->nj + j] = K.S[j][k];
        if (spheres) world_spheres(r, &K, spheres + (size_t)b * 3 * r->ns);
        if (bounds)
            for (int l = 0; l < r->nl; ++l) {
                const P7 P = link_pose(r, &K, l);
                const double lc[3] = {r->link_bound_centers[3 * l], r->link_bound_centers[3 * l + 1],
                                      r->link_bound_centers[3 * l + 2]};
                double wc[3];
                qrot(P.q, lc, wc);
                for (int k = 0; k < 3; ++k) bounds[((size_t)b * r->nl + l) * 3 + k] = wc[k] + P.t[k];
            }
    }
    return 0;
}

/* robo/robot_kernels.py:668-737 */
int or_link_jacobian(const OrRobot* r, int32_t B, const float* q, const float* base, int32_t link, int32_t body,
                     double* J) {
    Kin K;
    double qq[MAXD];
    const int floating = base != NULL;
    const int D = (floating ? 6 : 0) + r->na;
    for (int b = 0; b < B; ++b) {
        for (int a = 0; a < r->na; ++a) qq[a] = q[(size_t)b * r->na + a];
        const P7 bp = base_of(base, b);
        fk_one(r, qq, &bp, &K);
        const P7 F = link_pose(r, &K, link);
        const P7 Fi = inverse(&F);
        double* o = J + (size_t)b * 6 * D;
        for (int c = 0; c < D; ++c) {
            double v[3], w[3];
            if (c < (floating ? 6 : 0) && body) {
                const P7 FB = compose(&Fi, &bp);
                double e[3] = {0, 0, 0}, Re[3];
                e[c % 3] = 1.0;
                qrot(FB.q, e, Re);
                if (c < 3) {
                    for (int k = 0; k < 3; ++k) {
                        v[k] = Re[k];
                        w[k] = 0.0;
                    }
                } else {
                    for (int k = 0; k < 3; ++k) w[k] = Re[k];
                    cross3(FB.t, Re, v);
                }
            } else {
                column_twist(r, &K, floating, c, link, v, w);
                if (body && c >= (floating ? 6 : 0)) {
                    double tw[3], vv[3];
                    cross3(F.t, w, tw);
                    for (int k = 0; k < 3; ++k) vv[k] = v[k] - tw[k];
                    qrot(Fi.q, vv, v);
                    double ww[3];
                    qrot(Fi.q, w, ww);
                    for (int k = 0; k < 3; ++k) w[k] = ww[k];
                }
            }
            for (int k = 0; k < 3; ++k) {
                o[k * D + c] = v[k];
                o[(3 + k) * D + c] = w[k];
            }
        }
    }
    return 0;
}

int or_residual_jacobian(const OrRobot* r, const OrTerm* terms, int32_t nterms, int32_t floating, int32_t B,
                         const float* q, const float* base, double* res, double* J) {
    const int R = or_residual_dim(r, terms, nterms);
    const int D = (floating ? 6 : 0) + r->na;
    Kin K;
    double qq[MAXD];
    double* rtmp = (double*)malloc(sizeof(double) * (R > 0 ? R : 1));
    for (int b = 0; b < B; ++b) {
        for (int a = 0; a < r->na; ++a) qq[a] = q[(size_t)b * r->na + a];
        const P7 bp = base_of(floating ? base : NULL, b);
        fk_one(r, qq, &bp, &K);
        eval_terms(r, terms, nterms, floating, &K, qq, b, B, res ? res + (size_t)b * R : rtmp,
                   J ? J + (size_t)b * R * D : NULL, NULL, NULL);
    }
    free(rtmp);
    return 0;
}

/* H = J^T J, g = J^T r, cost = 0.5 r^T r with J columns scaled by the mask
 * (lm_optimizer.py:145-189, 872-880) */
static void normal_one(const double* res, const double* J, int R, int D, const float* mask, double* H, double* g,
                       double* cost) {
    double c = 0.0;
    for (int i = 0; i < R; ++i) c += res[i] * res[i];
    *cost = 0.5 * c;
    for (int a = 0; a < D; ++a) {
        const double ma = mask ? mask[a] : 1.0;
        double ga = 0.0;
        for (int i = 0; i < R; ++i) ga += J[(size_t)i * D + a] * res[i];
        g[a] = ma * ga;
        for (int bcol = 0; bcol <= a; ++bcol) {
            const double mb = mask ? mask[bcol] : 1.0;
            double s = 0.0;
            for (int i = 0; i < R; ++i) s += J[(size_t)i * D + a] * J[(size_t)i * D + bcol];
            H[a * D + bcol] = H[bcol * D + a] = ma * mb * s;
        }
    }
}

int or_normal_equations(const OrRobot* r, const OrTerm* terms, int32_t nterms, int32_t floating, const float* mask,
                        int32_t B, const float* q, const float* base, double* H, double* g, double* cost) {
    const int R = or_residual_dim(r, terms, nterms);
    const int D = (floating ? 6 : 0) + r->na;
    double* res = (double*)malloc(sizeof(double) * (R > 0 ? R : 1));
    double* J = (double*)malloc(sizeof(double) * (size_t)(R > 0 ? R : 1) * D);
    Kin K;
    double qq[MAXD];
    for (int b = 0; b < B; ++b) {
        for (int a = 0; a < r->na; ++a) qq[a] = q[(size_t)b * r->na + a];
        const P7 bp = base_of(floating ? base : NULL, b);
        fk_one(r, qq, &bp, &K);
        eval_terms(r, terms, nterms, floating, &K, qq, b, B, res, J, NULL, NULL);
        normal_one(res, J, R, D, mask, H + (size_t)b * D * D, g + (size_t)b * D, cost + b);
    }
    free(res);
    free(J);
    return 0;
}

/* (H + lambda I) delta = -g by Cholesky; pred = 0.5 delta.(lambda delta - g)
 * (lm_optimizer.py:56-79).  Returns 0 when a pivot is not positive. */
static int chol_step(int D, const double* H, const double* g, double lam, double* delta, double* pred) {
    double L[MAXD * MAXD];
    for (int i = 0; i < D; ++i)
        for (int j = 0; j <= i; ++j) L[i * D + j] = H[i * D + j] + (i == j ? lam : 0.0);
    for (int k = 0; k < D; ++k) {
        double s = L[k * D + k];
        for (int m = 0; m < k; ++m) s -= L[k * D + m] * L[k * D + m];
        if (!(s > 0.0)) {
            for (int i = 0; i < D; ++i) delta[i] = 0.0;
            *pred = 0.0;
            return 0;
        }
        const double d = sqrt(s);
        L[k * D + k] = d;
        for (int i = k + 1; i < D; ++i) {
            double t = L[i * D + k];
            for (int m = 0; m < k; ++m) t -= L[i * D + m] * L[k * D + m];
            L[i * D + k] = t / d;
        }
    }
    double y[MAXD];
    for (int i = 0; i < D; ++i) {
        double s = -g[i];
        for (int m = 0; m < i; ++m) s -= L[i * D + m] * y[m];
        y[i] = s / L[i * D + i];
    }
    for (int i = D - 1; i >= 0; --i) {
        double s = y[i];
        for (int m = i + 1; m < D; ++m) s -= L[m * D + i] * delta[m];
        delta[i] = s / L[i * D + i];
    }
    double p = 0.0;
    for (int i = 0; i < D; ++i) p += delta[i] * (lam * delta[i] - g[i]);
    *pred = 0.5 * p;
    return 1;
}

int or_damped_solve(int32_t B, int32_t D, const double* H, const double* g, const double* lambda, double* delta,
                    double* pred, int32_t* spd) {
    if (D < 1 || D > MAXD) return -1;
    for (int b = 0; b < B; ++b) {
        const int ok = chol_step(D, H + (size_t)b * D * D, g + (size_t)b * D, lambda[b], delta + (size_t)b * D,
                                 pred + b);
        if (spd) spd[b] = ok;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* the LM loop (Optimizer.solve opt/optimizer.py:216-240, LMOptimizer._step_body
 * lm_optimizer.py:834-1005, accept lm_optimizer.py:294-334, integrate
 * robo/robot_kernels.py:563-644)                                             */
/* ------------------------------------------------------------------------ */
typedef struct {
    const OrRobot* r;
    const OrTerm* terms;
    int nterms, floating;
    const float* mask;
    const OrParams* p;
    int B;
    const float* q0;
    const float* base0;
    double *q, *base, *cost, *lambda;
    int *iters, *status;
    int b0, b1;
    /* all-problems cost rule: processed iteration by iteration across the range */
} Job;

typedef struct {
    double q[MAXD];
    P7 base;
    double H[MAXD * MAXD], g[MAXD], cost, lam, max_pos, max_rot;
    int iters, status, done;
} PState;

static void linearize(const Job* jb, PState* s, int b, double* res, double* J) {
    const OrRobot* r = jb->r;
    const int R = or_residual_dim(r, jb->terms, jb->nterms);
    const int D = (jb->floating ? 6 : 0) + r->na;
    Kin K;
    fk_one(r, s->q, &s->base, &K);
    eval_terms(r, jb->terms, jb->nterms, jb->floating, &K, s->q, b, jb->B, res, J, &s->max_pos, &s->max_rot);
    normal_one(res, J, R, D, jb->mask, s->H, s->g, &s->cost);
}

static double eval_cost(const Job* jb, const double* q, const P7* base, int b, double* res, double* mp, double* mr) {
    const OrRobot* r = jb->r;
    const int R = or_residual_dim(r, jb->terms, jb->nterms);
    Kin K;
    fk_one(r, q, base, &K);
    eval_terms(r, jb->terms, jb->nterms, jb->floating, &K, q, b, jb->B, res, NULL, mp, mr);
    double c = 0.0;
    for (int i = 0; i < R; ++i) c += res[i] * res[i];
    return 0.5 * c;
}

static int check_stop(const OrParams* p, PState* s) {
    int stop = 0;
    if ((p->stop_rules & 4) && s->max_pos <= p->pose_pos_tol && s->max_rot <= p->pose_rot_tol) stop = 1;
    if ((p->stop_rules & 8) && s->cost <= p->cost_tol) stop = 1;
    if (stop) s->status |= 1;
    return stop;
}

/* one iteration; returns 1 when the problem stops */
static int iterate(const Job* jb, PState* s, int b, double* res, double* J) {
    const OrRobot* r = jb->r;
    const OrParams* p = jb->p;
    const int D = (jb->floating ? 6 : 0) + r->na;
    const int boff = jb->floating ? 6 : 0;
    double delta[MAXD], pred;
    const int ok = chol_step(D, s->H, s->g, s->lam, delta, &pred);
    if (!ok) s->status |= 4;
    double dn = 0.0;
    for (int i = 0; i < D; ++i) dn += delta[i] * delta[i];
    dn = sqrt(dn);
    if ((p->stop_rules & 2) && ok && dn < p->step_tol) {
        s->status |= 1;
        return 1;
    }
    double qp[MAXD];
    for (int a = 0; a < r->na; ++a) qp[a] = s->q[a] + (jb->mask ? jb->mask[boff + a] : 1.0) * delta[boff + a];
    P7 bp = s->base;
    if (jb->floating) {
        double xi[6];
        for (int k = 0; k < 6; ++k) xi[k] = delta[k];
        if (jb->mask)
            for (int k = 3; k < 6; ++k) xi[k] *= jb->mask[k];
        const P7 E = se3_exp(xi, 1e-4);
        bp = compose(&s->base, &E);
        if (jb->mask)
            for (int k = 0; k < 3; ++k)
                if (jb->mask[k] == 0.0f) bp.t[k] = s->base.t[k];
    }
    double mp, mr;
    const double cnew = eval_cost(jb, qp, &bp, b, res, &mp, &mr);
    int acc = pred > 0.0;
    if (acc) {
        const double rho = (s->cost - cnew) / (pred + p->gain_ratio_epsilon);
        acc = rho >= p->rho_min;
    }
    if (acc) {
        for (int a = 0; a < r->na; ++a) s->q[a] = qp[a];
        s->base = bp;
        s->lam = fmax(s->lam / p->lambda_factor, p->lambda_min);
        linearize(jb, s, b, res, J);
    } else {
        s->lam = fmin(fmax(s->lam * p->lambda_factor, p->lambda_min), p->lambda_max);
    }
    s->iters += 1;
    int stop = check_stop(p, s);
    if (!stop && s->iters >= p->max_iter) {
        s->status |= 2;
        stop = 1;
    }
    return stop;
}

static void load_state(const Job* jb, PState* s, int b) {
    const OrRobot* r = jb->r;
    for (int a = 0; a < r->na; ++a) s->q[a] = jb->q0[(size_t)b * r->na + a];
    s->base = base_of(jb->floating ? jb->base0 : NULL, b);
    s->lam = jb->p->lambda_init;
    s->iters = 0;
    s->status = 0;
    s->done = 0;
}

static void store_state(const Job* jb, const PState* s, int b) {
    const OrRobot* r = jb->r;
    for (int a = 0; a < r->na; ++a) jb->q[(size_t)b * r->na + a] = s->q[a];
    if (jb->floating && jb->base) p7_to_d(&s->base, jb->base + (size_t)b * 7);
    if (jb->cost) jb->cost[b] = s->cost;
    if (jb->lambda) jb->lambda[b] = s->lam;
    if (jb->iters) jb->iters[b] = s->iters;
    if (jb->status) jb->status[b] = s->status;
}

static void* run_job(void* arg) {
    const Job* jb = (const Job*)arg;
    const OrRobot* r = jb->r;
    const int R = or_residual_dim(r, jb->terms, jb->nterms);
    const int D = (jb->floating ? 6 : 0) + r->na;
    double* res = (double*)malloc(sizeof(double) * (R > 0 ? R : 1));
    double* J = (double*)malloc(sizeof(double) * (size_t)(R > 0 ? R : 1) * D);
    PState* s = (PState*)malloc(sizeof(PState));
    for (int b = jb->b0; b < jb->b1; ++b) {
        load_state(jb, s, b);
        linearize(jb, s, b, res, J);
        if (!isfinite(s->cost)) s->status |= 8;
        int stop = (s->status & 8) || check_stop(jb->p, s) || jb->p->max_iter <= 0;
        if (jb->p->max_iter <= 0) s->status |= 2;
        while (!stop) stop = iterate(jb, s, b, res, J);
        store_state(jb, s, b);
    }
    free(s);
    free(res);
    free(J);
    return NULL;
}

/* the reference's all-problems rule (opt/optimizer.py:237-239) couples the
 * problems, so it runs iteration-synchronously on one thread */
static int solve_all_cost(const Job* jb) {
    const OrRobot* r = jb->r;
    const int R = or_residual_dim(r, jb->terms, jb->nterms);
    const int D = (jb->floating ? 6 : 0) + r->na;
    const int B = jb->B;
    double* res = (double*)malloc(sizeof(double) * (R > 0 ? R : 1));
    double* J = (double*)malloc(sizeof(double) * (size_t)(R > 0 ? R : 1) * D);
    PState* S = (PState*)malloc(sizeof(PState) * (size_t)(B > 0 ? B : 1));
    OrParams p1 = *jb->p;
    p1.stop_rules &= ~1;
    p1.max_iter = 1 << 30;
    Job j1 = *jb;
    j1.p = &p1;
    for (int b = 0; b < B; ++b) {
        load_state(&j1, S + b, b);
        linearize(&j1, S + b, b, res, J);
    }
    const int interval = jb->p->check_interval > 0 ? jb->p->check_interval : 1;
    for (int it = 0; it < jb->p->max_iter; ++it) {
        for (int b = 0; b < B; ++b) iterate(&j1, S + b, b, res, J);
        if ((it + 1) % interval == 0) {
            int all = 1;
            for (int b = 0; b < B; ++b)
                if (!(S[b].cost <= jb->p->cost_tol)) all = 0;
            if (all) break;
        }
    }
    for (int b = 0; b < B; ++b) store_state(jb, S + b, b);
    free(S);
    free(res);
    free(J);
    return 0;
}

int or_solve(const OrRobot* r, const OrTerm* terms, int32_t nterms, int32_t floating, const float* mask,
             const OrParams* p, int32_t B, const float* q0, const float* base0, double* q, double* base,
             double* cost, double* lambda, int32_t* iters, int32_t* status, int32_t nthreads) {
    Job base_job;
    memset(&base_job, 0, sizeof(base_job));
    base_job.r = r;
    base_job.terms = terms;
    base_job.nterms = nterms;
    base_job.floating = floating;
    base_job.mask = mask;
    base_job.p = p;
    base_job.B = B;
    base_job.q0 = q0;
    base_job.base0 = base0;
    base_job.q = q;
    base_job.base = base;
    base_job.cost = cost;
    base_job.lambda = lambda;
    base_job.iters = iters;
    base_job.status = status;
    if ((floating ? 6 : 0) + r->na > MAXD || r->nj > MAXJ || r->nl > MAXL || r->ns > 1024) return -1;
    if (p->stop_rules & 1) return solve_all_cost(&base_job);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > B) nthreads = B > 0 ? B : 1;
    pthread_t th[256];
    Job jobs[256];
    if (nthreads > 256) nthreads = 256;
    const int per = (B + nthreads - 1) / nthreads;
    int started = 0;
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = base_job;
        jobs[t].b0 = t * per;
        jobs[t].b1 = (t + 1) * per < B ? (t + 1) * per : B;
        if (jobs[t].b0 >= jobs[t].b1) break;
        if (nthreads == 1) {
            run_job(&jobs[t]);
        } else {
            pthread_create(&th[t], NULL, run_job, &jobs[t]);
            ++started;
        }
    }
    for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
    return 0;
}

/* accept/reject on scalars, lm_accept_reject_cost_kernel (lm_optimizer.py:338-362) */
int or_accept_reject(int32_t B, double* cost, const double* cost_new, const double* pred, double* lambda,
                     int32_t* accept, const OrParams* p) {
    for (int b = 0; b < B; ++b) {
        int acc = pred[b] > 0.0;
        if (acc) acc = (cost[b] - cost_new[b]) / (pred[b] + p->gain_ratio_epsilon) >= p->rho_min;
        accept[b] = acc;
        if (acc) {
            lambda[b] = fmax(lambda[b] / p->lambda_factor, p->lambda_min);
            cost[b] = cost_new[b];
        } else {
            lambda[b] = fmin(fmax(lambda[b] * p->lambda_factor, p->lambda_min), p->lambda_max);
        }
    }
    return 0;
}

/* helpers/ik/ik.py:60-82 */
int or_metrics(const OrRobot* r, int32_t B, const double* q, const double* base, int32_t nt, const int32_t* links,
               const float* targets, double pos_th, double rot_th, double* perr, double* rerr, int32_t* success) {
    Kin K;
    for (int b = 0; b < B; ++b) {
        P7 bp = p7_identity();
        if (base) {
            for (int k = 0; k < 3; ++k) bp.t[k] = base[(size_t)b * 7 + k];
            for (int k = 0; k < 4; ++k) bp.q[k] = base[(size_t)b * 7 + 3 + k];
        }
        fk_one(r, q + (size_t)b * r->na, &bp, &K);
        int ok = 1;
        for (int i = 0; i < nt; ++i) {
            const P7 L = link_pose(r, &K, links[i]);
            const P7 Li = inverse(&L);
            const P7 T = p7_from_f(targets + ((size_t)b * nt + i) * 7);
            const P7 E = compose(&Li, &T);
            const double pe = sqrt(dot3(E.t, E.t));
            double sn = sqrt(E.q[1] * E.q[1] + E.q[2] * E.q[2] + E.q[3] * E.q[3]);
            if (sn > 1.0) sn = 1.0;
            const double ae = 2.0 * asin(sn);
            perr[(size_t)b * nt + i] = pe;
            rerr[(size_t)b * nt + i] = ae;
            if (pe >= pos_th || ae >= rot_th) ok = 0;
        }
        success[b] = ok;
    }
    return 0;
}
