// ik_device.cuh — device routines of the fused LM-IK kernel.
//
// A *group* of G lanes (G = 8, 16 or 32, always inside one warp) owns one IK
// problem.  The routines below are written for the group: loops over joints,
// residual rows, normal-equation entries and Cholesky items are strided by the
// group lane, synchronisation is __syncwarp on the group's lane mask and
// reductions are width-G shuffles.  Tables come from the staged blob
// (ik_tables.h); the per-group workspace is a private slice of shared memory.
//
// Numerics: kinematics, residuals, the Jacobian and J^T J run in FP32; J^T J,
// J^T r and the cost use compensated (Neumaier/Kahan) accumulation across row
// chunks; the damped Cholesky factorisation, the solve, the predicted
// reduction and the gain ratio run in FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <utility>
#include <type_traits>
#include "ik_tables.h"

namespace b200ik {

// ---------------------------------------------------------------------------
// SE(3) on [x y z | qw qx qy qz] poses (lie/se3_kernels.py:70-167,324-346,
// xform/warp/rotation_conversions.py:169-279).  Quaternion products are
// standardised to w >= 0 like quaternion_multiply_func (:268-279).
// ---------------------------------------------------------------------------
struct Pose {
    float x, y, z, w, i, j, k;
};

__device__ __forceinline__ Pose pose_identity() { return Pose{0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f}; }

__device__ __forceinline__ Pose pose_load(const float* p) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    const float4 b = *reinterpret_cast<const float4*>(p + 4);
    return Pose{a.x, a.y, a.z, a.w, b.x, b.y, b.z};
}
__device__ __forceinline__ void pose_store(float* p, const Pose& P) {
    *reinterpret_cast<float4*>(p) = make_float4(P.x, P.y, P.z, P.w);
    *reinterpret_cast<float4*>(p + 4) = make_float4(P.i, P.j, P.k, 0.f);
}
__device__ __forceinline__ Pose pose_load7(const float* p) {  // unaligned 7-float pose
    return Pose{p[0], p[1], p[2], p[3], p[4], p[5], p[6]};
}

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float norm3(V3 a) { return sqrtf(dot(a, a)); }

// v' = v + 2 (w (u x v) + u x (u x v)), quaternion_apply_func :192-200
__device__ __forceinline__ V3 qrot(float w, float i, float j, float k, V3 v) {
    const V3 u{i, j, k};
    const V3 uv = cross(u, v);
    const V3 uuv = cross(u, uv);
    return v + 2.0f * (w * uv + uuv);
}
__device__ __forceinline__ V3 pose_apply(const Pose& P, V3 v) { return qrot(P.w, P.i, P.j, P.k, v) + V3{P.x, P.y, P.z}; }

__device__ __forceinline__ void qmul_std(float aw, float ai, float aj, float ak, float bw, float bi, float bj, float bk,
                                         float& w, float& i, float& j, float& k) {
    w = aw * bw - ai * bi - aj * bj - ak * bk;
    i = aw * bi + ai * bw + aj * bk - ak * bj;
    j = aw * bj - ai * bk + aj * bw + ak * bi;
    k = aw * bk + ai * bj - aj * bi + ak * bw;
    if (w < 0.f) {
        w = -w;
        i = -i;
        j = -j;
        k = -k;
    }
}

// A o B, se3_compose_func :88-109
__device__ __forceinline__ Pose compose(const Pose& A, const Pose& B) {
    Pose O;
    qmul_std(A.w, A.i, A.j, A.k, B.w, B.i, B.j, B.k, O.w, O.i, O.j, O.k);
    const V3 t = qrot(A.w, A.i, A.j, A.k, V3{B.x, B.y, B.z});
    O.x = A.x + t.x;
    O.y = A.y + t.y;
    O.z = A.z + t.z;
    return O;
}

// SE(3) exponential with regularised angle, se3_exp_map_func :126-167
__device__ __forceinline__ Pose se3_exp(const float xi[6], float eps) {
    const V3 tl{xi[0], xi[1], xi[2]};
    const V3 rl{xi[3], xi[4], xi[5]};
    const float angle_sq = dot(rl, rl);
    const float angle_sq_reg = angle_sq + eps * eps;
    const float angle_reg = sqrtf(angle_sq_reg);
    float sh, ch;
    sincosf(angle_reg * 0.5f, &sh, &ch);
    const float kk = sh / angle_reg;
    float qw = ch, qi = kk * rl.x, qj = kk * rl.y, qk = kk * rl.z;
    const float qn = sqrtf(qw * qw + qi * qi + qj * qj + qk * qk);
    qw /= qn;
    qi /= qn;
    qj /= qn;
    qk /= qn;
    float sa, ca;
    sincosf(angle_reg, &sa, &ca);
    const float A = sa / angle_reg;
    const float c1 = (1.0f - ca) / angle_sq_reg;
    const float c2 = (1.0f - A) / angle_sq_reg;
    // V = I + c1 K + c2 K^2 with K = hat(rl); V t = t + c1 (rl x t) + c2 (rl x (rl x t))
    const V3 kt = cross(rl, tl);
    const V3 kkt = cross(rl, kt);
    const V3 tr = tl + c1 * kt + c2 * kkt;
    return Pose{tr.x, tr.y, tr.z, qw, qi, qj, qk};
}

// axis-angle of a standardised quaternion, quaternion_to_axis_angle_func :228-247.
// With half = atan2(n, w), sin(half) = n / |q| exactly, which replaces the sine;
// `angle` (2 half) is the rotation angle.
__device__ __forceinline__ V3 quat_to_axis_angle(float w, float i, float j, float k, float& angle) {
    const float n2 = i * i + j * j + k * k;
    const float n = sqrtf(n2);
    const float half = atan2f(n, w);
    angle = 2.0f * half;
    float inv_s;  // 1 / (sin(half) / angle)
    if (fabsf(angle) < 1e-6f) {
        inv_s = 1.0f / (0.5f - angle * angle / 48.0f);
    } else {
        inv_s = angle * sqrtf(n2 + w * w) / n;
    }
    return V3{i * inv_s, j * inv_s, k * inv_s};
}

// T^-1 with the conjugate quaternion, se3_inverse_func (lie/se3_kernels.py:70-78)
__device__ __forceinline__ Pose pose_inverse(const Pose& T) {
    const V3 ti = qrot(T.w, -T.i, -T.j, -T.k, V3{T.x, T.y, T.z});
    return Pose{-ti.x, -ti.y, -ti.z, T.w, -T.i, -T.j, -T.k};
}

// SE(3) logarithm [V^-1(w) t; w] with V^-1 = I - W/2 + c2 W^2, W = hat(w)
// (se3_log_map_func, lie/se3_kernels.py:230-311; eps 1e-4 as frame_task.py:523)
__device__ __forceinline__ void se3_log(const Pose& E, float out[6], float& angle) {
    const V3 w = quat_to_axis_angle(E.w, E.i, E.j, E.k, angle);
    const float th = norm3(w);
    float c2 = 1.0f / 12.0f;
    if (!(th < 1e-4f)) {
        float sn, cs;
        sincosf(th, &sn, &cs);
        const float omc = 1.0f - cs;
        if (!(fabsf(omc) < 1e-4f)) c2 = (1.0f / (th * th)) * (1.0f - (th * sn) / (2.0f * omc));
    }
    const V3 t{E.x, E.y, E.z};
    const V3 wt = cross(w, t);
    const V3 wwt = cross(w, wt);
    out[0] = t.x - 0.5f * wt.x + c2 * wwt.x;
    out[1] = t.y - 0.5f * wt.y + c2 * wwt.y;
    out[2] = t.z - 0.5f * wt.z + c2 * wwt.z;
    out[3] = w.x;
    out[4] = w.y;
    out[5] = w.z;
}

// Six weighted rows w (.) log(T_frame^-1 T_target) of a frame entry into rp, folded into the
// compensated cost and the pose errors (frame_task.py:505-527).  Out of line: frame entries are
// rare, and the solve loops keep their instruction footprint without them.
__device__ __forceinline__ void frame_residual(const Pose& P, const float* tg, float wp, float wr, float* rp, float& ks,
                                            float& kc, float& max_pos, float& max_rot);

// 3x3 helpers, row-major
__device__ __forceinline__ void m3_hat(const V3& a, float H[9]) {
    H[0] = 0.f; H[1] = -a.z; H[2] = a.y;
    H[3] = a.z; H[4] = 0.f; H[5] = -a.x;
    H[6] = -a.y; H[7] = a.x; H[8] = 0.f;
}
__device__ __forceinline__ void m3_mul(const float A[9], const float B[9], float C[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
__device__ __forceinline__ V3 m3_vec(const float A[9], const V3& v) {
    return V3{A[0] * v.x + A[1] * v.y + A[2] * v.z, A[3] * v.x + A[4] * v.y + A[5] * v.z,
              A[6] * v.x + A[7] * v.y + A[8] * v.z};
}
// rotation matrix of a unit quaternion (quaternion_to_matrix_func, rotation_conversions.py:169-183)
__device__ __forceinline__ void m3_quat(float w, float x, float y, float z, float R[9]) {
    R[0] = 1.f - 2.f * (y * y + z * z); R[1] = 2.f * (x * y - w * z); R[2] = 2.f * (x * z + w * y);
    R[3] = 2.f * (x * y + w * z); R[4] = 1.f - 2.f * (x * x + z * z); R[5] = 2.f * (y * z - w * x);
    R[6] = 2.f * (x * z - w * y); R[7] = 2.f * (y * z + w * x); R[8] = 1.f - 2.f * (x * x + y * y);
}

// Jlog(F) Ad(T) = [[P, K], [0, P]] for twists [v; om]: with (w, p) the axis-angle and
// translation of F, A = Jl^-1(w)^T (so3_jac_left_inv_func, lie/so3_kernels.py:14-40) and B the
// upper-right block of the SE(3) jlog (se3_jlog_func, lie/se3_kernels.py:359-428), so that
// Jlog(F) = [[A, B], [0, A]], and T = (R, t) (se3_adjoint_func :314-346):
//   P = A R,   K = (A hat(t) + B) R.
__device__ __forceinline__ void se3_jlog_ad(const Pose& F, const Pose& Ti, float P[9], float K[9]) {
    float ang;
    const V3 w = quat_to_axis_angle(F.w, F.i, F.j, F.k, ang);
    const V3 p{F.x, F.y, F.z};
    const float th2 = dot(w, w);
    const bool taylor = th2 < 1e-4f;
    float W[9], W2[9], A[9], B[9];
    m3_hat(w, W);
    m3_mul(W, W, W2);
    float coeff = 1.0f / 12.0f;
    float th = 1.0f;
    if (!taylor) {
        th = sqrtf(th2);
        float sh, ch;
        sincosf(0.5f * th, &sh, &ch);
        coeff = (1.0f - th * ch / (2.0f * sh)) / th2;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) A[k] = ((k % 4) == 0 ? 1.f : 0.f) + 0.5f * W[k] + coeff * W2[k];
    float Hp[9];
    m3_hat(p, Hp);
    if (taylor) {
#pragma unroll
        for (int k = 0; k < 9; ++k) B[k] = 0.5f * Hp[k];
    } else {
        float st, ct;
        sincosf(th, &st, &ct);
        const float inv = 1.0f / th, inv2 = inv * inv;
        const float i22 = 1.0f / (2.0f * (1.0f - ct));
        const float beta = inv2 - st * inv * i22;
        const float bdot = -2.0f * inv2 * inv2 + (1.0f + st * inv) * inv2 * i22;
        const float wtp = dot(w, p);
        const V3 v3 = (bdot * wtp) * w - (th2 * bdot + 2.0f * beta) * p;
        const float vv[3] = {v3.x, v3.y, v3.z}, ww[3] = {w.x, w.y, w.z}, pp[3] = {p.x, p.y, p.z};
        float C[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                C[3 * i + j] = vv[i] * ww[j] + beta * ww[i] * pp[j] + (i == j ? wtp * beta : 0.f) + 0.5f * Hp[3 * i + j];
        m3_mul(C, A, B);
    }
    float R[9], Ht[9], AH[9];
    m3_quat(Ti.w, Ti.i, Ti.j, Ti.k, R);
    m3_hat(V3{Ti.x, Ti.y, Ti.z}, Ht);
    m3_mul(A, R, P);
    m3_mul(A, Ht, AH);
#pragma unroll
    for (int k = 0; k < 9; ++k) AH[k] += B[k];
    m3_mul(AH, R, K);
}

// Jacobian factors of a frame residual (frame_task.py:391-456): for a world twist [v; om] of a
// tangent column the six rows are -w (.) [P v + K om; P om], where with F = T_target^-1 T_frame,
// (w, p) its axis-angle and translation, A = Jl^-1(w)^T (so3_jac_left_inv_func,
// lie/so3_kernels.py:14-40), B the upper-right block of the SE(3) jlog (se3_jlog_func,
// lie/se3_kernels.py:359-428) and (t_i, R_i) = T_frame^-1 (se3_adjoint_func :314-346):
//   P = A R_i,   K = (A hat(t_i) + B) R_i.
__device__ __forceinline__ void frame_jacobian_factors(const Pose& Tf, const Pose& Tt, float P[9], float K[9]) {
    se3_jlog_ad(compose(pose_inverse(Tt), Tf), pose_inverse(Tf), P, K);
}

// ---------------------------------------------------------------------------
// compensated accumulation (Neumaier's variant of Kahan summation)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void kadd(float& s, float& c, float x) {
    const float t = s + x;
    if (fabsf(s) >= fabsf(x))
        c += (s - t) + x;
    else
        c += (x - t) + s;
    s = t;
}

__device__ __forceinline__ void frame_residual(const Pose& P, const float* tg, float wp, float wr, float* rp, float& ks,
                                            float& kc, float& max_pos, float& max_rot) {
    const Pose E = compose(pose_inverse(P), Pose{tg[0], tg[1], tg[2], tg[3], tg[4], tg[5], tg[6]});
    float lg[6], angle;
    se3_log(E, lg, angle);
    max_pos = fmaxf(max_pos, norm3(V3{E.x, E.y, E.z}));
    max_rot = fmaxf(max_rot, angle);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float r = (k < 3 ? wp : wr) * lg[k];
        rp[k] = r;
        kadd(ks, kc, r * r);
    }
}

// ---------------------------------------------------------------------------
// lane group
// ---------------------------------------------------------------------------
template <int G>
struct Group {
    int lane;       // 0..G-1
    int wbase;      // first warp lane of this group
    unsigned mask;  // warp lanes of this group
    __device__ __forceinline__ Group() {
        const int wl = threadIdx.x & 31;
        lane = wl & (G - 1);
        wbase = wl & ~(G - 1);
        mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << wbase);
    }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    __device__ __forceinline__ float sum(float v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
        return v;
    }
    __device__ __forceinline__ double sumd(double v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
        return v;
    }
    __device__ __forceinline__ float maxf(float v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(mask, v, o, G));
        return v;
    }
    __device__ __forceinline__ int bcast(int v, int src) const { return __shfl_sync(mask, v, src, G); }
    __device__ __forceinline__ unsigned ballot(bool p) const { return (__ballot_sync(mask, p) >> wbase) & ((G == 32) ? 0xffffffffu : ((1u << G) - 1u)); }
    __device__ __forceinline__ unsigned lt_mask() const { return (1u << lane) - 1u; }
};

// Compensated group sum: each lane holds (s, c); the group reduces pairs.
template <int G>
__device__ __forceinline__ float group_ksum(const Group<G>& g, float s, float c) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
        const float so = __shfl_xor_sync(g.mask, s, o, G);
        const float co = __shfl_xor_sync(g.mask, c, o, G);
        c += co;
        kadd(s, c, so);
    }
    return s + c;
}

// ---------------------------------------------------------------------------
// table / workspace views
// ---------------------------------------------------------------------------
// Table view: only the blob base is held; every sub-array is derived from the
// header's offsets (shared memory) where it is used, so the compiler can
// rematerialise addresses instead of pinning dozens of pointers in registers.
#define IK_TAB(type, name, field) \
    __device__ __forceinline__ const type* name() const { return reinterpret_cast<const type*>(base + h->field); }
struct Tabs {
    const TabHeader* h;
    const char* base;
    __device__ __forceinline__ void bind(const char* blob) {
        base = blob;
        h = reinterpret_cast<const TabHeader*>(blob);
    }
    IK_TAB(int, jtype, o_jtype)
    IK_TAB(int, jparent, o_jparent)
    IK_TAB(int, jact, o_jact)
    IK_TAB(int, jmimic, o_jmimic)
    IK_TAB(float, jmul, o_jmul)
    IK_TAB(float, joff, o_joff)
    IK_TAB(float, jaxis, o_jaxis)    // [nj*4]
    IK_TAB(float, jpt, o_jpt)        // [nj*8]
    IK_TAB(int, lpj, o_lpj)
    IK_TAB(unsigned long long, lanc, o_lanc)
    IK_TAB(float, lbound, o_lbound)  // [nl*4]
    IK_TAB(float, sph, o_sph)        // [ns*4]
    IK_TAB(int, sphlink, o_sphlink)
    IK_TAB(float, lim, o_lim)        // [na*2]
    IK_TAB(int, colstart, o_colstart)
    IK_TAB(int, coljoint, o_coljoint)
    IK_TAB(float, colmul, o_colmul)
    IK_TAB(int, jorder, o_jorder)
    IK_TAB(PoseEntry, pose, o_pose)
    IK_TAB(CollEntry, coll, o_coll)
    IK_TAB(JointRefEntry, jref, o_jref)
    IK_TAB(SceneEntry, scene, o_scene)
    IK_TAB(BaseRefEntry, bref, o_bref)
    IK_TAB(float, limw, o_limw)
    IK_TAB(float, mask, o_mask)
    IK_TAB(uint16_t, ab, o_ab)
    template <typename T>
    __device__ __forceinline__ const T* at(int off) const { return reinterpret_cast<const T*>(base + off); }
};
#undef IK_TAB

// Per-group workspace view: the current / proposed joint and base buffers are
// held (the accept path swaps them); the rest is derived from header offsets.
#define IK_WS(type, name, field) \
    __device__ __forceinline__ type* name() const { return reinterpret_cast<type*>(raw + h->field); }
struct Ws {
    char* raw;
    const TabHeader* h;
    float* q;      // current joints [na]
    float* qp;     // proposed joints [na]
    float* base;   // current base pose [8]
    float* basep;  // proposed base pose [8]
    __device__ __forceinline__ void bind(char* w, const TabHeader* hh) {
        raw = w;
        h = hh;
        q = reinterpret_cast<float*>(w + h->w_q);
        qp = reinterpret_cast<float*>(w + h->w_qp);
        base = reinterpret_cast<float*>(w + h->w_base);
        basep = reinterpret_cast<float*>(w + h->w_basep);
    }
    IK_WS(float, T0, w_T0)            // FK buffer A [nj*8]
    IK_WS(float, T1, w_T1)            // FK buffer B [nj*8] / motion subspace
    IK_WS(int, anc, w_anc)            // [2*nj]
    IK_WS(float, sph, w_sph)          // world spheres [ns*4]
    IK_WS(float, lbw, w_lbw)          // world link bounding centres [nl*4]
    IK_WS(float, tgt, w_tgt)          // pose targets [npose*8]
    IK_WS(float, rpose, w_rpose)      // pose residuals [npose*3]
    IK_WS(float, rlim, w_rlim)        // limit residuals [na]
    IK_WS(float, fM, w_fM)            // frame entries: Jacobian factors P, K [nframe*18]
    IK_WS(float, Jc, w_Jc)            // chunk rows [kChunkRows*Dp]: D Jacobian columns, then the residual
    IK_WS(float, rowmeta, w_rowmeta)  // chunk row records [kChunkRows*2]: sphere pair i | j << 16, residual
    IK_WS(float, Hs, w_Hs)            // normal equations [E] (packed lower H, then g)
    IK_WS(float, Hc, w_Hc)            // compensation terms [E]
    IK_WS(double, L, w_L)             // Cholesky factor [T]
    IK_WS(double, tmp, w_tmp)         // [D]
    IK_WS(double, y, w_y)             // [D]
    IK_WS(float, d32, w_d32)          // step in FP32 [D]
    IK_WS(float, misc, w_misc)        // [64]
};
#undef IK_WS

// slot record of the slots-mode self-collision term: sphere pair + residual
struct Slot {
    int32_t i, j;
    float r;
    int32_t lp;
};

// ---------------------------------------------------------------------------
// forward kinematics (robo/robot_kernels.py:265-297 local transforms,
// :390-478 pointer jumping over the joint tree).  Returns the buffer that holds
// T_world_joint; the other FK buffer is free afterwards.
// ---------------------------------------------------------------------------
template <int G>
__device__ __forceinline__ float* group_fk(const Group<G>& g, const Tabs& t, Ws& w, const float* q, const float* base) {
    const int nj = t.h->nj;
    float* src = w.T0();
    float* dst = w.T1();
    int* asrc = w.anc();
    int* adst = w.anc() + nj;
    for (int j = g.lane; j < nj; j += G) {
        float pos = 0.f;
        const int mim = t.jmimic()[j];
        const int act = t.jact()[j];
        if (mim >= 0)
            pos = q[mim] * t.jmul()[j] + t.joff()[j];
        else if (act >= 0)
            pos = q[act];
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
        pose_store(src + 8 * j, X);
        asrc[j] = t.jparent()[j];
    }
    g.sync();
    const int rounds = t.h->fk_rounds;
    for (int r = 0; r < rounds; ++r) {
        for (int j = g.lane; j < nj; j += G) {
            const int a = asrc[j];
            Pose X = pose_load(src + 8 * j);
            int na = -1;
            if (a >= 0) {
                X = compose(pose_load(src + 8 * a), X);
                na = asrc[a];
            }
            pose_store(dst + 8 * j, X);
            adst[j] = na;
        }
        g.sync();
        float* tf = src;
        src = dst;
        dst = tf;
        int* ti = asrc;
        asrc = adst;
        adst = ti;
    }
    if (base != nullptr) {
        const Pose B = pose_load(base);
        for (int j = g.lane; j < nj; j += G) pose_store(src + 8 * j, compose(B, pose_load(src + 8 * j)));
        g.sync();
    }
    return src;
}

__device__ __forceinline__ Pose link_pose(const Tabs& t, const float* Tj, const float* base, int link) {
    const int j = t.lpj()[link];
    if (j >= 0) return pose_load(Tj + 8 * j);
    return base ? pose_load(base) : pose_identity();
}

// world motion subspace column of joint j: [v; w] = Ad(T_world_joint) twist_j
__device__ __forceinline__ void joint_subspace(const Tabs& t, const float* Tj, int j, V3& v, V3& om) {
    const int ty = t.jtype()[j];
    v = V3{0.f, 0.f, 0.f};
    om = V3{0.f, 0.f, 0.f};
    if (ty == 0) return;
    const Pose P = pose_load(Tj + 8 * j);
    const V3 a{t.jaxis()[4 * j], t.jaxis()[4 * j + 1], t.jaxis()[4 * j + 2]};
    const V3 Ra = qrot(P.w, P.i, P.j, P.k, a);
    if (ty == 2) {
        om = Ra;
        v = cross(V3{P.x, P.y, P.z}, Ra);
    } else {
        v = Ra;
    }
}

// spatial column of tangent column c restricted to the ancestors of `link`
// (position_task.py:242-249; floating-base columns :261-272).
__device__ __forceinline__ void column_twist(const Tabs& t, const float* S, const float* base, int c, int link, V3& v,
                                             V3& om) {
    const int boff = t.h->base_off;
    if (c < boff) {
        const Pose B = pose_load(base);
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
    const int a = c - boff;
    v = V3{0.f, 0.f, 0.f};
    om = V3{0.f, 0.f, 0.f};
    const unsigned long long anc = t.lanc()[link];
    for (int idx = t.colstart()[a]; idx < t.colstart()[a + 1]; ++idx) {
        const int j = t.coljoint()[idx];
        if ((anc >> j) & 1ull) {
            const float m = t.colmul()[idx];
            const float* s = S + 8 * j;
            v = v + m * V3{s[0], s[1], s[2]};
            om = om + m * V3{s[3], s[4], s[5]};
        }
    }
}

// d(distance between sphere centres ci, cj)/d(column c), scaled
// (self_collision_task.py:260-321)
__device__ __forceinline__ float collision_column(const Tabs& t, const float* S, const float* base, int c, int li,
                                                  int lj, V3 ci, V3 cj, V3 n) {
    const int boff = t.h->base_off;
    if (c < boff) {
        if (c < 3) return 0.f;
        const Pose B = pose_load(base);
        const V3 e{c == 3 ? 1.f : 0.f, c == 4 ? 1.f : 0.f, c == 5 ? 1.f : 0.f};
        const V3 om = qrot(B.w, B.i, B.j, B.k, e);
        return dot(n, cross(om, ci - cj));
    }
    const int a = c - boff;
    const unsigned long long ai = t.lanc()[li], aj = t.lanc()[lj];
    float val = 0.f;
    for (int idx = t.colstart()[a]; idx < t.colstart()[a + 1]; ++idx) {
        const int j = t.coljoint()[idx];
        const bool bi = (ai >> j) & 1ull, bj = (aj >> j) & 1ull;
        if (!bi && !bj) continue;
        const float* s = S + 8 * j;
        const V3 v{s[0], s[1], s[2]}, om{s[3], s[4], s[5]};
        V3 col_i{0.f, 0.f, 0.f}, col_j{0.f, 0.f, 0.f};
        if (bi) col_i = v + cross(om, ci);
        if (bj) col_j = v + cross(om, cj);
        val += t.colmul()[idx] * dot(n, col_i - col_j);
    }
    return val;
}

// ---------------------------------------------------------------------------
// Scene collision over primitive geometry (scene_collision_task.py:276-650).
// ---------------------------------------------------------------------------
// d(point)/d(tangent column c) of a point p fixed to `link`
// (scene_distance_task.py:44-70): base columns Ad(T_world_base) e_c, joint
// columns the contributing joints' world twists v + om x p.
__device__ __forceinline__ V3 point_column(const Tabs& t, const float* S, const float* base, int c, int link, V3 p) {
    const int boff = t.h->base_off;
    if (c < boff) {
        const Pose B = pose_load(base);
        const V3 e{c % 3 == 0 ? 1.f : 0.f, c % 3 == 1 ? 1.f : 0.f, c % 3 == 2 ? 1.f : 0.f};
        const V3 Re = qrot(B.w, B.i, B.j, B.k, e);
        if (c < 3) return Re;
        return cross(Re, V3{p.x - B.x, p.y - B.y, p.z - B.z});
    }
    const int a = c - boff;
    const unsigned long long anc = t.lanc()[link];
    V3 col{0.f, 0.f, 0.f};
    for (int idx = t.colstart()[a]; idx < t.colstart()[a + 1]; ++idx) {
        const int j = t.coljoint()[idx];
        if (!((anc >> j) & 1ull)) continue;
        const float* s = S + 8 * j;
        const V3 v{s[0], s[1], s[2]}, om{s[3], s[4], s[5]};
        const V3 cj = v + cross(om, p);
        const float m = t.colmul()[idx];
        col = V3{col.x + m * cj.x, col.y + m * cj.y, col.z + m * cj.z};
    }
    return col;
}

// Nearest primitive of scene `sid` to world point p: the first of strictly
// least signed distance in query order, its world normal
// (geom/sdf_kernels.py:223-344); an empty scene gives 1e6 and a zero normal
// (geom/geoms.py:29).
struct SdfHit {
    float dist;
    V3 n;
};
__device__ __forceinline__ SdfHit scene_query(const Tabs& t, const SceneEntry& se, int sid, V3 p) {
    const float4* el = t.at<float4>(se.o_elem);
    const int* off = t.at<int>(se.o_off);
    SdfHit hit{1.0e6f, V3{0.f, 0.f, 0.f}};
    for (int e = off[sid]; e < off[sid + 1]; ++e) {
        const float4 r0 = el[5 * e], r1 = el[5 * e + 1], r2 = el[5 * e + 2], prm = el[5 * e + 3], ts = el[5 * e + 4];
        const float s = ts.y;
        V3 ql{fmaf(r0.x, p.x, fmaf(r0.y, p.y, fmaf(r0.z, p.z, r0.w))),
              fmaf(r1.x, p.x, fmaf(r1.y, p.y, fmaf(r1.z, p.z, r1.w))),
              fmaf(r2.x, p.x, fmaf(r2.y, p.y, fmaf(r2.z, p.z, r2.w)))};
        if (s != 1.f) ql = V3{ql.x / s, ql.y / s, ql.z / s};
        float un;
        V3 nl{0.f, 0.f, 1.f};
        const int type = (int)ts.x;
        if (type == IK_GEOM_BOX) {
            const V3 qv{fabsf(ql.x) - prm.x, fabsf(ql.y) - prm.y, fabsf(ql.z) - prm.z};
            const float qmax = fmaxf(fmaxf(qv.x, qv.y), qv.z);
            const V3 qp{fmaxf(qv.x, 0.f), fmaxf(qv.y, 0.f), fmaxf(qv.z, 0.f)};
            un = norm3(qp) + fminf(qmax, 0.f);
            if (qmax < 0.f) {  // inside: the nearest face
                if (qv.x >= qv.y && qv.x >= qv.z)
                    nl = V3{ql.x < 0.f ? -1.f : 1.f, 0.f, 0.f};
                else if (qv.y >= qv.z)
                    nl = V3{0.f, ql.y < 0.f ? -1.f : 1.f, 0.f};
                else
                    nl = V3{0.f, 0.f, ql.z < 0.f ? -1.f : 1.f};
            } else {
                const V3 d{ql.x - fminf(fmaxf(ql.x, -prm.x), prm.x), ql.y - fminf(fmaxf(ql.y, -prm.y), prm.y),
                           ql.z - fminf(fmaxf(ql.z, -prm.z), prm.z)};
                const float dl = norm3(d);
                if (dl > 1.0e-10f) nl = V3{d.x / dl, d.y / dl, d.z / dl};
            }
        } else if (type == IK_GEOM_SPHERE) {
            const float ql2 = norm3(ql);
            un = ql2 - prm.x;
            nl = ql2 > 1.0e-10f ? V3{ql.x / ql2, ql.y / ql2, ql.z / ql2} : V3{1.f, 0.f, 0.f};
        } else if (type == IK_GEOM_PLANE) {
            un = ql.z;
        } else {  // capsule along local z
            const float tz = fminf(fmaxf(ql.z, -prm.y), prm.y);
            const V3 d{ql.x, ql.y, ql.z - tz};
            const float dl = norm3(d);
            un = dl - prm.x;
            nl = dl > 1.0e-10f ? V3{d.x / dl, d.y / dl, d.z / dl} : V3{1.f, 0.f, 0.f};
        }
        const float dist = un * s;
        if (dist < hit.dist) {
            hit.dist = dist;
            // world normal R n_local: the rows of R^T are the columns of R
            hit.n = V3{r0.x * nl.x + r1.x * nl.y + r2.x * nl.z, r0.y * nl.x + r1.y * nl.y + r2.y * nl.z,
                       r0.z * nl.x + r1.z * nl.y + r2.z * nl.z};
        }
    }
    return hit;
}

// Penalty of signed distance sd and its derivative (terms/sphere_collision_kernels.py:17-41).
__device__ __forceinline__ float2 scene_penalty(float sd, float margin, int mode) {
    if (mode == IK_PENALTY_SURFACE_DISTANCE) return make_float2(fabsf(sd), sd > 0.f ? 1.f : (sd < 0.f ? -1.f : 0.f));
    if (mode == IK_PENALTY_PLAIN) return sd < margin ? make_float2(margin - sd, -1.f) : make_float2(0.f, 0.f);
    if (sd < 0.f) return make_float2(0.5f * margin - sd, -1.f);
    if (sd <= margin) {
        const float diff = sd - margin;
        const float inv = 1.f / (margin + 1e-6f);
        return make_float2(0.5f * inv * diff * diff, inv * diff);
    }
    return make_float2(0.f, 0.f);
}

// Row k of a scene term at the current sphere centres: the weighted residual,
// whether its Jacobian row is non-zero, and the factor `scale` with which
// row = scale * n . d(centre)/d(tangent) (scene_collision_task.py:34-82).
struct SceneRow {
    float r, scale;
    V3 n, p;
    int link;
    bool act;
};
__device__ __forceinline__ SceneRow scene_row(const Tabs& t, const Ws& w, const SceneEntry& se, int sid, int k) {
    const int s = t.at<int>(se.o_q)[k];
    const float wk = t.at<float>(se.o_w)[k];
    const float4 c = *reinterpret_cast<const float4*>(w.sph() + 4 * s);
    SceneRow o;
    o.p = V3{c.x, c.y, c.z};
    o.link = t.sphlink()[s];
    const SdfHit hit = scene_query(t, se, sid, o.p);
    o.n = hit.n;
    const float sd = hit.dist - c.w;
    const float2 pp = scene_penalty(sd, se.margin, se.penalty);
    float res = pp.x, sc = pp.y;
    if (se.use_sqrt) {
        if (pp.x > 0.f) sc *= 0.5f / sqrtf(pp.x + se.eps);
        res = sqrtf(pp.x + se.eps);
    }
    o.r = wk * res;
    o.scale = wk * sc;
    o.act = se.penalty == IK_PENALTY_SURFACE_DISTANCE || sd <= se.margin;
    return o;
}

// Base-reference block at base pose Tb: weighted residual w (.) log(Tb T_ref^-1) and, when J
// is given, its 6x6 base Jacobian w (.) Jlog(E) Ad(T_ref) (smoothness_task.py:369-460) in J[6 * k + c].
__device__ __forceinline__ void base_ref_rows(const BaseRefEntry& be, const Ws& w, const Pose& Tb, float r[6],
                                              float* J) {
    const Pose Tr = pose_load(reinterpret_cast<const float*>(w.raw) + be.ws_ref);
    const Pose E = compose(Tb, pose_inverse(Tr));
    float lg[6], ang;
    se3_log(E, lg, ang);
#pragma unroll
    for (int k = 0; k < 6; ++k) r[k] = be.w[k] * lg[k];
    if (!J) return;
    float Pm[9], Km[9];
    se3_jlog_ad(E, Tr, Pm, Km);
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            J[6 * k + c] = be.w[k] * Pm[3 * k + c];
            J[6 * k + 3 + c] = be.w[k] * Km[3 * k + c];
            J[6 * (k + 3) + c] = 0.f;
            J[6 * (k + 3) + 3 + c] = be.w[k + 3] * Pm[3 * k + c];
        }
}

__device__ __forceinline__ int scene_of(const Ws& w, const SceneEntry& se) {
    return reinterpret_cast<const int*>(w.misc())[se.misc];
}

// ---------------------------------------------------------------------------
// Broad phase of a collision term: link pairs whose bounding spheres come
// within the margin (+ `inflate`), in link-pair order, into `list` (at most
// `cap`).  With inflate = 0 and the exact distance this is the reference's
// selection test (self_collision_task.py:73-87); the all-pairs mode uses a
// small positive inflate, which keeps every sphere pair that can penetrate
// (a link's bounding sphere contains its spheres).  Returns the count.
// ---------------------------------------------------------------------------
template <int G>
__device__ __forceinline__ int group_broad_phase(const Group<G>& g, const Tabs& t, const Ws& w, const CollEntry& ce, int* list,
                                 int stride, int cap, bool exact) {
    const int* lp = t.at<int>(ce.o_lp);
    int count = 0;
    for (int b0 = 0; b0 < ce.nlp; b0 += G) {
        const int l = b0 + g.lane;
        bool act = false;
        if (l < ce.nlp) {
            const float4 a = *reinterpret_cast<const float4*>(w.lbw() + 4 * lp[2 * l]);
            const float4 b = *reinterpret_cast<const float4*>(w.lbw() + 4 * lp[2 * l + 1]);
            const V3 d{a.x - b.x, a.y - b.y, a.z - b.z};
            if (exact) {
                act = (a.w + b.w + ce.margin - norm3(d)) > 0.f;
            } else {
                const float thr = a.w + b.w + ce.margin + 1e-5f;
                act = thr > 0.f && dot(d, d) < thr * thr;
            }
        }
        const unsigned bal = g.ballot(act);
        const int pos = count + __popc(bal & g.lt_mask());
        if (act && pos < cap) list[pos * stride] = l;
        count += __popc(bal);
    }
    g.sync();
    return min(count, cap);
}

// Visit the sphere pairs of a collision term in G-wide batches: every lane of
// the group calls fn(p) once per batch (p = -1 for a lane without a pair), so
// ballots inside fn see the whole group.  A term with many sphere pairs per
// link pair first drops the link pairs whose bounding spheres stay apart.
template <int G, typename Fn>
__device__ __forceinline__ void group_for_pairs(const Group<G>& g, const Tabs& t, const Ws& w, const CollEntry& ce,
                                                Fn fn) {
    const int* lpoff = t.at<int>(ce.o_lpoff);
    if (ce.nsp > 32 * ce.nlp) {
        int* list = reinterpret_cast<int*>(w.raw + ce.ws_slots);
        const int n = group_broad_phase<G>(g, t, w, ce, list, 1, ce.nlp, false);
        for (int k = 0; k < n; ++k) {
            const int l = list[k];
            const int end = lpoff[l + 1];
            for (int b0 = lpoff[l]; b0 < end; b0 += G) {
                const int p = b0 + g.lane;
                fn(p < end ? p : -1);
            }
        }
    } else {
        for (int b0 = 0; b0 < ce.nsp; b0 += G) {
            const int p = b0 + g.lane;
            fn(p < ce.nsp ? p : -1);
        }
    }
}

// All-pairs terms whose pairs fit 64 G-wide batches keep a per-lane bit mask of
// active pairs (flat scan); larger terms with many pairs per link pair are pruned.
template <int G>
__device__ __forceinline__ bool pairs_by_mask(const CollEntry& ce) {
    return ce.nsp <= 64 * G && !(ce.nsp > 32 * ce.nlp);
}

// Penetration of sphere pair `pk` (i | j << 16): margin - surface distance, or
// a value <= 0 without the square root when the pair is clearly apart.
__device__ __forceinline__ float pair_penetration(const Ws& w, int pk, float margin) {
    const float4 a = *reinterpret_cast<const float4*>(w.sph() + 4 * (pk & 0xffff));
    const float4 b = *reinterpret_cast<const float4*>(w.sph() + 4 * (pk >> 16));
    const V3 d{a.x - b.x, a.y - b.y, a.z - b.z};
    const float thr = margin + a.w + b.w;
    const float d2 = dot(d, d);
    if (!(thr > 0.f) || d2 >= thr * thr * 1.0001f) return -1.f;
    return margin - (sqrtf(d2) - a.w - b.w);
}

// ---------------------------------------------------------------------------
// evaluation of every residual at one point (the cost pass of _accept_body,
// lm_optimizer.py:964-982): FK, spheres, pose/limit/collision residuals,
// cost = 0.5 |r|^2 and the pose errors of the metrics kernel (helpers/ik/ik.py:60-82).
// ---------------------------------------------------------------------------
// Row a of a joint-reference entry at joint value qa: residual r and the one
// Jacobian entry js (column a).
//  linear (o_vlim == 0): r = w (q - ref), js = w — smoothness_task.py:350-366,
//    configuration_task.py:322-334;
//  velocity hinge: qd = (q - prev) / dt, r = w max(0, |qd| - vmax),
//    js = w sign(qd) / dt while |qd| > vmax, else 0 — velocity_limit_task.py:188-232.
struct JrRow {
    float r, js;
};
__device__ __forceinline__ JrRow jref_row(const Tabs& t, const Ws& w, const JointRefEntry& jr, float qa, int a) {
    const float wa = t.at<float>(jr.o_w)[a];
    const float d = qa - reinterpret_cast<const float*>(w.raw)[jr.ws_ref + a];
    if (jr.o_vlim == 0) return JrRow{wa * d, wa};
    const float qd = d / jr.dt;
    const float vmax = t.at<float>(jr.o_vlim)[a];
    if (fabsf(qd) > vmax) return JrRow{wa * (fabsf(qd) - vmax), wa * (qd > 0.f ? 1.f : -1.f) / jr.dt};
    return JrRow{0.f, 0.f};
}

struct EvalOut {
    float cost;
    float max_pos;  // largest position error over position entries [m]
    float max_rot;  // largest angle error over rotation entries [rad]
    float* Tj;      // FK buffer holding T_world_joint
    float* S;       // the other FK buffer
    int nslots;     // filled slots summed over slot-mode terms
};

// F: the tables may hold frame entries (false compiles the frame paths out)
template <int G, bool F = true>
__device__ __forceinline__ EvalOut group_eval(const Group<G>& g, const Tabs& t, Ws& w, const float* q, const float* base) {
    const TabHeader* h = t.h;
    EvalOut o;
    o.Tj = group_fk<G>(g, t, w, q, base);
    o.S = (o.Tj == w.T0()) ? w.T1() : w.T0();
    float* Tj = o.Tj;
    const bool need_sph = h->ncoll > 0 || (F && h->nscene > 0);
    if (need_sph) {
        for (int s = g.lane; s < h->ns; s += G) {
            const Pose P = link_pose(t, Tj, base, t.sphlink()[s]);
            const float* c = t.sph() + 4 * s;
            const V3 wc = pose_apply(P, V3{c[0], c[1], c[2]});
            *reinterpret_cast<float4*>(w.sph() + 4 * s) = make_float4(wc.x, wc.y, wc.z, c[3]);
        }
        bool need_lbw = false;  // link bounding spheres feed the pruned scans only
        for (int ci = 0; ci < h->ncoll; ++ci)
            need_lbw = need_lbw || t.coll()[ci].mode == 0 || !pairs_by_mask<G>(t.coll()[ci]);
        if (need_lbw) {
            for (int l = g.lane; l < h->nl; l += G) {
                const Pose P = link_pose(t, Tj, base, l);
                const float* c = t.lbound() + 4 * l;
                const V3 wc = pose_apply(P, V3{c[0], c[1], c[2]});
                *reinterpret_cast<float4*>(w.lbw() + 4 * l) = make_float4(wc.x, wc.y, wc.z, c[3]);
            }
        }
        g.sync();
    }
    float ks = 0.f, kc = 0.f;
    float max_pos = 0.f, max_rot = 0.f;
    // pose entries
    for (int e = g.lane; e < h->npose; e += G) {
        const PoseEntry& pe = t.pose()[e];
        const Pose P = link_pose(t, Tj, base, pe.link);
        const float* tg = w.tgt() + 8 * e;
        float* rp = w.rpose() + pe.r0;
        if (F && pe.kind == kPoseFrame) {
            frame_residual(P, tg, pe.w[0], pe.w[1], rp, ks, kc, max_pos, max_rot);
            continue;
        }
        V3 r;
        if (pe.kind == kPosePosition) {
            const V3 err{tg[0] - P.x, tg[1] - P.y, tg[2] - P.z};
            max_pos = fmaxf(max_pos, norm3(err));
            r = V3{pe.w[0] * err.x, pe.w[1] * err.y, pe.w[2] * err.z};
        } else {
            float qw, qi, qj, qk;
            qmul_std(P.w, P.i, P.j, P.k, tg[3], -tg[4], -tg[5], -tg[6], qw, qi, qj, qk);
            float angle;
            const V3 aa = quat_to_axis_angle(qw, qi, qj, qk, angle);
            max_rot = fmaxf(max_rot, angle);
            r = V3{pe.w[0] * aa.x, pe.w[1] * aa.y, pe.w[2] * aa.z};
        }
        rp[0] = r.x;
        rp[1] = r.y;
        rp[2] = r.z;
        kadd(ks, kc, r.x * r.x);
        kadd(ks, kc, r.y * r.y);
        kadd(ks, kc, r.z * r.z);
    }
    // joint limits, position_limit.py:509-534 ("abs")
    if (h->has_limit) {
        for (int a = g.lane; a < h->na; a += G) {
            const float v = q[a];
            const float lo = t.lim()[2 * a], hi = t.lim()[2 * a + 1];
            const float err = fmaxf(0.f, v - hi) + fmaxf(0.f, lo - v);
            const float r = t.limw()[a] * err;
            w.rlim()[a] = r;
            kadd(ks, kc, r * r);
        }
    }
    // joint references (smoothness, rest) and velocity limits
    for (int je = 0; F && je < h->njref; ++je) {
        const JointRefEntry& jr = t.jref()[je];
        for (int a = g.lane; a < h->na; a += G) {
            const float r = jref_row(t, w, jr, q[a], a).r;
            kadd(ks, kc, r * r);
        }
    }
    // self collision, self_collision_task.py:73-256
    o.nslots = 0;
    for (int ci = 0; ci < h->ncoll; ++ci) {
        const CollEntry& ce = t.coll()[ci];
        const int* spk = t.at<int>(ce.o_sp);
        const int* lpoff = t.at<int>(ce.o_lpoff);
        if (ce.mode == 1) {
            if (pairs_by_mask<G>(ce)) {
                // flat scan; each lane records which of its pairs are active (one bit per
                // G-wide batch) so the linearisation of this point needs no rescan
                unsigned long long amask = 0ull;
                int bit = 0;
                for (int b0 = 0; b0 < ce.nsp; b0 += G, ++bit) {
                    const int p = b0 + g.lane;
                    if (p < ce.nsp) {
                        const float pen = pair_penetration(w, spk[p], ce.margin);
                        if (pen > 0.f) {
                            const float r = ce.weight * pen;
                            kadd(ks, kc, r * r);
                            amask |= 1ull << bit;
                        }
                    }
                }
                reinterpret_cast<unsigned long long*>(w.raw + ce.ws_slots)[g.lane] = amask;
            } else {
                group_for_pairs<G>(g, t, w, ce, [&](int p) {
                    if (p >= 0) {
                        const float pen = pair_penetration(w, spk[p], ce.margin);
                        if (pen > 0.f) {
                            const float r = ce.weight * pen;
                            kadd(ks, kc, r * r);
                        }
                    }
                });
            }
        } else {
            Slot* slots = reinterpret_cast<Slot*>(w.raw + ce.ws_slots);
            // the first K penetrating link pairs in link-pair order take the slots
            const int nsl = group_broad_phase<G>(g, t, w, ce, &slots[0].lp, 4, ce.K, true);
            // narrow phase: first strict minimum of the surface distance per kept link pair
            for (int k = g.lane; k < nsl; k += G) {
                const int l = slots[k].lp;
                float best = 1.0e10f;
                int bp = lpoff[l];
                for (int p = lpoff[l]; p < lpoff[l + 1]; ++p) {
                    const int pk = spk[p];
                    const float4 a = *reinterpret_cast<const float4*>(w.sph() + 4 * (pk & 0xffff));
                    const float4 b = *reinterpret_cast<const float4*>(w.sph() + 4 * (pk >> 16));
                    const float s = norm3(V3{a.x - b.x, a.y - b.y, a.z - b.z}) - a.w - b.w;
                    if (s < best) {
                        best = s;
                        bp = p;
                    }
                }
                const int pk = spk[bp];
                const int si = pk & 0xffff, sj = pk >> 16;
                const float4 a = *reinterpret_cast<const float4*>(w.sph() + 4 * si);
                const float4 b = *reinterpret_cast<const float4*>(w.sph() + 4 * sj);
                const float surf = norm3(V3{a.x - b.x, a.y - b.y, a.z - b.z}) - a.w - b.w;
                const float r = ce.weight * fmaxf(0.f, ce.margin - surf);
                slots[k].i = si;
                slots[k].j = sj;
                slots[k].r = r;
                kadd(ks, kc, r * r);
            }
            reinterpret_cast<int*>(w.misc())[8 + ci] = nsl;
            o.nslots += nsl;
        }
    }
    // floating-base reference blocks (smoothness / rest)
    for (int k = 0; F && base && k < h->nbref; ++k) {
        float r[6];
        base_ref_rows(t.bref()[k], w, pose_load(base), r, nullptr);
        if (g.lane < 6) kadd(ks, kc, r[g.lane] * r[g.lane]);
    }
    // scene collision, scene_collision_task.py:550-592
    for (int k = 0; F && k < h->nscene; ++k) {
        const SceneEntry& se = t.scene()[k];
        const int sid = scene_of(w, se);
        for (int i = g.lane; i < se.nq; i += G) {
            const float r = scene_row(t, w, se, sid, i).r;
            kadd(ks, kc, r * r);
        }
    }
    o.cost = 0.5f * group_ksum<G>(g, ks, kc);
    o.max_pos = g.maxf(max_pos);
    o.max_rot = g.maxf(max_rot);
    g.sync();
    return o;
}

// ---------------------------------------------------------------------------
// linearisation at the last evaluated point: motion subspace, Jacobian rows in
// chunks, compensated J^T J / J^T r accumulation, joint-limit diagonal and the
// active-DOF mask (lm_optimizer.py:145-189, 872-880; position_task.py:216-272;
// rotation_task.py:353-401; position_limit.py:538-573;
// self_collision_task.py:325-385).  Result: w.Hs()[0:T] packed lower J^T J,
// w.Hs()[T:T+D] J^T r.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int tri(int i, int j) { return (i * (i + 1)) / 2 + j; }

// compile-time loop: f(std::integral_constant<int, I>) for I = 0..N-1
template <typename F, int... I>
__device__ __forceinline__ void sfor_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void sfor(F&& f) {
    sfor_impl(f, std::make_integer_sequence<int, N>{});
}

// J^T J and J^T r of one chunk.  The residual is column D of the chunk, so the
// lower triangle of [J r]^T [J r] holds both.  For D >= 16 each lane owns 4x4 tiles of that
// (D+1)-square triangle and keeps them in registers over the chunk's rows (two
// 16-byte loads per row and tile), then merges them into the compensated sums.
// Every entry is summed over rows in ascending order, as a per-entry loop would.
constexpr int kTile = 4;

template <int G>
__device__ __forceinline__ void group_accumulate_chunk(const Group<G>& g, const Tabs& t, Ws& w, int nrows) {
    const TabHeader* h = t.h;
    const int D = h->D, Dp = h->Dp, T = h->T;
    if (D < 4 * kTile) {
        // small systems: one entry per lane at a time keeps all G lanes busy
        const int E = h->E;
        const float* Jr = w.Jc();
        for (int e = g.lane; e < E; e += G) {
            int a, b;
            if (e < T) {
                const unsigned ab = t.ab()[e];
                a = (int)(ab >> 8);
                b = (int)(ab & 0xff);
            } else {
                a = e - T;
                b = D;
            }
            float s = 0.f;
            for (int r = 0; r < nrows; ++r) s = fmaf(Jr[r * Dp + a], Jr[r * Dp + b], s);
            float hs = w.Hs()[e], hc = w.Hc()[e];
            kadd(hs, hc, s);
            w.Hs()[e] = hs;
            w.Hc()[e] = hc;
        }
        g.sync();
        return;
    }
    const int nb = (D + kTile) / kTile;  // tile rows of the (D+1)-square triangle
    const int ntiles = nb * (nb + 1) / 2;
    const float* Jc = w.Jc();
    for (int tl = g.lane; tl < ntiles; tl += G) {
        const unsigned ab = t.ab()[tl];
        const int bi = (int)(ab >> 8), bj = (int)(ab & 0xff);
        float acc[kTile][kTile];
        sfor<kTile>([&](auto U) {
            sfor<kTile>([&](auto V) { acc[decltype(U)::value][decltype(V)::value] = 0.f; });
        });
        for (int r = 0; r < nrows; ++r) {
            const float4 x = *reinterpret_cast<const float4*>(Jc + r * Dp + kTile * bi);
            const float4 y = *reinterpret_cast<const float4*>(Jc + r * Dp + kTile * bj);
            const float xa[kTile] = {x.x, x.y, x.z, x.w};
            const float ya[kTile] = {y.x, y.y, y.z, y.w};
            sfor<kTile>([&](auto U) {
                constexpr int u = decltype(U)::value;
                sfor<kTile>([&](auto V) {
                    constexpr int v = decltype(V)::value;
                    acc[u][v] = fmaf(xa[u], ya[v], acc[u][v]);
                });
            });
        }
        sfor<kTile>([&](auto U) {
            constexpr int u = decltype(U)::value;
            sfor<kTile>([&](auto V) {
                constexpr int v = decltype(V)::value;
                const int ra = kTile * bi + u, cb = kTile * bj + v;
                if (ra <= D && cb <= ra && cb < D) {
                    const int e = (ra < D) ? tri(ra, cb) : T + cb;
                    float hs = w.Hs()[e], hc = w.Hc()[e];
                    kadd(hs, hc, acc[u][v]);
                    w.Hs()[e] = hs;
                    w.Hc()[e] = hc;
                }
            });
        });
    }
    g.sync();
}

__device__ __forceinline__ int pose_entry_rows(const PoseEntry& pe) { return pe.kind == kPoseFrame ? 6 : 3; }

// The six Jacobian entries of a frame entry for one column with world twist [v; om].
__device__ __forceinline__ void frame_rows(const float* f, V3 v, V3 om, float wp, float wr, float* J, int Dp) {
    const V3 top = m3_vec(f, v) + m3_vec(f + 9, om);
    const V3 bot = m3_vec(f, om);
    J[0] = -wp * top.x;
    J[Dp] = -wp * top.y;
    J[2 * Dp] = -wp * top.z;
    J[3 * Dp] = -wr * bot.x;
    J[4 * Dp] = -wr * bot.y;
    J[5 * Dp] = -wr * bot.z;
}

// Pose entries [e0, e1) whose rows fit one chunk, starting at e0.
__device__ __forceinline__ int pose_chunk_end(const Tabs& t, int e0) {
    const int npose = t.h->npose;
    int e1 = e0, rows = 0;
    while (e1 < npose && rows + pose_entry_rows(t.pose()[e1]) <= kChunkRows) rows += pose_entry_rows(t.pose()[e1++]);
    return e1;
}

// Jacobian factors of every frame entry at the current point (see frame_jacobian_factors).
template <int G, bool F = true>
__device__ __forceinline__ void group_frame_factors(const Group<G>& g, const Tabs& t, Ws& w, const float* Tj,
                                                    const float* base) {
    if (!F || t.h->nframe == 0) return;
    for (int e = g.lane; e < t.h->npose; e += G) {
        const PoseEntry& pe = t.pose()[e];
        if (pe.kind != kPoseFrame) continue;
        const float* tg = w.tgt() + 8 * e;
        float* f = w.fM() + 18 * pe.fm;
        frame_jacobian_factors(link_pose(t, Tj, base, pe.link), Pose{tg[0], tg[1], tg[2], tg[3], tg[4], tg[5], tg[6]},
                               f, f + 9);
    }
    g.sync();
}

// Build the Jacobian of pose entries [e0, e1) into the chunk (3 rows each, 6 for a frame entry).
// A lane owns a tangent column and walks the entries: a column driven by one
// joint (the usual case) loads that joint's twist once and only tests, per
// entry, whether the joint is an ancestor of the entry's link.
template <int G, bool F = true>
__device__ __forceinline__ void group_pose_rows(const Group<G>& g, const Tabs& t, Ws& w, const float* Tj, const float* S,
                                const float* base, int e0, int e1) {
    const int D = t.h->D, Dp = t.h->Dp, boff = t.h->base_off;
    const int rbase = t.pose()[e0].r0;
    for (int c = g.lane; c < D; c += G) {
        bool single = false;
        int j1 = 0;
        V3 v1{0.f, 0.f, 0.f}, om1{0.f, 0.f, 0.f};
        if (c >= boff) {
            const int a = c - boff;
            const int s0 = t.colstart()[a];
            if (t.colstart()[a + 1] - s0 == 1) {
                single = true;
                j1 = t.coljoint()[s0];
                const float m = t.colmul()[s0];
                const float* sj = S + 8 * j1;
                v1 = V3{0.f, 0.f, 0.f} + m * V3{sj[0], sj[1], sj[2]};
                om1 = V3{0.f, 0.f, 0.f} + m * V3{sj[3], sj[4], sj[5]};
            }
        }
        for (int el = e0; el < e1; ++el) {
            const PoseEntry& pe = t.pose()[el];
            V3 v, om;
            if (single) {
                const bool anc = (t.lanc()[pe.link] >> j1) & 1ull;
                v = anc ? v1 : V3{0.f, 0.f, 0.f};
                om = anc ? om1 : V3{0.f, 0.f, 0.f};
            } else {
                column_twist(t, S, base, c, pe.link, v, om);
            }
            float* J = w.Jc() + (pe.r0 - rbase) * Dp + c;
            if (F && pe.kind == kPoseFrame) {
                frame_rows(w.fM() + 18 * pe.fm, v, om, pe.w[0], pe.w[1], J, Dp);
            } else if (pe.kind == kPosePosition) {
                const int jl = t.lpj()[pe.link];
                const float* pp = jl >= 0 ? Tj + 8 * jl : base;
                const V3 p = pp ? V3{pp[0], pp[1], pp[2]} : V3{0.f, 0.f, 0.f};
                const V3 pv = v + cross(om, p);
                J[0] = -pe.w[0] * pv.x;
                J[Dp] = -pe.w[1] * pv.y;
                J[2 * Dp] = -pe.w[2] * pv.z;
            } else {
                J[0] = pe.w[0] * om.x;
                J[Dp] = pe.w[1] * om.y;
                J[2 * Dp] = pe.w[2] * om.z;
            }
        }
    }
    const int nrows = (e1 < t.h->npose ? t.pose()[e1].r0 : t.h->pose_rows) - rbase;
    for (int r = g.lane; r < nrows; r += G) w.Jc()[r * Dp + D] = w.rpose()[rbase + r];
    g.sync();
}

// Chunk row record of a collision row: sphere pair (i | j << 16) and residual.
__device__ __forceinline__ void rowmeta_put(Ws& w, int r, int si, int sj, float res) {
    float* m = w.rowmeta() + 2 * r;
    m[0] = __int_as_float(si | (sj << 16));
    m[1] = res;
}

// Build collision rows from rowmeta (sphere pair, residual) records into the chunk.
template <int G>
__device__ __forceinline__ void group_collision_rows(const Group<G>& g, const Tabs& t, Ws& w, const float* S, const float* base,
                                     const CollEntry& ce, int nrows) {
    const int D = t.h->D, Dp = t.h->Dp;
    const int items = nrows * D;
    for (int it = g.lane; it < items; it += G) {
        const int r = it / D, c = it - r * D;
        const int pk = __float_as_int(w.rowmeta()[2 * r]);
        const int si = pk & 0xffff, sj = pk >> 16;
        const float4 a = *reinterpret_cast<const float4*>(w.sph() + 4 * si);
        const float4 b = *reinterpret_cast<const float4*>(w.sph() + 4 * sj);
        const V3 ci{a.x, a.y, a.z}, cj{b.x, b.y, b.z};
        const V3 diff = ci - cj;
        const float dist = norm3(diff);
        const float surf = dist - a.w - b.w;
        const float pen = ce.margin - surf;
        float val = 0.f;
        if (pen > 0.f) {
            const float inv = 1.f / fmaxf(1e-8f, dist);
            const V3 n{diff.x * inv, diff.y * inv, diff.z * inv};
            val = -ce.weight * collision_column(t, S, base, c, t.sphlink()[si], t.sphlink()[sj], ci, cj, n);
        }
        w.Jc()[r * Dp + c] = val;
    }
    for (int r = g.lane; r < nrows; r += G) w.Jc()[r * Dp + D] = w.rowmeta()[2 * r + 1];
    g.sync();
}

template <int G, bool F = true>
__device__ __forceinline__ void group_linearize(const Group<G>& g, const Tabs& t, Ws& w, const EvalOut& ev, const float* base) {
    const TabHeader* h = t.h;
    const int D = h->D, T = h->T, E = h->E;
    float* S = ev.S;
    const float* Tj = ev.Tj;
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
    for (int e = g.lane; e < E; e += G) {
        w.Hs()[e] = 0.f;
        w.Hc()[e] = 0.f;
    }
    g.sync();
    // pose rows, as many whole entries per chunk as fit
    group_frame_factors<G, F>(g, t, w, Tj, base);
    for (int e0 = 0; e0 < h->npose;) {
        const int e1 = pose_chunk_end(t, e0);
        group_pose_rows<G, F>(g, t, w, Tj, S, base, e0, e1);
        group_accumulate_chunk<G>(g, t, w, (e1 < h->npose ? t.pose()[e1].r0 : h->pose_rows) - t.pose()[e0].r0);
        e0 = e1;
    }
    // collision rows
    for (int ci = 0; ci < h->ncoll; ++ci) {
        const CollEntry& ce = t.coll()[ci];
        if (ce.mode == 0) {
            const Slot* slots = reinterpret_cast<const Slot*>(w.raw + ce.ws_slots);
            const int nsl = reinterpret_cast<const int*>(w.misc())[8 + ci];
            for (int k0 = 0; k0 < nsl; k0 += kChunkRows) {
                const int nr = min(kChunkRows, nsl - k0);
                for (int r = g.lane; r < nr; r += G) {
                    rowmeta_put(w, r, slots[k0 + r].i, slots[k0 + r].j, slots[k0 + r].r);
                }
                g.sync();
                group_collision_rows<G>(g, t, w, S, base, ce, nr);
                group_accumulate_chunk<G>(g, t, w, nr);
            }
        } else {
            const int* spk = t.at<int>(ce.o_sp);
            int total = kChunkRows + 1;
            unsigned long long amask = 0ull;
            int off = 0;
            if (pairs_by_mask<G>(ce)) {
                // rows from the evaluation's activity masks: exclusive scan of the lane counts
                amask = reinterpret_cast<const unsigned long long*>(w.raw + ce.ws_slots)[g.lane];
                const int cnt = __popcll(amask);
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < G; o <<= 1) {
                    const int v = __shfl_up_sync(g.mask, incl, o, G);
                    if (g.lane >= o) incl += v;
                }
                total = __shfl_sync(g.mask, incl, G - 1, G);
                off = incl - cnt;
            }
            if (total <= kChunkRows) {
                while (amask) {
                    const int bit = __ffsll((long long)amask) - 1;
                    amask &= amask - 1ull;
                    const int pk = spk[bit * G + g.lane];
                    rowmeta_put(w, off++, pk & 0xffff, pk >> 16, ce.weight * pair_penetration(w, pk, ce.margin));
                }
                g.sync();
                if (total > 0) {
                    group_collision_rows<G>(g, t, w, S, base, ce, total);
                    group_accumulate_chunk<G>(g, t, w, total);
                }
            } else {
                int filled = 0;
                group_for_pairs<G>(g, t, w, ce, [&](int p) {
                    bool act = false;
                    float r = 0.f;
                    int pk = 0;
                    if (p >= 0) {
                        pk = spk[p];
                        const float pen = pair_penetration(w, pk, ce.margin);
                        act = pen > 0.f;
                        r = ce.weight * pen;
                    }
                    const unsigned bal = g.ballot(act);
                    if (act) {
                        rowmeta_put(w, (filled + __popc(bal & g.lt_mask())), pk & 0xffff, pk >> 16, r);
                    }
                    filled += __popc(bal);
                    if (filled > kChunkRows - G) {
                        g.sync();
                        group_collision_rows<G>(g, t, w, S, base, ce, filled);
                        group_accumulate_chunk<G>(g, t, w, filled);
                        filled = 0;
                    }
                });
                if (filled > 0) {
                    g.sync();
                    group_collision_rows<G>(g, t, w, S, base, ce, filled);
                    group_accumulate_chunk<G>(g, t, w, filled);
                }
            }
        }
    }
    // floating-base reference blocks: six rows on the base columns
    for (int k = 0; F && base && k < h->nbref; ++k) {
        if (g.lane < 6) {
            float r[6], J6[36];
            base_ref_rows(t.bref()[k], w, pose_load(base), r, J6);
            float* J = w.Jc() + g.lane * h->Dp;
            for (int c = 0; c < h->D; ++c) J[c] = c < 6 ? J6[6 * g.lane + c] : 0.f;
            J[h->D] = r[g.lane];
        }
        g.sync();
        group_accumulate_chunk<G>(g, t, w, 6);
    }
    // scene-collision rows with a non-zero Jacobian, compacted into chunks
    for (int k = 0; F && k < h->nscene; ++k) {
        const SceneEntry& se = t.scene()[k];
        const int sid = scene_of(w, se);
        const int D = h->D, Dp = h->Dp;
        int filled = 0;
        for (int b0 = 0; b0 < se.nq; b0 += G) {
            const int i = b0 + g.lane;
            SceneRow sr;
            sr.act = false;
            if (i < se.nq) sr = scene_row(t, w, se, sid, i);
            const unsigned bal = g.ballot(sr.act);
            if (sr.act) {
                float* J = w.Jc() + (filled + __popc(bal & g.lt_mask())) * Dp;
                for (int c = 0; c < D; ++c) J[c] = sr.scale * dot(sr.n, point_column(t, S, base, c, sr.link, sr.p));
                J[D] = sr.r;
            }
            filled += __popc(bal);
            if (filled > kChunkRows - G) {
                g.sync();
                group_accumulate_chunk<G>(g, t, w, filled);
                filled = 0;
            }
        }
        if (filled > 0) {
            g.sync();
            group_accumulate_chunk<G>(g, t, w, filled);
        }
    }
    // finalise: fold compensation, joint-limit diagonal, active-DOF mask
    const int boff = h->base_off;
    for (int e = g.lane; e < E; e += G) {
        float v = w.Hs()[e] + w.Hc()[e];
        int a, b;
        if (e < T) {
            const unsigned ab = t.ab()[e];
            a = ab >> 8;
            b = ab & 0xff;
            if (h->has_limit && a == b && a >= boff) {
                const int k = a - boff;
                const float qv = w.q[k];
                const float lo = t.lim()[2 * k], hi = t.lim()[2 * k + 1];
                const float sg = qv > hi ? 1.f : (qv < lo ? -1.f : 0.f);
                const float js = t.limw()[k] * sg;
                v += js * js;
            }
            if (F && a == b && a >= boff)
                for (int je = 0; je < h->njref; ++je) {
                    const float js = jref_row(t, w, t.jref()[je], w.q[a - boff], a - boff).js;
                    v += js * js;
                }
        } else {
            a = e - T;
            b = a;
            if (h->has_limit && a >= boff) {
                const int k = a - boff;
                const float qv = w.q[k];
                const float lo = t.lim()[2 * k], hi = t.lim()[2 * k + 1];
                const float sg = qv > hi ? 1.f : (qv < lo ? -1.f : 0.f);
                v += t.limw()[k] * sg * w.rlim()[k];
            }
            if (F && a >= boff)
                for (int je = 0; je < h->njref; ++je) {
                    const JrRow row = jref_row(t, w, t.jref()[je], w.q[a - boff], a - boff);
                    v += row.js * row.r;
                }
        }
        if (h->mask_any) v *= (e < T) ? t.mask()[a] * t.mask()[b] : t.mask()[a];
        w.Hs()[e] = v;
    }
    g.sync();
}

// ---------------------------------------------------------------------------
// damped FP64 Cholesky solve (lm_optimizer.py:56-79 / 145-189):
//   (H + lambda I) delta = -g,  pred = 0.5 delta . (lambda delta - g)
// H packed lower in `Hp` (fp32), g in Hp[T:].  Step in w.y() (fp64) and w.d32().
// Returns false when a pivot is not positive (delta = 0, pred = 0).
// ---------------------------------------------------------------------------

constexpr int kSmallD = 8;  // systems up to this size are factorised in registers

__host__ __device__ constexpr int ctri(int i, int j) { return (i * (i + 1)) / 2 + j; }

// D <= kSmallD: every lane factorises the system in FP64 registers at its
// exact size N = D — left-looking Cholesky, forward and back substitution
// fully unrolled — so the solve needs no shared memory and no
// synchronisation; all lanes hold the same step.
template <int G, int N>
__device__ __forceinline__ bool group_small_solve_n(const Group<G>& g, const Tabs& t, Ws& w, const float* Hp,
                                                    float lambda_f, double& pred, double& dnorm) {
    const int D = N, T = t.h->T;
    const double lam = (double)lambda_f;
    double a[ctri(N, 0)];
    double y[N];
    sfor<N>([&](auto I) {
        constexpr int i = decltype(I)::value;
        sfor<i + 1>([&](auto J) {
            constexpr int j = decltype(J)::value;
            a[ctri(i, j)] = (double)Hp[ctri(i, j)] + ((i == j) ? lam : 0.0);
        });
        y[i] = -(double)Hp[T + i];
    });
    bool ok = true;
    sfor<N>([&](auto K) {
        constexpr int k = decltype(K)::value;
        double s = a[ctri(k, k)];
        sfor<k>([&](auto M) { constexpr int m = decltype(M)::value; s -= a[ctri(k, m)] * a[ctri(k, m)]; });
        ok = ok && (s > 0.0);
        const double inv = rsqrt(s);
        a[ctri(k, k)] = inv;
        sfor<N - k - 1>([&](auto I0) {
            constexpr int i = k + 1 + decltype(I0)::value;
            double v = a[ctri(i, k)];
            sfor<k>([&](auto M) { constexpr int m = decltype(M)::value; v -= a[ctri(i, m)] * a[ctri(k, m)]; });
            a[ctri(i, k)] = v * inv;
        });
    });
    if (!ok) {
        for (int i = g.lane; i < D; i += G) w.d32()[i] = 0.f;
        pred = 0.0;
        dnorm = 0.0;
        g.sync();
        return false;
    }
    sfor<N>([&](auto I) {
        constexpr int i = decltype(I)::value;
        double v = y[i];
        sfor<i>([&](auto M) { constexpr int m = decltype(M)::value; v -= a[ctri(i, m)] * y[m]; });
        y[i] = v * a[ctri(i, i)];
    });
    sfor<N>([&](auto I0) {
        constexpr int i = N - 1 - decltype(I0)::value;
        double v = y[i];
        sfor<N - 1 - i>([&](auto M0) {
            constexpr int m = i + 1 + decltype(M0)::value;
            v -= a[ctri(m, i)] * y[m];
        });
        y[i] = v * a[ctri(i, i)];
    });
    double pp = 0.0, nn = 0.0;
    sfor<N>([&](auto I) {
        constexpr int i = decltype(I)::value;
        pp += y[i] * (lam * y[i] - (double)Hp[T + i]);
        nn += y[i] * y[i];
    });
    pred = 0.5 * pp;
    dnorm = sqrt(nn);
    sfor<N>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if ((i % G) == g.lane) w.d32()[i] = (float)y[i];
    });
    g.sync();
    return true;
}

template <int G>
__device__ __forceinline__ bool group_small_solve(const Group<G>& g, const Tabs& t, Ws& w, const float* Hp, float lambda_f,
                                                  double& pred, double& dnorm) {
    switch (t.h->D) {
        case 1: return group_small_solve_n<G, 1>(g, t, w, Hp, lambda_f, pred, dnorm);
        case 2: return group_small_solve_n<G, 2>(g, t, w, Hp, lambda_f, pred, dnorm);
        case 3: return group_small_solve_n<G, 3>(g, t, w, Hp, lambda_f, pred, dnorm);
        case 4: return group_small_solve_n<G, 4>(g, t, w, Hp, lambda_f, pred, dnorm);
        case 5: return group_small_solve_n<G, 5>(g, t, w, Hp, lambda_f, pred, dnorm);
        case 6: return group_small_solve_n<G, 6>(g, t, w, Hp, lambda_f, pred, dnorm);
        case 7: return group_small_solve_n<G, 7>(g, t, w, Hp, lambda_f, pred, dnorm);
        default: return group_small_solve_n<G, 8>(g, t, w, Hp, lambda_f, pred, dnorm);
    }
}

// D > kSmallD: blocked right-looking factorisation in shared memory.  Per
// block of kCholBlock columns every lane factorises the diagonal block
// redundantly in registers, lanes solve the panel rows they own, then update
// the trailing triangle element-parallel; two group syncs per block instead of
// three per column.  The subtractions run in the same order as a column-by-
// column right-looking factorisation.  The diagonal is stored as 1/L_kk.
// Both triangular solves keep the right-hand side in registers of the lanes
// that own its rows and broadcast each solved entry by shuffle (no syncs).
constexpr int kCholBlock = 4;

template <int G>
__device__ __forceinline__ bool group_damped_solve(const Group<G>& g, const Tabs& t, Ws& w, const float* Hp, float lambda_f,
                                   double& pred, double& dnorm) {
    const int D = t.h->D, T = t.h->T;
    if (D <= kSmallD) return group_small_solve<G>(g, t, w, Hp, lambda_f, pred, dnorm);
    constexpr int B = kCholBlock;
    double* L = w.L();
    const double lam = (double)lambda_f;
    for (int e = g.lane; e < T; e += G) {
        const unsigned ab = t.ab()[e];
        double v = (double)Hp[e];
        if ((ab >> 8) == (ab & 0xff)) v += lam;
        L[e] = v;
    }
    g.sync();
    bool ok = true;
    for (int k0 = 0; k0 < D; k0 += B) {
        const int bs = min(B, D - k0);
        // diagonal block, identity-padded past D
        double d[ctri(B, 0)];
        sfor<B>([&](auto I) {
            constexpr int i = decltype(I)::value;
            sfor<i + 1>([&](auto J) {
                constexpr int j = decltype(J)::value;
                d[ctri(i, j)] = (i < bs) ? L[tri(k0 + i, k0 + j)] : ((i == j) ? 1.0 : 0.0);
            });
        });
        sfor<B>([&](auto C) {
            constexpr int c = decltype(C)::value;
            double s = d[ctri(c, c)];
            sfor<c>([&](auto M) { constexpr int m = decltype(M)::value; s -= d[ctri(c, m)] * d[ctri(c, m)]; });
            ok = ok && (s > 0.0);
            const double inv = rsqrt(s);
            d[ctri(c, c)] = inv;
            sfor<B - c - 1>([&](auto I0) {
                constexpr int i = c + 1 + decltype(I0)::value;
                double v = d[ctri(i, c)];
                sfor<c>([&](auto M) { constexpr int m = decltype(M)::value; v -= d[ctri(i, m)] * d[ctri(c, m)]; });
                d[ctri(i, c)] = v * inv;
            });
        });
        if (!ok) break;  // every lane factorised the same block: a uniform decision
        // panel rows below the block
        for (int i = k0 + bs + g.lane; i < D; i += G) {
            double* row = L + tri(i, k0);
            double p[B];
            sfor<B>([&](auto C) {
                constexpr int c = decltype(C)::value;
                if (c < bs) {
                    double v = row[c];
                    sfor<c>([&](auto M) { constexpr int m = decltype(M)::value; v -= p[m] * d[ctri(c, m)]; });
                    p[c] = v * d[ctri(c, c)];
                    row[c] = p[c];
                }
            });
        }
        if (g.lane == 0) {
            sfor<B>([&](auto I) {
                constexpr int i = decltype(I)::value;
                sfor<i + 1>([&](auto J) {
                    constexpr int j = decltype(J)::value;
                    if (i < bs) L[tri(k0 + i, k0 + j)] = d[ctri(i, j)];
                });
            });
        }
        g.sync();
        // trailing triangle (i, j), k0+bs <= j <= i < D
        const int base = k0 + bs, n = D - base;
        const int nu = n * (n + 1) / 2;
        for (int u = g.lane; u < nu; u += G) {
            const unsigned ab = t.ab()[u];
            const int i = base + (int)(ab >> 8), j = base + (int)(ab & 0xff);
            const double* li = L + tri(i, k0);
            const double* lj = L + tri(j, k0);
            double v = L[tri(i, j)];
            sfor<B>([&](auto C) {
                constexpr int c = decltype(C)::value;
                if (c < bs) v -= li[c] * lj[c];
            });
            L[tri(i, j)] = v;
        }
        g.sync();
    }
    if (!ok) {
        for (int i = g.lane; i < D; i += G) w.d32()[i] = 0.f;
        pred = 0.0;
        dnorm = 0.0;
        g.sync();
        return false;
    }
    // right-hand side -g in the registers of the lanes owning its rows (i = lane + G r)
    constexpr int R = (kMaxDim + G - 1) / G;
    double yv[R];
    sfor<R>([&](auto Rr) {
        constexpr int r = decltype(Rr)::value;
        const int i = g.lane + G * r;
        yv[r] = (i < D) ? -(double)Hp[T + i] : 0.0;
    });
    // forward substitution L z = -g
    for (int k = 0; k < D; ++k) {
        const int rk = k / G;
        double yk = 0.0;
        sfor<R>([&](auto Rr) {
            constexpr int r = decltype(Rr)::value;
            if (r == rk) yk = yv[r];
        });
        const double zk = __shfl_sync(g.mask, yk, k % G, G) * L[tri(k, k)];
        sfor<R>([&](auto Rr) {
            constexpr int r = decltype(Rr)::value;
            const int i = g.lane + G * r;
            if (i > k && i < D) yv[r] -= L[tri(i, k)] * zk;
            else if (i == k) yv[r] = zk;
        });
    }
    // back substitution L^T x = z
    for (int k = D - 1; k >= 0; --k) {
        const int rk = k / G;
        double zk = 0.0;
        sfor<R>([&](auto Rr) {
            constexpr int r = decltype(Rr)::value;
            if (r == rk) zk = yv[r];
        });
        const double xk = __shfl_sync(g.mask, zk, k % G, G) * L[tri(k, k)];
        sfor<R>([&](auto Rr) {
            constexpr int r = decltype(Rr)::value;
            const int i = g.lane + G * r;
            if (i < k) yv[r] -= L[tri(k, i)] * xk;
            else if (i == k) yv[r] = xk;
        });
    }
    double pp = 0.0, nn = 0.0;
    sfor<R>([&](auto Rr) {
        constexpr int r = decltype(Rr)::value;
        const int i = g.lane + G * r;
        if (i < D) {
            const double x = yv[r];
            pp += x * (lam * x - (double)Hp[T + i]);
            nn += x * x;
            w.d32()[i] = (float)x;
        }
    });
    pred = 0.5 * g.sumd(pp);
    dnorm = sqrt(g.sumd(nn));
    g.sync();
    return true;
}

// ---------------------------------------------------------------------------
// integrate, robo/robot_kernels.py:563-644 (q + mask * delta; base * exp(delta_base))
// ---------------------------------------------------------------------------
template <int G>
__device__ __forceinline__ void group_integrate(const Group<G>& g, const Tabs& t, Ws& w, const float* q, const float* base, float* qo,
                                float* baseo) {
    const TabHeader* h = t.h;
    const int boff = h->base_off;
    for (int a = g.lane; a < h->na; a += G) {
        const float m = h->mask_any ? t.mask()[boff + a] : 1.f;
        qo[a] = q[a] + m * w.d32()[boff + a];
    }
    if (boff && g.lane == 0) {
        float xi[6];
        for (int k = 0; k < 6; ++k) xi[k] = w.d32()[k];
        if (h->mask_any)
            for (int k = 3; k < 6; ++k) xi[k] *= t.mask()[k];
        const Pose B = pose_load(base);
        Pose N = compose(B, se3_exp(xi, 1e-4f));
        if (h->mask_any) {
            if (t.mask()[0] == 0.f) N.x = B.x;
            if (t.mask()[1] == 0.f) N.y = B.y;
            if (t.mask()[2] == 0.f) N.z = B.z;
        }
        pose_store(baseo, N);
    }
    g.sync();
}

}  // namespace b200ik
