// ik_tables.h — the packed table blob one IK problem class runs on.
//
// The host lowers a robot (RobotSpec tables, robokit robo/robot_spec.py:65-139)
// and a term list (terms/dense/*.py) into ONE contiguous blob.  Every CTA of a
// solver launch stages the blob into shared memory with 16-byte loads and then
// reads the kinematic tree, the term rows and the per-group workspace layout
// from it.  Offsets are byte offsets from the blob start, each 16-byte aligned.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define IK_HD __host__ __device__
#else
#define IK_HD
#endif

namespace b200ik {

constexpr int kMaxJoints = 64;     // joint bit masks are one uint64
constexpr int kMaxLinks = 128;
constexpr int kMaxDim = 64;        // tangent dimension (6 base + actuated)
constexpr int kMaxSpheres = 1024;
constexpr int kChunkRows = 32;     // Jacobian rows staged per accumulation chunk

// Stride between the workspaces of consecutive lane groups of G lanes: whole
// 128-byte lines plus 4 G bytes, so the groups of one warp sit on different
// shared-memory banks (G < 32).
IK_HD inline constexpr int ws_stride(int ws_bytes, int G) { return ((ws_bytes + 127) & ~127) + (G < 32 ? 4 * G : 0); }

// pose-entry kinds
constexpr int kPosePosition = 0;
constexpr int kPoseRotation = 1;
constexpr int kPoseFrame = 2;   // six rows: SE(3) log of T_frame^-1 T_target (frame_task.py:505-527)

// One block of three residual rows: a PositionTask or RotationTask frame.
struct PoseEntry {
    int32_t link;         // link index of the frame
    int32_t kind;         // kPosePosition / kPoseRotation / kPoseFrame
    int32_t term;         // term index in the user's list
    int32_t frame;        // frame index inside the term
    int32_t num_frames;   // frames of the owning term (target row stride)
    int32_t out_row;      // first row in the reference layout
    int32_t target_rows;  // rows of the target array (broadcast rule)
    int32_t r0;           // first row of this entry among all pose rows
    float w[4];           // row weights (3 used); a frame entry: w[0] translation, w[1] rotation rows
    const float* targets; // device pointer [target_rows, num_frames, 7]
    int32_t fm;           // frame entry: slot of its Jacobian factors in the workspace, else -1
    int32_t pad1;
};
static_assert(sizeof(PoseEntry) == 64, "PoseEntry layout");

// One SelfCollisionTask (sphere representation).
struct CollEntry {
    int32_t mode;         // IK_PAIRS_SLOTS / IK_PAIRS_ALL
    int32_t K;            // slots (max_active_pairs)
    int32_t nlp;          // link pairs
    int32_t nsp;          // sphere pairs
    int32_t out_row;      // first row in the reference layout
    int32_t o_lp;         // int32 [nlp*2] link pairs
    int32_t o_lpoff;      // int32 [nlp+1] CSR offsets into sphere pairs
    int32_t o_sp;         // int32 [nsp] sphere pairs packed (i | j << 16)
    int32_t ws_slots;     // workspace offset of the slot list (slots mode)
    int32_t rows;         // residual rows this term owns in the reference layout
    float margin;
    float weight;
    int32_t t_mask;       // lane-per-problem workspace: first 32-bit activity word (all-pairs mode)
    int32_t pad[3];
};
static_assert(sizeof(CollEntry) == 64, "CollEntry layout");

// One joint-reference term: rows w_a (q_a - ref_a) (SmoothnessTask with the
// previous state, smoothness_task.py:350-366; ConfigurationTask toward a rest
// configuration, configuration_task.py:25-120; joints only).
struct JointRefEntry {
    int32_t out_row;      // first row in the reference layout
    int32_t target_rows;  // rows of the reference array (broadcast rule as for pose targets)
    int32_t o_w;          // blob offset of the weights [na]
    int32_t ws_ref;       // workspace float offset of this problem's reference [na]
    const float* ref;     // device pointer [target_rows, na]
    int32_t o_vlim;       // blob offset of the velocity limits [na]; 0 (the header) = a linear row
    float dt;             // velocity rows: the time step
};
static_assert(sizeof(JointRefEntry) == 32, "JointRefEntry layout");

// One SceneCollisionTask over primitive geometry (scene_collision_task.py:276-650):
// robot sphere centres against the primitives of the problem's scene.
// Primitive records: 5 float4 each — the three rows of the inverse pose
// [R^T | -R^T t], the parameters, and (type, scale, 0, 0) — sorted by scene
// (stable, so a point meets them in query order); CSR offsets per scene.
struct SceneEntry {
    int32_t out_row;      // first row in the reference layout
    int32_t nq;           // robot spheres queried (one row each)
    int32_t o_q;          // int32 [nq] sphere indices
    int32_t o_w;          // float [nq] weights
    int32_t o_elem;       // float4 [nelem * 5] primitive records
    int32_t o_off;        // int32 [nscenes + 1] CSR offsets into the records
    int32_t nscenes;
    int32_t penalty;      // IK_PENALTY_*
    int32_t use_sqrt;     // residual sqrt(penalty + eps)
    float margin;         // activation distance
    float eps;
    int32_t scene_rows;   // rows of scene_idx (0: scene 0 for every problem)
    const int32_t* scene_idx;  // device [scene_rows]
    int32_t misc;         // workspace misc slot holding the problem's scene index
    int32_t pad;
};
static_assert(sizeof(SceneEntry) == 64, "SceneEntry layout");

// One base-reference block: rows w_k log(T_world_base T_ref^-1)_k (SmoothnessTask with a
// floating-base previous state, smoothness_task.py:369-402, 426-460; ConfigurationTask toward a
// rest base pose, configuration_task.py:337-384).
struct BaseRefEntry {
    int32_t out_row;      // first of the six rows
    int32_t target_rows;  // rows of the reference array (broadcast rule as for pose targets)
    int32_t ws_ref;       // workspace float offset of this problem's reference pose [8]
    int32_t pad;
    float w[6];
    const float* ref;     // device [target_rows, 7]
};
static_assert(sizeof(BaseRefEntry) == 48, "BaseRefEntry layout");

struct TabHeader {
    int32_t bytes;        // blob size, multiple of 16
    int32_t nj, nl, na, ns;
    int32_t fk_rounds;    // pointer-jumping rounds = ceil(log2(max depth))
    int32_t D;            // tangent dimension
    int32_t base_off;     // 6 with a floating base, else 0
    int32_t R_ref;        // residual rows in the reference layout
    int32_t npose, ncoll, has_limit, limit_row;
    int32_t mask_any;     // 1 if an active-DOF mask is present
    int32_t E;            // D(D+1)/2 + D accumulated normal-equation entries
    int32_t T;            // D(D+1)/2
    // robot tables
    int32_t o_jtype, o_jparent, o_jact, o_jmimic, o_jmul, o_joff, o_jaxis, o_jpt;
    int32_t o_lpj, o_lanc, o_lbound, o_sph, o_sphlink, o_lim;
    int32_t o_colstart, o_coljoint, o_colmul;
    int32_t o_jorder;     // joints in topological order (parents first)
    // problem tables
    int32_t o_pose, o_coll, o_limw, o_mask, o_ab;
    // per-group workspace layout (byte offsets inside one group's workspace)
    int32_t ws_bytes;
    int32_t w_T0, w_T1, w_anc, w_sph, w_lbw, w_tgt, w_rpose, w_rlim;
    int32_t w_Jc, w_rc, w_rowmeta, w_Hs, w_Hc, w_L, w_tmp, w_y;
    int32_t w_q, w_qp, w_base, w_basep, w_d32, w_misc;
    int32_t Dp;           // padded row stride of the Jacobian chunk
    int32_t max_slots;    // sum of slot-mode K over collision terms
    int32_t pose_rows;    // rows of all pose entries (3 per position/rotation entry, 6 per frame entry)
    int32_t nframe;       // frame entries
    int32_t w_fM;         // workspace: 18 floats per frame entry (Jacobian factors P, K)
    int32_t njref;        // joint-reference terms
    int32_t o_jref;       // blob offset of the JointRefEntry table
    int32_t w_jref;       // workspace: the references [njref * na]
    // lane-per-problem workspace (float offsets; float k of lane t at [k * blockDim + t])
    int32_t thread_ok;    // 1 when the lane-per-problem kernels can run this problem
    int32_t t_floats;
    int32_t t_Tj, t_S, t_sph, t_tgt, t_Hs, t_Hc, t_q, t_qp, t_base, t_basep;
    int32_t nscene;       // scene-collision terms (at most IK_SCENE_MAX_TERMS)
    int32_t o_scene;      // blob offset of the SceneEntry table
    int32_t nbref;        // base-reference blocks
    int32_t o_bref;       // blob offset of the BaseRefEntry table
    int32_t w_bref;       // workspace: the reference poses [nbref * 8]
    int32_t pad2;
};

}  // namespace b200ik
