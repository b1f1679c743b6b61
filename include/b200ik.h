/*
 * b200ik.h — C ABI of libb200ik.so, the sm_100a batched Levenberg–Marquardt
 * inverse-kinematics library.
 *
 * Every entry point returns an int status: 0 on success, a negative IK_E_*
 * code on an API error (the message is kept per host thread and returned by
 * ik_last_error()).  Per-problem numerical outcomes (converged, iteration cap,
 * non-SPD normal matrix, non-finite input) are written to an int32 status array
 * on the device instead.  No C++ exception crosses this boundary.
 *
 * Pointers named d_* are device pointers owned by the caller; the library
 * never retains them beyond the call, except the pose-target pointers a term
 * descriptor names, which are read at every solve (like the target arrays a
 * reference term keeps, robokit terms/dense/position_task.py:77).  All calls are
 * stream-ordered on the caller's stream (a cudaStream_t passed as void*, 0 for
 * the legacy default stream) and do not synchronise the device.
 *
 * Pose layout everywhere: 7 floats [x, y, z, qw, qx, qy, qz], the reference's
 * vec7 (robokit AGENTS.md "SE(3)"; xform/warp/rotation_conversions.py:268).
 * Tangent layout of one problem: [6 floating-base twist entries, if floating |
 * one entry per actuated joint] (robo/robot_state.py:178-181).
 */
#ifndef B200IK_H
#define B200IK_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define IK_OK 0
#define IK_E_INVALID (-1)     /* bad argument / inconsistent tables           */
#define IK_E_CAPACITY (-2)    /* batch larger than the problem's capacity     */
#define IK_E_OOM (-3)         /* device allocation failed                     */
#define IK_E_CUDA (-4)        /* a CUDA runtime call failed                   */
#define IK_E_UNSUPPORTED (-5) /* a size beyond the kernel's compiled limits   */
#define IK_E_NO_DEVICE (-6)   /* no CUDA device visible                       */

/* per-problem status bits written by the solvers */
#define IK_ST_RUNNING 0
#define IK_ST_CONVERGED 1   /* a per-problem stop rule fired                  */
#define IK_ST_MAX_ITER 2    /* iteration cap reached                          */
#define IK_ST_NOT_SPD 4     /* some damped normal matrix had a pivot <= 0     */
#define IK_ST_NONFINITE 8   /* non-finite cost at the start point             */
#define IK_ST_FLAGS 0xff    /* status bits; the rest counts accepted steps    */
#define IK_ST_ACCEPTS(s) ((s) >> 8)

/* joint types, robo/robot_spec.py:34-41 */
#define IK_JOINT_FIXED 0
#define IK_JOINT_PRISMATIC 1
#define IK_JOINT_REVOLUTE 2

/* term kinds */
#define IK_TERM_POSITION 1       /* terms/dense/position_task.py:18            */
#define IK_TERM_ROTATION 2       /* terms/dense/rotation_task.py:25            */
#define IK_TERM_POSITION_LIMIT 3 /* terms/dense/position_limit.py:185 ("abs")  */
#define IK_TERM_SELF_COLLISION 4 /* terms/dense/self_collision_task.py:593     */
#define IK_TERM_FRAME 5          /* terms/dense/frame_task.py:47 ("log" mode): six rows per frame,
                                    weights [num_frames*2] = (position, orientation) per frame */
#define IK_TERM_JOINT_REF 6      /* w_a (q_a - ref_a), one row per actuated joint: SmoothnessTask
                                    (smoothness_task.py:22) / ConfigurationTask (configuration_task.py:25),
                                    joints only; weights [na]; d_targets = references [target_rows, na] */
#define IK_TERM_VELOCITY_LIMIT 7 /* w_a max(0, |q_a - prev_a| / dt - vmax_a), one row per actuated joint:
                                    VelocityLimitTask (velocity_limit_task.py:14); weights [na];
                                    d_targets = previous joints [target_rows, na]; dt, velocity_limits */
#define IK_TERM_BASE_REF 9        /* w_k log(T_world_base T_ref^-1)_k, six rows [v; om]: the floating-base
                                     block of SmoothnessTask / ConfigurationTask (smoothness_task.py:369-402,
                                     configuration_task.py:337-368); weights [6];
                                     d_targets = reference base poses [target_rows, 7]; floating base only */
#define IK_TERM_SCENE_COLLISION 8 /* terms/dense/scene_collision_task.py:276 with primitive geometry
                                     (geom/geoms.py:372-500): one row per queried robot sphere,
                                     w * penalty(sdf(centre) - radius); weights [num_query_spheres] */

/* scene-collision penalties (terms/sphere_collision_kernels.py:17-41) */
#define IK_PENALTY_SMOOTH 0
#define IK_PENALTY_PLAIN 1
#define IK_PENALTY_SURFACE_DISTANCE 2

/* scene primitives (geom/geoms.py:372-500, geom/sdf_kernels.py:223-344) and the
 * host record of one primitive: IK_GEOM_FLOATS floats
 *   [0] type IK_GEOM_*, [1] scene index, [2] uniform scale (1 = none), [3] 0,
 *   [4..7] parameters: box half extents (x, y, z); sphere radius; plane none;
 *          capsule radius, half height (axis local z),
 *   [8..14] pose [x y z qw qx qy qz] of the primitive in the world, [15] 0. */
#define IK_GEOM_BOX 0
#define IK_GEOM_SPHERE 1
#define IK_GEOM_PLANE 2
#define IK_GEOM_CAPSULE 3
#define IK_GEOM_FLOATS 16
#define IK_SCENE_MAX_TERMS 8

/* self-collision pair modes */
#define IK_PAIRS_SLOTS 0 /* reference: <= K link pairs, most penetrating sphere pair each */
#define IK_PAIRS_ALL 1   /* every filtered sphere pair is one residual row              */

/* stop rules (bitmask) */
#define IK_STOP_NONE 0
#define IK_STOP_ALL_COST 1 /* reference rule: stop once every problem's cost <= cost_tol (opt/optimizer.py:237-239) */
#define IK_STOP_STEP 2     /* per problem: ||delta||_2 < step_tol                                             */
#define IK_STOP_POSE 4     /* per problem: every pose target within pose_pos_tol [m] and pose_rot_tol [rad]   */
#define IK_STOP_COST 8     /* per problem: cost <= cost_tol                                                   */

/* ---- robot model ------------------------------------------------------- */
/* The kinematic tables of robo/robot_spec.py:65-139 (RobotSpec) after
 * parsing; arrays are host pointers copied at ik_robot_create. */
typedef struct IkRobotDesc {
    int32_t num_joints;   /* all joints, fixed included (<= 64)                 */
    int32_t num_links;    /* (<= 128)                                           */
    int32_t num_actuated; /* (<= 64 together with a floating base's 6)          */
    int32_t num_spheres;  /* collision spheres, 0 if none (<= 256)              */
    const int32_t* joint_types;       /* [nj]                                     */
    const float* joint_axes;          /* [nj*3]                                   */
    const float* parent_transforms;   /* [nj*7] joint origin in its parent joint  */
    const int32_t* parent_joints;     /* [nj] -1 = attached to the base link      */
    const int32_t* actuated_indices;  /* [nj] -1 = not actuated                   */
    const int32_t* mimic_indices;     /* [nj] actuated index mimicked, -1 = none  */
    const float* mimic_multipliers;   /* [nj]                                     */
    const float* mimic_offsets;       /* [nj]                                     */
    const int32_t* link_parent_joints;/* [nl] -1 = base link                      */
    const float* actuated_limits;     /* [na*2] lower, upper                      */
    const float* sphere_centers;      /* [ns*3] link-local                        */
    const float* sphere_radii;        /* [ns]                                     */
    const int32_t* sphere_links;      /* [ns]                                     */
    const float* link_bound_centers;  /* [nl*3] link-local bounding-sphere centre */
    const float* link_bound_radii;    /* [nl]                                     */
} IkRobotDesc;

typedef struct IkRobot IkRobot;
typedef struct IkProblem IkProblem;

/* ---- cost terms -------------------------------------------------------- */
typedef struct IkTermDesc {
    int32_t kind;                 /* IK_TERM_*                                         */
    /* pose terms */
    int32_t num_frames;
    const int32_t* frame_links;   /* [num_frames] link indices                         */
    const float* weights;         /* position/rotation: [num_frames*3]; limit: [na];
                                     self-collision: [1]                                 */
    const float* d_targets;       /* device [capacity rows, num_frames, 7] pose targets  */
    int32_t target_rows;          /* rows of d_targets; problem b reads row
                                     b / max(1, batch / target_rows) (reference n_repeat,
                                     position_task.py:201-202)                           */
    /* self-collision */
    float margin;
    int32_t max_active_pairs;     /* K, slots mode                                      */
    int32_t pair_mode;            /* IK_PAIRS_*                                         */
    int32_t num_link_pairs;
    const int32_t* link_pairs;        /* [num_link_pairs*2] (link a, link b)            */
    const int32_t* link_pair_offsets; /* [num_link_pairs+1] CSR into sphere_pairs        */
    int32_t num_sphere_pairs;
    const int32_t* sphere_pairs;      /* [num_sphere_pairs*2] grouped by link pair       */
    /* velocity limit */
    float dt;                         /* > 0                                              */
    const float* velocity_limits;     /* host [na]                                        */
    /* scene collision (margin above is the activation distance) */
    int32_t num_query_spheres;        /* robot spheres queried, one row each               */
    const int32_t* query_spheres;     /* host [num_query_spheres] sphere indices           */
    int32_t num_geoms;
    const float* geoms;               /* host [num_geoms * IK_GEOM_FLOATS], query order: a point
                                         keeps the first primitive of strictly least distance */
    int32_t num_scenes;
    int32_t penalty;                  /* IK_PENALTY_*                                       */
    int32_t residual_sqrt;            /* residual_mode "sqrt_abs": sqrt(penalty + eps)      */
    float residual_eps;
    const int32_t* d_scene_indices;   /* device [scene_rows]: scene of problem row b / max(1,
                                         batch / scene_rows); NULL = scene 0 for all        */
    int32_t scene_rows;
} IkTermDesc;

/* LMOptimizerConfig (opt/lm_optimizer.py:503-523) + OptimizerConfig
 * (opt/optimizer.py:160-167) + the per-problem stop rules. */
typedef struct IkLmParams {
    int32_t max_iter;
    float lambda_init;        /* lm_lambda                                   */
    float lambda_factor;
    float lambda_min;
    float lambda_max;
    float rho_min;
    float gain_ratio_epsilon;
    int32_t stop_rules;       /* IK_STOP_* bitmask                           */
    float cost_tol;
    float step_tol;
    float pose_pos_tol;
    float pose_rot_tol;
    int32_t check_interval;   /* early_stopping_interval of IK_STOP_ALL_COST (>= 1) */
} IkLmParams;

/* ---- lifecycle ----------------------------------------------------------- */
const char* ik_last_error(void);
int ik_version(void);
int ik_device_count(int* out);
int ik_set_device(int device);

int ik_robot_create(const IkRobotDesc* desc, IkRobot** out);
int ik_robot_destroy(IkRobot* robot);

/* A problem = robot + term list + tangent layout, with device buffers sized
 * for `capacity` problems (opt/optimizer.py:313-333: buffers are sized at the
 * first solve and smaller batches use a prefix).  `active_dof_mask` is a host
 * float array [tangent_dim] or NULL (opt/optimizer.py:203). */
int ik_problem_create(IkRobot* robot, int32_t capacity, int32_t floating_base, const IkTermDesc* terms,
                      int32_t num_terms, const float* active_dof_mask, IkProblem** out);
int ik_problem_destroy(IkProblem* problem);
int ik_problem_info(const IkProblem* problem, int32_t* tangent_dim, int32_t* residual_dim, int32_t* capacity);
/* Re-point a pose term's targets (set_target / resolve in the reference). */
int ik_problem_set_targets(IkProblem* problem, int32_t term_index, const float* d_targets, int32_t target_rows);

/* ---- solvers -------------------------------------------------------------- */
/* Whole LM solve, the plain form: one kernel launch per iteration over the
 * fixed batch, LMOptimizer.solve (opt/optimizer.py:216-240,
 * opt/lm_optimizer.py:834-1005).  d_q [batch*na] and d_base [batch*7] (NULL
 * without a floating base) are read as the start point and overwritten with
 * the solution.  Outputs: d_cost [batch] final cost 0.5*|r|^2, d_lambda [batch]
 * final damping, d_iters [batch] iterations run, d_status [batch] IK_ST_* bits
 * in bits 0-7 and the number of accepted steps in bits 8-31 (IK_ST_ACCEPTS).
 * Any output may be NULL. */
int ik_solve_plain(IkProblem* problem, int32_t batch, float* d_q, float* d_base, const IkLmParams* params,
                   float* d_cost, float* d_lambda, int32_t* d_iters, int32_t* d_status, void* stream);

/* The same solve with the LM loop of each problem inside one persistent
 * launch: groups of lanes pull problems from a device work queue and iterate
 * each to its stop rule (IK_STOP_ALL_COST is not available here). */
int ik_solve_persistent(IkProblem* problem, int32_t batch, float* d_q, float* d_base, const IkLmParams* params,
                        float* d_cost, float* d_lambda, int32_t* d_iters, int32_t* d_status, void* stream);

/* The persistent solve with no device allocation.  This entry point has no
 * counterpart in the reference.  It is for callers that may not allocate
 * device memory once running: a real-time control loop that forbids
 * allocation after start-up, or a plug-in whose host framework owns every
 * device buffer.  It takes the robot and term descriptors directly (as
 * ik_robot_create and ik_problem_create do), lowers them on the host every
 * call, and keeps the table blob and the work-queue counter in a static
 * device array of the library (IK_NOALLOC_MAX_TABLE_BYTES for the tables plus
 * 256 B); the counter is zeroed on `stream` before each launch.  Tables larger
 * than the limit are refused with IK_E_UNSUPPORTED.
 * - The first call on a device looks up that array's address (once per
 *   device, with the device current); make it before any stream capture.
 * - The array is shared by all calls on a device: calls that overlap in time
 *   race on it and must be serialised by the caller.
 * Arguments and outputs are those of ik_problem_create + ik_solve_persistent. */
#define IK_NOALLOC_MAX_TABLE_BYTES (224 * 1024)
int ik_solve_persistent_noalloc(const IkRobotDesc* robot, int32_t floating_base, const IkTermDesc* terms,
                                int32_t num_terms, const float* active_dof_mask, int32_t batch, float* d_q,
                                float* d_base, const IkLmParams* params, float* d_cost, float* d_lambda,
                                int32_t* d_iters, int32_t* d_status, void* stream);

/* Pick the lane-group width (8, 16 or 32 lanes per problem; 0 = automatic)
 * and the resident groups per SM of the persistent form (0 = automatic). */
int ik_problem_set_schedule(IkProblem* problem, int32_t group_lanes, int32_t blocks_per_sm);
int ik_problem_get_schedule(const IkProblem* problem, int32_t* group_lanes, int32_t* blocks_per_sm);

/* ---- serving: continuous batching of requests ------------------------------
 * The reference solves one batch per call (opt/optimizer.py:216-240); callers
 * that receive IK requests over time (helpers/ik/ik.py:98-304 per request)
 * wait for each batch.  A server keeps problem types resident and overlaps
 * requests on the GPU: each type runs a persistent kernel whose lane groups
 * take the next waiting problem as soon as theirs stops, so requests that
 * arrive while others run are admitted as slots free up.  Inputs and results
 * pass through mapped pinned host memory: submit, poll and fetch make no CUDA
 * call except to relaunch a type's kernel after it exited idle.
 * A server is used by one host thread. */
typedef struct IkServer IkServer;
/* budget_bytes bounds the memory of all types' slots (host-mapped inputs and
 * outputs plus device tables); idle_us = how long a kernel with no work
 * waits before it exits (0 = 200 us). */
int ik_server_create(int64_t budget_bytes, int32_t idle_us, IkServer** out);
/* Stops the kernels (after their running problems finish) and frees all. */
int ik_server_destroy(IkServer* server);
/* Register a problem type: robot + terms as for ik_problem_create, LM
 * parameters, and `slots` = problems of this type that may be admitted at
 * once.  The d_targets of pose terms are ignored: each request brings its
 * own targets.  Joint-reference, velocity-limit and base-reference terms must
 * have target_rows == 1 (one reference shared by every problem, read in place),
 * scene terms scene_rows <= 1; others fail with IK_E_UNSUPPORTED.  IK_E_OOM
 * when the slots do not fit the budget. */
int ik_server_add_type(IkServer* server, IkRobot* robot, int32_t floating_base, const IkTermDesc* terms,
                       int32_t num_terms, const float* active_dof_mask, const IkLmParams* params, int32_t slots,
                       int32_t* type_id);
/* Submit `batch` problems of a type from host arrays (copied before return):
 * h_q0 [batch, na], h_base0 [batch, 7] or NULL, h_targets = one array per
 * pose term in term order, [batch, num_frames, 7].  A request that does not
 * fit the free slots waits on the host and is admitted in arrival order as
 * fetched requests release theirs.  IK_E_CAPACITY if batch > slots. */
int ik_server_submit(IkServer* server, int32_t type, int32_t batch, const float* h_q0, const float* h_base0,
                     const float* const* h_targets, int64_t* request_id);
/* Report up to max_done newly finished requests (non-blocking). */
int ik_server_poll(IkServer* server, int64_t* done_ids, int32_t max_done, int32_t* num_done);
/* Copy a finished request's results (any pointer may be NULL) and release its
 * slots: q [batch, na], base [batch, 7], cost, iterations, status as in
 * ik_solve_persistent. */
int ik_server_fetch(IkServer* server, int64_t request_id, float* h_q, float* h_base, float* h_cost,
                    int32_t* h_iters, int32_t* h_status);
/* Free slots, waiting and running requests, and kernel launches of a type. */
int ik_server_info(IkServer* server, int32_t type, int32_t* free_slots, int32_t* pending, int32_t* inflight,
                   int64_t* launches);

/* ---- single-stage kernels (parity and the per-term reference API) ---------- */
/* Forward kinematics, Robot.forward_kinematics (robo/robot.py:131) with the
 * motion subspace (robo/robot_kernels.py:651-664) and the collision spheres
 * (robo/robot.py:428).  Outputs may be NULL: T_joint [B,nj,7], T_link [B,nl,7],
 * S_world [B,6,nj], spheres [B,ns,3], link_bounds [B,nl,3]. */
int ik_fk(IkRobot* robot, int32_t batch, const float* d_q, const float* d_base, float* d_T_joint, float* d_T_link,
          float* d_S_world, float* d_spheres, float* d_link_bounds, void* stream);

/* Link Jacobian, RobotState.get_link_jacobian (robo/robot_state.py:192,
 * robo/robot_kernels.py:668-737): out [B,6,tangent], frame 0 spatial, 1 body. */
int ik_link_jacobian(IkRobot* robot, int32_t batch, const float* d_q, const float* d_base, int32_t link,
                     int32_t body_frame, float* d_J, void* stream);

/* Weighted residuals and Jacobians of every term in the reference's row
 * layout (terms in order, LMOptimizer._default_offsets, lm_optimizer.py:594-602):
 * d_r [B,R], d_J [B,R,tangent] (either may be NULL). */
int ik_residual_jacobian(IkProblem* problem, int32_t batch, const float* d_q, const float* d_base, float* d_r,
                         float* d_J, void* stream);

/* Normal equations as the fused kernel forms them (lm_optimizer.py:145-189):
 * d_H [B,D,D], d_g [B,D], d_cost [B]. */
int ik_normal_equations(IkProblem* problem, int32_t batch, const float* d_q, const float* d_base, float* d_H,
                        float* d_g, float* d_cost, void* stream);

/* Damped FP64 Cholesky step (lm_optimizer.py:56-79): delta = -(H + lambda I)^-1 g,
 * pred = 0.5 * delta . (lambda delta - g).  d_H [B,D,D], d_g [B,D], d_lambda [B]
 * in; d_delta [B,D], d_pred [B] out; d_spd [B] (may be NULL) 1 if factorable. */
int ik_damped_solve(int32_t batch, int32_t dim, const float* d_H, const float* d_g, const float* d_lambda,
                    float* d_delta, float* d_pred, int32_t* d_spd, void* stream);

/* One LM iteration with the reference's buffers (LMOptimizer._step_body):
 * in/out d_q, d_base, d_lambda; out d_cost (the `costs` buffer after the step:
 * the proposal's cost if accepted, else the start point's), d_delta [B,D],
 * d_pred [B], d_cost_new [B] (the proposal's cost), d_accept [B]. */
int ik_step(IkProblem* problem, int32_t batch, float* d_q, float* d_base, float* d_lambda, const IkLmParams* params,
            float* d_cost, float* d_delta, float* d_pred, float* d_cost_new, int32_t* d_accept, void* stream);

/* Gain-ratio accept/reject and lambda update on scalars
 * (lm_accept_reject_cost_kernel, lm_optimizer.py:338-362), FP64 ratio. */
int ik_accept_reject(int32_t batch, float* d_cost, const float* d_cost_new, const float* d_pred, float* d_lambda,
                     int32_t* d_accept, const IkLmParams* params, void* stream);

/* IK accuracy metrics (helpers/ik/ik.py:60-82): per target position error [m]
 * and angle error [rad], success when every target is under both thresholds. */
int ik_metrics(IkRobot* robot, int32_t batch, const float* d_q, const float* d_base, int32_t num_targets,
               const int32_t* d_target_links, const float* d_targets, float pos_threshold, float rot_threshold,
               float* d_pos_err, float* d_rot_err, int32_t* d_success, void* stream);

/* Integrate a tangent step, RobotState.integrate (robo/robot_state.py:238-312):
 * q' = q + mask*delta, base' = base * exp(delta_base) (eps 1e-4). */
int ik_integrate(int32_t batch, int32_t num_actuated, int32_t floating_base, const float* d_q, const float* d_base,
                 const float* d_delta, const float* d_mask, float* d_q_out, float* d_base_out, void* stream);

/* Strided row copy: dst[r*dst_stride + c] = src[r*src_stride + c], c < width
 * (the row_offset writes of compute_weighted_residual, task.py:150-167, and
 * RobotState.get_T_world_link, robo/robot_state.py:186-190). */
int ik_copy_rows(int32_t rows, int32_t width, const float* d_src, int64_t src_stride, float* d_dst, int64_t dst_stride,
                 void* stream);

/* Row gather, RobotState.gather (robo/robot_state.py:478-520): d_dst[r*width + c] =
 * d_src[d_index[r]*width + c].  An index outside [0, src_rows) leaves its row
 * unwritten and adds one to *d_bad (when d_bad is not NULL). */
int ik_gather_rows(int32_t rows, int32_t width, const int32_t* d_index, int32_t src_rows, const float* d_src,
                   float* d_dst, int32_t* d_bad, void* stream);

/* Masked row copy, RobotState.accept (robo/robot_state.py:448-476,
 * robot_kernels.py:744-767): rows with d_mask[r] == 1 copy `width` floats. */
int ik_masked_copy_rows(int32_t rows, int32_t width, const int32_t* d_mask, const float* d_src, float* d_dst,
                        void* stream);

/* Cost of every row of a residual block, the reference's
 * aggregate_residuals_to_costs_kernel (opt/optimizer.py:21-33):
 * d_out[r] = (accumulate ? d_out[r] : 0) + sum_{i<width} d_x[r*stride + i]^2,
 * one FP32 running sum per row in column order.  Used by IKSolver.compute_costs
 * (helpers/ik/ik.py:373-385, opt/population_solver.py:555-574). */
int ik_row_sumsq(int32_t rows, int32_t width, const float* d_x, int64_t stride, float* d_out, int32_t accumulate,
                 void* stream);

/* Homogeneous transforms, 4x4 row-major floats, to and from poses
 * [x, y, z, qw, qx, qy, qz] with qw >= 0: the se3_from_matrix / se3_to_matrix
 * conversions of IKSolver.solve_torch (helpers/ik/ik.py:306-347). */
int ik_pose_from_matrix(int32_t n, const float* d_mats, float* d_poses, void* stream);
int ik_matrix_from_pose(int32_t n, const float* d_poses, float* d_mats, void* stream);

/* Keep the best `keep` of every instance's `num_candidates` candidates by cost
 * (ascending, equal costs in candidate order, NaN last), the select of
 * PopulationSolver (opt/population_solver.py:490-528).  Inputs are
 * instance-major [batch*num_candidates]; outputs [batch*keep] gather q
 * (num_actuated per row), base (7 per row; d_base may be NULL), cost and the
 * picked candidate index (any output but q may be NULL). */
int ik_select_best(int32_t batch, int32_t num_candidates, int32_t keep, const float* d_cost, const float* d_q,
                   const float* d_base, int32_t num_actuated, float* d_q_out, float* d_base_out, float* d_cost_out,
                   int32_t* d_index_out, void* stream);

/* Keep the previous solution where it scores no worse, IKSolver.solve
 * (helpers/ik/ik.py:43-56, 259-289): rows with d_prev_cost[b] <= d_cost[b] copy
 * d_prev_q (num_actuated per row) and, when both are given, d_prev_base (7 per
 * row) over d_q / d_base.  Costs are left as they are. */
int ik_keep_previous(int32_t batch, int32_t num_actuated, const float* d_prev_cost, const float* d_cost,
                     const float* d_prev_q, const float* d_prev_base, float* d_q, float* d_base, void* stream);

/* Clamp joints to [lo, hi], RobotState.clamp_q (robo/robot_state.py:314-333,
 * robot_kernels.py:593-609); entries whose d_mask is 0 are left (mask may be NULL). */
int ik_clamp_q(int32_t batch, int32_t num_actuated, float* d_q, const float* d_limits, const float* d_mask,
               void* stream);

/* ---- device memory, streams, events (the package imports no torch) ------ */
int ik_malloc(void** d_ptr, size_t bytes);
int ik_free(void* d_ptr);
int ik_malloc_host(void** h_ptr, size_t bytes); /* pinned */
int ik_free_host(void* h_ptr);
int ik_memcpy_htod(void* d_dst, const void* h_src, size_t bytes, void* stream);
int ik_memcpy_dtoh(void* h_dst, const void* d_src, size_t bytes, void* stream);
int ik_memcpy_dtod(void* d_dst, const void* d_src, size_t bytes, void* stream);
int ik_memset(void* d_ptr, int value, size_t bytes, void* stream);
int ik_stream_create(void** stream);
int ik_stream_destroy(void* stream);
int ik_stream_synchronize(void* stream);
int ik_device_synchronize(void);
int ik_event_create(void** event);
int ik_event_destroy(void* event);
int ik_event_record(void* event, void* stream);
int ik_event_elapsed_ms(void* start, void* stop, float* ms);
/* CUDA graphs of library calls: every call made on `stream` between begin and
 * end (by this host thread) is recorded instead of run; launch replays them.
 * The whole-solve "full" graph of OptimizerConfig.cuda_graph_mode
 * (opt/optimizer.py:160-174, opt/population_solver.py:84-85).  The stream must
 * be one from ik_stream_create; nothing may synchronise inside the capture.
 * Pointers and sizes are frozen into the graph: replay it on the same buffers. */
int ik_graph_begin(void* stream);
int ik_graph_end(void* stream, void** graph);
int ik_graph_launch(void* graph, void* stream);
int ik_graph_destroy(void* graph);
/* Count of this library's kernel launches since load (for launch accounting). */
int ik_launch_count(int64_t* out);
/* Measured CUDA-core FMA throughput (fp64 = 0: FP32, 1: FP64) in TFLOP/s on
 * the current device; independent FMA chains on every SM, best of 3 timed
 * launches.  The roofline denominator of the IK kernels.  Synchronises. */
int ik_measure_fma_peak(int32_t fp64, float* tflops);

#ifdef __cplusplus
}
#endif
#endif /* B200IK_H */
