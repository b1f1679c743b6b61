/*
 * ik_oracle.h — FP64 CPU restatement of robokit's batched LM-IK path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the GPU kernels are
 * compared against (tests/, __graft_entry__.smoke()) and the timed CPU
 * baseline of bench.py; nothing in the shipped package links or calls it.
 *
 * Inputs use the reference's float32 tables (RobotSpecTensors,
 * robo/robot_spec_tensors.py:35-191); all arithmetic is double.
 */
#ifndef IK_ORACLE_H
#define IK_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrRobot {
    int32_t nj, nl, na, ns;
    const int32_t* joint_types;
    const float* joint_axes;        /* [nj*3] */
    const float* parent_transforms; /* [nj*7] */
    const int32_t* parent_joints;
    const int32_t* actuated_indices;
    const int32_t* mimic_indices;
    const float* mimic_multipliers;
    const float* mimic_offsets;
    const int32_t* link_parent_joints; /* [nl] */
    const float* actuated_limits;      /* [na*2] */
    const float* sphere_centers;       /* [ns*3] */
    const float* sphere_radii;
    const int32_t* sphere_links;
    const float* link_bound_centers;   /* [nl*3] */
    const float* link_bound_radii;
} OrRobot;

typedef struct OrTerm {
    int32_t kind; /* 1 position, 2 rotation, 3 joint limit, 4 self collision, 5 frame ("log"),
                     6 joint reference (smoothness / configuration, joints only),
                     7 velocity limit, 8 scene collision over primitives,
                     9 floating-base reference (targets: [target_rows, 7] poses, weights [6]) */
    int32_t num_frames;
    const int32_t* frame_links;
    const float* weights;
    const float* targets; /* host [target_rows, num_frames, 7]; kinds 6, 7: [target_rows, na] */
    int32_t target_rows;
    float margin;
    int32_t max_active_pairs;
    int32_t pair_mode; /* 0 slots, 1 all sphere pairs */
    int32_t num_link_pairs;
    const int32_t* link_pairs;
    const int32_t* link_pair_offsets;
    int32_t num_sphere_pairs;
    const int32_t* sphere_pairs;
    float dt;                     /* kind 7 */
    const float* velocity_limits; /* kind 7: [na] */
    /* kind 8 (margin above is the activation distance) */
    int32_t num_query_spheres;
    const int32_t* query_spheres;
    int32_t num_geoms;
    const float* geoms;           /* [num_geoms * 16]: type, scene, scale, 0, params[4], pose[7], 0 */
    int32_t num_scenes;
    int32_t penalty;              /* 0 smooth, 1 plain, 2 surface distance */
    int32_t residual_sqrt;
    float residual_eps;
    const int32_t* scene_indices; /* host [scene_rows] or NULL */
    int32_t scene_rows;
} OrTerm;

typedef struct OrParams {
    int32_t max_iter;
    double lambda_init, lambda_factor, lambda_min, lambda_max, rho_min, gain_ratio_epsilon;
    int32_t stop_rules; /* 1 all-cost, 2 step, 4 pose, 8 cost */
    double cost_tol, step_tol, pose_pos_tol, pose_rot_tol;
    int32_t check_interval;
} OrParams;

int or_residual_dim(const OrRobot* r, const OrTerm* terms, int32_t nterms);

int or_fk(const OrRobot* r, int32_t B, const float* q, const float* base, double* T_joint, double* T_link,
          double* S_world, double* spheres, double* bounds);
int or_link_jacobian(const OrRobot* r, int32_t B, const float* q, const float* base, int32_t link, int32_t body,
                     double* J);
int or_residual_jacobian(const OrRobot* r, const OrTerm* terms, int32_t nterms, int32_t floating, int32_t B,
                         const float* q, const float* base, double* res, double* J);
int or_normal_equations(const OrRobot* r, const OrTerm* terms, int32_t nterms, int32_t floating, const float* mask,
                        int32_t B, const float* q, const float* base, double* H, double* g, double* cost);
int or_damped_solve(int32_t B, int32_t D, const double* H, const double* g, const double* lambda, double* delta,
                    double* pred, int32_t* spd);
int or_solve(const OrRobot* r, const OrTerm* terms, int32_t nterms, int32_t floating, const float* mask,
             const OrParams* p, int32_t B, const float* q0, const float* base0, double* q, double* base,
             double* cost, double* lambda, int32_t* iters, int32_t* status, int32_t nthreads);
int or_accept_reject(int32_t B, double* cost, const double* cost_new, const double* pred, double* lambda,
                     int32_t* accept, const OrParams* p);
int or_metrics(const OrRobot* r, int32_t B, const double* q, const double* base, int32_t nt, const int32_t* links,
               const float* targets, double pos_th, double rot_th, double* perr, double* rerr, int32_t* success);

#ifdef __cplusplus
}
#endif
#endif
