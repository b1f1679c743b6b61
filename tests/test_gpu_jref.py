"""Joint-reference terms (SmoothnessTask, ConfigurationTask: r = w (q - ref)) on the GPU against the FP64 oracle,
and the IKSolver's previous-state rule."""

import numpy as np
import pytest

import oracle
from robokit_b200 import _native as N
from robokit_b200.helpers.ik import IKContext, IKSolver, IKSolverConfig, presets
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
from robokit_b200.opt.population_solver import PopulationSolverConfig, Stage
from robokit_b200.terms.dense import (ConfigurationTask, PositionLimit, PositionTask, RotationTask, SmoothnessTask,
                                      VelocityLimitTask)

pytestmark = pytest.mark.gpu


def _view(spec, B, floating):
    class _V:
        pass

    v = _V()
    v.spec, v.batch_size, v.has_floating_base = spec, B, floating
    return v


@pytest.mark.parametrize("floating", [False, True])
def test_joint_reference_rows_match_the_oracle(gpu, panda_spec, floating):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_spec)
    rng = np.random.default_rng(11)
    B = 48
    na = panda_spec.num_actuated_joints
    hand = panda_spec.link_names.index("panda_hand")
    q = (panda_spec.midrange_q + rng.normal(0, 0.4, (B, na))).astype(np.float32)
    prev = (q + rng.normal(0, 0.2, (B, na))).astype(np.float32)
    rest = rng.normal(0, 0.5, (3, na)).astype(np.float32)  # 3 rows shared by B // 3 problems each
    base = None
    if floating:
        base = rng.normal(size=(B, 7)).astype(np.float32)
        base[:, :3] *= 0.2
        base[:, 3:] /= np.linalg.norm(base[:, 3:], axis=1, keepdims=True)
    tg = rng.normal(size=(B, 1, 7)).astype(np.float32)
    tg[..., 3:] /= np.linalg.norm(tg[..., 3:], axis=-1, keepdims=True)
    w = np.linspace(0.5, 2.0, na).astype(np.float32)
    terms = [PositionTask(robot, hand, tg, weight=3.0),
             SmoothnessTask(robot, prev_var=robot.state(prev), weight=w),
             ConfigurationTask(robot, rest_q=rest, weight=0.7, mask=(np.arange(na) % 2).astype(np.float32)),
             ConfigurationTask(robot, rest_q="midrange", weight=0.25),
             VelocityLimitTask(robot, dt=0.1, prev_state_var=robot.state(prev), weight=w[::-1].copy())]
    st = robot.state(q, base)
    vv = VarValues({VarKey.ROBOT: st})
    D = st.tangent_dim
    R = sum(t.residual_dim for t in terms)
    r = N.DeviceArray.zeros((B, R))
    J = N.DeviceArray.zeros((B, R, D))
    off = 0
    for t in terms:
        t.compute_weighted_residual(vv, out_residual=r, row_offset=off)
        t.compute_weighted_jacobian(vv, out_jacobian=J, row_offset=off)
        off += t.residual_dim
    ro, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(panda_spec),
                                      oracle.Terms([t.host_desc(_view(panda_spec, B, floating)) for t in terms]), q,
                                      base)
    np.testing.assert_allclose(r.numpy(), ro, rtol=1e-5, atol=2e-6)
    np.testing.assert_allclose(J.numpy(), Jo, rtol=1e-5, atol=2e-6)
    # the smoothness rows are exactly w (q - prev); some velocity rows are active, some not
    np.testing.assert_allclose(r.numpy()[:, 3:3 + na], w * (q - prev), rtol=1e-6, atol=1e-7)
    vel = r.numpy()[:, -na:]
    assert (vel > 0).any() and (vel == 0).any()


@pytest.mark.parametrize("form", ["persistent", "plain"])
def test_lm_with_joint_references_matches_the_oracle(gpu, panda_arm_spec, form):
    """LM with a pose, a limit, a smoothness and a rest term: per-problem costs agree with the FP64 oracle."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    hand = panda_arm_spec.link_names.index("panda_hand")
    B = 256
    qs = robot.sample_q(B, seed=21)
    T = robot.forward_kinematics(robot.state(qs)).get_T_world_link(hand).numpy().reshape(B, 1, 7)
    rng = np.random.default_rng(2)
    lo, hi = panda_arm_spec.float32_actuated_limits().T
    q0 = np.clip(qs + rng.normal(0, 0.3, qs.shape), lo, hi).astype(np.float32)
    prev = np.clip(qs + rng.normal(0, 0.1, qs.shape), lo, hi).astype(np.float32)
    terms = [PositionTask(robot, hand, T, weight=10.0), RotationTask(robot, hand, T, weight=5.0),
             PositionLimit(robot, 10.0), SmoothnessTask(robot, prev_var=robot.state(prev), weight=0.3),
             ConfigurationTask(robot, rest_q="midrange", weight=0.05),
             VelocityLimitTask(robot, dt=0.05, prev_state_var=robot.state(prev), velocity_limits=[2.0] * 7,
                               weight=1.0)]
    opt = LMOptimizer(terms, LMOptimizerConfig(max_iter=30, lm_lambda=1e-2, lambda_factor=2.0,
                                               early_stopping_interval=0, form=form))
    st = robot.state(q0)
    opt.solve(VarValues({VarKey.ROBOT: st}))
    rob = oracle.Robot.from_spec(panda_arm_spec)
    o = oracle.solve(rob, oracle.Terms([t.host_desc(_view(panda_arm_spec, B, False)) for t in terms]),
                     oracle.params(max_iter=30, lambda_init=1e-2, lambda_factor=2.0), q0, None, threads=8)
    # the regularised problems have one minimum near the start: both land on the same cost
    ot = oracle.Terms([t.host_desc(_view(panda_arm_spec, B, False)) for t in terms])
    cost_g = 0.5 * (oracle.residual_jacobian(rob, ot, st.q.numpy(), None)[0] ** 2).sum(axis=1)
    cost_o = 0.5 * (oracle.residual_jacobian(rob, ot, o["q"], None)[0] ** 2).sum(axis=1)
    close = np.abs(cost_g - cost_o) <= 1e-3 * np.maximum(1e-3, cost_o)
    assert close.mean() >= 0.9, close.mean()


def test_smoothness_without_a_previous_state_adds_zero_rows(gpu, panda_arm_spec):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    B, na = 8, panda_arm_spec.num_actuated_joints
    q = robot.sample_q(B, seed=3)
    t = SmoothnessTask(robot, weight=2.0)
    r = t.compute_weighted_residual(VarValues({VarKey.ROBOT: robot.state(q)}))
    assert r.shape == (B, na) and not np.any(r.numpy())
    t.set_prev_state(robot.state(q[:1] * 0.5))  # one row broadcast over the batch
    r = t.compute_weighted_residual(VarValues({VarKey.ROBOT: robot.state(q)}))
    np.testing.assert_allclose(r.numpy(), 2.0 * (q - 0.5 * q[:1]), rtol=1e-6, atol=1e-7)


def test_keep_previous_kernel(gpu):
    rng = np.random.default_rng(0)
    B, na = 1000, 7
    prev_cost = rng.random(B).astype(np.float32)
    cost = rng.random(B).astype(np.float32)
    cost[:10] = prev_cost[:10]  # ties keep the previous state
    cost[10] = np.nan
    prev_q, q = rng.random((B, na)).astype(np.float32), rng.random((B, na)).astype(np.float32)
    d = {k: N.DeviceArray.from_numpy(v) for k, v in dict(pc=prev_cost, c=cost, pq=prev_q, q=q).items()}
    N.check(N.lib().ik_keep_previous(B, na, d["pc"].ptr, d["c"].ptr, d["pq"].ptr, None, d["q"].ptr, None, None))
    keep = prev_cost <= cost
    np.testing.assert_array_equal(d["q"].numpy(), np.where(keep[:, None], prev_q, q))
    assert keep[:10].all() and not keep[10]
    assert N.lib().ik_keep_previous(B, na, d["pc"].ptr, d["c"].ptr, d["pq"].ptr, d["pq"].ptr, d["q"].ptr, None,
                                    None) != 0


def test_iksolver_keeps_a_previous_solution_that_scores_no_worse(gpu, panda_arm_spec):
    """solve(prev_state=...) keeps prev for a target where it costs no more than the new solution, else moves."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    hand = panda_arm_spec.link_names.index("panda_hand")
    B = 64
    qs = robot.sample_q(B, seed=8)
    T = robot.forward_kinematics(robot.state(qs)).get_T_world_link(hand).numpy().reshape(B, 1, 7)
    two = IKSolverConfig(solver=PopulationSolverConfig(stages=[Stage(6, 8, LMOptimizerConfig(lm_lambda=1.0)),
                                                               Stage(0, 2)]))
    two.add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
    with pytest.raises(ValueError):
        IKSolver(two, robot, "panda_hand").solve(T, prev_state=robot.state(qs))  # two solutions per target
    ik = IKSolver(presets.single_candidate, robot, "panda_hand")
    first = ik.solve(T, prev_state=robot.state(qs)).q.numpy().copy()
    # the previous state is an exact solution with no smoothness cost: kept unless the solve found a point
    # whose cost is strictly lower (only at the level of FP32 rounding of the pose residual)
    kept = (first == qs).all(axis=1)
    prev_cost, cost = ik._prev_cost.numpy(), ik.costs.numpy()
    assert kept.mean() >= 0.5, kept.mean()
    assert (prev_cost[kept] <= cost[kept]).all() and (prev_cost[~kept] > cost[~kept]).all()
    far = np.clip(qs + 0.6, *panda_arm_spec.float32_actuated_limits().T).astype(np.float32)
    moved = ik.solve(T, prev_state=robot.state(far)).q.numpy()
    assert np.abs(moved - far).max() > 1e-3
    # 30 iterations from the midrange with the pull toward a far previous state: most targets still reached
    assert ik.compute_metrics_numpy(robot.state(moved), T).success.mean() >= 0.7


def test_iksolver_smooth_preset_stays_near_the_previous_state(gpu, panda_arm_spec):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    hand = panda_arm_spec.link_names.index("panda_hand")
    B = 128
    qs = robot.sample_q(B, seed=13)
    T = robot.forward_kinematics(robot.state(qs)).get_T_world_link(hand).numpy().reshape(B, 1, 7)
    lo, hi = panda_arm_spec.float32_actuated_limits().T
    prev = np.clip(qs + np.random.default_rng(4).normal(0, 0.05, qs.shape), lo, hi).astype(np.float32)
    ik = IKSolver(presets.smooth, robot, "panda_hand")
    plain = IKSolver(presets.basic, robot, "panda_hand")
    a = ik.solve(T, prev_state=robot.state(prev)).q.numpy()
    b = plain.solve(T).q.numpy()
    assert ik.compute_metrics_numpy(robot.state(a), T).success.mean() >= 0.9
    # the smoothness pull keeps the redundant arm near prev more often than an unregularised solve
    assert np.median(np.abs(a - prev).max(axis=1)) <= np.median(np.abs(b - prev).max(axis=1))


def _unit_poses(rng, n, scale=0.2):
    p = rng.normal(size=(n, 7)).astype(np.float32)
    p[:, :3] *= scale
    p[:, 3] += 2.0
    p[:, 3:] /= np.linalg.norm(p[:, 3:], axis=1, keepdims=True)
    return p


def test_base_reference_rows_match_the_oracle(gpu, panda_spec):
    """Floating-base blocks of SmoothnessTask (previous base pose) and ConfigurationTask (rest base pose):
    residual and Jacobian rows against the oracle."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_spec)
    rng = np.random.default_rng(17)
    B = 48
    na = panda_spec.num_actuated_joints
    q = (panda_spec.midrange_q + rng.normal(0, 0.3, (B, na))).astype(np.float32)
    base = _unit_poses(rng, B)
    prev_base = _unit_poses(rng, B)
    rest_base = _unit_poses(rng, 2)  # 2 rows shared by B // 2 problems each
    terms = [SmoothnessTask(robot, prev_var=robot.state(q + 0.1, prev_base), weight=0.5,
                            base_weight=[1, 2, 3, 0.5, 0.25, 4]),
             ConfigurationTask(robot, rest_q="midrange", T_world_base_rest=rest_base, weight=0.2, base_weight=1.5),
             ConfigurationTask(robot, T_world_base_rest=rest_base[:1], include_joints=False)]
    st = robot.state(q, base)
    vv = VarValues({VarKey.ROBOT: st})
    D = st.tangent_dim
    R = sum(t.residual_dim for t in terms)
    assert R == (na + 6) * 2 + 6
    r = N.DeviceArray.zeros((B, R))
    J = N.DeviceArray.zeros((B, R, D))
    off = 0
    for t in terms:
        t.compute_weighted_residual(vv, out_residual=r, row_offset=off)
        t.compute_weighted_jacobian(vv, out_jacobian=J, row_offset=off)
        off += t.residual_dim
    ro, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(panda_spec),
                                      oracle.Terms([t.host_desc(_view(panda_spec, B, True)) for t in terms]), q, base)
    np.testing.assert_allclose(r.numpy(), ro, rtol=1e-4, atol=2e-5)
    np.testing.assert_allclose(J.numpy(), Jo, rtol=1e-3, atol=1e-4)


def test_lm_with_base_smoothness_matches_the_oracle(gpu, panda_arm_spec):
    """A floating-base arm reaching FK targets with base smoothness toward a previous base pose: per-problem
    costs agree with the oracle."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    hand = panda_arm_spec.link_names.index("panda_hand")
    B = 128
    rng = np.random.default_rng(5)
    qs = robot.sample_q(B, seed=41)
    base_s = _unit_poses(rng, B, 0.1)
    T = robot.forward_kinematics(robot.state(qs, base_s)).get_T_world_link(hand).numpy().reshape(B, 1, 7)
    lo, hi = panda_arm_spec.float32_actuated_limits().T
    q0 = np.clip(qs + rng.normal(0, 0.2, qs.shape), lo, hi).astype(np.float32)
    prev = robot.state(q0.copy(), base_s + np.r_[0.03, -0.02, 0.01, 0, 0, 0, 0].astype(np.float32))
    terms = [PositionTask(robot, hand, T, weight=10.0), RotationTask(robot, hand, T, weight=5.0),
             SmoothnessTask(robot, prev_var=prev, weight=0.2, base_weight=2.0)]
    opt = LMOptimizer(terms, LMOptimizerConfig(max_iter=30, lm_lambda=1e-2, lambda_factor=2.0,
                                               early_stopping_interval=0, form="persistent"))
    st = robot.state(q0, base_s.copy())
    opt.solve(VarValues({VarKey.ROBOT: st}))
    rob = oracle.Robot.from_spec(panda_arm_spec)
    ot = oracle.Terms([t.host_desc(_view(panda_arm_spec, B, True)) for t in terms])
    o = oracle.solve(rob, ot, oracle.params(max_iter=30, lambda_init=1e-2, lambda_factor=2.0), q0, base_s, threads=8)
    cost_g = 0.5 * (oracle.residual_jacobian(rob, ot, st.q.numpy(), st.T_world_base.numpy())[0] ** 2).sum(axis=1)
    cost_o = 0.5 * (oracle.residual_jacobian(rob, ot, o["q"], o["base"])[0] ** 2).sum(axis=1)
    close = np.abs(cost_g - cost_o) <= 1e-3 * np.maximum(1e-3, cost_o)
    assert close.mean() >= 0.85, close.mean()
