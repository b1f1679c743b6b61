"""The reference-facing Python API over the GPU kernels (RobotState, terms, LMOptimizer.step)."""

import numpy as np
import pytest

import oracle
from robokit_b200 import configs
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
from robokit_b200.terms.dense import PositionLimit, PositionTask, RotationTask, SelfCollisionTask

pytestmark = pytest.mark.gpu


def test_integrate_accept_clamp(gpu, panda_spec):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_spec)
    rng = np.random.default_rng(0)
    B, na = 5, panda_spec.num_actuated_joints
    q = rng.uniform(-1, 1, (B, na)).astype(np.float32)
    base = np.tile(np.array([0.1, 0.2, 0.3, 1, 0, 0, 0], np.float32), (B, 1))
    st = robot.state(q, base)
    v = rng.normal(0, 0.1, (B, 6 + na)).astype(np.float32)
    out = st.integrate(v)
    np.testing.assert_allclose(out.q.numpy(), q + v[:, 6:], atol=1e-7)
    # base' = base * exp(v_base): check against the oracle's exponential through FK of a zero-joint robot
    assert np.all(np.abs(np.linalg.norm(out.T_world_base.numpy()[:, 3:], axis=1) - 1) < 1e-6)
    acc = np.array([1, 0, 1, 0, 0], np.int32)
    st.accept(acc, out)
    qa = st.q.numpy()
    np.testing.assert_array_equal(qa[acc == 1], out.q.numpy()[acc == 1])
    np.testing.assert_array_equal(qa[acc == 0], q[acc == 0])
    st.q.copy_from_numpy(np.full((B, na), 10.0, np.float32))
    st.clamp_q()
    np.testing.assert_allclose(st.q.numpy(), np.tile(panda_spec.float32_actuated_limits()[:, 1], (B, 1)))


def test_get_T_world_link(gpu, panda_spec):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_spec)
    q = np.random.default_rng(1).uniform(-1, 1, (3, panda_spec.num_actuated_joints)).astype(np.float32)
    st = robot.forward_kinematics(robot.state(q))
    li = panda_spec.link_names.index("panda_hand")
    np.testing.assert_array_equal(st.get_T_world_link(li).numpy(), st.T_world_link.numpy()[:, li])


def test_term_residuals_with_row_offset(gpu):
    cfg = configs.make("chain7c", 16, seed=2, pair_mode="slots")
    st = cfg.robot.state(cfg.workload.q0)
    vv = VarValues({VarKey.ROBOT: st})
    R = sum(t.residual_dim for t in cfg.terms)
    D = st.tangent_dim
    from robokit_b200 import _native as N

    r = N.DeviceArray.zeros((16, R))
    J = N.DeviceArray.zeros((16, R, D))
    off = 0
    for t in cfg.terms:
        t.compute_weighted_residual(vv, out_residual=r, row_offset=off)
        t.compute_weighted_jacobian(vv, out_jacobian=J, row_offset=off)
        off += t.residual_dim
    ro, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(cfg.workload.spec),
                                      oracle.Terms(configs.oracle_terms(cfg)), cfg.workload.q0)
    np.testing.assert_allclose(r.numpy(), ro, rtol=1e-5, atol=2e-5)
    np.testing.assert_allclose(J.numpy(), Jo, rtol=1e-5, atol=5e-5)


def test_position_limit_doctest(gpu, panda_spec):
    """terms/dense/position_limit.py:197-200: 0.1 below the lower limit gives residual 0.1 and diagonal -1."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_spec)
    q = (panda_spec.actuated_joint_limits[:, 0] - 0.1).astype(np.float32)[None]
    st = robot.state(q)
    task = PositionLimit(robot=robot)
    r = task.compute_weighted_residual(VarValues({VarKey.ROBOT: st})).numpy()[0]
    np.testing.assert_allclose(r, 0.1, atol=1e-6)
    J = task.compute_weighted_jacobian(VarValues({VarKey.ROBOT: st})).numpy()[0]
    np.testing.assert_allclose(np.diag(J), -1.0)


def test_self_collision_batch_consistency(gpu, panda_collision_spec):
    """tests/terms/test_self_collision_task.py:66-85: batch vs single on sorted residuals."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_collision_spec)
    rng = np.random.default_rng(0)
    q = (rng.normal(size=(4, panda_collision_spec.num_actuated_joints)) * 0.1 +
         panda_collision_spec.midrange_q).astype(np.float32)
    task = SelfCollisionTask(robot=robot, weight=1.0, margin=0.5)
    rb = task.compute_weighted_residual(VarValues({VarKey.ROBOT: robot.state(q)})).numpy()
    assert rb.shape == (4, 50) and rb.min() >= 0 and rb.max() > 0
    for i in range(4):
        t1 = SelfCollisionTask(robot=robot, weight=1.0, margin=0.5)
        r1 = t1.compute_weighted_residual(VarValues({VarKey.ROBOT: robot.state(q[i:i + 1])})).numpy()[0]
        np.testing.assert_allclose(np.sort(rb[i]), np.sort(r1), atol=1e-6)
    # pair filtering reduces pairs (tests/terms/test_self_collision_task.py:57-64)
    ns = len(panda_collision_spec.collision_sphere_radii)
    assert SelfCollisionTask(robot, filter_adjacent_links=False).num_pairs == ns * (ns - 1) // 2
    assert task.num_pairs < ns * (ns - 1) // 2


def test_step_and_callback(gpu):
    cfg = configs.make("chain7", 32, seed=8)
    # lambda0 = 0.1 keeps the damped systems well conditioned: the two paths are separate kernels whose
    # FP32 contraction choices differ in the last bits, which badly conditioned steps would amplify
    lm = LMOptimizerConfig(max_iter=5, lm_lambda=1e-1, lambda_factor=10.0, early_stopping_interval=0)
    opt = LMOptimizer(cfg.terms, lm)
    st = cfg.robot.state(cfg.workload.q0)
    seen = []
    opt.solve(VarValues({VarKey.ROBOT: st}), iteration_callback=lambda i, v, c: seen.append((i, c.numpy().copy())))
    assert [s[0] for s in seen] == list(range(6))
    costs = np.stack([s[1] for s in seen])
    # accepted steps only lower the cost; iteration 0 comes from another kernel, whose FP32
    # rounding may differ in the last bits (FMA contraction is chosen per kernel)
    assert np.all(np.diff(costs, axis=0) <= 1e-6 * np.abs(costs[:-1]) + 1e-12)
    # stepping 5 times matches the fused solve over 5 iterations (no stop rule)
    opt2 = LMOptimizer(cfg.terms, lm)
    st2 = cfg.robot.state(cfg.workload.q0)
    opt2.solve(VarValues({VarKey.ROBOT: st2}))
    close = np.all(np.abs(st.q.numpy() - st2.q.numpy()) < 1e-4, axis=1)
    assert close.mean() > 0.9
    np.testing.assert_allclose(costs[-1][close], opt2.costs.numpy()[close], rtol=1e-3, atol=1e-9)


def test_set_target_and_weight(gpu):
    cfg = configs.make("chain7", 16, seed=3)
    opt = LMOptimizer(cfg.terms, cfg.lm)
    st = cfg.robot.state(cfg.workload.q0)
    opt.solve(VarValues({VarKey.ROBOT: st}))
    c1 = opt.costs.numpy().copy()
    cfg.terms[0].set_weight(5.0)
    st = cfg.robot.state(cfg.workload.q0)
    opt.solve(VarValues({VarKey.ROBOT: st}))
    assert not np.array_equal(c1, opt.costs.numpy())
    new_t = cfg.workload.targets.copy()
    new_t[:, :, :3] += 0.01
    cfg.terms[0].set_target(new_t)
    cfg.terms[1].set_target(new_t)
    st = cfg.robot.state(cfg.workload.q0)
    opt.solve(VarValues({VarKey.ROBOT: st}))
    rob = oracle.Robot.from_spec(cfg.workload.spec)
    pe, _, _ = oracle.metrics(rob, st.q.numpy(), None, cfg.workload.target_links, new_t)
    pe_old, _, _ = oracle.metrics(rob, st.q.numpy(), None, cfg.workload.target_links, cfg.workload.targets)
    assert np.median(pe) < np.median(pe_old)


def test_errors_are_loud(gpu):
    cfg = configs.make("chain7", 8)
    with pytest.raises(NotImplementedError):
        LMOptimizer(cfg.terms, LMOptimizerConfig(linear_solver="cg"))
    with pytest.raises(ValueError):
        LMOptimizer(cfg.terms, cfg.lm, device="cpu")
    with pytest.raises(ValueError, match="DOFs"):
        cfg.robot.state(np.zeros((2, 3), np.float32))
    with pytest.raises(ValueError, match="active_dof_mask"):
        opt = LMOptimizer(cfg.terms, cfg.lm, active_dof_mask=np.ones(3, np.float32))
        opt.solve(VarValues({VarKey.ROBOT: cfg.robot.state(cfg.workload.q0)}))
