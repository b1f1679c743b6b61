"""FrameTask ("log" residual, six rows per frame) on the GPU against the FP64 oracle."""

import numpy as np
import pytest

import oracle
from robokit_b200 import _native as N
from robokit_b200.helpers.ik import IKContext, IKSolver, IKSolverConfig
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
from robokit_b200.opt.population_solver import PopulationSolverConfig, Stage
from robokit_b200.terms.dense import FrameTask, PositionLimit, PositionTask, RotationTask

pytestmark = pytest.mark.gpu


def _targets(rng, B, nf):
    t = rng.normal(size=(B, nf, 7)).astype(np.float32)
    t[..., :3] *= 0.4
    t[..., 3:] /= np.linalg.norm(t[..., 3:], axis=-1, keepdims=True)
    return t


@pytest.mark.parametrize("floating", [False, True])
def test_frame_residual_and_jacobian_match_the_oracle(gpu, panda_spec, floating):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_spec)
    rng = np.random.default_rng(5)
    B = 64
    links = [panda_spec.link_names.index("panda_hand"), panda_spec.link_names.index("panda_link4")]
    tg = _targets(rng, B, 2)
    na = panda_spec.num_actuated_joints
    q = (panda_spec.midrange_q + rng.normal(0, 0.4, (B, na))).astype(np.float32)
    base = None
    if floating:
        base = rng.normal(size=(B, 7)).astype(np.float32)
        base[:, :3] *= 0.2
        base[:, 3:] /= np.linalg.norm(base[:, 3:], axis=1, keepdims=True)
    terms = [FrameTask(robot, links, tg, position_weight=[2.0, 1.0], orientation_weight=[0.5, 3.0]),
             PositionTask(robot, links[0], tg[:, :1], weight=1.5)]
    st = robot.state(q, base)
    vv = VarValues({VarKey.ROBOT: st})
    D = st.tangent_dim
    r = N.DeviceArray.zeros((B, 15))
    J = N.DeviceArray.zeros((B, 15, D))
    off = 0
    for t in terms:
        t.compute_weighted_residual(vv, out_residual=r, row_offset=off)
        t.compute_weighted_jacobian(vv, out_jacobian=J, row_offset=off)
        off += t.residual_dim
    from robokit_b200 import configs  # noqa: F401  (oracle lowering helpers live with the terms)

    class _V:
        spec, batch_size, has_floating_base = panda_spec, B, floating

    ro, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(panda_spec),
                                      oracle.Terms([t.host_desc(_V) for t in terms]), q, base)
    np.testing.assert_allclose(r.numpy(), ro, rtol=1e-4, atol=2e-5)
    np.testing.assert_allclose(J.numpy(), Jo, rtol=1e-4, atol=2e-4)


def test_lm_with_frame_task_reaches_fk_targets(gpu, panda_arm_spec):
    """Full-pose targets from FK: LM on a FrameTask converges like the FP64 oracle."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    hand = panda_arm_spec.link_names.index("panda_hand")
    B = 256
    qs = robot.sample_q(B, seed=9)
    T = robot.forward_kinematics(robot.state(qs)).get_T_world_link(hand).numpy().reshape(B, 1, 7)
    q0 = np.clip(qs + np.random.default_rng(1).normal(0, 0.3, qs.shape),
                 *panda_arm_spec.float32_actuated_limits().T).astype(np.float32)
    terms = [FrameTask(robot, hand, T, position_weight=10.0, orientation_weight=5.0), PositionLimit(robot, 10.0)]
    opt = LMOptimizer(terms, LMOptimizerConfig(max_iter=40, lm_lambda=1e-2, lambda_factor=2.0,
                                               early_stopping_interval=0, form="persistent"))
    st = robot.state(q0)
    opt.solve(VarValues({VarKey.ROBOT: st}))

    class _V:
        spec, batch_size, has_floating_base = panda_arm_spec, B, False

    rob = oracle.Robot.from_spec(panda_arm_spec)
    o = oracle.solve(rob, oracle.Terms([t.host_desc(_V) for t in terms]),
                     oracle.params(max_iter=40, lambda_init=1e-2, lambda_factor=2.0), q0, None, threads=8)
    pe_g, re_g, ok_g = oracle.metrics(rob, st.q.numpy(), None, [hand], T, 1e-3, 0.01)
    pe_o, re_o, ok_o = oracle.metrics(rob, o["q"], None, [hand], T, 1e-3, 0.01)
    assert ok_g.mean() > 0.8 and abs(ok_g.mean() - ok_o.mean()) <= 0.05, (ok_g.mean(), ok_o.mean())


def test_iksolver_with_a_frame_template(gpu, panda_arm_spec):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    hand = panda_arm_spec.link_names.index("panda_hand")
    cfg = IKSolverConfig(solver=PopulationSolverConfig(stages=[Stage(6, 32, LMOptimizerConfig(lm_lambda=10.0)),
                                                               Stage(10, 4, LMOptimizerConfig(lm_lambda=1.0)),
                                                               Stage(0, 1)], cuda_graph_mode="full"))
    cfg.add(FrameTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, position_weight=20.0,
                      orientation_weight=10.0)).add(PositionLimit(weight=50.0))
    ik = IKSolver(cfg, robot, "panda_hand")
    B = 64
    qs = robot.sample_q(B, seed=4)
    T = robot.forward_kinematics(robot.state(qs)).get_T_world_link(hand).numpy().reshape(B, 1, 7)
    assert ik.compute_metrics_numpy(ik.solve(T), T).success.mean() >= 0.9


def _compose(a, b):
    """vec7 a * b (translation a.t + R_a b.t, quaternion a.q b.q), numpy, per row."""
    def qmul(p, r):
        w1, x1, y1, z1 = np.moveaxis(p, -1, 0)
        w2, x2, y2, z2 = np.moveaxis(r, -1, 0)
        return np.stack([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                         w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2], -1)

    v = np.concatenate([np.zeros(b.shape[:-1] + (1,)), b[..., :3]], -1)
    conj = a[..., 3:] * [1, -1, -1, -1]
    rt = qmul(qmul(a[..., 3:], v), conj)[..., 1:]
    return np.concatenate([a[..., :3] + rt, qmul(a[..., 3:], b[..., 3:])], -1)


def test_log_residual_of_the_reference_frame_test(gpu, panda_spec):
    """tests/terms/test_frame_task.py:14-43 (its default-log half): targets offset from two links by a
    translation along x and a rotation about x give log rows [2 dx, 0, 0, 3 a, 0, 0] per frame."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_spec)
    frames = [robot.link_names.index("panda_hand"), robot.link_names.index("panda_link5")]
    q = np.tile(panda_spec.midrange_q, (6, 1)).astype(np.float32)
    state = robot.state(q=q)
    robot.forward_kinematics(state)
    reference = state.T_world_link.numpy()[:2][:, frames].astype(np.float64)
    delta = np.zeros((2, 2, 7))
    delta[:, :, 0] = np.array([0.004, 0.006])[:, None]
    angle = np.array([0.04, 0.06])[:, None]
    delta[:, :, 3], delta[:, :, 4] = np.cos(angle / 2), np.sin(angle / 2)
    target = _compose(reference, delta).astype(np.float32)  # rows broadcast over the 6 problems (3 each)
    task = FrameTask(robot, frames, target, position_weight=2.0, orientation_weight=3.0)
    residual = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state})).numpy().reshape(6, 2, 6)
    expected = np.repeat([[0.008, 0.12] * 2, [0.012, 0.18] * 2], 3, axis=0)
    np.testing.assert_allclose(residual[:, :, [0, 3]].reshape(6, 4), expected, atol=1e-6)
    np.testing.assert_allclose(residual[:, :, [1, 2, 4, 5]], 0.0, atol=1e-6)


def test_jacobian_fixed_base_of_the_reference_frame_test(gpu, panda_spec):
    """tests/terms/test_frame_task.py:45-72: position and rotation Jacobians at the link's own pose, against
    the exact FP64 oracle in place of Warp autodiff."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_spec)
    rng = np.random.RandomState(42)
    q = (rng.randn(panda_spec.num_actuated_joints) * 0.1 + panda_spec.midrange_q).astype(np.float32)
    state = robot.state(q=q)
    robot.forward_kinematics(state)
    hand = robot.link_names.index("panda_hand")
    target = state.get_T_world_link(hand).numpy().reshape(1, 1, 7)
    tasks = [PositionTask(robot, [hand], target, weight=5.0, fixed_target=True),
             RotationTask(robot, [hand], target, weight=2.0, fixed_target=True)]
    analytic = np.concatenate([t.compute_weighted_jacobian_analytic(VarValues({VarKey.ROBOT: state})).numpy()
                               for t in tasks], axis=1)

    class _V:
        spec, batch_size, has_floating_base = panda_spec, 1, False

    _, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(panda_spec),
                                     oracle.Terms([t.host_desc(_V) for t in tasks]), q[None])
    assert analytic.shape == Jo.shape
    assert np.allclose(analytic, Jo, atol=1e-4, rtol=1e-4)
