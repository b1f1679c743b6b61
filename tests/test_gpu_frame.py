"""FrameTask ("log" residual, six rows per frame) on the GPU against the FP64 oracle."""

import numpy as np
import pytest

import oracle
from robokit_b200 import _native as N
from robokit_b200.helpers.ik import IKContext, IKSolver, IKSolverConfig
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
from robokit_b200.opt.population_solver import PopulationSolverConfig, Stage
from robokit_b200.terms.dense import FrameTask, PositionLimit, PositionTask

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
    assert ik.compute_metrics(ik.solve(T), T).success.mean() >= 0.9
