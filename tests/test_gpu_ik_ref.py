"""The reference's IKSolver tests (tests/helpers/ik/test_ik.py) on the Panda, through this library's API.

Each test names the reference test it follows.  Robots whose descriptions are not here (G1, Fetch, YuMi,
the Ability hand) are replaced by the Panda with the same configuration; the Fetch's mobile base becomes the
Panda with a floating base.
"""

import numpy as np
import pytest

import oracle
from robokit_b200 import _native as N
from robokit_b200.helpers.ik import IKContext, IKSolver, IKSolverConfig, presets
from robokit_b200.helpers.ik.ik import IKMetrics
from robokit_b200.opt import LMOptimizerConfig
from robokit_b200.opt.population_solver import PopulationSolverConfig, Stage
from robokit_b200.opt.sampler import RobertsSamplerConfig
from robokit_b200.robo.robot_spec import matrix_to_quaternion, quaternion_to_matrix
from robokit_b200.terms.dense import (ConfigurationTask, PositionLimit, PositionTask, RotationTask, SmoothnessTask,
                                      VelocityLimitTask)

pytestmark = pytest.mark.gpu

HAND = "panda_hand"


def _robot(spec):
    from robokit_b200.robo.robot import Robot

    return Robot(spec)


def basic_config():
    return (IKSolverConfig()
            .add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
            .add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
            .add(PositionLimit(weight=50.0)))


def advanced_config():
    return (basic_config()
            .add(ConfigurationTask(rest_q=IKContext.REST_Q, T_world_base_rest=IKContext.REST_BASE, weight=0.1,
                                   base_weight=0.0))
            .add(SmoothnessTask(prev_var=IKContext.PREVIOUS_STATE, weight=0.3))
            .add(VelocityLimitTask(prev_state_var=IKContext.PREVIOUS_STATE, dt=0.1, weight=1.0)))


def mobile_config():
    return (IKSolverConfig(enable_T_world_base=True, sampler=RobertsSamplerConfig(keep_first=True, seed=42, scale=0.1))
            .add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
            .add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=5.0))
            .add(PositionLimit(weight=50.0))
            .add(ConfigurationTask(rest_q=IKContext.REST_Q, T_world_base_rest=IKContext.REST_BASE, weight=0.01,
                                   base_weight=[0.01, 0.01, 100.0, 100.0, 100.0, 0.01])))


def _initial_targets(robot, links, B):
    """FK of the zero configuration at every target link, tiled over the batch (test_ik.py:138-149)."""
    st = robot.forward_kinematics(robot.state(robot.spec.zero_q[None].astype(np.float32)))
    idx = [robot.link_names.index(x) for x in links]
    poses = np.stack([st.get_T_world_link(i).numpy()[0] for i in idx])
    return np.ascontiguousarray(np.tile(poses[None], (B, 1, 1)), np.float32)


def _errors(robot, state, links, T):
    st = robot.forward_kinematics(state)
    out = []
    for i, name in enumerate(links):
        got = st.get_T_world_link(robot.link_names.index(name)).numpy()
        tgt = T[:, i] if T.ndim == 3 else T
        pos = np.linalg.norm(got[:, :3] - tgt[:, :3], axis=1)
        q1 = got[:, 3:] / np.linalg.norm(got[:, 3:], axis=1, keepdims=True)
        q2 = tgt[:, 3:] / np.linalg.norm(tgt[:, 3:], axis=1, keepdims=True)
        rot = 2 * np.arccos(np.clip(np.abs(np.sum(q1 * q2, axis=1)), -1, 1))
        out.append((pos, rot))
    return out


def _within_limits(robot, q):
    lim = robot.spec.actuated_joint_limits
    return np.all(q >= lim[:, 0] - 1e-3) and np.all(q <= lim[:, 1] + 1e-3)


@pytest.mark.parametrize("name,B,builder", [("basic", 1, basic_config), ("advanced", 1, advanced_config),
                                             ("batch", 10, basic_config), ("mobile", 1, mobile_config)])
def test_ik_examples(gpu, panda_arm_spec, name, B, builder):
    """TestIKExamples.test_ik_initialization / test_ik_solve (test_ik.py:223-255)."""
    robot = _robot(panda_arm_spec)
    ik = IKSolver(builder(), robot=robot, target_links=[HAND])
    assert ik.num_joints == robot.num_actuated_joints and ik.num_targets == 1
    T = _initial_targets(robot, [HAND], B)
    state = ik.solve(T)
    q = state.q.numpy()
    assert q.shape == (B, robot.num_actuated_joints) and _within_limits(robot, q)
    (pos, rot), = _errors(robot, state, [HAND], T)
    assert np.all(pos < 0.01) and np.all(rot < 0.1)


def test_metrics_match_numpy_and_reuse_buffers(gpu, panda_arm_spec):
    """TestIKMetrics.test_matches_numpy_and_reuses_buffers (test_ik.py:258-295)."""
    robot = _robot(panda_arm_spec)
    ik = IKSolver(basic_config(), robot=robot, target_links=[HAND])
    T = _initial_targets(robot, [HAND], 4)
    Td = N.DeviceArray.from_numpy(T)
    metrics = ik.compute_metrics(ik.solve(Td), Td)
    assert isinstance(metrics, IKMetrics) and metrics.position_error_m.shape == (4, 1)
    assert np.all(metrics.success.numpy()) and np.all(metrics.position_error_m.numpy() < 0.005)
    shifted = T.copy()
    shifted[:, :, 0] += 0.05  # a 5 cm offset reads as 5 cm of error; out= writes in place
    same = ik.compute_metrics(ik.solve(Td), N.DeviceArray.from_numpy(shifted), out=metrics)
    assert same.success is metrics.success
    np.testing.assert_allclose(metrics.position_error_m.numpy()[:, 0], 0.05, atol=2e-3, rtol=0)
    assert not np.any(metrics.success.numpy())
    state = ik.solve(Td)
    host = ik.compute_metrics_numpy(state, shifted)
    np.testing.assert_allclose(host.position_error_m,
                               ik.compute_metrics(state, N.DeviceArray.from_numpy(shifted)).position_error_m.numpy())
    assert host.success.dtype == bool and not np.any(host.success)
    assert np.all(ik.compute_metrics_numpy(state, T).success)


def test_score_terms_rank_the_candidates(gpu, panda_arm_spec):
    """TestIKScoreTask.test_ik_score_task (test_ik.py:298-346), the Fetch replaced by a floating Panda: a solve
    with score terms runs with a previous state, and its reported costs are the score terms' 0.5 |r|^2 at the
    returned solutions."""
    robot = _robot(panda_arm_spec)
    config = (IKSolverConfig(enable_T_world_base=True,
                             solver=PopulationSolverConfig(stages=[Stage(4, 8, LMOptimizerConfig(lm_lambda=10.0)),
                                                                   Stage(6, 2, LMOptimizerConfig(lm_lambda=1.0)),
                                                                   Stage(0, 1)], cuda_graph_mode="none"))
              .add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
              .add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
              .add(PositionLimit(weight=50.0))
              .add(ConfigurationTask(rest_q=IKContext.REST_Q, T_world_base_rest=IKContext.REST_BASE, weight=0.0,
                                     base_weight=[0.0, 0.0, 100.0, 100.0, 100.0, 0.0]))
              .add(SmoothnessTask(prev_var=IKContext.PREVIOUS_STATE, weight=0.2, base_weight=0.2)))
    config.add_score(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=1.0),
                     name="score_position")
    config.add_score(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=0.5),
                     name="score_rotation")
    assert config.task("score_position").weight == 1.0
    ik = IKSolver(config, robot=robot, target_links=HAND)
    B = 16
    q = robot.sample_q(B, seed=5)
    T = robot.forward_kinematics(robot.state(q)).get_T_world_link(robot.link_names.index(HAND)).numpy()
    T = T.reshape(B, 1, 7)
    prev = robot.state(np.tile(robot.spec.zero_q.astype(np.float32), (B, 1)),
                       np.tile(np.array([0, 0, 0, 1, 0, 0, 0], np.float32), (B, 1)))
    sol = ik.solve(T, prev_state=prev)
    cost = ik.costs.numpy().copy()
    qs, bs = sol.q.numpy().copy(), sol.T_world_base.numpy().copy()
    st = robot.state(qs, bs)
    from robokit_b200.opt import VarKey, VarValues

    vv = VarValues({VarKey.ROBOT: st})
    hand = [robot.link_names.index(HAND)]
    r = np.concatenate([PositionTask(robot, hand, T.reshape(B, 7), weight=1.0).compute_weighted_residual(vv).numpy(),
                        RotationTask(robot, hand, T.reshape(B, 7), weight=0.5).compute_weighted_residual(vv).numpy()],
                       axis=1)
    solved = ~np.all(qs == robot.spec.zero_q.astype(np.float32), axis=1)  # rows that kept prev_state report
    assert solved.sum() >= B - 2  # the solve's cost, not prev_state's (helpers/ik/ik.py:277-289)
    np.testing.assert_allclose(cost[solved], 0.5 * np.sum(r.astype(np.float64) ** 2, axis=1)[solved], rtol=2e-4,
                               atol=1e-9)


def test_score_terms_equal_to_the_objective_change_nothing(gpu, panda_arm_spec):
    """Ranking by score terms identical to the optimization terms keeps the same candidates as ranking by the
    optimizer's cost (opt/population_solver.py:415-434)."""
    robot = _robot(panda_arm_spec)
    B = 64
    q = robot.sample_q(B, seed=11)
    T = robot.forward_kinematics(robot.state(q)).get_T_world_link(robot.link_names.index(HAND)).numpy().reshape(B, 1, 7)
    plain = IKSolver(basic_config(), robot=robot, target_links=HAND)
    scored_cfg = basic_config()
    for t in basic_config().terms:
        scored_cfg.add_score(t)
    scored = IKSolver(scored_cfg, robot=robot, target_links=HAND)
    a = plain.solve(T).q.numpy().copy()
    b = scored.solve(T).q.numpy().copy()
    np.testing.assert_allclose(a, b, atol=1e-6)
    np.testing.assert_allclose(plain.costs.numpy(), scored.costs.numpy(), rtol=1e-5, atol=1e-10)


def test_rank_final_sorts_the_solutions(gpu, panda_arm_spec):
    """rank_final returns every instance's final solutions best first (opt/population_solver.py:385-404)."""
    robot = _robot(panda_arm_spec)
    B, K = 32, 4

    def cfg(rank):
        c = basic_config()
        c.solver = PopulationSolverConfig(stages=[Stage(6, 16, LMOptimizerConfig(lm_lambda=10.0)),
                                                  Stage(4, K, LMOptimizerConfig(lm_lambda=1.0))],
                                          cuda_graph_mode="full", rank_final=rank)
        return c

    q = robot.sample_q(B, seed=13)
    T = robot.forward_kinematics(robot.state(q)).get_T_world_link(robot.link_names.index(HAND)).numpy().reshape(B, 1, 7)
    plain, ranked = IKSolver(cfg(False), robot, HAND), IKSolver(cfg(True), robot, HAND)
    qa, ca = plain.solve(T).q.numpy().copy(), plain.costs.numpy().copy()
    qb, cb = ranked.solve(T).q.numpy().copy(), ranked.costs.numpy().copy()
    assert qb.shape == (B * K, robot.num_actuated_joints)
    ca, cb = ca.reshape(B, K), cb.reshape(B, K)
    assert np.all(np.diff(cb, axis=1) >= 0)
    order = np.argsort(ca, axis=1, kind="stable")
    np.testing.assert_array_equal(np.take_along_axis(ca, order, axis=1), cb)
    rows = (np.arange(B)[:, None] * K + order).reshape(-1)
    np.testing.assert_array_equal(qa[rows], qb)
    again = ranked.solve(T).q.numpy()  # the captured graph replays the ranking
    np.testing.assert_array_equal(again, qb)


def test_multi_step_solve(gpu, panda_arm_spec):
    """TestIKMultiStepSolve.test_ik_multi_step_solve (test_ik.py:349-378): a solve, then a 1 cm move solved from
    the previous solution."""
    robot = _robot(panda_arm_spec)
    ik = IKSolver(advanced_config(), robot=robot, target_links=[HAND])
    prev = robot.state(robot.spec.zero_q[None].astype(np.float32))
    T = _initial_targets(robot, [HAND], 1)
    state = ik.solve(T, prev_state=prev)
    (pos, rot), = _errors(robot, state, [HAND], T)
    assert pos[0] < 0.01 and rot[0] < 0.1
    moved = T.copy()
    moved[:, :, 0] += 0.01
    state2 = ik.solve(moved, prev_state=robot.state(state.q.numpy().copy()))
    (pos, rot), = _errors(robot, state2, [HAND], moved)
    assert pos[0] < 0.02 and rot[0] < 0.2


def test_solve_torch_matrix_interface(gpu, panda_arm_spec):
    """TestIKInterfaces.test_ik_batch_torch_matrix_interface (test_ik.py:382-410)."""
    import torch

    robot = _robot(panda_arm_spec)
    ik = IKSolver(presets.basic, robot=robot, target_links=HAND)
    B = 10
    wxyz = np.array([0.0, 0.707, 0.0, 0.707], np.float32)
    wxyz /= np.linalg.norm(wxyz)
    M = np.eye(4, dtype=np.float32)
    M[:3, :3] = quaternion_to_matrix(wxyz)
    M[:3, 3] = [0.5, 0.0, 0.5]
    result = ik.solve_torch(torch.tensor(np.tile(M, (B, 1, 1)), device="cuda"))
    q = result.q.cpu().numpy()
    assert result.T_world_base is None
    assert q.shape == (B, robot.num_actuated_joints) and _within_limits(robot, q)
    T = np.concatenate([M[:3, 3], wxyz])[None].repeat(B, 0)
    (pos, _), = _errors(robot, robot.state(q), [HAND], T)
    assert np.all(pos < 0.01)


def test_solve_torch_floating_base_returns_matrices(gpu, panda_arm_spec):
    """solve_torch with a floating base returns the base as 4x4 matrices of the solved base poses."""
    import torch

    robot = _robot(panda_arm_spec)
    ik = IKSolver(mobile_config(), robot=robot, target_links=HAND)
    T = _initial_targets(robot, [HAND], 3)
    T[:, 0, 0] += np.array([0.3, 0.6, 0.9], np.float32)
    mats = np.zeros((3, 4, 4), np.float32)
    for i in range(3):
        mats[i, :3, :3] = quaternion_to_matrix(T[i, 0, 3:])
        mats[i, :3, 3] = T[i, 0, :3]
        mats[i, 3, 3] = 1
    res = ik.solve_torch(torch.tensor(mats, device="cuda"))
    assert res.T_world_base.shape == (3, 4, 4)
    Tb = res.T_world_base.cpu().numpy()
    base = np.concatenate([Tb[:, :3, 3], np.stack([matrix_to_quaternion(m[:3, :3]) for m in Tb])], axis=1)
    (pos, _), = _errors(robot, robot.state(res.q.cpu().numpy(), base.astype(np.float32)), [HAND], T)
    assert np.all(pos < 0.01)
    np.testing.assert_allclose(Tb[:, 3], np.tile([0, 0, 0, 1], (3, 1)), atol=0)


def test_pose_matrix_conversions_match_numpy(gpu):
    """The device pose <-> matrix conversions against the host ones, including the branches of Shepperd's method
    (rotations near pi about each axis)."""
    rng = np.random.default_rng(0)
    n = 512
    q = rng.normal(size=(n, 4))
    q[:8] = [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1], [0.01, 1, 0.02, 0], [0.01, 0, 1, 0.03],
             [0.02, 0.01, 0, 1], [0.5, 0.5, 0.5, 0.5]]
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q[q[:, 0] < 0] *= -1
    t = rng.normal(size=(n, 3))
    M = np.zeros((n, 4, 4))
    for i in range(n):
        M[i, :3, :3] = quaternion_to_matrix(q[i])
    M[:, :3, 3], M[:, 3, 3] = t, 1
    dm = N.DeviceArray.from_numpy(M.astype(np.float32))
    dp = N.DeviceArray.empty((n, 7))
    N.check(N.lib().ik_pose_from_matrix(n, dm.ptr, dp.ptr, None))
    p = dp.numpy()
    np.testing.assert_allclose(p[:, :3], t, atol=1e-6)
    np.testing.assert_allclose(p[:, 3:], q, atol=2e-6)
    back = N.DeviceArray.empty((n, 4, 4))
    N.check(N.lib().ik_matrix_from_pose(n, dp.ptr, back.ptr, None))
    np.testing.assert_allclose(back.numpy(), M, atol=2e-6)


def test_multiple_final_solutions(gpu, panda_arm_spec):
    """TestIKInterfaces.test_ik_returns_multiple_final_solutions (test_ik.py:412-439)."""
    robot = _robot(panda_arm_spec)
    config = basic_config()
    config.solver = PopulationSolverConfig(stages=[Stage(2, 8, LMOptimizerConfig(lm_lambda=10.0)),
                                                   Stage(0, 2, LMOptimizerConfig(lm_lambda=1.0))],
                                           cuda_graph_mode="none")
    ik = IKSolver(config, robot=robot, target_links=HAND)
    T = _initial_targets(robot, [HAND], 2)
    state = ik.solve(T)
    assert ik.num_solutions == 2 and state.q.shape == (4, robot.num_actuated_joints)
    with pytest.raises(ValueError, match="prev_state requires"):
        ik.solve(T, prev_state=robot.state(np.zeros((2, robot.num_actuated_joints), np.float32)))


def test_solve_numpy_interface(gpu, panda_arm_spec):
    """TestIKInterfaces.test_ik_basic_solve_numpy_interface (test_ik.py:441-464)."""
    robot = _robot(panda_arm_spec)
    ik = IKSolver(presets.basic, robot=robot, target_links=HAND)
    pose = np.array([0.5, 0.2, 0.5, 0.0, 0.0, 1.0, 0.0], np.float32)
    state = ik.solve_numpy(pose)
    q = state.q.numpy()
    assert q.shape == (1, robot.num_actuated_joints) and _within_limits(robot, q)
    (pos, _), = _errors(robot, state, [HAND], pose[None])
    assert pos[0] < 0.01


def test_continuous_tracking(gpu, panda_arm_spec):
    """TestIKContinuousTracking.test_ik_advanced_config_continuous_tracking (test_ik.py:525-544)."""
    robot = _robot(panda_arm_spec)
    init_ik = IKSolver(presets.basic, robot=robot, target_links=HAND)
    tracking = IKSolver(advanced_config(), robot=robot, target_links=HAND)
    pose = np.array([[0.5, 0.2, 0.5, 0.0, 0.0, 1.0, 0.0]], np.float32)
    state = robot.state(init_ik.solve(pose[:, None]).q.numpy().copy())
    for _ in range(10):
        state = robot.state(tracking.solve(pose[:, None], prev_state=state, init_state=state).q.numpy().copy())
    (pos, _), = _errors(robot, state, [HAND], pose)
    assert pos[0] < 0.01


def test_hysteresis(gpu, panda_arm_spec):
    """TestIKContinuousTracking.test_ik_hysteresis (test_ik.py:546-586): a static target keeps the previous
    solution (ties keep it), a moved one is still tracked."""
    robot = _robot(panda_arm_spec)
    ik = IKSolver(basic_config(), robot=robot, target_links=HAND)
    ik.warmup(batch_size=1)
    T = _initial_targets(robot, [HAND], 1)  # the zero-q hand pose: the flattest null space
    na = ik.num_joints
    rest = robot.state(np.zeros((1, na), np.float32))
    out = robot.state(np.zeros((1, na), np.float32))
    prev, qs = None, []
    for _ in range(50):
        ik.solve(T, init_state=prev if prev is not None else rest, rest_state=rest, prev_state=prev, out_state=out)
        qs.append(out.q.numpy()[0].copy())
        prev = robot.state(out.q.numpy().copy())
    idle = np.array(qs[10:])
    assert float((idle.max(0) - idle.min(0)).max()) < 1e-4
    moved = T.copy()
    moved[0, 0, 0] += 0.05
    state = ik.solve(moved, init_state=prev, rest_state=rest, prev_state=prev)
    (pos, _), = _errors(robot, state, [HAND], moved)
    assert pos[0] < 0.01


def test_set_weight_per_link(gpu, panda_arm_spec):
    """set_weight by name with per-link weights (helpers/ik/ik.py:180-198; the G1 test at test_ik.py:592-646
    zeroes the left hand's weights the same way): a link weighted zero stops pulling."""
    robot = _robot(panda_arm_spec)
    links = ["panda_link4", HAND]
    ik = IKSolver(basic_config(), robot=robot, target_links=links)
    assert [t.name for t in ik.config.terms] == ["position_task_0", "rotation_task_0", "position_limit_0"]
    B = 32
    q = robot.sample_q(B, seed=17)
    T = _initial_targets(robot, links, B)
    hand = robot.forward_kinematics(robot.state(q)).get_T_world_link(robot.link_names.index(HAND)).numpy()
    T[:, 1] = hand
    T[:, 0, :3] += np.array([0.0, 0.0, 0.6], np.float32)  # link 4 out of reach: it fights the hand
    before = ik.compute_metrics_numpy(ik.solve(T), T).position_error_m[:, 1]
    ik.set_weight("position_task_0", [0.0, 20.0])
    ik.set_weight("rotation_task_0", [0.0, 10.0])
    after = ik.compute_metrics_numpy(ik.solve(T), T).position_error_m[:, 1]
    assert np.median(before) > 0.02 and np.mean(after < 0.005) >= 0.9
    with pytest.raises(KeyError, match="No term named"):
        ik.set_weight("nope", 1.0)
    with pytest.raises(TypeError, match="per-link weights"):
        ik.set_weight("position_limit_0", [1.0, 1.0])
    with pytest.raises(ValueError, match="weight sequence length"):
        ik.set_weight("position_task_0", [1.0])


def test_weight_sequence_length_is_checked(gpu, panda_arm_spec):
    robot = _robot(panda_arm_spec)
    cfg = IKSolverConfig().add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET,
                                            weight=[1.0, 2.0, 3.0]))
    with pytest.raises(ValueError, match="weight sequence length 3 != 1"):
        IKSolver(cfg, robot=robot, target_links=HAND)


def test_unknown_link_raises(gpu, panda_arm_spec):
    """TestIKConfigValidation.test_unknown_link_raises (test_ik.py:755-760)."""
    robot = _robot(panda_arm_spec)
    with pytest.raises(ValueError, match="not in robot.link_names"):
        IKSolver(presets.basic, robot=robot, target_links="definitely_not_a_link")
    with pytest.raises(ValueError, match="out of range"):
        IKSolver(presets.basic, robot=robot, target_links=len(robot.link_names))


def test_target_contract(gpu, panda_arm_spec):
    """TestIKTargetValidation (test_ik.py:763-850): dtype, logical shape, target count, the adapters' shapes and
    compute_costs' use of the same contract."""
    import torch

    robot = _robot(panda_arm_spec)
    ik = IKSolver(presets.basic, robot=robot, target_links=HAND)
    with pytest.raises(TypeError, match="float32 poses"):
        ik.solve(N.DeviceArray.zeros((1, 1)))
    with pytest.raises(TypeError, match="float32 poses"):
        ik.solve(N.DeviceArray.zeros((1, 1, 7), np.int32))
    with pytest.raises(ValueError, match="logical shape"):
        ik.solve(N.DeviceArray.zeros(7))
    with pytest.raises(ValueError, match="target count"):
        ik.solve(N.DeviceArray.zeros((1, 2, 7)))
    with pytest.raises(ValueError, match="must be on cuda"):
        ik.solve(torch.zeros((1, 1, 7)))
    with pytest.raises(ValueError, match=r"shape \(\.\.\., 7\)"):
        ik.solve_numpy(np.zeros((1, 6), np.float32))
    with pytest.raises(ValueError, match=r"shape \(\.\.\., 4, 4\)"):
        ik.solve_torch(torch.zeros((1, 3, 3)))  # the shape is checked before the device
    state = robot.state(np.zeros((1, robot.num_actuated_joints), np.float32))
    with pytest.raises(TypeError, match="float32 poses"):
        ik.compute_costs(state, N.DeviceArray.zeros((1, 1)))


def test_compute_costs_per_term(gpu, panda_arm_spec):
    """compute_costs (helpers/ik/ik.py:373-385): |r|^2 of each term by cost_name, against the FP64 oracle's
    residuals of the same terms."""
    robot = _robot(panda_arm_spec)
    cfg = advanced_config()
    ik = IKSolver(cfg, robot=robot, target_links=HAND)
    B = 24
    q = robot.sample_q(B, seed=23)
    T = robot.forward_kinematics(robot.state(robot.sample_q(B, seed=24))).get_T_world_link(
        robot.link_names.index(HAND)).numpy().reshape(B, 1, 7)
    lim = robot.spec.actuated_joint_limits
    q[:4] = lim[:, 1] + 0.2  # outside the limits: the limit term is non-zero
    prev_q = robot.sample_q(B, seed=25)
    costs = ik.compute_costs(robot.state(q), T, prev_state=robot.state(prev_q))
    assert set(costs) == {"position_task", "rotation_task", "position_limit", "configuration_task",
                          "smoothness_task", "velocity_limit_task"}

    class _V:
        spec, batch_size, has_floating_base = panda_arm_spec, B, False

    rob = oracle.Robot.from_spec(panda_arm_spec)
    for t in ik._terms:
        r, _ = oracle.residual_jacobian(rob, oracle.Terms([t.host_desc(_V)]), q, None)
        want = np.sum(r ** 2, axis=1)
        np.testing.assert_allclose(costs[t.cost_name].numpy(), want, rtol=2e-5, atol=1e-6, err_msg=t.cost_name)
    assert costs["position_limit"].numpy()[:4].min() > 0


@pytest.mark.parametrize("preset,scale", [("single_candidate", 1.0), ("smooth", 0.5)])
def test_keep_previous_prices_on_the_reference_scale(gpu, panda_arm_spec, preset, scale):
    """prev_state is priced as the reference does (helpers/ik/ik.py:257-289): |r|^2 against a final LM stage's
    0.5 |r|^2, 0.5 |r|^2 (the select's scale) after a final select stage; kept exactly where that price is no
    more than the solve's cost."""
    robot = _robot(panda_arm_spec)
    B = 64
    q = robot.sample_q(B, seed=31)
    T = robot.forward_kinematics(robot.state(q)).get_T_world_link(robot.link_names.index(HAND)).numpy().reshape(B, 1, 7)
    rng = np.random.default_rng(0)
    lim = robot.spec.actuated_joint_limits
    prev_q = np.clip(q + 0.02 * rng.random((B, 1)) ** 2 * rng.normal(size=q.shape), lim[:, 0], lim[:, 1])
    prev_q = prev_q.astype(np.float32)
    ik = IKSolver(getattr(presets, preset), robot, HAND)
    sol = ik.solve(T, prev_state=robot.state(prev_q)).q.numpy().copy()
    pc, cost = ik._prev_cost.numpy(), ik.costs.numpy()

    class _V:
        spec, batch_size, has_floating_base = panda_arm_spec, B, False

    r, _ = oracle.residual_jacobian(oracle.Robot.from_spec(panda_arm_spec),
                                    oracle.Terms([t.host_desc(_V) for t in ik._terms]), prev_q, None)
    np.testing.assert_allclose(pc, scale * np.sum(r ** 2, axis=1), rtol=1e-4, atol=2e-7)  # FP32 residuals
    kept = np.all(sol == prev_q, axis=1)
    np.testing.assert_array_equal(kept, pc <= cost)


# --- heterogeneous scenes (test_ik.py:852-955, tests/helpers/motion_plan/hetero_scenes.py:1-100) -----------------
# The reference's icosphere meshes are replaced by analytic spheres of the same radii.
SCENE_IDS = [0, 0, 0, 1, 2, 2, 2, 2]
SCENE_SPECS = [
    {"boxes": [((0.05, 0.05, 0.3), (0.45, 0.16, 0.3)), ((0.05, 0.05, 0.3), (0.45, -0.16, 0.3))], "planes": [],
     "spheres": []},
    {"boxes": [((0.08, 0.35, 0.04), (0.45, 0.0, 0.25))], "planes": [], "spheres": [(0.11, (0.45, 0.0, 0.5))]},
    {"boxes": [((0.05, 0.05, 0.25), (0.45, 0.0, 0.28))], "planes": [-0.05],
     "spheres": [(0.1, (0.4, 0.22, 0.42)), (0.1, (0.4, -0.22, 0.42))]},
]


def _at(centers):
    return [[*c, 1.0, 0.0, 0.0, 0.0] for c in centers]


def _build_scene(ids):
    """One Scene over the listed scene specs, one geometry per primitive type (empty types left out)."""
    from robokit_b200.geom import BoxGeom, PlaneGeom, Scene, SphereGeom

    specs = [SCENE_SPECS[i] for i in ids]
    scene = Scene(len(specs))
    he = [h for s in specs for h, _ in s["boxes"]]
    off = np.cumsum([0] + [len(s["boxes"]) for s in specs])
    scene.add(BoxGeom(he, off, poses=_at([c for s in specs for _, c in s["boxes"]])))
    if any(s["planes"] for s in specs):
        off = np.cumsum([0] + [len(s["planes"]) for s in specs])
        scene.add(PlaneGeom(off, poses=_at([(0.0, 0.0, z) for s in specs for z in s["planes"]])))
    if any(s["spheres"] for s in specs):
        off = np.cumsum([0] + [len(s["spheres"]) for s in specs])
        scene.add(SphereGeom([r for s in specs for r, _ in s["spheres"]], off,
                             poses=_at([c for s in specs for _, c in s["spheres"]])))
    return scene


def _penetration(robot, scene, q):
    """Deepest penetration of a collision sphere into the scene at each row of q (the "plain" penalty at
    margin 0 is max(0, -signed distance))."""
    from robokit_b200.opt import VarKey, VarValues
    from robokit_b200.terms.dense import SceneCollisionTask

    t = SceneCollisionTask(robot, scene, weight=1.0, margin=0.0, penalty="plain")
    return t.compute_weighted_residual(VarValues({VarKey.ROBOT: robot.state(np.atleast_2d(q))})).numpy().max(axis=1)


def _sample_targets(robot):
    """A collision-free configuration per query in its own scene and its hand pose (hetero_scenes.py:113-133)."""
    rng = np.random.default_rng(0)
    lim = robot.spec.actuated_joint_limits
    hand = robot.link_names.index(HAND)
    start = np.tile(robot.spec.midrange_q.astype(np.float32), (len(SCENE_IDS), 1))
    poses = []
    for sid in SCENE_IDS:
        scene = _build_scene([sid])
        while True:
            q = rng.uniform(lim[:, 0] * 0.6, lim[:, 1] * 0.6).astype(np.float32)
            if _penetration(robot, scene, q)[0] == 0.0:
                break
        poses.append(robot.forward_kinematics(robot.state(q[None])).get_T_world_link(hand).numpy()[0])
    return start, np.asarray(poses, np.float32)


def _collision_config(robot, scene, scene_indices, solver, scale):
    from robokit_b200.terms.dense import SceneCollisionTask

    cfg = (IKSolverConfig(solver=solver, sampler=RobertsSamplerConfig(keep_first=True, scale=scale))
           .add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
           .add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
           .add(PositionLimit(weight=50.0)))
    for geometry in scene.geoms:
        cfg.add(SceneCollisionTask(robot, scene=scene, geometry=geometry, scene_indices=scene_indices, weight=100.0,
                                   margin=0.02))
    return cfg


def test_heterogeneous_collision_ik_matches_single_scenes(gpu, panda_collision_spec):
    """TestHeterogeneousCollisionIK.test_matches_single_scene (test_ik.py:852-889): one candidate, batched over
    three scenes, equals each query solved alone in its own scene."""
    robot = _robot(panda_collision_spec)
    start, T = _sample_targets(robot)
    solver = PopulationSolverConfig(stages=[Stage(40, 1, LMOptimizerConfig(lm_lambda=1.0))], cuda_graph_mode="none")
    idx = N.DeviceArray.from_numpy(np.asarray(SCENE_IDS, np.int32))
    ik = IKSolver(_collision_config(robot, _build_scene([0, 1, 2]), idx, solver, 0.0), robot, HAND)
    batched = ik.solve(T[:, None], init_state=robot.state(start), scene_indices=idx).q.numpy().copy()
    for i, sid in enumerate(SCENE_IDS):
        one = IKSolver(_collision_config(robot, _build_scene([sid]), None, solver, 0.0), robot, HAND)
        qi = one.solve(T[i:i + 1, None], init_state=robot.state(start[i:i + 1])).q.numpy()
        np.testing.assert_allclose(batched[i], qi[0], atol=1e-4, err_msg=f"query {i} (scene {sid})")


def test_heterogeneous_collision_ik_is_collision_free(gpu, panda_collision_spec):
    """TestHeterogeneousCollisionIK.test_collision_free_per_scene (test_ik.py:924-955)."""
    robot = _robot(panda_collision_spec)
    start, T = _sample_targets(robot)
    idx = N.DeviceArray.from_numpy(np.asarray(SCENE_IDS, np.int32))
    ik = IKSolver(_collision_config(robot, _build_scene([0, 1, 2]), idx, presets.smooth.solver, 1.0), robot, HAND)
    q = ik.solve(T[:, None], init_state=robot.state(start), scene_indices=idx).q.numpy().copy()
    (pos, _), = _errors(robot, robot.state(q), [HAND], T)
    for i, sid in enumerate(SCENE_IDS):
        assert _penetration(robot, _build_scene([sid]), q[i])[0] <= 0.001, f"query {i} collides in scene {sid}"
        assert pos[i] < 0.02, f"query {i} missed its target by {pos[i] * 1000:.1f} mm"


@pytest.mark.parametrize("mode", ["none", "iter", "full"])
def test_prev_state_with_scene_collision(gpu, panda_collision_spec, mode):
    """TestIKPreviousStateWithSceneCollision (test_ik.py:958-986): pricing prev_state (one row per target) before
    the multi-candidate solve leaves the candidates' collision term intact."""
    from robokit_b200.geom import Scene, SphereGeom
    from robokit_b200.terms.dense import SceneCollisionTask

    robot = _robot(panda_collision_spec)
    scene = Scene(1).add(SphereGeom([0.05], [0, 1], poses=[[2.0, 2.0, 2.0, 1.0, 0.0, 0.0, 0.0]]))
    cfg = IKSolverConfig()
    cfg.solver = PopulationSolverConfig(stages=cfg.solver.stages, cuda_graph_mode=mode)
    cfg = (cfg.add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
           .add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
           .add(SceneCollisionTask(scene=IKContext.SCENE, scene_indices=IKContext.SCENE_INDICES, weight=100.0)))
    ik = IKSolver(cfg, robot, HAND, scene=scene)
    q = robot.spec.midrange_q.astype(np.float32)[None]
    state = robot.state(q)
    pose = robot.forward_kinematics(robot.state(q)).get_T_world_link(robot.link_names.index(HAND)).numpy()
    solved = ik.solve(pose[:, None], prev_state=state, init_state=state).q.numpy()
    np.testing.assert_allclose(solved, q, atol=1e-4)
