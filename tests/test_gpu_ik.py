"""IKSolver over a candidate population: select kernel, presets on the Panda, stage plumbing, metrics."""

import ctypes

import numpy as np
import pytest

import oracle
from robokit_b200 import _native as N
from robokit_b200.helpers.ik import IKSolver, presets
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues

pytestmark = pytest.mark.gpu


def test_select_best_matches_a_stable_sort(gpu):
    rng = np.random.default_rng(0)
    B, C, K, na = 37, 70, 5, 3
    cost = rng.integers(0, 20, size=(B, C)).astype(np.float32)  # many ties
    cost[rng.random((B, C)) < 0.05] = np.nan
    q = rng.normal(size=(B * C, na)).astype(np.float32)
    dc, dq = N.DeviceArray.from_numpy(cost.reshape(-1)), N.DeviceArray.from_numpy(q)
    qo, co, io = N.DeviceArray.empty((B * K, na)), N.DeviceArray.empty(B * K), N.DeviceArray.empty(B * K, np.int32)
    N.check(N.lib().ik_select_best(B, C, K, dc.ptr, dq.ptr, None, na, qo.ptr, None, co.ptr, io.ptr, None))
    key = np.where(np.isnan(cost), np.inf, cost)
    want = np.argsort(key, axis=1, kind="stable")[:, :K]
    np.testing.assert_array_equal(io.numpy().reshape(B, K), want)
    rows = (np.arange(B)[:, None] * C + want).reshape(-1)
    np.testing.assert_array_equal(qo.numpy(), q[rows])
    with pytest.raises(ValueError):
        N.check(N.lib().ik_select_best(B, C, C + 1, dc.ptr, dq.ptr, None, na, qo.ptr, None, None, None, None))


def _targets(robot, B, seed, link):
    q = robot.sample_q(B, seed=seed)
    st = robot.forward_kinematics(robot.state(q))
    return st.get_T_world_link(link).numpy().reshape(B, 1, 7)


def test_basic_preset_solves_panda_targets(gpu, panda_arm_spec):
    """presets.basic (64 -> 4 -> 1 candidates) on FK-sampled Panda targets, scored at 5 mm / 0.05 rad
    like scripts/benchmark/ik/helper.py:63-64."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    link = panda_arm_spec.link_names.index("panda_hand")
    ik = IKSolver(presets.basic, robot, "panda_hand")
    assert ik.num_solutions == 1
    T = _targets(robot, 128, 42, link)
    sol = ik.solve(T)
    assert sol.q.shape == (128, 7)
    m = ik.compute_metrics_numpy(sol, T)
    assert m.success.mean() >= 0.95, m.success.mean()
    # the metrics kernel against the FP64 oracle
    rob = oracle.Robot.from_spec(panda_arm_spec)
    pe, re, ok = oracle.metrics(rob, sol.q.numpy(), None, [link], T, 0.005, 0.05)
    np.testing.assert_allclose(m.position_error_m, pe, atol=2e-5)
    np.testing.assert_allclose(m.orientation_error_rad, re, atol=2e-4)
    # a second solve on new targets reuses the buffers
    T2 = _targets(robot, 128, 43, link)
    assert ik.compute_metrics_numpy(ik.solve(T2), T2).success.mean() >= 0.95
    with pytest.raises(ValueError, match="Batch size mismatch"):
        ik.solve(T2[:64])


def test_single_stage_equals_the_optimizer(gpu, panda_arm_spec):
    """One candidate, one stage: the solve is an LMOptimizer solve from the joint midrange (bitwise), its
    smoothness term pulling toward the zero previous state the solver holds until a prev_state is given."""
    from robokit_b200.robo.robot import Robot
    from robokit_b200.terms.dense import PositionLimit, PositionTask, RotationTask, SmoothnessTask

    robot = Robot(panda_arm_spec)
    link = panda_arm_spec.link_names.index("panda_hand")
    T = _targets(robot, 64, 7, link)
    sol = IKSolver(presets.single_candidate, robot, link).solve(T).q.numpy()
    terms = [PositionTask(robot, [link], T, weight=20.0), RotationTask(robot, [link], T, weight=10.0),
             PositionLimit(robot, weight=50.0),
             SmoothnessTask(robot, prev_var=robot.state(np.zeros((64, 7), np.float32)), weight=0.1)]
    opt = LMOptimizer(terms, LMOptimizerConfig(max_iter=30, lm_lambda=1.0, early_stopping_interval=0,
                                               form="persistent"))
    st = robot.state(np.tile(panda_arm_spec.midrange_q, (64, 1)).astype(np.float32))
    opt.solve(VarValues({VarKey.ROBOT: st}))
    np.testing.assert_array_equal(sol, st.q.numpy())


def test_graph_replay_equals_direct_launches(gpu, panda_arm_spec):
    """cuda_graph_mode "full" (one captured graph per solve) gives the solutions of direct launches, bitwise."""
    import copy

    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    link = panda_arm_spec.link_names.index("panda_hand")
    direct_cfg = copy.deepcopy(presets.basic)
    direct_cfg.solver.cuda_graph_mode = "none"
    graph = IKSolver(presets.basic, robot, "panda_hand")
    direct = IKSolver(direct_cfg, robot, "panda_hand")
    for seed in (11, 12, 13):  # the first graph solve runs directly, the next two replay the graph
        T = _targets(robot, 96, seed, link)
        n0 = N.launch_count()
        a = graph.solve(T).q.numpy()
        n1 = N.launch_count()
        b = direct.solve(T).q.numpy()
        np.testing.assert_array_equal(a, b)
        assert n1 > n0  # replayed kernels are counted
    assert graph._graph is not None and direct._graph is None


def test_init_state_seeds_around_a_previous_solution(gpu, panda_arm_spec):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    link = panda_arm_spec.link_names.index("panda_hand")
    ik = IKSolver(presets.basic, robot, "panda_hand")
    T = _targets(robot, 32, 21, link)
    first = ik.solve(T)
    prev = robot.state(first.q.numpy())
    again = ik.solve(T, init_state=prev, init_sample_range=0.05)
    m = ik.compute_metrics_numpy(again, T)
    assert m.success.mean() >= 0.95
    with pytest.raises(ValueError, match="init_state batch size"):
        ik.solve(T, init_state=robot.state(first.q.numpy()[:8]))


def test_roberts_sampler_fill_and_sample(gpu, panda_arm_spec):
    """tests/opt/test_sampler.py:27-54 on device arrays: fill tiles the scaled offsets, rejects a wrong width,
    and sample() spreads a state in place."""
    from robokit_b200 import _native as N
    from robokit_b200.opt.sampler import RobertsSampler, RobertsSamplerConfig
    from robokit_b200.robo.robot import Robot

    s = RobertsSampler(num_candidates=4, scale=[0.5, 0.5], keep_first=True)
    t = N.DeviceArray.zeros((8, 2))
    s.fill(t)
    np.testing.assert_array_equal(t.numpy(), s.tangent(2))
    with pytest.raises(ValueError, match="tangent_dim"):
        s.fill(N.DeviceArray.zeros((4, 3)))
    robot = Robot(panda_arm_spec)
    q = np.tile(panda_arm_spec.midrange_q, (8, 1)).astype(np.float32)
    vv = VarValues({VarKey.ROBOT: robot.state(q)})
    smp = RobertsSamplerConfig(scale=0.1, keep_first=True).build(vv, 4)
    smp.sample(vv)
    moved = vv.get(VarKey.ROBOT).q.numpy()
    np.testing.assert_allclose(moved, q + smp.tangent(2), atol=1e-6)
