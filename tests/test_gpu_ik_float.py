"""IKSolver with a floating base (enable_T_world_base) and active joint / base masks."""

import numpy as np
import pytest

from robokit_b200.helpers.ik import IKContext, IKSolver, IKSolverConfig, presets
from robokit_b200.opt import LMOptimizerConfig
from robokit_b200.opt.population_solver import PopulationSolverConfig, Stage
from robokit_b200.opt.sampler import RobertsSamplerConfig
from robokit_b200.terms.dense import (ConfigurationTask, PositionLimit, PositionTask, RotationTask, SmoothnessTask)

pytestmark = pytest.mark.gpu


def _config(**kw):
    cfg = IKSolverConfig(sampler=RobertsSamplerConfig(keep_first=True, scale=1.0), enable_T_world_base=True, **kw)
    cfg.add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
    cfg.add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
    cfg.add(PositionLimit(weight=50.0))
    return cfg


def _targets(robot, B, seed, base=None):
    hand = robot.spec.link_names.index("panda_hand")
    qs = robot.sample_q(B, seed=seed)
    return robot.forward_kinematics(robot.state(qs, base)).get_T_world_link(hand).numpy().reshape(B, 1, 7)


def test_floating_base_solver_reaches_targets_beyond_the_fixed_arm(gpu, panda_arm_spec):
    """Targets from arms on shifted bases: the floating-base solver moves its base and reaches them."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    B = 64
    rng = np.random.default_rng(3)
    base = np.tile(np.array([0, 0, 0, 1, 0, 0, 0], np.float32), (B, 1))
    base[:, :2] = rng.uniform(-0.6, 0.6, (B, 2))
    T = _targets(robot, B, 5, base)
    ik = IKSolver(_config(), robot, "panda_hand")
    sol = ik.solve(T)
    assert sol.has_floating_base and sol.q.shape == (B, 7)
    assert ik.compute_metrics_numpy(sol, T).success.mean() >= 0.9
    fixed = IKSolver(presets.basic, robot, "panda_hand")
    assert fixed.compute_metrics_numpy(fixed.solve(T), T).success.mean() < 0.9  # some targets out of a fixed arm's reach


def test_locked_base_and_joint_masks(gpu, panda_arm_spec):
    """A locked base stays at identity; a locked joint stays at its seed (the midrange)."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    B = 32
    T = _targets(robot, B, 9)
    ik = IKSolver(_config(base_active_mask=(0.0, 0.0, 0.0, 0.0, 0.0, 0.0)), robot, "panda_hand")
    sol = ik.solve(T)
    np.testing.assert_array_equal(sol.T_world_base.numpy(), np.tile([0, 0, 0, 1, 0, 0, 0], (B, 1)))
    assert ik.compute_metrics_numpy(sol, T).success.mean() >= 0.9
    mask = np.ones(7, np.float32)
    mask[6] = 0.0
    ik.set_active_joint_mask(mask)
    sol2 = ik.solve(T)
    np.testing.assert_array_equal(sol2.q.numpy()[:, 6], np.full(B, panda_arm_spec.midrange_q[6], np.float32))
    with pytest.raises(ValueError):
        IKSolver(presets.basic, robot, "panda_hand").set_active_base_mask([1] * 6)


def test_floating_previous_and_rest_states(gpu, panda_arm_spec):
    """Smoothness on the previous base and a rest-base ConfigurationTask through IKContext placeholders."""
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_arm_spec)
    B = 32
    T = _targets(robot, B, 21)
    cfg = IKSolverConfig(solver=PopulationSolverConfig(stages=[Stage(30, 1, LMOptimizerConfig(lm_lambda=1.0))]),
                         enable_T_world_base=True)
    cfg.add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
    cfg.add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
    cfg.add(PositionLimit(weight=50.0))
    cfg.add(SmoothnessTask(prev_var=IKContext.PREVIOUS_STATE, weight=0.1, base_weight=5.0))
    cfg.add(ConfigurationTask(T_world_base_rest=IKContext.REST_BASE, include_joints=False, base_weight=1.0))
    ik = IKSolver(cfg, robot, "panda_hand")
    first = ik.solve(T)
    assert ik.compute_metrics_numpy(first, T).success.mean() >= 0.8
    first_q, first_base = first.q.numpy().copy(), first.T_world_base.numpy().copy()  # solve reuses its buffers
    prev = robot.state(first_q, first_base)
    again = ik.solve(T, prev_state=prev)
    # the keep-previous rule on joints and base: kept exactly where the previous state costs no more
    same = np.all(again.q.numpy() == prev.q.numpy(), axis=1) & np.all(
        again.T_world_base.numpy() == prev.T_world_base.numpy(), axis=1)
    prev_cost, cost = ik._prev_cost.numpy(), ik.costs.numpy()
    assert (prev_cost[same] <= cost[same]).all() and (prev_cost[~same] > cost[~same]).all()
    assert ik.compute_metrics_numpy(again, T).success.mean() >= 0.8
    rest = robot.state(first_q, np.tile([0.3, 0, 0, 1, 0, 0, 0], (B, 1)).astype(np.float32))
    moved = ik.solve(T, rest_state=rest)
    # the rest base pulls the base toward x = 0.3
    assert np.mean(moved.T_world_base.numpy()[:, 0]) > np.mean(first_base[:, 0]) + 0.01
