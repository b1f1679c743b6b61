"""The reference's term-optimization tests (tests/terms/test_task_optimization.py) through this library's LM.

Part A: each term alone (with a joint-limit term) lowers its cost under LMOptimizer.  Part B: two instances,
four candidates each, converge to their own targets.  The box mesh of the collision case is a BoxGeom of the
same size; the base-position-limit and centre-of-mass cases are outside the IK path.
"""

import numpy as np
import pytest

from robokit_b200 import _native as N
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
from robokit_b200.terms.dense import (ConfigurationTask, FrameTask, PositionLimit, PositionTask, RotationTask,
                                      SceneCollisionTask, SelfCollisionTask, SmoothnessTask, VelocityLimitTask)

pytestmark = pytest.mark.gpu


def _robot(spec):
    from robokit_b200.robo.robot import Robot

    return Robot(spec)


def _initial_cost(terms, state):
    """|r|^2 over the terms at a one-row state (test_task_optimization.py:26-32)."""
    return sum(float(np.sum(t.compute_weighted_residual(VarValues({VarKey.ROBOT: state})).numpy() ** 2))
               for t in terms)


def _solve(terms, state, max_iter=30, lm_lambda=1.0):
    opt = LMOptimizer(terms=terms, config=LMOptimizerConfig(max_iter=max_iter, lm_lambda=lm_lambda))
    vv, costs = opt.solve(VarValues({VarKey.ROBOT: state}))
    return vv.get(VarKey.ROBOT), costs.numpy().copy()


def _hand_target(robot, q):
    hand = robot.link_names.index("panda_hand")
    pose = robot.forward_kinematics(robot.state(np.atleast_2d(q).astype(np.float32))).get_T_world_link(hand).numpy()
    return hand, pose


def _q(robot, q):
    return robot.state(np.atleast_2d(np.asarray(q, np.float32)))


@pytest.mark.parametrize("kind", ["position", "rotation", "frame", "fixed_frame"])
def test_pose_terms_reduce_cost(gpu, panda_spec, kind):
    """TestOptimizationEffectiveness.test_position_task / rotation / frame / fixed frames
    (test_task_optimization.py:47-127)."""
    robot = _robot(panda_spec)
    hand, pose = _hand_target(robot, panda_spec.midrange_q)
    T = pose.reshape(1, 1, 7)
    tasks = {"position": lambda: [PositionTask(robot, hand, T, weight=10.0)],
             "rotation": lambda: [RotationTask(robot, hand, T, weight=5.0)],
             "frame": lambda: [FrameTask(robot, hand, T, position_weight=10.0, orientation_weight=5.0)],
             "fixed_frame": lambda: [PositionTask(robot, [hand], T, weight=10.0, fixed_target=True),
                                     RotationTask(robot, [hand], T, weight=5.0, fixed_target=True)]}[kind]()
    init = _initial_cost(tasks, _q(robot, panda_spec.zero_q))
    assert init > 0.01
    _, final = _solve([*tasks, PositionLimit(robot, weight=2.0)], _q(robot, panda_spec.zero_q))
    assert final[0] < 0.1 * init


def test_configuration_task_reduces_cost(gpu, panda_spec):
    """test_task_optimization.py:223-237."""
    robot = _robot(panda_spec)
    start = panda_spec.zero_q + 0.5
    task = ConfigurationTask(robot=robot, rest_q=panda_spec.midrange_q.astype(np.float32), weight=1.0)
    init = _initial_cost([task], _q(robot, start))
    assert init > 0.01
    _, final = _solve([task], _q(robot, start))
    assert final[0] < 0.01 * init


def test_position_limit_reduces_cost(gpu, panda_spec):
    """test_task_optimization.py:239-253: a start 10 rad outside the limits."""
    robot = _robot(panda_spec)
    start = panda_spec.midrange_q + 10.0
    task = PositionLimit(robot=robot, weight=1.0)
    init = _initial_cost([task], _q(robot, start))
    assert init > 1.0
    _, final = _solve([task], _q(robot, start))
    assert final[0] < 0.01 * init


def test_smoothness_task_reduces_cost(gpu, panda_spec):
    """test_task_optimization.py:255-270."""
    robot = _robot(panda_spec)
    prev = _q(robot, panda_spec.zero_q)
    start = panda_spec.zero_q + 0.5
    task = SmoothnessTask(robot=robot, prev_var=prev, weight=1.0)
    init = _initial_cost([task], _q(robot, start))
    assert init > 0.01
    _, final = _solve([task], _q(robot, start))
    assert final[0] < 0.01 * init


def test_velocity_limit_task_reduces_cost(gpu, panda_spec):
    """test_task_optimization.py:272-288: a 2 rad step over dt = 0.01 s."""
    robot = _robot(panda_spec)
    prev = _q(robot, panda_spec.zero_q)
    start = panda_spec.zero_q + 2.0
    task = VelocityLimitTask(robot=robot, dt=0.01, prev_state_var=prev, weight=1.0)
    init = _initial_cost([task], _q(robot, start))
    assert init > 0.1
    _, final = _solve([task], _q(robot, start), max_iter=50)
    assert final[0] < 0.5 * init


def test_scene_collision_task_reduces_cost(gpu, panda_collision_spec):
    """test_task_optimization.py:309-337, the 0.3 m box mesh as a BoxGeom of half extent 0.15 m."""
    from robokit_b200.geom import BoxGeom, Scene

    robot = _robot(panda_collision_spec)
    scene = Scene(1).add(BoxGeom([[0.15, 0.15, 0.15]], [0, 1]))
    task = SceneCollisionTask(robot=robot, scene=scene, weight=5.0, margin=0.1,
                              sphere_indices=list(range(min(6, len(panda_collision_spec.collision_sphere_radii)))))
    q0 = panda_collision_spec.midrange_q
    init = _initial_cost([task], _q(robot, q0))
    assert init > 0.001
    _, final = _solve([task, PositionLimit(robot, weight=2.0)], _q(robot, q0), max_iter=50)
    assert final[0] < 0.9 * init


def test_self_collision_task_reduces_cost(gpu, panda_collision_spec):
    """test_task_optimization.py:339-357: a 0.5 m margin keeps the residual non-zero."""
    robot = _robot(panda_collision_spec)
    task = SelfCollisionTask(robot=robot, weight=5.0, margin=0.5)
    q0 = panda_collision_spec.zero_q
    init = _initial_cost([task], _q(robot, q0))
    assert init > 0.01
    _, final = _solve([task, PositionLimit(robot, weight=2.0)], _q(robot, q0), max_iter=50)
    assert final[0] < 0.5 * init


# --- part B: two instances, four candidates each (test_task_optimization.py:360-520) -----------------------------
C, B = 4, 2


def _two_targets(robot, spec, offset):
    lim = spec.actuated_joint_limits
    qs = np.stack([spec.midrange_q, np.clip(spec.midrange_q + offset, lim[:, 0], lim[:, 1])]).astype(np.float32)
    return _hand_target(robot, qs)


def _check(achieved, targets, atol):
    for inst in range(B):
        for s in range(C):
            np.testing.assert_allclose(achieved[inst * C + s], targets[inst], atol=atol,
                                       err_msg=f"instance {inst}, candidate {s}")


@pytest.mark.parametrize("kind,offset,start,iters,atol", [("position", 0.3, "zero", 50, 0.02),
                                                         ("rotation", 0.4, "zero", 50, None),
                                                         ("frame", 0.2, "mid", 100, 0.05),
                                                         ("fixed_frame", 0.2, "mid", 100, 0.05)])
def test_instances_reach_their_own_targets(gpu, panda_spec, kind, offset, start, iters, atol):
    """TestMultiInstanceTargetIsolation (test_task_optimization.py:361-480): targets repeated per candidate,
    instance-major; every candidate of an instance converges to that instance's target."""
    robot = _robot(panda_spec)
    hand, poses = _two_targets(robot, panda_spec, offset)
    T = N.DeviceArray.from_numpy(np.repeat(poses, C, axis=0).reshape(B * C, 1, 7))
    task = {"position": lambda: [PositionTask(robot, hand, T, weight=10.0)],
            "rotation": lambda: [RotationTask(robot, hand, T, weight=5.0)],
            "frame": lambda: [FrameTask(robot, hand, T, position_weight=10.0, orientation_weight=5.0)],
            "fixed_frame": lambda: [PositionTask(robot, [hand], T, weight=10.0, fixed_target=True),
                                    RotationTask(robot, [hand], T, weight=5.0, fixed_target=True)]}[kind]()
    q0 = panda_spec.zero_q if start == "zero" else panda_spec.midrange_q
    final, _ = _solve([*task, PositionLimit(robot, weight=2.0)], _q(robot, np.tile(q0, (B * C, 1))), max_iter=iters)
    got = robot.forward_kinematics(final).get_T_world_link(hand).numpy()
    if kind == "rotation":
        for inst in range(B):
            for s in range(C):
                assert abs(float(np.dot(got[inst * C + s, 3:], poses[inst, 3:]))) > 0.99
    else:
        _check(got[:, :3], poses[:, :3], atol)
