"""The reference's tests/terms/test_terms.py through this library: integration of fixed and floating bases,
analytic Jacobians of the frame and scene-collision terms (against the exact FP64 oracle here, where the
reference uses Warp autodiff, same tolerances), and the multi-seed consistency of every dense term: candidates
that hold the same q give the same rows.  The 2 m box mesh of the collision case is a BoxGeom of half extent 1 m.
"""

import numpy as np
import pytest

import oracle
from robokit_b200 import _native as N
from robokit_b200.opt import VarKey, VarValues
from robokit_b200.terms.dense import (ConfigurationTask, FrameTask, PositionTask, RotationTask, SceneCollisionTask,
                                      SmoothnessTask, VelocityLimitTask)

pytestmark = pytest.mark.gpu

ID7 = np.array([0, 0, 0, 1, 0, 0, 0], np.float32)


def _robot(spec):
    from robokit_b200.robo.robot import Robot

    return Robot(spec)


class _View:
    def __init__(self, spec, B, floating):
        self.spec, self.batch_size, self.has_floating_base = spec, B, floating


def test_integrate_fixed_base_preserves_world_base(gpu, panda_spec):
    """TestWarpIntegration.test_integrate_fixed_base_preserves_world_base (test_terms.py:21-30)."""
    robot = _robot(panda_spec)
    state = robot.state(panda_spec.zero_q[None].astype(np.float32))
    expected = np.array([[0.2, -0.1, 0.3, 1.0, 0.0, 0.0, 0.0]], np.float32)
    state.T_world_base.assign(expected)
    out = robot.state(state.q.numpy())
    state.integrate(np.zeros((1, robot.num_actuated_joints), np.float32), out=out)
    np.testing.assert_array_equal(out.T_world_base.numpy(), expected)


def test_integrate_floating_base(gpu, panda_spec):
    """TestWarpIntegration.test_integrate_floating_base (test_terms.py:32-50)."""
    robot = _robot(panda_spec)
    state = robot.state(panda_spec.zero_q[None].astype(np.float32), ID7[None])
    v = np.zeros((1, 6 + robot.num_actuated_joints), np.float32)
    v[0, 0] = 0.1
    assert state.integrate(v).T_world_base.numpy()[0, 0] > 0


def test_frame_task_jacobian(gpu, panda_spec):
    """TestWarpAutodiffJacobian.test_frame_task_jacobian (test_terms.py:54-85), floating base at identity."""
    robot = _robot(panda_spec)
    rng = np.random.default_rng(0)
    q = (rng.normal(size=robot.num_actuated_joints) * 0.1 + panda_spec.midrange_q).astype(np.float32)[None]
    state = robot.forward_kinematics(robot.state(q, ID7[None]))
    ee = robot.link_names.index("panda_hand")
    T = np.array([[[0.5, 0.0, 0.5, 0.0, 1.0, 0.0, 0.0]]], np.float32)
    task = FrameTask(robot=robot, frame_index=ee, T_world_target=T, position_weight=1.0, orientation_weight=1.0)
    J = task.compute_weighted_jacobian_analytic(VarValues({VarKey.ROBOT: state})).numpy()
    _, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(panda_spec),
                                     oracle.Terms([task.host_desc(_View(panda_spec, 1, True))]), q, ID7[None])
    np.testing.assert_allclose(J, Jo, atol=1e-4, rtol=1e-4)


def test_collision_task_jacobian(gpu, panda_collision_spec):
    """TestWarpAutodiffJacobian.test_collision_task_jacobian (test_terms.py:87-120)."""
    from robokit_b200.geom import BoxGeom, Scene

    robot = _robot(panda_collision_spec)
    rng = np.random.default_rng(0)
    q = (rng.normal(size=robot.num_actuated_joints) * 0.1 + panda_collision_spec.midrange_q).astype(np.float32)[None]
    state = robot.forward_kinematics(robot.state(q))
    scene = Scene(1).add(BoxGeom([[1.0, 1.0, 1.0]], [0, 1]))
    ns = len(panda_collision_spec.collision_sphere_radii)
    task = SceneCollisionTask(robot=robot, scene=scene, weight=1.0, margin=0.01, sphere_indices=list(range(min(6, ns))))
    vv = VarValues({VarKey.ROBOT: state})
    r = task.compute_weighted_residual(vv).numpy()
    J = task.compute_weighted_jacobian_analytic(vv).numpy()
    ro, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(panda_collision_spec),
                                      oracle.Terms([task.host_desc(_View(panda_collision_spec, 1, False))]), q, None)
    assert np.all(r > 0)  # every queried sphere is inside the box
    np.testing.assert_allclose(r, ro, atol=3e-4, rtol=3e-4)
    np.testing.assert_allclose(J, Jo, atol=3e-4, rtol=3e-4)


# --- TestMultiSeedConsistency (test_terms.py:122-290) ------------------------------------------------------------
C, B = 4, 2


def _expanded(robot, seed):
    rng = np.random.default_rng(seed)
    lim = robot.spec.actuated_joint_limits
    q = rng.uniform(lim[:, 0], lim[:, 1], size=(B, robot.num_actuated_joints)).astype(np.float32)
    return q, robot.forward_kinematics(robot.state(np.repeat(q, C, axis=0))), rng


def _consistent(a, name):
    assert a.shape[0] == B * C
    for i in range(B):
        for s in range(1, C):
            np.testing.assert_allclose(a[i * C + s], a[i * C], atol=1e-5, rtol=1e-5,
                                       err_msg=f"{name}: instance {i}, candidate {s}")


@pytest.mark.parametrize("kind", ["position", "rotation", "frame", "configuration", "velocity", "smoothness"])
def test_multi_seed_consistency(gpu, panda_spec, kind):
    robot = _robot(panda_spec)
    q, state, rng = _expanded(robot, 42 + ["position", "rotation", "frame", "configuration", "velocity",
                                            "smoothness"].index(kind))
    link7 = robot.link_names.index("panda_link7")
    T = robot.forward_kinematics(robot.state(q)).get_T_world_link(link7).numpy().reshape(B, 1, 7)
    lim = robot.spec.actuated_joint_limits
    prev = robot.state(rng.uniform(lim[:, 0], lim[:, 1], size=(B, robot.num_actuated_joints)).astype(np.float32))
    vv = VarValues({VarKey.ROBOT: state})
    extra = {}
    if kind == "position":
        task = PositionTask(robot, link7, T, weight=1.0)
    elif kind == "rotation":
        task = RotationTask(robot, link7, T, weight=1.0)
    elif kind == "frame":
        task = FrameTask(robot, link7, T, position_weight=1.0, orientation_weight=1.0)
    elif kind == "configuration":
        task = ConfigurationTask(robot=robot, rest_q=panda_spec.midrange_q.astype(np.float32), weight=0.1)
        task.set_target(N.DeviceArray.from_numpy(q))
    elif kind == "velocity":
        task = VelocityLimitTask(robot=robot, dt=0.1, weight=1.0)
        task.set_prev_state(prev)
    else:
        task = SmoothnessTask(robot=robot, weight=1.0)
        extra = {"prev_var": prev}
    r = task.compute_weighted_residual(vv, **extra).numpy()
    J = task.compute_weighted_jacobian(vv, **extra).numpy()
    _consistent(r, f"{kind} residual")
    _consistent(J, f"{kind} jacobian")
    if kind == "configuration":  # each instance's rest is its own q: the rows read the per-instance reference
        np.testing.assert_allclose(r, 0.0, atol=1e-6)
    if kind in ("smoothness", "velocity"):
        assert np.any(r != 0)  # the rows read the per-instance previous state, not zeros
