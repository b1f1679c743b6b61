"""The reference's own pose and limit term tests (tests/terms/test_position_task.py, test_rotation_task.py,
test_position_limit.py) run against this library; where they compare with Warp autodiff, the exact FP64
Jacobian of the oracle stands in, at the same tolerance."""

import numpy as np
import pytest

import oracle
from robokit_b200.opt import VarKey, VarValues
from robokit_b200.terms.dense import PositionLimit, PositionTask, RotationTask

pytestmark = pytest.mark.gpu

T0 = np.array([[0.5, 0.0, 0.5, 1.0, 0.0, 0.0, 0.0]], np.float32)
T1 = np.array([[0.3, 0.2, 0.4, 0.0, 1.0, 0.0, 0.0]], np.float32)
TGT = np.array([[0.5, 0.0, 0.5, 0.0, 1.0, 0.0, 0.0]], np.float32)


@pytest.fixture
def panda_robot(gpu, panda_spec):
    from robokit_b200.robo.robot import Robot

    return Robot(panda_spec)


def _state(robot):
    rng = np.random.RandomState(42)
    q = (rng.randn(robot.num_actuated_joints) * 0.1 + robot.spec.midrange_q).astype(np.float32)
    state = robot.state(q=q)
    robot.forward_kinematics(state)
    return state, q


def _oracle_jacobian(robot, task, q):
    class _V:
        spec, batch_size, has_floating_base = robot.spec, 1, False

    _, J = oracle.residual_jacobian(oracle.Robot.from_spec(robot.spec), oracle.Terms([task.host_desc(_V)]), q[None])
    return J


def _quat_err_rotvec(qa, qt):
    """Rotation vector of R_a R_t^-1 for wxyz quaternions (scipy Rotation convention of the reference test)."""
    w1, x1, y1, z1 = qa
    w2, x2, y2, z2 = qt[0], -qt[1], -qt[2], -qt[3]
    q = np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                  w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2])
    if q[0] < 0:
        q = -q
    s = np.linalg.norm(q[1:])
    ang = 2 * np.arctan2(s, q[0])
    return q[1:] * (ang / s if s > 1e-12 else 2.0)


def test_position_residual_is_world_frame_position_error(panda_robot):  # test_position_task.py:13-35
    robot = panda_robot
    state, _ = _state(robot)
    ee = robot.link_names.index("panda_hand")
    task = PositionTask(robot, ee, TGT.reshape(1, 1, 7), weight=2.0)
    res = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state})).numpy()
    ee_pos = state.T_world_link.numpy()[0, ee, :3]
    assert np.allclose(res[0], 2.0 * (TGT[0, :3] - ee_pos), atol=1e-5)


def test_position_jacobian_analytic_vs_exact(panda_robot):  # :37-59
    robot = panda_robot
    state, q = _state(robot)
    ee = robot.link_names.index("panda_hand")
    task = PositionTask(robot, ee, TGT.reshape(1, 1, 7), weight=2.0)
    analytic = task.compute_weighted_jacobian_analytic(VarValues({VarKey.ROBOT: state})).numpy()
    assert np.allclose(analytic, _oracle_jacobian(robot, task, q), atol=1e-4, rtol=1e-4)


def test_position_per_link_weights_residual(panda_robot):  # :62-83
    robot = panda_robot
    state, _ = _state(robot)
    i0, i1 = robot.link_names.index("panda_link4"), robot.link_names.index("panda_hand")
    task = PositionTask(robot, [i0, i1], np.stack([T0, T1], axis=1), weight=[2.0, 0.0])
    res = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state})).numpy()[0]
    ee0 = state.T_world_link.numpy()[0, i0, :3]
    assert np.allclose(res[:3], 2.0 * (T0[0, :3] - ee0), atol=1e-5)
    assert np.allclose(res[3:6], 0.0, atol=1e-7)


def test_position_set_weight_dynamic(panda_robot):  # :85-107
    robot = panda_robot
    state, _ = _state(robot)
    i0, i1 = robot.link_names.index("panda_link4"), robot.link_names.index("panda_hand")
    task = PositionTask(robot, [i0, i1], np.stack([T0, T1], axis=1), weight=1.0)
    task.set_weight([0.0, 3.0])
    res = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state})).numpy()[0]
    ee1 = state.T_world_link.numpy()[0, i1, :3]
    assert np.allclose(res[:3], 0.0, atol=1e-7)
    assert np.allclose(res[3:6], 3.0 * (T1[0, :3] - ee1), atol=1e-5)


def test_position_per_link_weights_jacobian(panda_robot):  # :109-131
    robot = panda_robot
    state, q = _state(robot)
    i0, i1 = robot.link_names.index("panda_link4"), robot.link_names.index("panda_hand")
    task = PositionTask(robot, [i0, i1], np.stack([T0, T1], axis=1), weight=[2.0, 0.5])
    analytic = task.compute_weighted_jacobian_analytic(VarValues({VarKey.ROBOT: state})).numpy()
    assert np.allclose(analytic, _oracle_jacobian(robot, task, q), atol=1e-4, rtol=1e-4)


def test_rotation_residual_is_world_frame_rotation_error(panda_robot):  # test_rotation_task.py:14-38
    robot = panda_robot
    state, _ = _state(robot)
    ee = robot.link_names.index("panda_hand")
    task = RotationTask(robot, ee, TGT.reshape(1, 1, 7), weight=3.0)
    res = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state})).numpy()
    qa = state.T_world_link.numpy()[0, ee, 3:7].astype(np.float64)
    expected = 3.0 * _quat_err_rotvec(qa, TGT[0, 3:7].astype(np.float64))
    assert np.allclose(res[0], expected, atol=1e-5)


def test_rotation_jacobian_analytic_vs_exact_near_identity(panda_robot):  # :40-66
    robot = panda_robot
    state, q = _state(robot)
    ee = robot.link_names.index("panda_hand")
    cur = state.T_world_link.numpy()[0, ee].reshape(1, 1, 7)
    task = RotationTask(robot, ee, cur, weight=2.0)  # target at the current pose: the near-identity branch
    analytic = task.compute_weighted_jacobian_analytic(VarValues({VarKey.ROBOT: state})).numpy()
    assert np.allclose(analytic, _oracle_jacobian(robot, task, q), atol=1e-4, rtol=1e-4)


def test_rotation_per_link_weights_residual(panda_robot):  # :68-88
    robot = panda_robot
    state, _ = _state(robot)
    i0, i1 = robot.link_names.index("panda_link4"), robot.link_names.index("panda_hand")
    task = RotationTask(robot, [i0, i1], np.stack([T0, T1], axis=1), weight=[2.0, 0.0])
    res = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state})).numpy()[0]
    q0 = state.T_world_link.numpy()[0, i0, 3:7].astype(np.float64)
    assert np.allclose(res[:3], 2.0 * _quat_err_rotvec(q0, T0[0, 3:7].astype(np.float64)), atol=1e-5)
    assert np.allclose(res[3:6], 0.0, atol=1e-7)


def test_position_limit_fixed_base(panda_robot):  # test_position_limit.py:21-37
    robot = panda_robot
    state = robot.state(q=robot.spec.zero_q)
    limit = PositionLimit(robot=robot, weight=1.0)
    residual = limit.compute_weighted_residual(VarValues({VarKey.ROBOT: state}))
    jacobian = limit.compute_weighted_jacobian(VarValues({VarKey.ROBOT: state}))
    na = robot.num_actuated_joints
    assert residual.shape == (1, na) and jacobian.shape == (1, na, na)
    assert np.all(residual.numpy() >= 0)
    lo, hi = robot.spec.float32_actuated_limits().T
    np.testing.assert_allclose(residual.numpy()[0], np.maximum(0, lo) + np.maximum(0, -hi), atol=1e-6)
