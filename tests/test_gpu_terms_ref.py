"""The reference's own tests of the temporal and rest terms (tests/terms/test_smoothness_task.py,
test_configuration_task.py, test_velocity_limit_task.py), run against this library's API."""

import numpy as np
import pytest

from robokit_b200.opt import VarKey, VarValues
from robokit_b200.terms.dense import ConfigurationTask, SmoothnessTask, VelocityLimitTask

pytestmark = pytest.mark.gpu

_ID = np.array([0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0], np.float32).reshape(1, 7)


@pytest.fixture
def panda_robot(gpu, panda_spec):
    from robokit_b200.robo.robot import Robot

    return Robot(panda_spec)


def test_smoothness_task_fixed_base(panda_robot):  # test_smoothness_task.py:24-39
    robot = panda_robot
    state_prev = robot.state(q=robot.spec.zero_q)
    state_curr = robot.state(q=robot.spec.zero_q + 0.1)
    smooth_task = SmoothnessTask(robot=robot, weight=0.5)
    residual = smooth_task.compute_weighted_residual(VarValues({VarKey.ROBOT: state_curr}), state_prev)
    assert residual.shape == (1, robot.num_actuated_joints)
    assert np.allclose(residual.numpy(), 0.1 * 0.5, atol=1e-5)
    # the previous state was for that call only
    assert not np.any(smooth_task.compute_weighted_residual(VarValues({VarKey.ROBOT: state_curr})).numpy())


def test_smoothness_task_floating_base_residual_dim_is_static(panda_robot):  # :52-75
    robot = panda_robot
    state_prev = robot.state(q=robot.spec.zero_q, T_world_base=_ID)
    state_curr = robot.state(q=robot.spec.zero_q + 0.1, T_world_base=_ID)
    smooth_task = SmoothnessTask(robot=robot, prev_var=state_prev, weight=0.5, base_weight=0.2)
    before = smooth_task.residual_dim
    residual = smooth_task.compute_weighted_residual(VarValues({VarKey.ROBOT: state_curr}))
    jacobian = smooth_task.compute_weighted_jacobian(VarValues({VarKey.ROBOT: state_curr}))
    na = robot.num_actuated_joints
    assert before == na + 6 and smooth_task.residual_dim == before
    assert residual.shape == (1, before) and jacobian.shape == (1, before, 6 + na)
    np.testing.assert_allclose(residual.numpy()[0, :na], 0.05, atol=1e-6)
    np.testing.assert_allclose(residual.numpy()[0, na:], 0.0, atol=1e-6)  # same base


def test_smoothness_task_residual_dim_static_after_set_prev_state_with_floating_base(panda_robot):  # :77-96
    robot = panda_robot
    state_prev = robot.state(q=robot.spec.zero_q, T_world_base=_ID)
    state_curr = robot.state(q=robot.spec.zero_q + 0.1, T_world_base=_ID)
    smooth_task = SmoothnessTask(robot=robot, prev_var=None, weight=0.5, base_weight=None)
    before = smooth_task.residual_dim
    smooth_task.set_prev_state(state_prev)
    residual = smooth_task.compute_weighted_residual(VarValues({VarKey.ROBOT: state_curr}))
    jacobian = smooth_task.compute_weighted_jacobian(VarValues({VarKey.ROBOT: state_curr}))
    na = robot.num_actuated_joints
    assert before == na and smooth_task.residual_dim == before
    assert residual.shape == (1, before) and jacobian.shape == (1, before, 6 + na)


def test_smoothness_task_base_enabled_rejects_nonfloating_var(panda_robot):  # :98-121
    robot = panda_robot
    state_prev = robot.state(q=robot.spec.zero_q, T_world_base=_ID)
    state_curr = robot.state(q=robot.spec.zero_q + 0.1)
    smooth_task = SmoothnessTask(robot=robot, prev_var=state_prev, weight=0.5, base_weight=0.2)
    with pytest.raises(ValueError, match="configured with base residuals"):
        smooth_task.compute_weighted_residual(VarValues({VarKey.ROBOT: state_curr}))


def test_configuration_task_fixed_base(panda_robot):  # test_configuration_task.py:12-25
    robot = panda_robot
    rest_q = robot.spec.midrange_q
    state = robot.state(q=(rest_q + 0.1).astype(np.float32))
    task = ConfigurationTask(robot=robot, rest_q=rest_q, weight=0.1)
    residual = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state}))
    assert residual.shape == (1, robot.num_actuated_joints)
    assert np.allclose(residual.numpy(), 0.1 * 0.1, atol=1e-5)


def test_configuration_task_fixed_base_batched(panda_robot):  # :27-49
    robot = panda_robot
    batch_size, num_candidates = 4, 2
    total = batch_size * num_candidates
    rest_q = robot.spec.midrange_q
    state = robot.state(q=np.tile(rest_q + 0.1, (total, 1)).astype(np.float32))
    task = ConfigurationTask(robot=robot, rest_q=rest_q, weight=0.1)
    residual = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state}))
    assert residual.shape == (total, robot.num_actuated_joints)
    assert np.allclose(residual.numpy(), 0.1 * 0.1, atol=1e-5)
    from robokit_b200 import _native as N

    task.set_target(N.DeviceArray.from_numpy(np.tile(rest_q + 0.05, (batch_size, 1)).astype(np.float32)))
    residual2 = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state}))
    assert np.allclose(residual2.numpy(), 0.05 * 0.1, atol=1e-5)


def test_configuration_task_base_only(panda_robot):  # :51-68
    robot = panda_robot
    state = robot.state(q=robot.spec.zero_q, T_world_base=_ID)
    task = ConfigurationTask(robot=robot, T_world_base_rest=_ID, weight=0.0, base_weight=1.0, include_joints=False)
    residual = task.compute_weighted_residual(VarValues({VarKey.ROBOT: state}))
    jacobian = task.compute_weighted_jacobian_analytic(VarValues({VarKey.ROBOT: state}))
    assert residual.shape == (1, 6)
    assert jacobian.shape == (1, 6, state.tangent_dim)
    assert np.allclose(residual.numpy(), 0.0)


def test_velocity_limit_task(panda_robot):  # test_velocity_limit_task.py:11-30
    robot = panda_robot
    state_prev = robot.state(q=robot.spec.zero_q)
    state_curr = robot.state(q=robot.spec.zero_q + 0.5)  # large change
    vel_task = VelocityLimitTask(robot=robot, dt=0.1, weight=1.0)
    residual = vel_task.compute_weighted_residual(VarValues({VarKey.ROBOT: state_curr}), state_prev)
    jacobian = vel_task.compute_weighted_jacobian(VarValues({VarKey.ROBOT: state_curr}), state_prev)
    na = robot.num_actuated_joints
    assert residual.shape == (1, na)
    assert np.all(residual.numpy() >= 0)
    assert jacobian.shape == (1, na, na)
    # 0.5 rad in 0.1 s = 5 rad/s against limits of 2.175-2.61 rad/s (0.2 for the finger)
    vmax = robot.spec.actuated_joint_velocity_limits
    np.testing.assert_allclose(residual.numpy()[0], np.maximum(0, 5.0 - vmax), rtol=1e-5, atol=1e-5)
