"""The reference's own SelfCollisionTask tests (tests/terms/test_self_collision_task.py:13-100, sphere
representation) run against this library; the exact FP64 oracle Jacobian stands in for Warp autodiff."""

import copy

import numpy as np
import pytest

import oracle
from robokit_b200.opt import VarKey, VarValues
from robokit_b200.terms.dense import SelfCollisionTask

pytestmark = pytest.mark.gpu


@pytest.fixture
def panda_robot_with_collision(gpu, panda_collision_spec):
    from robokit_b200.robo.robot import Robot

    return Robot(panda_collision_spec)


def _residual(task, robot, q, base=None):
    return task.compute_weighted_residual(VarValues({VarKey.ROBOT: robot.state(q=q, T_world_base=base)})).numpy()


def test_residual_shape_and_nonneg(panda_robot_with_collision):
    robot = panda_robot_with_collision
    task = SelfCollisionTask(robot=robot, weight=1.0, margin=0.0)
    residual = _residual(task, robot, robot.spec.midrange_q.astype(np.float32))[0]
    assert residual.shape == (task.residual_dim,) and float(np.min(residual)) >= 0.0


def test_residual_positive_when_colliding(panda_robot_with_collision):
    robot = panda_robot_with_collision
    task = SelfCollisionTask(robot=robot, weight=1.0, margin=1.0)  # a large margin forces contacts at midrange
    assert float(np.max(_residual(task, robot, robot.spec.midrange_q.astype(np.float32))[0])) > 0.0


def test_jacobian_analytic_vs_exact(panda_robot_with_collision):
    robot = panda_robot_with_collision
    rng = np.random.RandomState(42)
    q = (rng.randn(robot.num_actuated_joints).astype(np.float32) * 0.1 + robot.spec.midrange_q).astype(np.float32)
    base = np.array([[0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0]], np.float32)
    task = SelfCollisionTask(robot=robot, weight=1.0, margin=0.5)
    st = robot.state(q=q, T_world_base=base)
    analytic = task.compute_weighted_jacobian_analytic(VarValues({VarKey.ROBOT: st})).numpy()
    residual = task.compute_weighted_residual(VarValues({VarKey.ROBOT: st})).numpy()

    class _V:
        spec, batch_size, has_floating_base = robot.spec, 1, True

    ro, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(robot.spec), oracle.Terms([task.host_desc(_V)]),
                                      q[None], base)
    assert analytic.shape == Jo.shape
    # slot rows hold the same pairs in the same order (first K penetrating link pairs in link-pair order)
    np.testing.assert_allclose(residual, ro, atol=3e-4, rtol=3e-4)
    assert np.allclose(analytic, Jo, atol=3e-4, rtol=3e-4)


def test_pair_filtering_reduces_pairs(panda_robot_with_collision):
    robot = panda_robot_with_collision
    filtered = SelfCollisionTask(robot=robot, filter_adjacent_links=True)
    every = SelfCollisionTask(robot=robot, filter_adjacent_links=False)
    n = len(robot.spec.local_collision_sphere_centers)
    assert every.num_pairs == n * (n - 1) // 2
    assert filtered.num_pairs < every.num_pairs


def test_batch_consistency(panda_robot_with_collision):
    robot = panda_robot_with_collision
    rng = np.random.RandomState(0)
    q = (rng.randn(4, robot.num_actuated_joints).astype(np.float32) * 0.1 + robot.spec.midrange_q).astype(np.float32)
    batch = _residual(SelfCollisionTask(robot=robot, weight=1.0, margin=0.5), robot, q)
    for i in range(4):
        single = _residual(SelfCollisionTask(robot=robot, weight=1.0, margin=0.5), robot, q[i])[0]
        assert np.allclose(np.sort(batch[i]), np.sort(single), atol=1e-6)


def test_stub_built_by_set_robot_matches_constructed(panda_robot_with_collision):
    robot = panda_robot_with_collision
    q = robot.spec.midrange_q.astype(np.float32)
    stub = copy.deepcopy(SelfCollisionTask(weight=3.0, margin=0.5))
    stub.set_robot(robot)
    built = SelfCollisionTask(robot=robot, weight=3.0, margin=0.5)
    residual = _residual(stub, robot, q)[0]
    expected = _residual(built, robot, q)[0]
    assert stub.num_pairs == built.num_pairs > 0
    assert float(np.max(residual)) > 0.0
    assert np.allclose(np.sort(residual), np.sort(expected), atol=1e-6)
