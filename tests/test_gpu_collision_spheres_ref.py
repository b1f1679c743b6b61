"""The reference's collision-sphere tests (tests/robo/test_collision_spheres.py) through this library.

World sphere centres come from the same forward-kinematics launch as the link poses; the reference point is
each sphere's local centre moved by its link's world pose, computed here on the host in FP64.
"""

import numpy as np
import pytest

from robokit_b200.robo.robot_spec import quaternion_to_matrix

pytestmark = pytest.mark.gpu


def _robot(spec):
    from robokit_b200.robo.robot import Robot

    return Robot(spec)


def _reference_centers(T_world_link, local, links):
    """se3_apply of each sphere's link pose to its local centre (test_collision_spheres.py:10-26)."""
    out = np.zeros((T_world_link.shape[0], len(links), 3))
    for b in range(T_world_link.shape[0]):
        for i, (c, l) in enumerate(zip(local, links)):
            T = T_world_link[b, l].astype(np.float64)
            out[b, i] = quaternion_to_matrix(T[3:]) @ c + T[:3]
    return out


@pytest.mark.parametrize("rows", [1, 4])
def test_world_collision_spheres_match_the_link_poses(gpu, panda_collision_spec, rows):
    """test_world_collision_spheres_correctness_single / _batch_shape_and_values (test_collision_spheres.py:29-62)."""
    robot = _robot(panda_collision_spec)
    spec = panda_collision_spec
    assert spec.has_collision_spheres
    state = robot.state() if rows == 1 else robot.state(robot.sample_q(num_samples=rows, seed=0))
    state = robot.transform_collision_spheres(robot.forward_kinematics(state))
    got = state.collision_sphere_centers_world.numpy()
    assert got.shape == (rows, spec.local_collision_sphere_centers.shape[0], 3)
    ref = _reference_centers(state.T_world_link.numpy(), spec.local_collision_sphere_centers,
                             spec.collision_spheres_link_indices)
    np.testing.assert_allclose(got, ref, atol=1e-5)


def test_world_collision_spheres_change_with_the_base(gpu, panda_collision_spec):
    """test_world_collision_spheres_changes_with_base_transform (test_collision_spheres.py:64-80)."""
    robot = _robot(panda_collision_spec)
    q = panda_collision_spec.zero_q[None].astype(np.float32)
    a = robot.transform_collision_spheres(robot.forward_kinematics(robot.state(q))).collision_sphere_centers_world
    base = np.array([[1.0, 2.0, 3.0, 0.7071, 0.0, 0.7071, 0.0]], np.float32)
    sb = robot.transform_collision_spheres(robot.forward_kinematics(robot.state(q, base)))
    b = sb.collision_sphere_centers_world.numpy()
    assert a.numpy().shape == b.shape and not np.allclose(a.numpy(), b)
    ref = _reference_centers(sb.T_world_link.numpy(), panda_collision_spec.local_collision_sphere_centers,
                             panda_collision_spec.collision_spheres_link_indices)
    np.testing.assert_allclose(b, ref, atol=1e-5)


def test_world_collision_spheres_invalidated_by_integrate(gpu, panda_collision_spec):
    """test_world_collision_spheres_invalidation_on_integrate (test_collision_spheres.py:82-97)."""
    robot = _robot(panda_collision_spec)
    state = robot.transform_collision_spheres(robot.forward_kinematics(robot.state()))
    assert state.is_collision_spheres_computed
    nxt = state.integrate(np.zeros((state.batch_size, state.tangent_dim), np.float32))
    assert not nxt.is_collision_spheres_computed
    nxt = robot.transform_collision_spheres(robot.forward_kinematics(nxt))
    assert nxt.is_collision_spheres_computed
    assert nxt.collision_sphere_centers_world.numpy().shape[0] == nxt.num_elements


def test_world_collision_spheres_empty_without_spheres(gpu, panda_spec):
    """test_world_collision_spheres_zero_length_when_not_loaded (test_collision_spheres.py:99-106)."""
    robot = _robot(panda_spec)
    assert not panda_spec.has_collision_spheres
    state = robot.forward_kinematics(robot.state())
    assert state.collision_sphere_centers_world.shape[1] == 0
    assert not state.is_collision_spheres_computed


def test_link_bounding_spheres_contain_their_spheres(gpu, panda_collision_spec):
    """test_link_bounding_spheres_lazy_field (test_collision_spheres.py:108-123)."""
    spec = panda_collision_spec
    centers, radii = spec.local_link_bounding_sphere_centers, spec.link_bounding_sphere_radii
    assert centers.shape == (spec.num_links, 3) and radii.shape == (spec.num_links,)
    for c, r, link in zip(spec.local_collision_sphere_centers, spec.collision_sphere_radii,
                          spec.collision_spheres_link_indices):
        assert np.linalg.norm(c - centers[link]) + r <= radii[link] + 1e-5
