"""The reference's RobotState tests (tests/robo/test_robot_state.py) through this library's RobotState.

Poses are float32 rows [x, y, z, qw, qx, qy, qz] where the reference has one wp_vec7 element, so a buffer the
reference shapes (B, links) is (B, links, 7) here.  Trajectory states (a frame axis) are outside the IK path.
"""

import numpy as np
import pytest

from robokit_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def robot(panda_spec):
    from robokit_b200.robo.robot import Robot

    return Robot(panda_spec)


def _q(values, na):
    """One row per value, every joint at that value."""
    return np.tile(np.asarray(values, np.float32)[:, None], (1, na))


def test_typed_transform_buffers(gpu, robot):
    """TestTypedTransformBuffers (test_robot_state.py:9-22)."""
    state = robot.state()
    s = robot.spec
    assert state.T_world_base.shape == (1, 7)
    assert state.T_world_joint.shape == (1, s.num_joints, 7)
    assert state.T_world_link.shape == (1, s.num_links, 7)
    np.testing.assert_allclose(state.T_world_base.numpy(), [[0, 0, 0, 1, 0, 0, 0]])


def test_gather_basic(gpu, robot):
    """TestGather.test_gather_basic (test_robot_state.py:26-37)."""
    na = robot.num_actuated_joints
    state = robot.forward_kinematics(robot.state(_q([0.1, 0.2, 0.3], na)))
    g = state.gather(np.array([2, 0], np.int32))
    assert g.q.shape == (2, na)
    np.testing.assert_allclose(g.q.numpy(), [[0.3] * na, [0.1] * na], atol=1e-6)


def test_gather_marks_fk_stale(gpu, robot):
    """TestGather.test_gather_marks_fk_stale (test_robot_state.py:39-72)."""
    na = robot.num_actuated_joints
    home = np.zeros(na)
    home[:min(na, 7)] = [0.0, -1.2, 0.0, -2.0, 0.0, 1.0, 0.0][:na]
    q = np.stack([home, np.linspace(0.1, 0.8, na), np.full(na, 0.2)]).astype(np.float32)
    state = robot.forward_kinematics(robot.state(q))
    g = state.gather(N.DeviceArray.from_numpy(np.array([1, 2, 0], np.int32)))
    assert not g.is_fk_computed
    g = robot.forward_kinematics(g)
    assert g.T_world_link.shape == (3, robot.spec.num_links, 7)
    np.testing.assert_allclose(g.T_world_link.numpy(), state.T_world_link.numpy()[[1, 2, 0]], atol=1e-6)


def test_gather_with_dest(gpu, robot):
    """TestGather.test_gather_with_dest (test_robot_state.py:74-90)."""
    na = robot.num_actuated_joints
    state = robot.forward_kinematics(robot.state(_q([0.1, 0.2, 0.3, 0.4], na)))
    dest = robot.state(N.DeviceArray.empty((2, na)))
    g = state.gather(np.array([3, 1], np.int32), out=dest)
    assert g is dest
    np.testing.assert_allclose(g.q.numpy(), [[0.4] * na, [0.2] * na], atol=1e-6)


def test_gather_rejects_an_index_outside_the_batch(gpu, robot):
    state = robot.state(_q([0.1, 0.2], robot.num_actuated_joints))
    with pytest.raises(IndexError, match="outside a batch of 2"):
        state.gather(np.array([0, 2], np.int32))
    with pytest.raises(IndexError):
        state.gather(np.array([-1], np.int32))


def test_accept_basic(gpu, robot):
    """TestAccept.test_accept_basic (test_robot_state.py:93-122)."""
    na = robot.num_actuated_joints
    src = robot.forward_kinematics(robot.state(_q([0.1, 0.2, 0.3], na)))
    dst = robot.forward_kinematics(robot.state(_q([0.9, 0.8, 0.7], na)))
    dst.accept(np.array([1, 0, 1], np.int32), src)
    np.testing.assert_allclose(dst.q.numpy(), [[0.1] * na, [0.8] * na, [0.3] * na], atol=1e-6)
    np.testing.assert_allclose(dst.T_world_link.numpy()[[0, 2]], src.T_world_link.numpy()[[0, 2]], atol=1e-6)
    assert dst.is_fk_computed and not dst.is_motion_subspace_computed


def test_accept_floating_base_stale_fk(gpu, robot):
    """TestAccept.test_accept_floating_base_stale_fk (test_robot_state.py:124-140)."""
    na = robot.num_actuated_joints
    base = np.tile(np.array([0, 0, 0, 1, 0, 0, 0], np.float32), (3, 1))
    moved = base + np.array([0.5, 0, 0, 0, 0, 0, 0], np.float32)
    dst = robot.state(np.zeros((3, na), np.float32), base)
    src = robot.state(np.full((3, na), 0.1, np.float32), moved)
    assert not dst.is_fk_computed
    dst.accept(np.array([1, 0, 1], np.int32), src)
    np.testing.assert_allclose(dst.q.numpy(), [[0.1] * na, [0.0] * na, [0.1] * na])
    np.testing.assert_allclose(dst.T_world_base.numpy(), [moved[0], base[1], moved[2]])


@pytest.mark.parametrize("floating", [False, True])
def test_unevaluated_copies(gpu, robot, floating):
    """TestLazyTransformBuffers.test_unevaluated_copies (test_robot_state.py:140-161), single-pose states."""
    na = robot.num_actuated_joints
    q = np.arange(3 * na, dtype=np.float32).reshape(3, na) / 100
    base = np.tile(np.array([0, 0, 0, 1, 0, 0, 0], np.float32), (3, 1))
    state = robot.state(q, base if floating else None)
    copies = [state.clone(), state.view(2), state.gather(np.array([2, 0], np.int32))]
    for c in [state, *copies]:
        assert "T_world_joint" not in c.__dict__ and "T_world_link" not in c.__dict__
    np.testing.assert_array_equal(copies[0].q.numpy(), q)
    np.testing.assert_array_equal(copies[1].q.numpy(), q[:2])
    np.testing.assert_array_equal(copies[2].q.numpy(), q[[2, 0]])
    assert copies[0].q.ptr != state.q.ptr and copies[1].q.ptr == state.q.ptr
    robot.forward_kinematics(copies[2])
    assert "T_world_joint" not in state.__dict__ and "T_world_link" not in state.__dict__


def test_copies_and_shared_views(gpu, robot):
    """TestLazyTransformBuffers.test_copies_and_shared_views (test_robot_state.py:163-194), single-pose states."""
    na = robot.num_actuated_joints
    state = robot.state(np.arange(3 * na, dtype=np.float32).reshape(3, na) / 100)
    view = state.view(2)
    for name in ("T_world_joint", "T_world_link"):
        assert name not in state.__dict__
        assert getattr(view, name).ptr == getattr(state, name).ptr
    robot.forward_kinematics(state)
    clone = state.clone()
    idx = np.array([2, 0], np.int32)
    gathered = state.gather(idx, q_only=False)
    for name in ("T_world_joint", "T_world_link"):
        expected = getattr(state, name).numpy()
        np.testing.assert_array_equal(getattr(view, name).numpy(), expected[:2])
        np.testing.assert_array_equal(getattr(clone, name).numpy(), expected)
        np.testing.assert_array_equal(getattr(gathered, name).numpy(), expected[[2, 0]])
        assert getattr(clone, name).ptr != getattr(state, name).ptr
    assert clone.is_fk_computed and gathered.is_fk_computed
    q_only = state.gather(idx)
    assert "T_world_joint" not in q_only.__dict__ and "T_world_link" not in q_only.__dict__
    robot.forward_kinematics(q_only)
    np.testing.assert_array_equal(q_only.T_world_link.numpy(), gathered.T_world_link.numpy())
    cold = robot.state(np.zeros((3, na), np.float32))
    cold.gather(idx, out=gathered, q_only=False)
    for name in ("T_world_joint", "T_world_link"):
        np.testing.assert_array_equal(getattr(gathered, name).numpy(), getattr(cold, name).numpy()[[2, 0]])
    assert not gathered.is_fk_computed


def test_fk_on_a_view_writes_the_source_rows(gpu, robot):
    """A view's forward kinematics lands in its rows of the source's buffers (the storage sharing the reference's
    graph-replay test relies on, test_robot_state.py:196-208)."""
    na = robot.num_actuated_joints
    state = robot.state(np.zeros((4, na), np.float32))
    robot.forward_kinematics(state)
    state.q.assign(np.full((4, na), 0.2, np.float32))
    view = state.view(2, offset=1)
    robot.forward_kinematics(view)
    expected = robot.forward_kinematics(robot.state(np.full((1, na), 0.2, np.float32))).T_world_link.numpy()[0]
    got = state.T_world_link.numpy()
    np.testing.assert_array_equal(got[1], expected)
    np.testing.assert_array_equal(got[2], expected)
    zero = robot.forward_kinematics(robot.state(np.zeros((1, na), np.float32))).T_world_link.numpy()[0]
    np.testing.assert_array_equal(got[0], zero)
    np.testing.assert_array_equal(got[3], zero)


def _frees_without_gc(build):
    """tests/test_frees_without_gc.py:24-29: the object dies by refcount alone, with the collector off."""
    import gc
    import weakref

    gc.disable()
    try:
        ref = weakref.ref(build())
        return ref() is None
    finally:
        gc.enable()


def test_solved_optimizer_and_ik_solver_free_without_gc(gpu, panda_arm_spec):
    """A solved LMOptimizer and an IKSolver that captured its solve graph hold no reference cycles, so their device
    buffers, problems and graphs are released as soon as the last reference goes."""
    from robokit_b200.helpers.ik import IKSolver, presets
    from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
    from robokit_b200.robo.robot import Robot
    from robokit_b200.terms.dense import PositionLimit, PositionTask

    robot = Robot(panda_arm_spec)
    hand = robot.link_names.index("panda_hand")
    q = robot.sample_q(8, seed=1)
    T = robot.forward_kinematics(robot.state(q)).get_T_world_link(hand).numpy().reshape(8, 1, 7)

    def optimizer():
        opt = LMOptimizer([PositionTask(robot, hand, T, weight=1.0), PositionLimit(robot, weight=1.0)],
                          LMOptimizerConfig(max_iter=5))
        opt.solve(VarValues({VarKey.ROBOT: robot.state(np.zeros_like(q))}))
        return opt

    def solver():
        ik = IKSolver(presets.basic, robot, "panda_hand")
        ik.solve(T)
        ik.solve(T)  # the second solve replays the captured graph
        return ik

    assert _frees_without_gc(optimizer)
    assert _frees_without_gc(solver)
