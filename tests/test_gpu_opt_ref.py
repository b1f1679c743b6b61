"""The reference's own LMOptimizer tests (tests/opt/test_optimizer.py) run against this library.  The UR10
of the originals has no URDF here; the Panda stands in where the test is about the optimizer, not the robot."""

import numpy as np
import pytest

from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
from robokit_b200.terms.dense import FrameTask, PositionLimit, PositionTask

pytestmark = pytest.mark.gpu


def _target_pose(values=(0.5, 0.3, 0.4, 1.0, 0.0, 0.0, 0.0), batch_size=1):
    return np.tile(np.asarray(values, np.float32), (batch_size, 1))[:, None]


@pytest.fixture
def panda(gpu, panda_spec):
    from robokit_b200.robo.robot import Robot

    return Robot(panda_spec)


def test_mobile_ik_with_base_pose(panda):  # test_optimizer.py:165-228
    robot = panda
    base = np.array([0.3, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0], np.float32).reshape(1, 7)
    q = robot.spec.midrange_q.reshape(1, -1).astype(np.float32)
    target = np.array([0.6, 0.0, 0.55, 0.0, 0.707, 0.0, -0.707], np.float32).reshape(1, 1, 7)
    frame_index = robot.link_names.index("panda_hand")
    terms = [FrameTask(robot=robot, frame_index=frame_index, T_world_target=target, position_weight=10.0,
                       orientation_weight=2.0),
             PositionLimit(robot=robot, weight=2.0)]
    cfg = LMOptimizerConfig(max_iter=50, lm_lambda=1.0, lambda_factor=2.0, lambda_min=1e-6, lambda_max=1e6)
    opt = LMOptimizer(terms=terms, config=cfg)
    state = robot.state(q=q, T_world_base=base)
    state = opt.solve(VarValues({VarKey.ROBOT: state}))[0].get(VarKey.ROBOT)
    state = robot.forward_kinematics(state)
    T = state.get_T_world_link(frame_index).numpy()
    assert np.allclose(T[..., :3], target[:, 0, :3], atol=1e-3)
    assert np.abs(np.sum(T[..., 3:] * target[:, 0, 3:])) > 0.999
    assert state.T_world_base is not None and state.q.shape == (1, robot.num_actuated_joints)


def _frame_task(robot, batch_size=1, pw=1.0, ow=0.5):
    return FrameTask(robot=robot, frame_index=robot.link_names.index("panda_hand"),
                     T_world_target=_target_pose(batch_size=batch_size), position_weight=pw, orientation_weight=ow)


def test_max_iter_zero_populates_current_cost(panda):  # :257-320
    robot = panda
    task = _frame_task(robot)
    q0 = robot.spec.zero_q.reshape(1, -1).astype(np.float32)
    r = task.compute_weighted_residual(VarValues({VarKey.ROBOT: robot.state(q=q0)})).numpy()
    expected = 0.5 * float(np.sum(r ** 2))
    assert expected > 1e-3
    for form in ("plain", "persistent"):
        opt = LMOptimizer(terms=[task], config=LMOptimizerConfig(max_iter=0, early_stopping_interval=0, form=form))
        _, costs = opt.solve(VarValues({VarKey.ROBOT: robot.state(q=q0)}))
        assert costs is opt.costs
        assert abs(float(costs.numpy()[0]) - expected) / expected < 1e-3


def test_smaller_batch_runs_as_a_prefix(panda):  # :322-335
    robot = panda
    opt = LMOptimizer(terms=[_frame_task(robot, 2, 10.0, 2.0)], config=LMOptimizerConfig(max_iter=5,
                                                                                       early_stopping_interval=0))
    opt.solve(VarValues({VarKey.ROBOT: robot.state(q=np.tile(robot.spec.zero_q, (2, 1)).astype(np.float32))}))
    assert opt.costs.shape == (2,)
    opt.terms = [_frame_task(robot, 1, 10.0, 2.0)]
    opt.solve(VarValues({VarKey.ROBOT: robot.state(q=robot.spec.zero_q.reshape(1, -1).astype(np.float32))}))
    assert opt.costs.shape == (1,)


@pytest.mark.parametrize("graph", ["none", "iter"])
def test_growing_past_capacity_raises(panda, graph):  # :337-354
    robot = panda
    opt = LMOptimizer(terms=[_frame_task(robot, 1, 10.0, 2.0)],
                      config=LMOptimizerConfig(max_iter=5, early_stopping_interval=0, cuda_graph_mode=graph))
    opt.solve(VarValues({VarKey.ROBOT: robot.state(q=robot.spec.zero_q.reshape(1, -1).astype(np.float32))}))
    opt.terms = [_frame_task(robot, 2, 10.0, 2.0)]
    with pytest.raises(ValueError, match="batch size 2 exceeds"):
        opt.solve(VarValues({VarKey.ROBOT: robot.state(q=np.tile(robot.spec.zero_q, (2, 1)).astype(np.float32))}))


def test_lm_optimizer_rejects_active_dof_mask_shape(panda):  # :356-364
    robot = panda
    state = robot.state(q=np.zeros((1, robot.num_actuated_joints), np.float32))
    opt = LMOptimizer(PositionLimit(robot=robot), active_dof_mask=np.ones(state.tangent_dim + 1, np.float32))
    with pytest.raises(ValueError, match="active_dof_mask"):
        opt.reset(VarValues({VarKey.ROBOT: state}))


def test_active_dof_mask_matches_reduced_problem(panda):  # :366-429 (one step(), whose delta this API exposes)
    robot = panda
    task = _frame_task(robot, 1, 10.0, 2.0)
    q0 = robot.spec.midrange_q.reshape(1, -1).astype(np.float32)
    D = robot.state(q=q0).tangent_dim
    frozen = 1
    mask = np.ones(D, np.float32)
    mask[frozen] = 0.0
    lam = 1e-2
    opt = LMOptimizer(terms=[task], config=LMOptimizerConfig(max_iter=1, lm_lambda=lam, early_stopping_interval=0),
                      active_dof_mask=mask)
    vv = VarValues({VarKey.ROBOT: robot.state(q=q0)})
    opt.reset(vv)
    opt.step(vv)
    ref = VarValues({VarKey.ROBOT: robot.state(q=q0)})
    J = task.compute_weighted_jacobian(ref).numpy()[0]
    r = task.compute_weighted_residual(ref).numpy()[0]
    Jm = J * mask[None]
    expected = np.linalg.solve(Jm.T @ Jm + lam * np.eye(D), -Jm.T @ r)
    got = opt.delta.numpy()[0]
    assert abs(got[frozen]) < 1e-6
    assert np.max(np.abs(got[mask.astype(bool)] - expected[mask.astype(bool)])) < 1e-4


def test_active_dof_mask_freezes_world_base_translation(panda):  # :431-463 (the LM part)
    robot = panda
    target = _target_pose((1.5, 0.0, 0.5, 1.0, 0.0, 0.0, 0.0))
    task = PositionTask(robot=robot, frame_index=robot.link_names.index("panda_hand"), T_world_target=target,
                        weight=1.5)
    base = np.array([[0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0]], np.float32)
    q0 = robot.spec.midrange_q.reshape(1, -1).astype(np.float32)
    D = 6 + robot.num_actuated_joints
    mask = np.ones(D, np.float32)
    mask[0] = mask[1] = 0.0
    opt = LMOptimizer(terms=[task], config=LMOptimizerConfig(max_iter=20, lm_lambda=1.0, early_stopping_interval=0),
                      active_dof_mask=mask)
    state = robot.state(q=q0, T_world_base=base.copy())
    opt.solve(VarValues({VarKey.ROBOT: state}))
    assert np.linalg.norm(state.T_world_base.numpy()[0, :2]) < 1e-4
