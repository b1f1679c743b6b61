"""PopulationSolver (opt/population_solver.py:148-404) on the IK path against its definition: LM stages on the
candidates, each instance's best kept between stages by a stable sort of the costs, the cheapest returned."""

from dataclasses import replace

import numpy as np
import pytest

import oracle
from robokit_b200.opt import (LMOptimizer, LMOptimizerConfig, PopulationSolver, PopulationSolverConfig, Stage, VarKey,
                              VarValues)
from robokit_b200.terms.dense import PositionLimit, PositionTask, RotationTask

pytestmark = pytest.mark.gpu

B, C = 16, 8


def _setup(spec, seed=0):
    from robokit_b200.robo.robot import Robot

    robot = Robot(spec)
    hand = robot.link_names.index("panda_hand")
    T = robot.forward_kinematics(robot.state(robot.sample_q(B, seed=seed))).get_T_world_link(hand).numpy()
    terms = [PositionTask(robot, hand, T.reshape(B, 1, 7), weight=20.0),
             RotationTask(robot, hand, T.reshape(B, 1, 7), weight=10.0), PositionLimit(robot, weight=50.0)]
    q0 = robot.sample_q(B * C, seed=seed + 1)
    return robot, terms, q0


def _stage_lm(terms, lm, iters, robot, q):
    opt = LMOptimizer(terms, replace(lm, max_iter=iters, early_stopping_interval=0, form="persistent"))
    vv, cost = opt.solve(VarValues({VarKey.ROBOT: robot.state(q)}))
    return vv.get(VarKey.ROBOT).q.numpy().copy(), cost.numpy().copy()


def _keep(q, cost, width, keep):
    order = np.argsort(cost.reshape(B, width), axis=1, kind="stable")[:, :keep]
    rows = (np.arange(B)[:, None] * width + order).reshape(-1)
    return q[rows], cost[rows]


@pytest.mark.parametrize("mode", ["none", "full"])
def test_population_solver_matches_its_definition(gpu, panda_arm_spec, mode):
    robot, terms, q0 = _setup(panda_arm_spec)
    lm0, lm1 = LMOptimizerConfig(lm_lambda=10.0), LMOptimizerConfig(lm_lambda=1.0)
    cfg = PopulationSolverConfig(stages=[Stage(6, C, lm0), Stage(4, 2, lm1), Stage(0, 1)], cuda_graph_mode=mode)
    solver = PopulationSolver(terms, cfg)
    var = VarValues({VarKey.ROBOT: robot.state(q0)})
    for _ in range(2):  # the second solve replays the captured graph under "full"
        best, costs = solver.solve(var)
        q_best, c_best = best.get(VarKey.ROBOT).q.numpy().copy(), costs.numpy().copy()
        q1, c1 = _stage_lm(terms, lm0, 6, robot, q0)
        q1, _ = _keep(q1, c1, C, 2)
        q2, c2 = _stage_lm(terms, lm1, 4, robot, q1)
        want_q, want_c = _keep(q2, c2, 2, 1)
        np.testing.assert_array_equal(q_best, want_q)
        np.testing.assert_array_equal(c_best, want_c)
        assert solver.final_var.get(VarKey.ROBOT).batch_size == B


def test_population_solver_rank_final_and_costs(gpu, panda_arm_spec):
    robot, terms, q0 = _setup(panda_arm_spec, seed=4)
    cfg = PopulationSolverConfig(stages=[Stage(6, C, LMOptimizerConfig(lm_lambda=10.0)), Stage(3, 4)],
                                 cuda_graph_mode="none", rank_final=True)
    solver = PopulationSolver(terms, cfg)
    best, costs = solver.solve(VarValues({VarKey.ROBOT: robot.state(q0)}))
    final = solver.final_var.get(VarKey.ROBOT)
    assert final.batch_size == 4 * B
    fq = final.q.numpy()
    c = solver.compute_costs(solver.final_var)
    assert set(c) == {"position_task", "rotation_task", "position_limit"}
    total = sum(v.numpy() for v in c.values()).reshape(B, 4)
    assert np.all(np.diff(total, axis=1) >= -1e-6 * np.abs(total[:, 1:]) - 1e-12)  # best first per instance
    np.testing.assert_array_equal(best.get(VarKey.ROBOT).q.numpy(), fq[::4])
    np.testing.assert_allclose(costs.numpy(), 0.5 * total[:, 0], rtol=1e-5, atol=1e-12)

    class _V:
        spec, batch_size, has_floating_base = panda_arm_spec, 4 * B, False

    rob = oracle.Robot.from_spec(panda_arm_spec)
    for t in terms:
        r, _ = oracle.residual_jacobian(rob, oracle.Terms([t.host_desc(_V)]), fq, None)
        # FP32 residuals: a weight-20 position row carries ~1e-6 absolute rounding, ~3e-6 once squared
        np.testing.assert_allclose(c[t.cost_name].numpy(), np.sum(r ** 2, axis=1), rtol=2e-5, atol=1e-5)


def test_population_solver_rejects_a_ragged_batch(gpu, panda_arm_spec):
    robot, terms, q0 = _setup(panda_arm_spec)
    solver = PopulationSolver(terms, PopulationSolverConfig(stages=[Stage(2, C)]))
    with pytest.raises(ValueError, match="not a multiple of num_candidates"):
        solver.solve(VarValues({VarKey.ROBOT: robot.state(q0[:C * B - 1])}))
    with pytest.raises(ValueError, match="CUDA only"):
        PopulationSolver(terms, PopulationSolverConfig(), device="cpu")


def test_replay_solves_each_new_population(gpu, panda_arm_spec):
    """TestCpuReplay.test_replay_solves_each_new_population (tests/opt/test_population_solver.py:266-285) on the
    GPU: under "full" the recorded solve reads the population's buffers at replay, so new values written into
    the same var give that population's solution; a new var is recorded again."""
    robot, terms, q0 = _setup(panda_arm_spec, seed=7)
    stages = [Stage(3, C, LMOptimizerConfig(lm_lambda=10.0)), Stage(2, 1)]
    solver = PopulationSolver(terms, PopulationSolverConfig(stages=stages, cuda_graph_mode="full"))
    var = VarValues({VarKey.ROBOT: robot.state(q0)})
    solver.solve(var)
    q_new = robot.sample_q(B * C, seed=99)
    var.get(VarKey.ROBOT).q.assign(q_new)
    replayed = solver.solve(var)[0].get(VarKey.ROBOT).q.numpy().copy()
    fresh = PopulationSolver(terms, PopulationSolverConfig(stages=stages, cuda_graph_mode="none"))
    want = fresh.solve(VarValues({VarKey.ROBOT: robot.state(q_new)}))[0].get(VarKey.ROBOT).q.numpy()
    np.testing.assert_array_equal(replayed, want)
    other = solver.solve(VarValues({VarKey.ROBOT: robot.state(q0)}))[0].get(VarKey.ROBOT).q.numpy().copy()
    first = fresh.solve(VarValues({VarKey.ROBOT: robot.state(q0)}))[0].get(VarKey.ROBOT).q.numpy()
    np.testing.assert_array_equal(other, first)
