"""End-to-end LM solves on the GPU: parity with the oracle, forms, determinism, capacity, status."""

import numpy as np
import pytest

import oracle
from robokit_b200 import configs
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues

pytestmark = pytest.mark.gpu


def _solve(cfg, form="plain", q0=None, base0=None, group=0, **lm_overrides):
    wl = cfg.workload
    lm = cfg.lm if not lm_overrides and form == cfg.lm.form else \
        LMOptimizerConfig(**{**cfg.lm.__dict__, "form": form, **lm_overrides})
    opt = LMOptimizer(cfg.terms, lm)
    st = cfg.robot.state(wl.q0 if q0 is None else q0, wl.base0 if base0 is None else base0)
    vv = VarValues({VarKey.ROBOT: st})
    if group:
        opt.reset(vv)
        opt.set_schedule(group)
    opt.solve(vv)
    base = st.T_world_base.numpy() if st.has_floating_base else None
    return st.q.numpy(), base, opt.costs.numpy(), opt.iterations.numpy(), opt.status.numpy()


def _oracle_solve(cfg, **over):
    lm = cfg.lm
    rules = 0
    if lm.step_tol:
        rules |= 2
    if lm.pose_tol:
        rules |= 4
    kw = dict(max_iter=lm.max_iter, lambda_init=lm.lm_lambda, lambda_factor=lm.lambda_factor,
              lambda_min=lm.lambda_min, lambda_max=lm.lambda_max, rho_min=lm.rho_min,
              gain_ratio_epsilon=lm.gain_ratio_epsilon, stop_rules=rules, step_tol=lm.step_tol or 0.0)
    kw.update(over)
    rob = oracle.Robot.from_spec(cfg.workload.spec)
    out = oracle.solve(rob, oracle.Terms(configs.oracle_terms(cfg)), oracle.params(**kw), cfg.workload.q0,
                       cfg.workload.base0, threads=8)
    return rob, out


def _success(rob, cfg, q, base, pos=1e-3, rot=0.01):
    pe, re, ok = oracle.metrics(rob, q, base, cfg.workload.target_links, cfg.workload.targets, pos, rot)
    return pe, re, ok


@pytest.mark.parametrize("name,B,tol", [("chain7", 512, 0.05), ("chain7c", 512, 0.06), ("humanoid", 256, 0.06)])
def test_end_to_end_matches_oracle(gpu, name, B, tol):
    """Success rate within `tol` of the FP64 oracle; where both succeed the final errors agree within 1e-4 m / 1e-3 rad."""
    cfg = configs.make(name, B, seed=11)
    q, base, cost, iters, status = _solve(cfg)
    rob, o = _oracle_solve(cfg)
    pe_g, re_g, ok_g = _success(rob, cfg, q, base)
    pe_o, re_o, ok_o = _success(rob, cfg, o["q"], o["base"])
    assert abs(ok_g.mean() - ok_o.mean()) <= tol, (ok_g.mean(), ok_o.mean())
    both = ok_g & ok_o
    assert both.sum() > 0.3 * B * min(ok_g.mean(), ok_o.mean()) / max(ok_g.mean(), 1e-9) or both.sum() > 10
    assert np.all(np.abs(pe_g[both] - pe_o[both]) < 1e-4)
    assert np.all(np.abs(re_g[both] - re_o[both]) < 1e-3)
    # with at most one redundant direction most trajectories make identical decisions, so final joint
    # vectors agree; the 35-DoF humanoid with 30 rows drifts along its null space and is compared by pose only
    if name != "humanoid":
        close = np.all(np.abs(q - o["q"]) < 1e-3, axis=1)
        assert close.mean() > 0.5, close.mean()


def test_hand_error_vs_fp64_oracle(gpu):
    """The hand config reports the per-problem keypoint error against the FP64 oracle's solution."""
    cfg = configs.make("hand", 256, seed=2)
    q, base, cost, iters, status = _solve(cfg)
    rob, o = _oracle_solve(cfg)
    links = cfg.workload.target_links
    kg = oracle.fk(rob, q, base)["T_link"][:, links, :3]
    ko = oracle.fk(rob, o["q"], o["base"])["T_link"][:, links, :3]
    err = np.linalg.norm(kg - ko, axis=2).max(axis=1)
    assert np.median(err) < 1e-4, np.median(err)
    assert np.mean(err < 1e-3) > 0.9
    np.testing.assert_allclose(np.median(cost), np.median(o["cost"]), rtol=0.05)


@pytest.mark.parametrize("name,B", [("chain7c", 300), ("humanoid", 100), ("hand", 100)])
def test_persistent_equals_plain(gpu, name, B):
    """Same per-problem arithmetic: the persistent work-queue form is bitwise equal to the plain form."""
    cfg = configs.make(name, B, seed=5)
    a = _solve(cfg, "plain", step_tol=1e-6)
    b = _solve(cfg, "persistent", step_tol=1e-6)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[2], b[2])
    np.testing.assert_array_equal(a[3], b[3])


def test_result_alone_equals_result_in_mix(gpu):
    """A problem solved alone, in a small batch, or inside a large mixed batch gives the same bits."""
    cfg = configs.make("chain7c", 200, seed=9)
    full = _solve(cfg, "persistent", step_tol=1e-6)
    idx = np.array([3, 17, 64, 101, 150, 199])
    from robokit_b200.terms.dense import PositionLimit, PositionTask, RotationTask, SelfCollisionTask

    wl = cfg.workload
    sub_targets = wl.targets[idx]
    ee = wl.target_links[0]
    terms = [PositionTask(cfg.robot, ee, sub_targets, weight=1.0), RotationTask(cfg.robot, ee, sub_targets, weight=1.0),
             SelfCollisionTask(cfg.robot, weight=1.0, margin=0.02, pair_mode="all"), PositionLimit(cfg.robot, weight=1.0)]
    lm = LMOptimizerConfig(**{**cfg.lm.__dict__, "form": "persistent"})
    for k, i in enumerate(idx):
        opt = LMOptimizer([t for t in terms], lm)
        # alone: one problem, its own target row
        t1 = [PositionTask(cfg.robot, ee, sub_targets[k:k + 1], weight=1.0),
              RotationTask(cfg.robot, ee, sub_targets[k:k + 1], weight=1.0), terms[2], terms[3]]
        opt = LMOptimizer(t1, lm)
        st = cfg.robot.state(wl.q0[i:i + 1])
        opt.solve(VarValues({VarKey.ROBOT: st}))
        np.testing.assert_array_equal(st.q.numpy()[0], full[0][i])
    opt = LMOptimizer(terms, lm)
    st = cfg.robot.state(wl.q0[idx])
    opt.solve(VarValues({VarKey.ROBOT: st}))
    np.testing.assert_array_equal(st.q.numpy(), full[0][idx])


def test_prefix_batch_matches_fresh_optimizer(gpu):
    """tests/opt/test_varied_batch.py:72-83: a capacity-N optimizer solving a prefix equals a fresh one."""
    cfg = configs.make("chain7", 64, seed=4)
    wl = cfg.workload
    lm = LMOptimizerConfig(max_iter=10, lm_lambda=1e-3, lambda_factor=10.0)
    from robokit_b200.terms.dense import PositionTask, RotationTask

    def terms(n):
        return [PositionTask(cfg.robot, wl.target_links[0], wl.targets[:n], weight=1.0),
                RotationTask(cfg.robot, wl.target_links[0], wl.targets[:n], weight=1.0)]

    big = LMOptimizer(terms(64), lm)
    big.solve(VarValues({VarKey.ROBOT: cfg.robot.state(wl.q0)}))
    for n in (16, 4, 64):
        st = cfg.robot.state(wl.q0[:n])
        big.solve(VarValues({VarKey.ROBOT: st}))
        q_prefix, c_prefix = st.q.numpy(), big.costs.numpy()
        fresh = LMOptimizer(terms(n), lm)
        st2 = cfg.robot.state(wl.q0[:n])
        fresh.solve(VarValues({VarKey.ROBOT: st2}))
        np.testing.assert_array_equal(q_prefix, st2.q.numpy())
        np.testing.assert_array_equal(c_prefix, fresh.costs.numpy())


def test_growing_past_capacity_raises(gpu):
    cfg = configs.make("chain7", 16, seed=4)
    opt = LMOptimizer(cfg.terms, cfg.lm)
    opt.solve(VarValues({VarKey.ROBOT: cfg.robot.state(cfg.workload.q0[:4])}))
    with pytest.raises(ValueError, match="batch"):
        opt.solve(VarValues({VarKey.ROBOT: cfg.robot.state(cfg.workload.q0)}))


def test_all_cost_rule_stops_like_the_reference(gpu):
    """opt/optimizer.py:237-239: iterate every problem until all costs <= cost_tol, then stop."""
    cfg = configs.make("chain7", 64, seed=1)
    lm = LMOptimizerConfig(max_iter=100, lm_lambda=1e-3, lambda_factor=10.0, early_stopping_interval=1,
                           cost_tol=1e5)
    opt = LMOptimizer(cfg.terms, lm)
    st = cfg.robot.state(cfg.workload.q0)
    opt.solve(VarValues({VarKey.ROBOT: st}))
    its = opt.iterations.numpy()
    assert np.all(its == 1), its  # every start cost is below 1e5, so the check after step 1 stops the solve
    lm2 = LMOptimizerConfig(max_iter=30, lm_lambda=1e-3, lambda_factor=10.0, early_stopping_interval=1,
                            cost_tol=1e-30)
    opt2 = LMOptimizer(cfg.terms, lm2)
    st2 = cfg.robot.state(cfg.workload.q0)
    opt2.solve(VarValues({VarKey.ROBOT: st2}))
    assert np.all(opt2.iterations.numpy() == 30)
    rob, o = _oracle_solve(cfg, max_iter=30, stop_rules=1, cost_tol=1e-30)
    assert np.all(o["iters"] == 30)


@pytest.mark.parametrize("name,widths", [("chain7c", (8, 16, 32)), ("humanoid", (16, 32))])
def test_group_widths_agree(gpu, name, widths):
    cfg = configs.make(name, 64, seed=3)
    res = [_solve(cfg, group=G, step_tol=1e-6) for G in widths]
    rob = oracle.Robot.from_spec(cfg.workload.spec)
    rates = [_success(rob, cfg, r[0], r[1])[2].mean() for r in res]
    assert max(rates) - min(rates) <= 0.1, rates
    if name != "humanoid":
        for r in res[1:]:
            close = np.all(np.abs(r[0] - res[0][0]) < 1e-3, axis=1)
            assert close.mean() > 0.7


def test_oversized_group_is_refused(gpu):
    """A width whose workspaces do not fit one block's shared memory is an error, not a silent change."""
    from robokit_b200 import _native as N

    from robokit_b200.robo.robot import Robot
    from robokit_b200.robo.synthetic import serial_chain
    from robokit_b200.terms.dense import PositionTask

    spec = serial_chain(seed=1, dofs=60)  # 60x60 normal equations: one 8-lane workspace is ~35 KB
    robot = Robot(spec)
    targets = np.tile(np.array([0.1, 0.2, 0.3, 1, 0, 0, 0], np.float32), (4, 1, 1))
    opt = LMOptimizer([PositionTask(robot, spec.num_links - 1, targets)], LMOptimizerConfig(max_iter=2))
    opt.reset(VarValues({VarKey.ROBOT: robot.state(np.zeros((4, 60), np.float32))}))
    with pytest.raises(N.NativeError, match="shared memory"):
        opt.set_schedule(8)
    opt.set_schedule(32)


def test_nonfinite_start_is_reported(gpu):
    from robokit_b200 import _native as N

    cfg = configs.make("chain7", 8, seed=0)
    tg = cfg.workload.targets.copy()
    tg[3, 0, 0] = np.nan
    from robokit_b200.terms.dense import PositionTask, RotationTask

    terms = [PositionTask(cfg.robot, cfg.workload.target_links[0], tg, weight=1.0),
             RotationTask(cfg.robot, cfg.workload.target_links[0], tg, weight=1.0)]
    opt = LMOptimizer(terms, LMOptimizerConfig(max_iter=5, early_stopping_interval=0))
    st = cfg.robot.state(cfg.workload.q0)
    opt.solve(VarValues({VarKey.ROBOT: st}))
    status = opt.status.numpy()
    assert status[3] & N.IK_ST_NONFINITE
    assert not (status[2] & N.IK_ST_NONFINITE)
    assert np.all(np.isfinite(st.q.numpy()))


def test_pose_stop_rule(gpu):
    cfg = configs.make("chain7", 128, seed=6)
    q, base, cost, iters, status = _solve(cfg, "persistent", pose_tol=(1e-4, 1e-4), max_iter=100)
    rob = oracle.Robot.from_spec(cfg.workload.spec)
    pe, re, ok = _success(rob, cfg, q, base, 1e-4 * 1.01, 1e-4 * 1.01)
    conv = (status & 1) != 0
    assert conv.mean() > 0.5
    assert np.all(ok[conv])
    assert np.all(iters[~conv] == 100)


@pytest.mark.parametrize("form", ["plain", "persistent"])
def test_graph_mode_equals_direct_launches(gpu, form):
    """cuda_graph_mode "full": the solve is recorded once and replayed; results equal direct launches bitwise."""
    cfg = configs.make("chain7c", 200, seed=6)
    outs = []
    for mode in ("none", "full"):
        lm = LMOptimizerConfig(**{**cfg.lm.__dict__, "form": form, "cuda_graph_mode": mode})
        opt = LMOptimizer(cfg.terms, lm)
        st = cfg.robot.state(cfg.workload.q0)
        res = []
        for _ in range(2):  # the second "full" solve replays the recorded graph
            st.q.copy_from_numpy(cfg.workload.q0)
            opt.solve(VarValues({VarKey.ROBOT: st}))
            res.append((st.q.numpy(), opt.costs.numpy(), opt.iterations.numpy()))
        outs.append(res)
        if mode == "full":
            assert opt._graph is not None
    for a, b in zip(outs[0], outs[1]):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
