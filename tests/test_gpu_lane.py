"""The one-lane-per-problem schedule of the whole-solve kernels (small systems, D <= 8)."""

import numpy as np
import pytest

import oracle
from robokit_b200 import _native as N
from robokit_b200 import configs
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues

pytestmark = pytest.mark.gpu


def _solve(cfg, form, lanes, **over):
    lm = LMOptimizerConfig(**{**cfg.lm.__dict__, "form": form, **over})
    opt = LMOptimizer(cfg.terms, lm)
    st = cfg.robot.state(cfg.workload.q0, cfg.workload.base0)
    vv = VarValues({VarKey.ROBOT: st})
    opt.reset(vv)
    opt.set_schedule(lanes)
    assert opt.problem.schedule()[0] == lanes
    opt.solve(vv)
    return st.q.numpy(), opt.costs.numpy(), opt.iterations.numpy(), opt.status.numpy()


def _oracle(cfg, **over):
    lm = cfg.lm
    kw = dict(max_iter=lm.max_iter, lambda_init=lm.lm_lambda, lambda_factor=lm.lambda_factor,
              lambda_min=lm.lambda_min, lambda_max=lm.lambda_max, rho_min=lm.rho_min,
              gain_ratio_epsilon=lm.gain_ratio_epsilon, stop_rules=2 if lm.step_tol else 0,
              step_tol=lm.step_tol or 0.0)
    kw.update(over)
    rob = oracle.Robot.from_spec(cfg.workload.spec)
    return rob, oracle.solve(rob, oracle.Terms(configs.oracle_terms(cfg)), oracle.params(**kw), cfg.workload.q0,
                             cfg.workload.base0, threads=8)


@pytest.mark.parametrize("name,B,tol", [("chain7", 512, 0.05), ("chain7c", 512, 0.06)])
def test_lane_schedule_matches_oracle(gpu, name, B, tol):
    """Success rate within `tol` of the FP64 oracle; where both succeed the final errors agree within 1e-4 m / 1e-3 rad."""
    cfg = configs.make(name, B, seed=11)
    q, cost, iters, status = _solve(cfg, "persistent", 1)
    rob, o = _oracle(cfg)
    wl = cfg.workload
    pe_g, re_g, ok_g = oracle.metrics(rob, q, None, wl.target_links, wl.targets, 1e-3, 0.01)
    pe_o, re_o, ok_o = oracle.metrics(rob, o["q"], None, wl.target_links, wl.targets, 1e-3, 0.01)
    assert abs(ok_g.mean() - ok_o.mean()) <= tol, (ok_g.mean(), ok_o.mean())
    both = ok_g & ok_o
    assert both.sum() > 10
    assert np.all(np.abs(pe_g[both] - pe_o[both]) <= 1e-4)
    assert np.all(np.abs(re_g[both] - re_o[both]) <= 1e-3)


@pytest.mark.parametrize("name", ["chain7", "chain7c"])
def test_lane_persistent_equals_lane_plain(gpu, name):
    """Both lane-per-problem forms run the same per-problem arithmetic: bitwise equal."""
    cfg = configs.make(name, 300, seed=5)
    a = _solve(cfg, "plain", 1, step_tol=1e-6)
    b = _solve(cfg, "persistent", 1, step_tol=1e-6)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_lane_and_group_schedules_agree(gpu):
    """The same problems under one lane and under 8-lane groups: same success rate, mostly the same solution."""
    cfg = configs.make("chain7c", 256, seed=3)
    a = _solve(cfg, "persistent", 1, step_tol=1e-6)
    b = _solve(cfg, "persistent", 8, step_tol=1e-6)
    rob = oracle.Robot.from_spec(cfg.workload.spec)
    wl = cfg.workload
    ra = oracle.metrics(rob, a[0], None, wl.target_links, wl.targets, 1e-3, 0.01)[2].mean()
    rb = oracle.metrics(rob, b[0], None, wl.target_links, wl.targets, 1e-3, 0.01)[2].mean()
    assert abs(ra - rb) <= 0.06, (ra, rb)
    close = np.all(np.abs(a[0] - b[0]) < 1e-3, axis=1)
    assert close.mean() > 0.7
    # a single step from the same point is the same step up to FP32 rounding, except for badly conditioned
    # normal equations (lambda = 1e-3 amplifies last-bit differences of J^T J, whose FK poses the two
    # schedules compose in a different order) and sphere pairs on the activity boundary
    c1 = _solve(cfg, "plain", 1, max_iter=1, step_tol=None)
    c8 = _solve(cfg, "plain", 8, max_iter=1, step_tol=None)
    same = np.isclose(c1[1], c8[1], rtol=1e-4, atol=1e-7) & np.all(np.abs(c1[0] - c8[0]) <= 1e-4, axis=1)
    assert same.mean() >= 0.95, same.mean()


def test_lane_schedule_is_refused_where_it_does_not_apply(gpu):
    for name, kw in (("chain7c", {"pair_mode": "slots"}), ("humanoid", {})):
        cfg = configs.make(name, 8, **kw)
        opt = LMOptimizer(cfg.terms, cfg.lm)
        opt.reset(VarValues({VarKey.ROBOT: cfg.robot.state(cfg.workload.q0, cfg.workload.base0)}))
        with pytest.raises(N.NativeError, match="one lane per problem"):
            opt.set_schedule(1)


def test_autotune_picks_a_schedule_and_keeps_the_inputs(gpu):
    cfg = configs.make("chain7", 2048, seed=4)
    opt = LMOptimizer(cfg.terms, LMOptimizerConfig(**{**cfg.lm.__dict__, "form": "persistent"}))
    st = cfg.robot.state(cfg.workload.q0)
    vv = VarValues({VarKey.ROBOT: st})
    res = opt.autotune(vv, lanes=(1, 8, 16))
    assert res["lanes"] in (1, 8, 16) and len(res["times_ms"]) == 3
    np.testing.assert_array_equal(st.q.numpy(), cfg.workload.q0.astype(np.float32))
    assert opt.problem.schedule()[0] == res["lanes"]
    opt.solve(vv)
    assert np.isfinite(opt.costs.numpy()).all()
