"""The allocation-free persistent solve, through the C ABI, against the regular persistent solve.

Collected last on purpose: it must pass both alone in a fresh process and
after every other test has run in the same process.
"""

import ctypes

import numpy as np
import pytest

from robokit_b200 import _native as N
from robokit_b200 import configs
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
from robokit_b200.terms.task import _VarStub

pytestmark = pytest.mark.gpu


class _Descs:
    """IkRobotDesc + IkTermDesc array for a config, with the host arrays they point at kept alive."""

    def __init__(self, cfg, floating):
        self.keep = []
        spec = cfg.robot.spec
        t = spec.native_tables()
        self.keep.append(t)
        self.robot = N.IkRobotDesc()
        self.robot.num_joints = spec.num_joints
        self.robot.num_links = spec.num_links
        self.robot.num_actuated = spec.num_actuated_joints
        self.robot.num_spheres = len(spec.collision_sphere_radii)
        for name, arr in t.items():
            setattr(self.robot, name, arr.ctypes.data if arr.size else None)
        B = cfg.workload.q0.shape[0]
        stub = _VarStub(cfg.robot, B, floating)
        self.terms = (N.IkTermDesc * max(1, len(cfg.terms)))()
        for i, term in enumerate(cfg.terms):
            d = term.native_desc(stub)
            td = self.terms[i]
            td.kind = d["kind"]
            td.num_frames = d.get("num_frames", 0)
            td.frame_links = self._arr(d.get("frame_links"), np.int32)
            td.weights = self._arr(d.get("weights"), np.float32)
            tg = d.get("targets")
            if tg is not None:
                self.keep.append(tg)
                td.d_targets = tg.ptr
                td.target_rows = tg.shape[0]
            td.margin = d.get("margin", 0.0)
            td.max_active_pairs = d.get("max_active_pairs", 0)
            td.pair_mode = d.get("pair_mode", 0)
            td.num_link_pairs = d.get("num_link_pairs", 0)
            td.link_pairs = self._arr(d.get("link_pairs"), np.int32)
            td.link_pair_offsets = self._arr(d.get("link_pair_offsets"), np.int32)
            td.num_sphere_pairs = d.get("num_sphere_pairs", 0)
            td.sphere_pairs = self._arr(d.get("sphere_pairs"), np.int32)
        self.num_terms = len(cfg.terms)

    def _arr(self, x, dt):
        if x is None:
            return None
        a = np.ascontiguousarray(x, dtype=dt)
        if a.size == 0:
            return None
        self.keep.append(a)
        return a.ctypes.data


def _persistent(cfg):
    lm = LMOptimizerConfig(**{**cfg.lm.__dict__, "form": "persistent"})
    opt = LMOptimizer(cfg.terms, lm)
    st = cfg.robot.state(cfg.workload.q0, cfg.workload.base0)
    opt.solve(VarValues({VarKey.ROBOT: st}))
    base = st.T_world_base.numpy() if st.has_floating_base else None
    return lm, st.q.numpy(), base, opt.costs.numpy(), opt.iterations.numpy(), opt.status.numpy()


def _noalloc(cfg, lm):
    floating = cfg.workload.base0 is not None
    descs = _Descs(cfg, floating)
    B = cfg.workload.q0.shape[0]
    q = N.DeviceArray.from_numpy(np.ascontiguousarray(cfg.workload.q0, np.float32))
    base = N.DeviceArray.from_numpy(np.ascontiguousarray(cfg.workload.base0, np.float32)) if floating else None
    cost, lam = N.DeviceArray.zeros(B), N.DeviceArray.zeros(B)
    iters, status = N.DeviceArray.zeros(B, np.int32), N.DeviceArray.zeros(B, np.int32)
    prm = lm.native_params()
    N.check(N.lib().ik_solve_persistent_noalloc(ctypes.byref(descs.robot), int(floating), descs.terms,
                                                descs.num_terms, None, B, q.ptr, base.ptr if base is not None else None,
                                                ctypes.byref(prm), cost.ptr, lam.ptr, iters.ptr, status.ptr, None))
    N.check(N.lib().ik_device_synchronize())
    return q.numpy(), base.numpy() if base is not None else None, cost.numpy(), iters.numpy(), status.numpy()


def _compare(ref, got):
    _, q_r, b_r, c_r, it_r, st_r = ref
    q_g, b_g, c_g, it_g, st_g = got
    # the same kernel source and the same tables; the tolerance only covers a
    # different choice of FMA contraction between the two compiled copies
    np.testing.assert_allclose(q_g, q_r, rtol=0, atol=1e-4)
    np.testing.assert_allclose(c_g, c_r, rtol=1e-4, atol=1e-9)
    if b_r is not None:
        np.testing.assert_allclose(b_g, b_r, rtol=0, atol=1e-4)
    assert np.mean(it_g == it_r) > 0.98
    assert np.mean((st_g & 0xff) == (st_r & 0xff)) > 0.98


def test_noalloc_matches_persistent_two_calls_in_a_row(gpu):
    """Two different problems back to back through the shared scratch: each matches ik_solve_persistent."""
    a = configs.make("chain7c", 512, seed=21, pair_mode="slots")
    b = configs.make("humanoid", 256, seed=22)
    ref_a, ref_b = _persistent(a), _persistent(b)
    _compare(ref_a, _noalloc(a, ref_a[0]))
    _compare(ref_b, _noalloc(b, ref_b[0]))
    # and once more with the first problem: nothing of the second call leaks into it
    _compare(ref_a, _noalloc(a, ref_a[0]))


def test_noalloc_refuses_oversized_tables(gpu):
    cfg = configs.make("chain7c", 4, seed=1, pair_mode="all")
    descs = _Descs(cfg, False)
    n = 70000  # 280 KB of sphere pairs: more than the scratch holds
    lp = np.array([0, cfg.robot.spec.num_links - 1], np.int32)
    off = np.array([0, n], np.int32)
    sp = np.tile(np.array([0, 1], np.int32), n)
    w = np.ones(1, np.float32)
    descs.keep += [lp, off, sp, w]
    t = N.IkTermDesc()
    t.kind = N.IK_TERM_SELF_COLLISION
    t.weights = w.ctypes.data
    t.margin = 0.01
    t.pair_mode = N.IK_PAIRS_ALL
    t.num_link_pairs = 1
    t.link_pairs = lp.ctypes.data
    t.link_pair_offsets = off.ctypes.data
    t.num_sphere_pairs = n
    t.sphere_pairs = sp.ctypes.data
    terms = (N.IkTermDesc * 1)(t)
    q = N.DeviceArray.from_numpy(np.ascontiguousarray(cfg.workload.q0, np.float32))
    prm = cfg.lm.native_params()
    rc = N.lib().ik_solve_persistent_noalloc(ctypes.byref(descs.robot), 0, terms, 1, None, 4, q.ptr, None,
                                             ctypes.byref(prm), None, None, None, None, None)
    assert rc == N.IK_E_UNSUPPORTED
    assert b"at most" in N.lib().ik_last_error()
