"""Continuous-batching IK server over the C ABI (``ik_server_*``), and the mixed request stream.

robokit solves one batch per ``LMOptimizer.solve`` call (opt/optimizer.py:216-240),
so a caller that receives IK requests over time batches them itself and waits
for each batch.  ``IKServer`` keeps problem types resident on the GPU and
overlaps requests: each type runs a persistent kernel whose lane groups take
the next waiting problem whenever theirs stops.  ``run_plain`` is the
comparison: requests that arrived while the GPU was busy are grouped by type
and solved as fixed batches with the plain form (one launch per iteration).

``run_served`` and ``run_plain`` replay the same seeded Poisson stream of
requests in real time and report solves/s and latency percentiles.
"""

from __future__ import annotations

import ctypes
import time
import weakref
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Sequence

import numpy as np

from . import _native as N
from .terms.task import lower_terms


def _destroy_server(handle: int) -> None:
    try:
        if N._lib is not None and handle:
            N._lib.ik_server_destroy(ctypes.c_void_p(handle))
    except Exception:
        pass


@dataclass
class _TypeInfo:
    robot: Any
    na: int
    floating: bool
    pose_frames: List[int]
    slots: int
    keep: List[Any] = field(default_factory=list)


class IKServer:
    """Resident problem types + continuous batching of requests on one GPU."""

    def __init__(self, budget_bytes: int = 8 << 30, idle_us: int = 200):
        N.load_library()
        h = ctypes.c_void_p(0)
        N.check(N.lib().ik_server_create(int(budget_bytes), int(idle_us), ctypes.byref(h)))
        self.handle = h.value
        self._fin = weakref.finalize(self, _destroy_server, self.handle)
        self.types: List[_TypeInfo] = []
        self._req: Dict[int, tuple] = {}

    def add_type(self, robot: Any, terms: Sequence[Any], lm_config: Any, slots: int, floating: bool = False,
                 active_dof_mask: Optional[np.ndarray] = None) -> int:
        """Register robot + terms + LM parameters; `slots` problems of this type may be in flight at once."""
        keep: List[Any] = []
        descs, ndesc = lower_terms(robot, list(terms), 1, floating, keep)
        pose_frames = [int(descs[i].num_frames) for i in range(ndesc)
                       if descs[i].kind in (N.IK_TERM_POSITION, N.IK_TERM_ROTATION, N.IK_TERM_FRAME)]
        mask = None
        if active_dof_mask is not None:
            mask = np.ascontiguousarray(active_dof_mask, np.float32)
            keep.append(mask)
        prm = lm_config.native_params()
        tid = ctypes.c_int32(0)
        N.check(N.lib().ik_server_add_type(self.handle, robot.handle, int(bool(floating)), descs, ndesc,
                                           N.np_ptr(mask), ctypes.byref(prm), int(slots), ctypes.byref(tid)))
        self.types.append(_TypeInfo(robot, robot.spec.num_actuated_joints, bool(floating), pose_frames, int(slots),
                                    keep))
        return tid.value

    def submit(self, type_id: int, q0: np.ndarray, targets: Sequence[np.ndarray],
               base0: Optional[np.ndarray] = None) -> int:
        """Submit q0 [n, na] with one target array [n, frames, 7] per pose term; returns the request id."""
        if not 0 <= type_id < len(self.types):
            raise ValueError(f"type {type_id} not registered")
        ti = self.types[type_id]
        q0 = np.ascontiguousarray(q0, np.float32)
        n = q0.shape[0]
        tg = [np.ascontiguousarray(t, np.float32) for t in targets]
        if len(tg) != len(ti.pose_frames):
            raise ValueError(f"expected {len(ti.pose_frames)} target arrays, got {len(tg)}")
        for t, f in zip(tg, ti.pose_frames):
            if t.shape != (n, f, 7):
                raise ValueError(f"targets must be [{n}, {f}, 7], got {t.shape}")
        b = None
        if ti.floating:
            if base0 is None:
                raise ValueError("a floating-base type needs base0")
            b = np.ascontiguousarray(base0, np.float32)
        ptrs = (ctypes.c_void_p * max(1, len(tg)))(*[t.ctypes.data for t in tg])
        rid = ctypes.c_int64(0)
        N.check(N.lib().ik_server_submit(self.handle, int(type_id), int(n), q0.ctypes.data, N.np_ptr(b), ptrs,
                                         ctypes.byref(rid)))
        self._req[rid.value] = (type_id, n)
        return rid.value

    def poll(self, max_done: int = 4096) -> List[int]:
        """Ids of requests that finished since the last poll (non-blocking)."""
        out = (ctypes.c_int64 * max_done)()
        n = ctypes.c_int32(0)
        N.check(N.lib().ik_server_poll(self.handle, out, int(max_done), ctypes.byref(n)))
        return [out[i] for i in range(n.value)]

    def fetch(self, request_id: int) -> Dict[str, np.ndarray]:
        """Results of a finished request; releases its slots."""
        type_id, n = self._req.pop(request_id)
        ti = self.types[type_id]
        q = np.empty((n, ti.na), np.float32)
        base = np.empty((n, 7), np.float32) if ti.floating else None
        cost = np.empty(n, np.float32)
        iters = np.empty(n, np.int32)
        status = np.empty(n, np.int32)
        N.check(N.lib().ik_server_fetch(self.handle, int(request_id), q.ctypes.data, N.np_ptr(base),
                                        cost.ctypes.data, iters.ctypes.data, status.ctypes.data))
        return {"q": q, "base": base, "cost": cost, "iterations": iters, "status": status}

    def info(self, type_id: int) -> Dict[str, int]:
        fs, pend, infl = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        lau = ctypes.c_int64()
        N.check(N.lib().ik_server_info(self.handle, int(type_id), ctypes.byref(fs), ctypes.byref(pend),
                                       ctypes.byref(infl), ctypes.byref(lau)))
        return {"free_slots": fs.value, "pending": pend.value, "inflight": infl.value, "launches": lau.value}

    def wait(self, ids: Sequence[int], timeout_s: float = 60.0) -> Dict[int, Dict[str, np.ndarray]]:
        """Poll until every request in `ids` finished; fetch and return their results."""
        want = set(ids)
        out: Dict[int, Dict[str, np.ndarray]] = {}
        t_end = time.time() + timeout_s
        while want:
            for r in self.poll():
                if r in want:
                    out[r] = self.fetch(r)
                    want.discard(r)
            if want and time.time() > t_end:
                raise TimeoutError(f"{len(want)} requests did not finish in {timeout_s} s")
        return out

    def close(self) -> None:
        self._fin()


# ---------------------------------------------------------------------------
# the mixed request stream
# ---------------------------------------------------------------------------
@dataclass
class StreamType:
    """One problem type of the stream: a config with a pool of seeded problems to draw requests from."""
    name: str
    cfg: Any
    lm: Any


@dataclass
class RequestSpec:
    t_arrive: float      # seconds after the stream start
    type_id: int
    start: int           # first problem of the type's pool
    batch: int


def mixed_types(pool: int = 4096, seed: int = 0, pos_tol: float = 1e-4, rot_tol: float = 1e-3,
                max_iter: int = 100) -> List[StreamType]:
    """The four robots of the mixed stream (7-DoF chain, 7-DoF chain + spheres, humanoid, hand), each with a
    pool of `pool` seeded problems, a cap of `max_iter` iterations and a per-problem stop at the pose
    tolerance (metres, radians)."""
    from . import configs
    from .opt import LMOptimizerConfig

    out = []
    for k, name in enumerate(("chain7", "chain7c", "humanoid", "hand")):
        cfg = configs.make(name, pool, seed=seed + k)
        lm = LMOptimizerConfig(**{**cfg.lm.__dict__, "max_iter": max_iter, "pose_tol": (pos_tol, rot_tol),
                                  "early_stopping_interval": 0, "form": "persistent"})
        out.append(StreamType(name, cfg, lm))
    return out


def make_server(types: Sequence[StreamType], budget_bytes: int = 8 << 30, slots: Optional[int] = None) -> IKServer:
    """A server with every stream type registered in order (slots default to each type's pool size)."""
    srv = IKServer(budget_bytes)
    for st in types:
        srv.add_type(st.cfg.robot, st.cfg.terms, st.lm, slots or st.cfg.batch,
                     floating=st.cfg.workload.base0 is not None)
    return srv


def make_stream(types: Sequence[StreamType], rate: float, duration: float, seed: int = 0,
                max_batch: int = 4096) -> List[RequestSpec]:
    """Poisson arrivals of `rate` problems/s for `duration` s; type uniform, batch log-uniform in [1, max_batch]."""
    rng = np.random.default_rng(seed)
    mean_batch = (max_batch - 1) / np.log(max_batch)
    req_rate = rate / mean_batch
    out: List[RequestSpec] = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / req_rate)
        if t >= duration:
            break
        k = int(rng.integers(len(types)))
        b = int(np.floor(np.exp(rng.uniform(0.0, np.log(max_batch + 1)))))
        b = max(1, min(max_batch, b))
        pool = types[k].cfg.batch
        b = min(b, pool)
        start = int(rng.integers(0, pool - b + 1))
        out.append(RequestSpec(t, k, start, b))
    return out


def _inputs(st: StreamType, r: RequestSpec):
    wl = st.cfg.workload
    sl = slice(r.start, r.start + r.batch)
    q0 = wl.q0[sl]
    base0 = wl.base0[sl] if wl.base0 is not None else None
    n_pose = sum(1 for t in st.cfg.terms if hasattr(t, "T_world_target"))
    tg = [wl.targets[sl]] * n_pose
    return q0, base0, tg


def _converged(types: Sequence[StreamType], r: RequestSpec, q: np.ndarray, base: Optional[np.ndarray],
               pos: float = 1e-3, rot: float = 0.01) -> int:
    st = types[r.type_id]
    wl = st.cfg.workload
    nt = len(wl.target_links)
    robot = st.cfg.robot
    B = r.batch
    qd = N.DeviceArray.from_numpy(np.ascontiguousarray(q, np.float32))
    bd = N.DeviceArray.from_numpy(np.ascontiguousarray(base, np.float32)) if base is not None else None
    links = N.DeviceArray.from_numpy(np.asarray(wl.target_links, np.int32))
    tg = N.DeviceArray.from_numpy(np.ascontiguousarray(wl.targets[r.start:r.start + B].reshape(B, nt, 7)))
    pe, re = N.DeviceArray.empty((B, nt)), N.DeviceArray.empty((B, nt))
    ok = N.DeviceArray.empty(B, np.int32)
    N.check(N.lib().ik_metrics(robot.handle, B, qd.ptr, N.ptr(bd), nt, links.ptr, tg.ptr, pos, rot, pe.ptr, re.ptr,
                               ok.ptr, None))
    return int(ok.numpy().sum())


def run_served(server: IKServer, types: Sequence[StreamType], reqs: Sequence[RequestSpec]) -> Dict[str, Any]:
    """Replay `reqs` in real time against `server` (types registered in the same order)."""
    inputs = [_inputs(types[r.type_id], r) for r in reqs]
    lat = np.zeros(len(reqs))
    results: Dict[int, Dict[str, np.ndarray]] = {}
    id_to_idx: Dict[int, int] = {}
    t0 = time.perf_counter()
    nxt = 0
    done = 0
    while done < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt].t_arrive <= now:
            q0, base0, tg = inputs[nxt]
            id_to_idx[server.submit(reqs[nxt].type_id, q0, tg, base0)] = nxt
            nxt += 1
        for rid in server.poll():
            i = id_to_idx.pop(rid)
            lat[i] = time.perf_counter() - t0 - reqs[i].t_arrive
            results[i] = server.fetch(rid)
            done += 1
    wall = time.perf_counter() - t0
    return _summary(types, reqs, results, lat, wall)


def run_plain(types: Sequence[StreamType], reqs: Sequence[RequestSpec]) -> Dict[str, Any]:
    """The same stream through the plain form (one launch per iteration): requests that arrived while the
    GPU was busy are grouped by type and solved as fixed batches of at most the type's pool size."""
    from .opt import LMOptimizer, VarKey, VarValues

    opts, pose_terms = [], []
    for st in types:
        opt = LMOptimizer(st.cfg.terms, type(st.lm)(**{**st.lm.__dict__, "form": "plain"}))
        wl = st.cfg.workload
        opt.solve(VarValues({VarKey.ROBOT: st.cfg.robot.state(wl.q0, wl.base0)}))  # buffers at the pool size
        opts.append(opt)
        pose_terms.append([t for t in st.cfg.terms if hasattr(t, "T_world_target")])
    inputs = [_inputs(types[r.type_id], r) for r in reqs]
    lat = np.zeros(len(reqs))
    results: Dict[int, Dict[str, np.ndarray]] = {}
    t0 = time.perf_counter()
    nxt = 0
    waiting: List[int] = []
    while len(results) < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt].t_arrive <= now:
            waiting.append(nxt)
            nxt += 1
        if not waiting:
            continue
        for k, st in enumerate(types):
            mine = [i for i in waiting if reqs[i].type_id == k]
            cap = st.cfg.batch
            while mine:
                group, total = [], 0
                while mine and total + reqs[mine[0]].batch <= cap:
                    total += reqs[mine[0]].batch
                    group.append(mine.pop(0))
                q0 = np.concatenate([inputs[i][0] for i in group])
                base0 = np.concatenate([inputs[i][1] for i in group]) if inputs[group[0]][1] is not None else None
                tg = np.ascontiguousarray(np.concatenate([inputs[i][2][0] for i in group]), np.float32)
                for t in pose_terms[k]:  # the first `total` target rows; problem p reads row p
                    N.check(N.lib().ik_memcpy_htod(t.T_world_target.ptr, tg.ctypes.data, tg.nbytes, None))
                state = st.cfg.robot.state(q0, base0)
                opts[k].solve(VarValues({VarKey.ROBOT: state}))
                q = state.q.numpy()
                base = state.T_world_base.numpy() if state.has_floating_base else None
                t_done = time.perf_counter() - t0
                off = 0
                for i in group:
                    n = reqs[i].batch
                    results[i] = {"q": q[off:off + n], "base": None if base is None else base[off:off + n]}
                    lat[i] = t_done - reqs[i].t_arrive
                    off += n
        waiting = []
    wall = time.perf_counter() - t0
    return _summary(types, reqs, results, lat, wall)


def _summary(types, reqs, results, lat, wall) -> Dict[str, Any]:
    if not reqs:
        return {"requests": 0, "problems": 0, "converged": 0, "wall_s": round(wall, 4), "solves_per_s": 0.0,
                "converged_per_s": 0.0, "p50_ms": None, "p99_ms": None, "max_ms": None}
    problems = sum(r.batch for r in reqs)
    conv = sum(_converged(types, reqs[i], results[i]["q"], results[i]["base"]) for i in range(len(reqs)))
    return {
        "requests": len(reqs),
        "problems": problems,
        "converged": conv,
        "wall_s": round(wall, 4),
        "solves_per_s": round(problems / wall, 1),
        "converged_per_s": round(conv / wall, 1),
        "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 3),
        "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 3),
        "max_ms": round(float(lat.max()) * 1e3, 3),
    }
