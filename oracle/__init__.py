"""FP64 CPU oracle of robokit's batched LM-IK path — TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package: it is the checker the CUDA path is
compared against, never something the product calls.  The arithmetic lives in
``ik_oracle.c`` (a restatement of the reference's algorithm, citing each
reference routine); this module only marshals arrays.

Parity pinning: the FK and link-Jacobian routines are checked against the
reference's golden files (panda entries of tests/robo/fk_ground_truth.json and
tests/robo/jacobian_ground_truth.json, extracted into tests/golden/) and the LM
accept/reject and step routines against the reference's unit-test recipes
(tests/opt/test_optimizer_acceptance.py, tests/opt/test_optimizer.py:366-429).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Any, Dict, List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "liboracle.so")


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "ik_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return LIB


class OrRobot(ctypes.Structure):
    _fields_ = [("nj", ctypes.c_int32), ("nl", ctypes.c_int32), ("na", ctypes.c_int32), ("ns", ctypes.c_int32)] + [
        (n, ctypes.c_void_p)
        for n in (
            "joint_types",
            "joint_axes",
            "parent_transforms",
            "parent_joints",
            "actuated_indices",
            "mimic_indices",
            "mimic_multipliers",
            "mimic_offsets",
            "link_parent_joints",
            "actuated_limits",
            "sphere_centers",
            "sphere_radii",
            "sphere_links",
            "link_bound_centers",
            "link_bound_radii",
        )
    ]


class OrTerm(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("num_frames", ctypes.c_int32),
        ("frame_links", ctypes.c_void_p),
        ("weights", ctypes.c_void_p),
        ("targets", ctypes.c_void_p),
        ("target_rows", ctypes.c_int32),
        ("margin", ctypes.c_float),
        ("max_active_pairs", ctypes.c_int32),
        ("pair_mode", ctypes.c_int32),
        ("num_link_pairs", ctypes.c_int32),
        ("link_pairs", ctypes.c_void_p),
        ("link_pair_offsets", ctypes.c_void_p),
        ("num_sphere_pairs", ctypes.c_int32),
        ("sphere_pairs", ctypes.c_void_p),
        ("dt", ctypes.c_float),
        ("velocity_limits", ctypes.c_void_p),
        ("num_query_spheres", ctypes.c_int32),
        ("query_spheres", ctypes.c_void_p),
        ("num_geoms", ctypes.c_int32),
        ("geoms", ctypes.c_void_p),
        ("num_scenes", ctypes.c_int32),
        ("penalty", ctypes.c_int32),
        ("residual_sqrt", ctypes.c_int32),
        ("residual_eps", ctypes.c_float),
        ("scene_indices", ctypes.c_void_p),
        ("scene_rows", ctypes.c_int32),
    ]


class OrParams(ctypes.Structure):
    _fields_ = [
        ("max_iter", ctypes.c_int32),
        ("lambda_init", ctypes.c_double),
        ("lambda_factor", ctypes.c_double),
        ("lambda_min", ctypes.c_double),
        ("lambda_max", ctypes.c_double),
        ("rho_min", ctypes.c_double),
        ("gain_ratio_epsilon", ctypes.c_double),
        ("stop_rules", ctypes.c_int32),
        ("cost_tol", ctypes.c_double),
        ("step_tol", ctypes.c_double),
        ("pose_pos_tol", ctypes.c_double),
        ("pose_rot_tol", ctypes.c_double),
        ("check_interval", ctypes.c_int32),
    ]


_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
    return _lib


def _p(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


class Robot:
    """Oracle view of a robot: float32/int32 tables (same layout as IkRobotDesc)."""

    def __init__(self, tables: Dict[str, np.ndarray], nj: int, nl: int, na: int, ns: int):
        self.t = {k: np.ascontiguousarray(v) for k, v in tables.items()}
        self.c = OrRobot(nj, nl, na, ns, *[_p(self.t[n]) for n, _ in OrRobot._fields_[4:]])
        self.nj, self.nl, self.na, self.ns = nj, nl, na, ns

    @classmethod
    def from_spec(cls, spec: Any) -> "Robot":
        return cls(spec.native_tables(), spec.num_joints, spec.num_links, spec.num_actuated_joints,
                   len(spec.collision_sphere_radii))


class Terms:
    """A list of term dicts lowered to OrTerm structs (arrays kept alive here)."""

    def __init__(self, terms: Sequence[Any]):
        self.keep: List[np.ndarray] = []
        flat: List[Dict[str, Any]] = []
        for t in terms:  # a term may hold several descriptors (joint rows, then base rows)
            flat.extend(t if isinstance(t, list) else [t])
        terms = flat
        arr = (OrTerm * max(1, len(terms)))()
        for i, t in enumerate(terms):
            def keep(x, dt):
                if x is None:
                    return None
                a = np.ascontiguousarray(x, dtype=dt)
                self.keep.append(a)
                return a.ctypes.data

            arr[i].kind = t["kind"]
            arr[i].num_frames = t.get("num_frames", 0)
            arr[i].frame_links = keep(t.get("frame_links"), np.int32)
            arr[i].weights = keep(t.get("weights"), np.float32)
            arr[i].targets = keep(t.get("targets"), np.float32)
            arr[i].target_rows = t.get("target_rows", 0)
            arr[i].margin = t.get("margin", 0.0)
            arr[i].max_active_pairs = t.get("max_active_pairs", 0)
            arr[i].pair_mode = t.get("pair_mode", 0)
            arr[i].num_link_pairs = t.get("num_link_pairs", 0)
            arr[i].link_pairs = keep(t.get("link_pairs"), np.int32)
            arr[i].link_pair_offsets = keep(t.get("link_pair_offsets"), np.int32)
            arr[i].num_sphere_pairs = t.get("num_sphere_pairs", 0)
            arr[i].sphere_pairs = keep(t.get("sphere_pairs"), np.int32)
            arr[i].dt = t.get("dt", 0.0)
            arr[i].velocity_limits = keep(t.get("velocity_limits"), np.float32)
            qs = t.get("query_spheres")
            arr[i].num_query_spheres = 0 if qs is None else len(qs)
            arr[i].query_spheres = keep(qs, np.int32)
            gm = t.get("geoms")
            arr[i].num_geoms = 0 if gm is None else int(np.asarray(gm).size // 16)
            arr[i].geoms = keep(gm, np.float32) if gm is not None and np.asarray(gm).size else None
            arr[i].num_scenes = t.get("num_scenes", 0)
            arr[i].penalty = t.get("penalty", 0)
            arr[i].residual_sqrt = int(bool(t.get("residual_sqrt", 0)))
            arr[i].residual_eps = t.get("residual_eps", 0.0)
            si = t.get("scene_indices")
            arr[i].scene_indices = keep(si, np.int32)
            arr[i].scene_rows = 0 if si is None else int(np.asarray(si).size)
        self.arr = arr
        self.n = len(terms)


def _f32(a: Optional[np.ndarray]) -> Optional[np.ndarray]:
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def fk(robot: Robot, q: np.ndarray, base: Optional[np.ndarray] = None) -> Dict[str, np.ndarray]:
    q = _f32(q).reshape(-1, robot.na)
    B = q.shape[0]
    base = _f32(base).reshape(B, 7) if base is not None else None
    out = dict(
        T_joint=np.zeros((B, robot.nj, 7)),
        T_link=np.zeros((B, robot.nl, 7)),
        S_world=np.zeros((B, 6, robot.nj)),
        spheres=np.zeros((B, robot.ns, 3)),
        link_bounds=np.zeros((B, robot.nl, 3)),
    )
    lib().or_fk(ctypes.byref(robot.c), B, _p(q), _p(base), *[_p(out[k]) for k in
                ("T_joint", "T_link", "S_world", "spheres", "link_bounds")])
    return out


def link_jacobian(robot: Robot, q: np.ndarray, base: Optional[np.ndarray], link: int, body: bool) -> np.ndarray:
    q = _f32(q).reshape(-1, robot.na)
    B = q.shape[0]
    base = _f32(base).reshape(B, 7) if base is not None else None
    D = (6 if base is not None else 0) + robot.na
    J = np.zeros((B, 6, D))
    lib().or_link_jacobian(ctypes.byref(robot.c), B, _p(q), _p(base), int(link), int(bool(body)), _p(J))
    return J


def residual_dim(robot: Robot, terms: Terms) -> int:
    return int(lib().or_residual_dim(ctypes.byref(robot.c), terms.arr, terms.n))


def residual_jacobian(robot: Robot, terms: Terms, q: np.ndarray, base: Optional[np.ndarray] = None):
    q = _f32(q).reshape(-1, robot.na)
    B = q.shape[0]
    floating = base is not None
    base = _f32(base).reshape(B, 7) if floating else None
    R = residual_dim(robot, terms)
    D = (6 if floating else 0) + robot.na
    r = np.zeros((B, R))
    J = np.zeros((B, R, D))
    lib().or_residual_jacobian(ctypes.byref(robot.c), terms.arr, terms.n, int(floating), B, _p(q), _p(base), _p(r),
                               _p(J))
    return r, J


def normal_equations(robot: Robot, terms: Terms, q: np.ndarray, base: Optional[np.ndarray] = None,
                     mask: Optional[np.ndarray] = None):
    q = _f32(q).reshape(-1, robot.na)
    B = q.shape[0]
    floating = base is not None
    base = _f32(base).reshape(B, 7) if floating else None
    D = (6 if floating else 0) + robot.na
    mask = _f32(mask)
    H = np.zeros((B, D, D))
    g = np.zeros((B, D))
    c = np.zeros(B)
    lib().or_normal_equations(ctypes.byref(robot.c), terms.arr, terms.n, int(floating), _p(mask), B, _p(q), _p(base),
                              _p(H), _p(g), _p(c))
    return H, g, c


def damped_solve(H: np.ndarray, g: np.ndarray, lam: np.ndarray):
    H = np.ascontiguousarray(H, np.float64)
    B, D = H.shape[0], H.shape[1]
    g = np.ascontiguousarray(g, np.float64).reshape(B, D)
    lam = np.ascontiguousarray(lam, np.float64).reshape(B)
    delta = np.zeros((B, D))
    pred = np.zeros(B)
    spd = np.zeros(B, np.int32)
    lib().or_damped_solve(B, D, _p(H), _p(g), _p(lam), _p(delta), _p(pred), _p(spd))
    return delta, pred, spd


def params(max_iter: int = 100, lambda_init: float = 1e-3, lambda_factor: float = 2.0, lambda_min: float = 1e-5,
           lambda_max: float = 1e10, rho_min: float = 1e-3, gain_ratio_epsilon: float = 1e-8, stop_rules: int = 0,
           cost_tol: float = 1e-9, step_tol: float = 0.0, pose_pos_tol: float = 0.0, pose_rot_tol: float = 0.0,
           check_interval: int = 1) -> OrParams:
    return OrParams(max_iter, lambda_init, lambda_factor, lambda_min, lambda_max, rho_min, gain_ratio_epsilon,
                    stop_rules, cost_tol, step_tol, pose_pos_tol, pose_rot_tol, check_interval)


def solve(robot: Robot, terms: Terms, prm: OrParams, q0: np.ndarray, base0: Optional[np.ndarray] = None,
          mask: Optional[np.ndarray] = None, threads: int = 1) -> Dict[str, np.ndarray]:
    q0 = _f32(q0).reshape(-1, robot.na)
    B = q0.shape[0]
    floating = base0 is not None
    base0 = _f32(base0).reshape(B, 7) if floating else None
    mask = _f32(mask)
    out = dict(q=np.zeros((B, robot.na)), base=np.zeros((B, 7)), cost=np.zeros(B), lam=np.zeros(B),
               iters=np.zeros(B, np.int32), status=np.zeros(B, np.int32))
    rc = lib().or_solve(ctypes.byref(robot.c), terms.arr, terms.n, int(floating), _p(mask), ctypes.byref(prm), B,
                        _p(q0), _p(base0), _p(out["q"]), _p(out["base"]), _p(out["cost"]), _p(out["lam"]),
                        _p(out["iters"]), _p(out["status"]), int(threads))
    if rc != 0:
        raise ValueError("oracle: unsupported sizes")
    if not floating:
        out["base"] = None
    return out


def metrics(robot: Robot, q: np.ndarray, base: Optional[np.ndarray], links: Sequence[int], targets: np.ndarray,
            pos_th: float = 5e-3, rot_th: float = 0.05):
    q = np.ascontiguousarray(q, np.float64).reshape(-1, robot.na)
    B = q.shape[0]
    base = None if base is None else np.ascontiguousarray(base, np.float64).reshape(B, 7)
    links = np.ascontiguousarray(links, np.int32)
    nt = len(links)
    targets = _f32(targets).reshape(B, nt, 7)
    pe = np.zeros((B, nt))
    re = np.zeros((B, nt))
    ok = np.zeros(B, np.int32)
    lib().or_metrics(ctypes.byref(robot.c), B, _p(q), _p(base), nt, _p(links), _p(targets), ctypes.c_double(pos_th),
                     ctypes.c_double(rot_th), _p(pe), _p(re), _p(ok))
    return pe, re, ok.astype(bool)


def accept_reject(cost: np.ndarray, cost_new: np.ndarray, pred: np.ndarray, lam: np.ndarray, prm: OrParams):
    """Returns (cost, lambda, accept) after the gain-ratio test."""
    cost = np.array(cost, np.float64).reshape(-1)
    B = cost.shape[0]
    cost_new = np.ascontiguousarray(cost_new, np.float64).reshape(B)
    pred = np.ascontiguousarray(pred, np.float64).reshape(B)
    lam = np.array(lam, np.float64).reshape(B)
    acc = np.zeros(B, np.int32)
    lib().or_accept_reject(B, _p(cost), _p(cost_new), _p(pred), _p(lam), _p(acc), ctypes.byref(prm))
    return cost, lam, acc


def _setup_signatures() -> None:
    L = lib()
    vp, i32, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double
    L.or_fk.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp]
    L.or_link_jacobian.argtypes = [vp, i32, vp, vp, i32, i32, vp]
    L.or_residual_dim.argtypes = [vp, vp, i32]
    L.or_residual_jacobian.argtypes = [vp, vp, i32, i32, i32, vp, vp, vp, vp]
    L.or_normal_equations.argtypes = [vp, vp, i32, i32, vp, i32, vp, vp, vp, vp, vp]
    L.or_damped_solve.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp]
    L.or_solve.argtypes = [vp, vp, i32, i32, vp, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, i32]
    L.or_metrics.argtypes = [vp, i32, vp, vp, i32, vp, vp, dbl, dbl, vp, vp, vp]
    L.or_accept_reject.argtypes = [i32, vp, vp, vp, vp, vp, vp]


_setup_done = False


def _ensure() -> None:
    global _setup_done
    if not _setup_done:
        _setup_signatures()
        _setup_done = True


for _name in ("fk", "link_jacobian", "residual_dim", "residual_jacobian", "normal_equations", "damped_solve", "solve",
              "metrics", "accept_reject"):
    _fn = globals()[_name]

    def _wrap(fn=_fn):
        def inner(*a, **k):
            _ensure()
            return fn(*a, **k)

        inner.__name__ = fn.__name__
        inner.__doc__ = fn.__doc__
        return inner

    globals()[_name] = _wrap()
