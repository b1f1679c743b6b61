"""Cost-term protocol (robokit terms/task.py:13-262, terms/robot_task.py).

A term here is a thin, configuration-only object.  The optimizer lowers its
term list into the device term table of libb200ik.so (``native_desc``); there
is no per-term kernel and no host fallback.  ``compute_weighted_residual`` /
``compute_weighted_jacobian`` evaluate one term on the GPU for the reference's
per-term API and for tests.
"""

from __future__ import annotations

import abc
import ctypes
import re
from enum import Enum
from typing import Any, Dict, List, Optional

import numpy as np

from .. import _native as N
from ..opt.var_values import VarKey, VarValues


class Context(Enum):
    """Base of the placeholder keys a helper fills in at build time (terms/task.py:13-14)."""


class Task(abc.ABC):
    name: str = ""
    var_key = VarKey.ROBOT

    @property
    def cost_name(self) -> str:
        """The class name in snake case (PositionTask -> position_task): the key of this term's cost in cost
        reports and the stem of the names a config gives its terms (terms/task.py:89-93)."""
        return re.sub(r"(?<!^)(?=[A-Z])", "_", type(self).__name__).lower()


class ResidualTask(Task):
    """Weighted residual term with an analytic Jacobian (terms/task.py:133-232)."""

    robot: Any = None
    _version: int = 0

    @property
    @abc.abstractmethod
    def residual_dim(self) -> int: ...

    @abc.abstractmethod
    def native_desc(self, var: Any) -> Dict[str, Any]:
        """Fields of IkTermDesc (include/b200ik.h) for this term; arrays are numpy."""

    def host_desc(self, var: Any) -> Dict[str, Any]:
        """Like native_desc, with host (numpy) arrays only — the oracle's view of the term."""
        return self.native_desc(var)

    def _touch(self) -> None:
        self._version = getattr(self, "_version", 0) + 1

    # -- single-term evaluation on the GPU -----------------------------------------
    def _single_problem(self, var: Any) -> "NativeProblem":
        key = (var.batch_size, var.has_floating_base, id(var.robot), getattr(self, "_version", 0))
        cache = self.__dict__.setdefault("_single", {})
        if key not in cache:
            cache.clear()
            cache[key] = NativeProblem(var.robot, [self], var.batch_size, var.has_floating_base, None)
        return cache[key]

    def _eval(self, var_values: VarValues, want_r: bool, want_j: bool):
        var = var_values.get(self.var_key)
        prob = self._single_problem(var)
        B, R, D = var.batch_size, self.residual_dim, var.tangent_dim
        r = N.DeviceArray.empty((B, R), np.float32) if want_r else None
        J = N.DeviceArray.empty((B, R, D), np.float32) if want_j else None
        N.check(N.lib().ik_residual_jacobian(prob.handle, B, var.q.ptr,
                                             var.T_world_base.ptr if var.has_floating_base else None,
                                             N.ptr(r), N.ptr(J), None))
        return r, J

    def compute_weighted_residual(self, var_values: VarValues, out_residual: Any = None, row_offset: int = 0):
        r, _ = self._eval(var_values, True, False)
        if out_residual is None:
            return r
        out = N.as_device(out_residual, np.float32)
        B, R = r.shape
        N.check(N.lib().ik_copy_rows(B, R, r.ptr, R, out.ptr + 4 * row_offset, out.shape[1], None))
        return out_residual

    def compute_weighted_jacobian(self, var_values: VarValues, out_jacobian: Any = None, row_offset: int = 0):
        _, J = self._eval(var_values, False, True)
        if out_jacobian is None:
            return J
        out = N.as_device(out_jacobian, np.float32)
        B, R, D = J.shape
        Rtot = out.shape[1]
        off = var_values.tangent_offset(self.var_key)
        N.check(N.lib().ik_copy_rows(B * R, D, J.ptr, D, out.ptr + 4 * (row_offset * out.shape[2] + off),
                                     out.shape[2], None) if Rtot == R else _copy_block(J, out, row_offset, off))
        return out_jacobian

    compute_weighted_jacobian_analytic = compute_weighted_jacobian


def _copy_block(J: N.DeviceArray, out: N.DeviceArray, row_offset: int, col_offset: int) -> int:
    B, R, D = J.shape
    Rtot, Dtot = out.shape[1], out.shape[2]
    for b in range(B):
        rc = N.lib().ik_copy_rows(R, D, J.ptr + 4 * b * R * D, D,
                                  out.ptr + 4 * (b * Rtot * Dtot + row_offset * Dtot + col_offset), Dtot, None)
        if rc:
            return rc
    return 0


def _destroy_problem(handle: int) -> None:
    try:
        if N._lib is not None and handle:
            N._lib.ik_problem_destroy(ctypes.c_void_p(handle))
    except Exception:
        pass


def lower_terms(robot: Any, terms: List[ResidualTask], capacity: int, floating: bool,
                keep: List[Any]) -> Any:
    """(IkTermDesc array, descriptor count) for `terms`; the host arrays it points at are appended to `keep`."""

    def arr(x: Any, dt: Any) -> Optional[int]:
        if x is None:
            return None
        a = np.ascontiguousarray(x, dtype=dt)
        if a.size == 0:
            return None
        keep.append(a)
        return a.ctypes.data

    var_stub = _VarStub(robot, capacity, floating)
    flat: List[Dict[str, Any]] = []
    for t in terms:  # a term may lower to several descriptors (joint rows, then base rows)
        d = t.native_desc(var_stub)
        flat.extend(d if isinstance(d, list) else [d])
    descs = (N.IkTermDesc * max(1, len(flat)))()
    for i, d in enumerate(flat):
        descs[i].kind = d["kind"]
        descs[i].num_frames = d.get("num_frames", 0)
        descs[i].frame_links = arr(d.get("frame_links"), np.int32)
        descs[i].weights = arr(d.get("weights"), np.float32)
        tg = d.get("targets")
        if tg is not None:
            keep.append(tg)
            descs[i].d_targets = tg.ptr
            descs[i].target_rows = tg.shape[0]
        descs[i].margin = d.get("margin", 0.0)
        descs[i].max_active_pairs = d.get("max_active_pairs", 0)
        descs[i].pair_mode = d.get("pair_mode", 0)
        descs[i].num_link_pairs = d.get("num_link_pairs", 0)
        descs[i].link_pairs = arr(d.get("link_pairs"), np.int32)
        descs[i].link_pair_offsets = arr(d.get("link_pair_offsets"), np.int32)
        descs[i].num_sphere_pairs = d.get("num_sphere_pairs", 0)
        descs[i].sphere_pairs = arr(d.get("sphere_pairs"), np.int32)
        descs[i].dt = d.get("dt", 0.0)
        descs[i].velocity_limits = arr(d.get("velocity_limits"), np.float32)
        qs = d.get("query_spheres")
        if qs is not None:
            descs[i].num_query_spheres = len(qs)
            descs[i].query_spheres = arr(qs, np.int32)
            gm = np.asarray(d.get("geoms"), np.float32)
            descs[i].num_geoms = gm.size // N.IK_GEOM_FLOATS
            descs[i].geoms = arr(gm, np.float32)
            descs[i].num_scenes = d["num_scenes"]
            descs[i].penalty = d["penalty"]
            descs[i].residual_sqrt = int(bool(d.get("residual_sqrt", 0)))
            descs[i].residual_eps = d.get("residual_eps", 0.0)
            si = d.get("scene_indices")
            if si is not None:
                keep.append(si)
                descs[i].d_scene_indices = si.ptr
                descs[i].scene_rows = si.shape[0]
    return descs, len(flat)


class NativeProblem:
    """An IkProblem: robot + lowered term list, sized for `capacity` problems."""

    def __init__(self, robot: Any, terms: List[ResidualTask], capacity: int, floating: bool,
                 active_dof_mask: Optional[np.ndarray]):
        import weakref

        self.keep: List[Any] = []
        descs, ndesc = lower_terms(robot, terms, capacity, floating, self.keep)
        mask = None
        if active_dof_mask is not None:
            mask = np.ascontiguousarray(active_dof_mask, np.float32)
            self.keep.append(mask)
        h = ctypes.c_void_p(0)
        N.check(N.lib().ik_problem_create(robot.handle, int(capacity), int(bool(floating)), descs, ndesc,
                                          N.np_ptr(mask), ctypes.byref(h)))
        self.handle = h.value
        self.robot = robot
        self.capacity = capacity
        self._fin = weakref.finalize(self, _destroy_problem, self.handle)
        D, R, C = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        N.check(N.lib().ik_problem_info(self.handle, ctypes.byref(D), ctypes.byref(R), ctypes.byref(C)))
        self.tangent_dim, self.residual_dim = D.value, R.value

    def set_schedule(self, group_lanes: int = 0, blocks_per_sm: int = 0) -> None:
        N.check(N.lib().ik_problem_set_schedule(self.handle, int(group_lanes), int(blocks_per_sm)))

    def schedule(self):
        g, b = ctypes.c_int32(), ctypes.c_int32()
        N.check(N.lib().ik_problem_get_schedule(self.handle, ctypes.byref(g), ctypes.byref(b)))
        return g.value, b.value


class _VarStub:
    def __init__(self, robot: Any, batch: int, floating: bool):
        self.robot = robot
        self.spec = robot.spec
        self.batch_size = batch
        self.has_floating_base = floating
