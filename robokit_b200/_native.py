"""ctypes binding of libb200ik.so (include/b200ik.h) and a torch-free device array.

The package talks to the GPU only through this module.  There is no CPU
fallback: if the shared library or a CUDA device is missing, every entry point
that needs them raises :class:`NativeError`.
"""

from __future__ import annotations

import ctypes
import os
import weakref
from typing import Any, Iterable, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libb200ik.so")

# status codes, joint types, term kinds, stop rules (include/b200ik.h)
IK_OK = 0
IK_E_INVALID = -1
IK_E_CAPACITY = -2
IK_E_OOM = -3
IK_E_CUDA = -4
IK_E_UNSUPPORTED = -5
IK_E_NO_DEVICE = -6

IK_ST_CONVERGED = 1
IK_ST_MAX_ITER = 2
IK_ST_NOT_SPD = 4
IK_ST_NONFINITE = 8

IK_TERM_POSITION = 1
IK_TERM_ROTATION = 2
IK_TERM_POSITION_LIMIT = 3
IK_TERM_SELF_COLLISION = 4
IK_TERM_FRAME = 5
IK_TERM_JOINT_REF = 6
IK_TERM_VELOCITY_LIMIT = 7
IK_TERM_SCENE_COLLISION = 8
IK_TERM_BASE_REF = 9
IK_PENALTY_SMOOTH, IK_PENALTY_PLAIN, IK_PENALTY_SURFACE_DISTANCE = 0, 1, 2
IK_GEOM_BOX, IK_GEOM_SPHERE, IK_GEOM_PLANE, IK_GEOM_CAPSULE = 0, 1, 2, 3
IK_GEOM_FLOATS = 16

IK_PAIRS_SLOTS = 0
IK_PAIRS_ALL = 1

IK_STOP_NONE = 0
IK_STOP_ALL_COST = 1
IK_STOP_STEP = 2
IK_STOP_POSE = 4
IK_STOP_COST = 8


class NativeError(RuntimeError):
    """An IK_E_* status from libb200ik.so, or the library could not be used."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class CapacityError(NativeError, ValueError):
    """Batch larger than the buffers were sized for (opt/optimizer.py:321-322 raises ValueError)."""


_i32p = ctypes.POINTER(ctypes.c_int32)
_f32p = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


class IkRobotDesc(ctypes.Structure):
    _fields_ = [
        ("num_joints", ctypes.c_int32),
        ("num_links", ctypes.c_int32),
        ("num_actuated", ctypes.c_int32),
        ("num_spheres", ctypes.c_int32),
        ("joint_types", _vp),
        ("joint_axes", _vp),
        ("parent_transforms", _vp),
        ("parent_joints", _vp),
        ("actuated_indices", _vp),
        ("mimic_indices", _vp),
        ("mimic_multipliers", _vp),
        ("mimic_offsets", _vp),
        ("link_parent_joints", _vp),
        ("actuated_limits", _vp),
        ("sphere_centers", _vp),
        ("sphere_radii", _vp),
        ("sphere_links", _vp),
        ("link_bound_centers", _vp),
        ("link_bound_radii", _vp),
    ]


class IkTermDesc(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("num_frames", ctypes.c_int32),
        ("frame_links", _vp),
        ("weights", _vp),
        ("d_targets", _vp),
        ("target_rows", ctypes.c_int32),
        ("margin", ctypes.c_float),
        ("max_active_pairs", ctypes.c_int32),
        ("pair_mode", ctypes.c_int32),
        ("num_link_pairs", ctypes.c_int32),
        ("link_pairs", _vp),
        ("link_pair_offsets", _vp),
        ("num_sphere_pairs", ctypes.c_int32),
        ("sphere_pairs", _vp),
        ("dt", ctypes.c_float),
        ("velocity_limits", _vp),
        ("num_query_spheres", ctypes.c_int32),
        ("query_spheres", _vp),
        ("num_geoms", ctypes.c_int32),
        ("geoms", _vp),
        ("num_scenes", ctypes.c_int32),
        ("penalty", ctypes.c_int32),
        ("residual_sqrt", ctypes.c_int32),
        ("residual_eps", ctypes.c_float),
        ("d_scene_indices", _vp),
        ("scene_rows", ctypes.c_int32),
    ]


class IkLmParams(ctypes.Structure):
    _fields_ = [
        ("max_iter", ctypes.c_int32),
        ("lambda_init", ctypes.c_float),
        ("lambda_factor", ctypes.c_float),
        ("lambda_min", ctypes.c_float),
        ("lambda_max", ctypes.c_float),
        ("rho_min", ctypes.c_float),
        ("gain_ratio_epsilon", ctypes.c_float),
        ("stop_rules", ctypes.c_int32),
        ("cost_tol", ctypes.c_float),
        ("step_tol", ctypes.c_float),
        ("pose_pos_tol", ctypes.c_float),
        ("pose_rot_tol", ctypes.c_float),
        ("check_interval", ctypes.c_int32),
    ]


# every symbol include/b200ik.h declares, with its ctypes signature
_SIGNATURES = {
    "ik_last_error": (ctypes.c_char_p, []),
    "ik_version": (ctypes.c_int, []),
    "ik_device_count": (ctypes.c_int, [_i32p]),
    "ik_set_device": (ctypes.c_int, [ctypes.c_int]),
    "ik_robot_create": (ctypes.c_int, [ctypes.POINTER(IkRobotDesc), ctypes.POINTER(_vp)]),
    "ik_robot_destroy": (ctypes.c_int, [_vp]),
    "ik_problem_create": (
        ctypes.c_int,
        [_vp, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(IkTermDesc), ctypes.c_int32, _vp, ctypes.POINTER(_vp)],
    ),
    "ik_problem_destroy": (ctypes.c_int, [_vp]),
    "ik_problem_info": (ctypes.c_int, [_vp, _i32p, _i32p, _i32p]),
    "ik_problem_set_targets": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, ctypes.c_int32]),
    "ik_problem_set_schedule": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32]),
    "ik_problem_get_schedule": (ctypes.c_int, [_vp, _i32p, _i32p]),
    "ik_solve_plain": (
        ctypes.c_int,
        [_vp, ctypes.c_int32, _vp, _vp, ctypes.POINTER(IkLmParams), _vp, _vp, _vp, _vp, _vp],
    ),
    "ik_solve_persistent": (
        ctypes.c_int,
        [_vp, ctypes.c_int32, _vp, _vp, ctypes.POINTER(IkLmParams), _vp, _vp, _vp, _vp, _vp],
    ),
    "ik_solve_persistent_noalloc": (
        ctypes.c_int,
        [ctypes.POINTER(IkRobotDesc), ctypes.c_int32, ctypes.POINTER(IkTermDesc), ctypes.c_int32, _vp,
         ctypes.c_int32, _vp, _vp, ctypes.POINTER(IkLmParams), _vp, _vp, _vp, _vp, _vp],
    ),
    "ik_server_create": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(_vp)]),
    "ik_server_destroy": (ctypes.c_int, [_vp]),
    "ik_server_add_type": (
        ctypes.c_int,
        [_vp, _vp, ctypes.c_int32, ctypes.POINTER(IkTermDesc), ctypes.c_int32, _vp, ctypes.POINTER(IkLmParams),
         ctypes.c_int32, _i32p],
    ),
    "ik_server_submit": (
        ctypes.c_int,
        [_vp, ctypes.c_int32, ctypes.c_int32, _vp, _vp, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int64)],
    ),
    "ik_server_poll": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int32, _i32p]),
    "ik_server_fetch": (ctypes.c_int, [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp]),
    "ik_server_info": (ctypes.c_int, [_vp, ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.POINTER(ctypes.c_int64)]),
    "ik_fk": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ik_link_jacobian": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, _vp, ctypes.c_int32, ctypes.c_int32, _vp, _vp]),
    "ik_residual_jacobian": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp]),
    "ik_normal_equations": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ik_damped_solve": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ik_step": (
        ctypes.c_int,
        [_vp, ctypes.c_int32, _vp, _vp, _vp, ctypes.POINTER(IkLmParams), _vp, _vp, _vp, _vp, _vp, _vp],
    ),
    "ik_accept_reject": (ctypes.c_int, [ctypes.c_int32, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(IkLmParams), _vp]),
    "ik_metrics": (
        ctypes.c_int,
        [_vp, ctypes.c_int32, _vp, _vp, ctypes.c_int32, _vp, _vp, ctypes.c_float, ctypes.c_float, _vp, _vp, _vp, _vp],
    ),
    "ik_integrate": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    ),
    "ik_row_sumsq": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _vp, ctypes.c_int64, _vp, ctypes.c_int32, _vp]),
    "ik_pose_from_matrix": (ctypes.c_int, [ctypes.c_int32, _vp, _vp, _vp]),
    "ik_matrix_from_pose": (ctypes.c_int, [ctypes.c_int32, _vp, _vp, _vp]),
    "ik_gather_rows": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _vp, ctypes.c_int32, _vp, _vp, _vp, _vp]),
    "ik_copy_rows": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _vp, ctypes.c_int64, _vp, ctypes.c_int64, _vp]),
    "ik_masked_copy_rows": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp, _vp]),
    "ik_select_best": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp],
    ),
    "ik_keep_previous": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ik_clamp_q": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp, _vp]),
    "ik_malloc": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_size_t]),
    "ik_free": (ctypes.c_int, [_vp]),
    "ik_malloc_host": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_size_t]),
    "ik_free_host": (ctypes.c_int, [_vp]),
    "ik_memcpy_htod": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t, _vp]),
    "ik_memcpy_dtoh": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t, _vp]),
    "ik_memcpy_dtod": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t, _vp]),
    "ik_memset": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_size_t, _vp]),
    "ik_stream_create": (ctypes.c_int, [ctypes.POINTER(_vp)]),
    "ik_stream_destroy": (ctypes.c_int, [_vp]),
    "ik_stream_synchronize": (ctypes.c_int, [_vp]),
    "ik_device_synchronize": (ctypes.c_int, []),
    "ik_event_create": (ctypes.c_int, [ctypes.POINTER(_vp)]),
    "ik_event_destroy": (ctypes.c_int, [_vp]),
    "ik_event_record": (ctypes.c_int, [_vp, _vp]),
    "ik_event_elapsed_ms": (ctypes.c_int, [_vp, _vp, _f32p]),
    "ik_graph_begin": (ctypes.c_int, [_vp]),
    "ik_graph_end": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "ik_graph_launch": (ctypes.c_int, [_vp, _vp]),
    "ik_graph_destroy": (ctypes.c_int, [_vp]),
    "ik_launch_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int64)]),
    "ik_measure_fma_peak": (ctypes.c_int, [ctypes.c_int32, _f32p]),
}

_lib: Optional[ctypes.CDLL] = None


def load_library(path: Optional[str] = None) -> ctypes.CDLL:
    """Load libb200ik.so (built in-tree by robokit_b200.build) and bind every symbol."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise NativeError(IK_E_UNSUPPORTED, f"{p} is missing: build it with robokit_b200.build.build_library()")
    lib = ctypes.CDLL(p)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def lib() -> ctypes.CDLL:
    return load_library()


def check(rc: int) -> None:
    if rc != IK_OK:
        msg = lib().ik_last_error().decode(errors="replace")
        if rc == IK_E_CAPACITY:
            raise CapacityError(rc, msg)
        if rc == IK_E_INVALID:
            raise ValueError(msg)
        raise NativeError(rc, msg)


def device_count() -> int:
    n = ctypes.c_int32(0)
    try:
        rc = lib().ik_device_count(ctypes.byref(n))
    except NativeError:
        return 0
    return int(n.value) if rc == IK_OK else 0


def synchronize() -> None:
    check(lib().ik_device_synchronize())


def launch_count() -> int:
    v = ctypes.c_int64(0)
    check(lib().ik_launch_count(ctypes.byref(v)))
    return int(v.value)


# ---------------------------------------------------------------------------
# device memory
# ---------------------------------------------------------------------------
def _free_ptr(ptr: int) -> None:
    try:
        if _lib is not None:
            _lib.ik_free(ctypes.c_void_p(ptr))
    except Exception:
        pass


class DeviceArray:
    """A contiguous device buffer with a shape and dtype (float32 / int32 / ...).

    Exposes ``__cuda_array_interface__`` so torch/cupy/numba users can wrap it
    without a copy, and accepts such objects through :meth:`from_cuda_array`.
    """

    __slots__ = ("ptr", "shape", "dtype", "_owner", "_fin", "__weakref__")

    def __init__(self, ptr: int, shape: Sequence[int], dtype: Any, owner: Any = None, owned: bool = False):
        self.ptr = int(ptr)
        self.shape = tuple(int(s) for s in shape)
        self.dtype = np.dtype(dtype)
        self._owner = owner
        self._fin = weakref.finalize(self, _free_ptr, self.ptr) if owned else None

    # -- construction -------------------------------------------------------
    @classmethod
    def empty(cls, shape: Sequence[int] | int, dtype: Any = np.float32) -> "DeviceArray":
        shape = (shape,) if isinstance(shape, int) else tuple(shape)
        nbytes = int(np.prod(shape, dtype=np.int64)) * np.dtype(dtype).itemsize
        p = ctypes.c_void_p(0)
        check(lib().ik_malloc(ctypes.byref(p), max(nbytes, 16)))
        return cls(p.value or 0, shape, dtype, owned=True)

    @classmethod
    def zeros(cls, shape: Sequence[int] | int, dtype: Any = np.float32) -> "DeviceArray":
        a = cls.empty(shape, dtype)
        a.zero_()
        return a

    @classmethod
    def from_numpy(cls, arr: np.ndarray, dtype: Any = None) -> "DeviceArray":
        arr = np.ascontiguousarray(arr, dtype=dtype if dtype is not None else arr.dtype)
        a = cls.empty(arr.shape, arr.dtype)
        a.copy_from_numpy(arr)
        return a

    @classmethod
    def from_cuda_array(cls, obj: Any) -> "DeviceArray":
        """Wrap any object with ``__cuda_array_interface__`` (no copy, no ownership)."""
        cai = obj.__cuda_array_interface__
        if cai.get("strides") not in (None,):
            itemsize = np.dtype(cai["typestr"]).itemsize
            expect, acc = [], itemsize
            for s in reversed(cai["shape"]):
                expect.append(acc)
                acc *= s
            if tuple(reversed(expect)) != tuple(cai["strides"]):
                raise ValueError("only C-contiguous device arrays can be wrapped")
        return cls(cai["data"][0], cai["shape"], np.dtype(cai["typestr"]), owner=obj)

    # -- properties ---------------------------------------------------------
    @property
    def size(self) -> int:
        return int(np.prod(self.shape, dtype=np.int64))

    @property
    def nbytes(self) -> int:
        return self.size * self.dtype.itemsize

    @property
    def ndim(self) -> int:
        return len(self.shape)

    @property
    def __cuda_array_interface__(self) -> dict:
        return {"shape": self.shape, "typestr": self.dtype.str, "data": (self.ptr, False), "version": 3, "strides": None}

    def __len__(self) -> int:
        return self.shape[0] if self.shape else 0

    def __repr__(self) -> str:
        return f"DeviceArray(shape={self.shape}, dtype={self.dtype.name}, ptr=0x{self.ptr:x})"

    # -- data movement -------------------------------------------------------
    def copy_from_numpy(self, arr: np.ndarray, stream: Optional[int] = None) -> "DeviceArray":
        arr = np.ascontiguousarray(arr, dtype=self.dtype)
        if arr.nbytes != self.nbytes:
            raise ValueError(f"size mismatch: {arr.shape} vs {self.shape}")
        check(lib().ik_memcpy_htod(self.ptr, arr.ctypes.data, arr.nbytes, stream))
        if stream is None:
            check(lib().ik_stream_synchronize(None))
        return self

    def numpy(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=self.dtype)
        if self.nbytes:
            check(lib().ik_memcpy_dtoh(out.ctypes.data, self.ptr, self.nbytes, None))
            check(lib().ik_stream_synchronize(None))
        return out

    def zero_(self) -> "DeviceArray":
        check(lib().ik_memset(self.ptr, 0, self.nbytes, None))
        return self

    def assign(self, other: "DeviceArray | np.ndarray") -> "DeviceArray":
        if isinstance(other, np.ndarray):
            return self.copy_from_numpy(other)
        if other.nbytes != self.nbytes:
            raise ValueError("size mismatch")
        check(lib().ik_memcpy_dtod(self.ptr, other.ptr, self.nbytes, None))
        return self

    def clone(self) -> "DeviceArray":
        out = DeviceArray.empty(self.shape, self.dtype)
        out.assign(self)
        return out

    def reshape(self, shape: Sequence[int]) -> "DeviceArray":
        shape = tuple(int(s) for s in shape)
        if int(np.prod(shape, dtype=np.int64)) != self.size:
            raise ValueError(f"cannot reshape {self.shape} to {shape}")
        return DeviceArray(self.ptr, shape, self.dtype, owner=self)

    def prefix(self, n: int) -> "DeviceArray":
        """Rows [0, n) sharing storage (the capacity-prefix views of opt/optimizer.py:313-333)."""
        if n > self.shape[0]:
            raise ValueError(f"prefix {n} exceeds {self.shape[0]} rows")
        return DeviceArray(self.ptr, (n,) + self.shape[1:], self.dtype, owner=self)

    def row_slice(self, start: int, stop: int) -> "DeviceArray":
        row = int(np.prod(self.shape[1:], dtype=np.int64)) * self.dtype.itemsize
        return DeviceArray(self.ptr + start * row, (stop - start,) + self.shape[1:], self.dtype, owner=self)


def as_device(x: Any, dtype: Any = np.float32) -> DeviceArray:
    """numpy / DeviceArray / __cuda_array_interface__ object -> DeviceArray of `dtype`."""
    if isinstance(x, DeviceArray):
        if x.dtype != np.dtype(dtype):
            raise TypeError(f"expected {np.dtype(dtype).name}, got {x.dtype.name}")
        return x
    if hasattr(x, "__cuda_array_interface__"):
        d = DeviceArray.from_cuda_array(x)
        if d.dtype != np.dtype(dtype):
            raise TypeError(f"expected {np.dtype(dtype).name}, got {d.dtype.name}")
        return d
    return DeviceArray.from_numpy(np.asarray(x, dtype=dtype))


def ptr(x: Optional[DeviceArray]) -> Optional[int]:
    return None if x is None else x.ptr


class Stream:
    def __init__(self):
        s = ctypes.c_void_p(0)
        check(lib().ik_stream_create(ctypes.byref(s)))
        self.handle = s.value
        self._fin = weakref.finalize(self, lambda h=self.handle: _lib and _lib.ik_stream_destroy(ctypes.c_void_p(h)))

    def synchronize(self) -> None:
        check(lib().ik_stream_synchronize(self.handle))


class Event:
    def __init__(self):
        e = ctypes.c_void_p(0)
        check(lib().ik_event_create(ctypes.byref(e)))
        self.handle = e.value
        self._fin = weakref.finalize(self, lambda h=self.handle: _lib and _lib.ik_event_destroy(ctypes.c_void_p(h)))

    def record(self, stream: Optional[Stream] = None) -> "Event":
        check(lib().ik_event_record(self.handle, stream.handle if stream else None))
        return self

    def elapsed_ms(self, end: "Event") -> float:
        v = ctypes.c_float(0.0)
        check(lib().ik_event_elapsed_ms(self.handle, end.handle, ctypes.byref(v)))
        return float(v.value)


class Graph:
    """Library calls recorded on a stream between capture() and end(), replayed by launch()."""

    def __init__(self, stream: "Stream"):
        self.stream = stream
        self.handle: Optional[int] = None
        self._fin = None

    def capture(self, body) -> "Graph":
        check(lib().ik_graph_begin(self.stream.handle))
        try:
            body()
        finally:
            g = ctypes.c_void_p(0)
            rc = lib().ik_graph_end(self.stream.handle, ctypes.byref(g))
        check(rc)
        self.handle = g.value
        self._fin = weakref.finalize(self, lambda h=self.handle: _lib and _lib.ik_graph_destroy(ctypes.c_void_p(h)))
        return self

    def launch(self) -> None:
        check(lib().ik_graph_launch(self.handle, self.stream.handle))


class PinnedBuffer:
    """Page-locked host memory viewed as a numpy array."""

    def __init__(self, shape: Sequence[int], dtype: Any = np.float32):
        self.shape = tuple(shape)
        self.dtype = np.dtype(dtype)
        nbytes = int(np.prod(self.shape, dtype=np.int64)) * self.dtype.itemsize
        p = ctypes.c_void_p(0)
        check(lib().ik_malloc_host(ctypes.byref(p), max(nbytes, 16)))
        self.ptr = p.value
        buf = (ctypes.c_char * max(nbytes, 16)).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=int(np.prod(self.shape))).reshape(self.shape)
        self._fin = weakref.finalize(self, lambda h=self.ptr: _lib and _lib.ik_free_host(ctypes.c_void_p(h)))


def np_ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


def keepalive(*arrays: Iterable[np.ndarray]) -> Tuple[np.ndarray, ...]:
    return tuple(arrays)  # type: ignore[arg-type]
