"""Dense residual terms of the IK path.

PositionTask (terms/dense/position_task.py:18-272), RotationTask
(terms/dense/rotation_task.py:25-401), FrameTask in "log" mode
(terms/dense/frame_task.py:47-621), PositionLimit in "abs" mode
(terms/dense/position_limit.py:185-573), the joint blocks of SmoothnessTask
(terms/dense/smoothness_task.py:22-460) and ConfigurationTask
(terms/dense/configuration_task.py:25-478), VelocityLimitTask
(terms/dense/velocity_limit_task.py:14-232), SceneCollisionTask over primitive
geometry (terms/dense/scene_collision_task.py:276-650), and SelfCollisionTask with sphere
geometry (terms/dense/self_collision_task.py:593-1152).  Constructor
signatures, defaults, residual_dim and set_weight / set_target follow the
reference; the arithmetic runs in libb200ik.so.
"""

from __future__ import annotations

from typing import Any, Dict, Literal, Optional, Sequence, Union

import numpy as np

from .. import _native as N
from ..robo.robot_spec import collision_pair_tables
from .task import Context, ResidualTask


def _host_pose_targets(T: Any, num_frames: int) -> np.ndarray:
    a = np.asarray(T, np.float32)
    if a.ndim == 1:
        a = a.reshape(1, 1, 7)
    elif a.ndim == 2:
        a = a.reshape(a.shape[0], 1, 7) if num_frames == 1 and a.shape[1] == 7 else a.reshape(1, -1, 7)
    if a.ndim != 3 or a.shape[2] != 7:
        raise ValueError(f"targets must be (rows, frames, 7) poses, got {np.asarray(T).shape}")
    return np.ascontiguousarray(a)


def _device_pose_targets(T: Any, num_frames: int) -> N.DeviceArray:
    """A device [rows, num_frames, 7] float32 copy of device targets (the reference clones, position_task.py:77)."""
    d = N.as_device(T, np.float32)
    rows = d.size // (7 * num_frames)
    if d.size != rows * num_frames * 7:
        raise ValueError(f"targets of shape {d.shape} do not hold {num_frames} poses per row")
    out = N.DeviceArray.empty((rows, num_frames, 7), np.float32)
    out.assign(d.reshape(out.shape))
    return out


class _PoseTask(ResidualTask):
    kind = 0
    default_weight = 1.0

    def __init__(self, robot: Any = None, frame_index: Any = None, T_world_target: Any = None,
                 weight: Union[float, Sequence[float]] = 1.0, fixed_target: bool = False, name: str = ""):
        self.name = name
        self.weight = weight
        self.fixed_target = fixed_target
        self.robot = robot
        self.frame_index_arg, self.T_world_target_arg = frame_index, T_world_target
        self._target_host: Optional[np.ndarray] = None
        self._target_dev: Optional[N.DeviceArray] = None
        if frame_index is None or T_world_target is None or any(
            isinstance(a, Context) for a in (frame_index, T_world_target)
        ):
            return  # configuration-time stub
        frames = [int(frame_index)] if isinstance(frame_index, (int, np.integer)) else [int(f) for f in frame_index]
        self.frame_indices = np.asarray(frames, np.int32)
        self.num_frames = len(frames)
        if isinstance(T_world_target, N.DeviceArray) or hasattr(T_world_target, "__cuda_array_interface__"):
            self._target_dev = _device_pose_targets(T_world_target, self.num_frames)
            shape = self._target_dev.shape
        else:
            self._target_host = _host_pose_targets(T_world_target, self.num_frames)
            shape = self._target_host.shape
        if shape[1] != self.num_frames:
            raise ValueError(f"Number of frame indices ({self.num_frames}) must match number of targets ({shape[1]})")
        self._set_weight_array(weight)

    @property
    def T_world_target(self) -> N.DeviceArray:
        """Device copy of the targets [rows, num_frames, 7] (copied to the GPU on first use)."""
        if self._target_dev is None:
            self._target_dev = N.DeviceArray.from_numpy(self._target_host)
        return self._target_dev

    def targets_numpy(self) -> np.ndarray:
        if self._target_dev is not None:
            return self._target_dev.numpy()
        return self._target_host

    def _set_weight_array(self, weight: Union[float, Sequence[float]]) -> None:
        if isinstance(weight, (int, float)):
            self.residual_weight = np.full(self.num_frames * 3, weight, np.float32)
        else:
            self.residual_weight = np.repeat(np.asarray(weight, np.float32), 3)

    def set_weight(self, weight: Union[float, Sequence[float]]) -> None:
        self.weight = weight
        self._set_weight_array(weight)
        self._touch()

    def set_target(self, T_world_target: Any) -> None:
        """Overwrite the target poses in place (same row count; position_task.py:103-105)."""
        cur = self._target_dev.shape if self._target_dev is not None else self._target_host.shape
        if isinstance(T_world_target, N.DeviceArray) or hasattr(T_world_target, "__cuda_array_interface__"):
            new = N.as_device(T_world_target, np.float32)
            if new.size != int(np.prod(cur)):
                raise ValueError(f"target shape {new.shape} differs from {cur}")
            self.T_world_target.assign(new.reshape(cur))
        else:
            new_h = _host_pose_targets(T_world_target, self.num_frames)
            if new_h.shape != tuple(cur):
                raise ValueError(f"target shape {new_h.shape} differs from {cur}")
            if self._target_dev is not None:
                self._target_dev.copy_from_numpy(new_h)
            else:
                self._target_host = new_h

    def bind_targets(self, targets: N.DeviceArray) -> None:
        """Read the targets from `targets` [rows, num_frames, 7] in place from now on (no copy per update)."""
        if targets.ndim != 3 or targets.shape[1:] != (self.num_frames, 7):
            raise ValueError(f"targets of shape {targets.shape} are not [rows, {self.num_frames}, 7]")
        self._target_dev = targets
        self._target_host = None
        self._touch()

    @property
    def residual_dim(self) -> int:
        return 3 * self.num_frames

    def _desc(self, var: Any, targets: Any) -> Dict[str, Any]:
        for f in self.frame_indices:
            if not 0 <= f < var.spec.num_links:
                raise ValueError(f"frame index {f} out of range")
        return dict(kind=self.kind, num_frames=self.num_frames, frame_links=self.frame_indices,
                    weights=self.residual_weight, targets=targets, target_rows=targets.shape[0])

    def native_desc(self, var: Any) -> Dict[str, Any]:
        return self._desc(var, self.T_world_target)

    def host_desc(self, var: Any) -> Dict[str, Any]:
        return self._desc(var, self.targets_numpy())


class PositionTask(_PoseTask):
    """w * (p_target - p_frame); Jacobian -w (v + w x p) (position_task.py:189-272)."""

    kind = N.IK_TERM_POSITION

    def __init__(self, robot: Any = None, frame_index: Any = None, T_world_target: Any = None,
                 weight: Union[float, Sequence[float]] = 20.0, fixed_target: bool = False, name: str = ""):
        super().__init__(robot, frame_index, T_world_target, weight, fixed_target, name)


class RotationTask(_PoseTask):
    """w * log(q_frame q_target^-1) in the world frame; Jacobian +w w (rotation_task.py:324-401)."""

    kind = N.IK_TERM_ROTATION

    def __init__(self, robot: Any = None, frame_index: Any = None, T_world_target: Any = None,
                 weight: Union[float, Sequence[float]] = 10.0, fixed_target: bool = False, name: str = ""):
        super().__init__(robot, frame_index, T_world_target, weight, fixed_target, name)


class FrameTask(_PoseTask):
    """w (.) log(T_frame^-1 T_target), six rows per frame; Jacobian -w (.) jlog Ad(T_frame^-1) S
    (frame_task.py:47-621, residual_mode "log")."""

    kind = N.IK_TERM_FRAME

    def __init__(self, robot: Any = None, frame_index: Any = None, T_world_target: Any = None,
                 position_weight: Union[float, Sequence[float]] = 1.0,
                 orientation_weight: Union[float, Sequence[float]] = 1.0,
                 residual_mode: Literal["log", "distance"] = "log", trajectory_frames: int = 1, name: str = ""):
        if residual_mode not in {"log", "distance"}:
            raise ValueError(f"Unsupported residual_mode: {residual_mode}")
        if residual_mode != "log":
            raise NotImplementedError("residual_mode='distance' is outside the IK hot path (log residuals only)")
        if trajectory_frames != 1:
            raise NotImplementedError("trajectory frames are outside the IK hot path")
        self.position_weight = position_weight
        self.orientation_weight = orientation_weight
        self.residual_mode = residual_mode
        super().__init__(robot, frame_index, T_world_target, 1.0, False, name)

    def _set_weight_array(self, weight: Any) -> None:
        pw = np.broadcast_to(np.asarray(self.position_weight, np.float32), (self.num_frames,))
        ow = np.broadcast_to(np.asarray(self.orientation_weight, np.float32), (self.num_frames,))
        self.residual_weight = np.ascontiguousarray(np.stack([pw, ow], axis=1).reshape(-1))

    def set_weight(self, position_weight: Any = None, orientation_weight: Any = None) -> None:
        if position_weight is not None:
            self.position_weight = position_weight
        if orientation_weight is not None:
            self.orientation_weight = orientation_weight
        self._set_weight_array(None)
        self._touch()

    @property
    def residual_dim(self) -> int:
        return 6 * self.num_frames


class PositionLimit(ResidualTask):
    """Joint-limit hinge w (max(0, q - hi) + max(0, lo - q)) (position_limit.py:185-573, mode "abs")."""

    def __init__(self, robot: Any = None, weight: Optional[Union[float, Sequence[float]]] = None,
                 residual_mode: Literal["abs", "sqrt_abs", "exp_barrier"] = "abs", residual_eps: float = 1e-6,
                 mask: Any = None, base_axis: Optional[int] = None, name: str = "", **unsupported: Any):
        if residual_mode not in {"abs", "sqrt_abs", "exp_barrier"}:
            raise ValueError(f"Unsupported residual_mode: {residual_mode}")
        if residual_mode != "abs":
            raise NotImplementedError(f"residual_mode={residual_mode!r} is outside the IK hot path (only 'abs')")
        if base_axis is not None or mask is not None or unsupported:
            raise NotImplementedError("base bounds, masks and warm-up ramps are outside the IK hot path")
        self.name = name
        self.weight = weight
        self.residual_mode = residual_mode
        self.robot = robot

    def set_weight(self, weight: Union[float, Sequence[float]]) -> None:
        self.weight = weight
        self._touch()

    @property
    def residual_dim(self) -> int:
        return self.robot.spec.num_actuated_joints

    def native_desc(self, var: Any) -> Dict[str, Any]:
        na = var.spec.num_actuated_joints
        w = np.zeros(na, np.float32)
        w[:] = 1.0 if self.weight is None else self.weight
        return dict(kind=N.IK_TERM_POSITION_LIMIT, weights=w)


def _ref_rows(ref: Any, na: int) -> Any:
    """A reference as [rows, na]: a DeviceArray (read in place) or a float32 numpy array."""
    if isinstance(ref, N.DeviceArray) or hasattr(ref, "__cuda_array_interface__"):
        d = N.as_device(ref, np.float32)
        if d.size % max(na, 1) or d.size == 0:
            raise ValueError(f"reference of shape {d.shape} does not hold rows of {na} joints")
        return d.reshape((d.size // na, na))
    a = np.ascontiguousarray(np.asarray(ref, np.float32).reshape(-1, na))
    if a.shape[0] == 0:
        raise ValueError("empty reference")
    return a


def _pose_rows(T: Any) -> Any:
    """Base poses as [rows, 7] [x y z qw qx qy qz]: a DeviceArray (read in place) or float32 numpy."""
    if isinstance(T, N.DeviceArray) or hasattr(T, "__cuda_array_interface__"):
        d = N.as_device(T, np.float32)
        if d.size % 7 or d.size == 0:
            raise ValueError(f"base poses of shape {d.shape} are not rows of 7")
        return d.reshape((d.size // 7, 7))
    a = np.asarray(T, np.float32)
    if a.shape[-2:] == (4, 4):
        from ..geom import _poses_vec7

        return _poses_vec7(a, a.reshape(-1, 4, 4).shape[0])
    return np.ascontiguousarray(a.reshape(-1, 7))


def _base_desc(weights: np.ndarray, ref: Any, host: bool) -> Dict[str, Any]:
    """Six rows w (.) log(T_world_base T_ref^-1) (kind IK_TERM_BASE_REF)."""
    if host:
        r = ref.numpy() if isinstance(ref, N.DeviceArray) else np.asarray(ref, np.float32)
        return dict(kind=N.IK_TERM_BASE_REF, weights=weights, targets=r, target_rows=r.shape[0])
    d = ref if isinstance(ref, N.DeviceArray) else N.DeviceArray.from_numpy(np.asarray(ref, np.float32))
    return dict(kind=N.IK_TERM_BASE_REF, weights=weights, targets=d)


_IDENTITY_POSE = np.array([[0, 0, 0, 1, 0, 0, 0]], np.float32)


class _JointRefTask(ResidualTask):
    """r_a = w_a (q_a - ref_a) over the actuated joints: a diagonal Jacobian block of w.

    The reference row of problem b is b // max(1, batch // rows), the reference's
    broadcast rule (smoothness_task.py:361-363, configuration_task.py:331-332)."""

    _ref: Any = None
    _ref_dev: Optional[N.DeviceArray] = None

    def _joint_weights(self, na: int) -> np.ndarray:
        w = np.zeros(na, np.float32)
        w[:] = self.weight
        return w

    @property
    def residual_dim(self) -> int:
        return self.robot.spec.num_actuated_joints

    def _reference(self, na: int) -> Any:
        raise NotImplementedError

    def _device_ref(self, na: int) -> N.DeviceArray:
        ref = self._reference(na)
        if isinstance(ref, N.DeviceArray):
            return ref
        if self._ref_dev is None or self._ref_dev.shape != ref.shape:
            self._ref_dev = N.DeviceArray.from_numpy(ref)
        else:
            self._ref_dev.copy_from_numpy(ref)
        return self._ref_dev

    def _check(self, var: Any) -> int:
        na = var.spec.num_actuated_joints
        if self.robot is not None and self.robot.spec.num_actuated_joints != na:
            raise ValueError("term built for another robot")
        return na

    def native_desc(self, var: Any) -> Dict[str, Any]:
        na = self._check(var)
        return dict(kind=N.IK_TERM_JOINT_REF, weights=self._joint_weights(na), targets=self._device_ref(na))

    def host_desc(self, var: Any) -> Dict[str, Any]:
        na = self._check(var)
        ref = self._reference(na)
        ref = ref.numpy() if isinstance(ref, N.DeviceArray) else ref
        return dict(kind=N.IK_TERM_JOINT_REF, weights=self._joint_weights(na), targets=ref, target_rows=ref.shape[0])


class _PrevStateEval:
    """The reference's evaluation signature with an optional previous state for this call only
    (smoothness_task.py:171-300, velocity_limit_task.py:99-185)."""

    def _with_prev(self, fn: Any, var_values: Any, prev_var: Any, out: Any, row_offset: int) -> Any:
        if prev_var is None:
            return fn(var_values, out, row_offset)
        saved = (self._prev_q, getattr(self, "_prev_base", None))
        self._prev_q = None  # fresh copies: a buffer bound in place is left as it is
        if hasattr(self, "_prev_base"):
            self._prev_base = None
        self.set_prev_state(prev_var)
        try:
            return fn(var_values, out, row_offset)
        finally:
            self._prev_q = saved[0]
            if hasattr(self, "_prev_base"):
                self._prev_base = saved[1]
            self._touch()

    def compute_weighted_residual(self, var_values: Any, prev_var: Any = None, out_residual: Any = None,
                                  row_offset: int = 0) -> Any:
        return self._with_prev(super().compute_weighted_residual, var_values, prev_var, out_residual, row_offset)

    def compute_weighted_jacobian(self, var_values: Any, prev_var: Any = None, out_jacobian: Any = None,
                                  row_offset: int = 0) -> Any:
        return self._with_prev(super().compute_weighted_jacobian, var_values, prev_var, out_jacobian, row_offset)

    compute_weighted_jacobian_analytic = compute_weighted_jacobian


class SmoothnessTask(_PrevStateEval, _JointRefTask):
    """Penalise change from a previous state, w (q - q_prev) on the joints and, with a floating-base
    previous state (or a base_weight), w_b (.) log(T_world_base T_prev^-1) on the base
    (smoothness_task.py:22-460).  Base weights default to the first joint's weight.  Without a
    previous state the term adds zero rows, as the reference's does.  The warm-up weight ramp is not
    supported."""

    def __init__(self, robot: Any = None, prev_var: Any = None, weight: Union[float, Sequence[float]] = 1.0,
                 base_weight: Optional[Union[float, Sequence[float]]] = None, name: str = "", warmup_frames: int = 0,
                 frame: Any = None):
        if warmup_frames and frame is not None:
            raise NotImplementedError("the warm-up weight ramp is outside the IK hot path")
        self.name = name
        self.weight = weight
        self.base_weight = base_weight
        self.warmup_frames, self.frame = warmup_frames, frame
        self.robot = robot
        self.prev_var = prev_var
        self._prev_q: Any = None
        self._prev_base: Any = None
        self._include_base = base_weight is not None or bool(getattr(prev_var, "has_floating_base", False))
        if prev_var is not None and not isinstance(prev_var, Context):
            self._prev_q = _ref_rows(prev_var.q, prev_var.spec.num_actuated_joints)
            if isinstance(self._prev_q, N.DeviceArray):  # the reference clones the state (smoothness_task.py:57)
                self._prev_q = self._prev_q.clone()
            if prev_var.has_floating_base:
                self._prev_base = _pose_rows(prev_var.T_world_base)
                if isinstance(self._prev_base, N.DeviceArray):
                    self._prev_base = self._prev_base.clone()

    @property
    def residual_dim(self) -> int:
        return self.robot.spec.num_actuated_joints + (6 if self._include_base else 0)

    def _base_weights(self, na: int) -> np.ndarray:
        w = np.zeros(6, np.float32)
        if self._prev_q is None:
            return w
        if self.base_weight is not None:
            w[:] = self.base_weight
        else:
            jw = super()._joint_weights(na)
            w[:] = jw[0] if na else 1.0
        return w

    def _descs(self, var: Any, host: bool) -> Any:
        d = (_JointRefTask.host_desc if host else _JointRefTask.native_desc)(self, var)
        if not self._include_base:
            return d
        if not var.has_floating_base or (self._prev_q is not None and self._prev_base is None):
            raise ValueError("SmoothnessTask is configured with base residuals but var/prev_var has no floating base.")
        ref = self._prev_base if self._prev_base is not None else _IDENTITY_POSE
        return [d, _base_desc(self._base_weights(var.spec.num_actuated_joints), ref, host)]

    def native_desc(self, var: Any) -> Any:
        return self._descs(var, False)

    def host_desc(self, var: Any) -> Any:
        return self._descs(var, True)

    @property
    def active(self) -> bool:
        return bool(np.any(self.weight))

    def _joint_weights(self, na: int) -> np.ndarray:
        w = super()._joint_weights(na)
        return w if self._prev_q is not None else np.zeros_like(w)

    def _reference(self, na: int) -> Any:
        return self._prev_q if self._prev_q is not None else np.zeros((1, na), np.float32)

    def set_weight(self, weight: Union[float, Sequence[float]]) -> None:
        self.weight = weight
        self._touch()

    def bind_previous(self, prev_q: N.DeviceArray, prev_base: Optional[N.DeviceArray] = None) -> None:
        """Read the previous joints from `prev_q` [rows, na] (and base poses from `prev_base` [rows, 7], which
        adds the base rows) in place from now on."""
        self._prev_q = prev_q
        if prev_base is not None:
            self._prev_base = prev_base
            self._include_base = True
        self._touch()

    def set_prev_state(self, prev_state: Any) -> None:
        """Copy a new previous state in place; a new row count rebuilds (smoothness_task.py:111-120)."""
        new = _ref_rows(prev_state.q, prev_state.spec.num_actuated_joints)
        newb = _pose_rows(prev_state.T_world_base) if prev_state.has_floating_base else None
        if (isinstance(self._prev_q, N.DeviceArray) and self._prev_q.shape == new.shape and
                (newb is None) == (self._prev_base is None) and
                (newb is None or (isinstance(self._prev_base, N.DeviceArray) and self._prev_base.shape == newb.shape))):
            self._prev_q.assign(new)
            if newb is not None:
                self._prev_base.assign(newb)
            return
        self._prev_q = new.clone() if isinstance(new, N.DeviceArray) else new
        self._prev_base = None if newb is None else (newb.clone() if isinstance(newb, N.DeviceArray) else newb)
        self._touch()  # the row layout stays as built: base rows only if configured (smoothness_task.py:111-120)


class ConfigurationTask(_JointRefTask):
    """Bias joints toward a rest configuration, w (q - rest_q) (configuration_task.py:25-478).

    ``rest_q`` is "midrange" (the joint-limit midpoints), an array of one or more
    rows, or None (the zero configuration); ``mask`` scales each joint's weight.
    With ``T_world_base_rest`` (rows of [x y z qw qx qy qz] or 4x4 poses) six more
    rows w_b (.) log(T_world_base T_rest^-1) bias a floating base toward it
    (base_weight, default 1); ``include_joints=False`` keeps only those."""

    def __init__(self, robot: Any = None, rest_q: Any = None, T_world_base_rest: Any = None,
                 weight: Union[float, Sequence[float]] = 1.0, base_weight: Any = None, include_joints: bool = True,
                 var_key: Any = None, name: str = "", mask: Any = None):
        if isinstance(rest_q, str) and rest_q != "midrange":
            raise ValueError(f"Unsupported rest_q: {rest_q}")
        if isinstance(mask, Context):
            raise NotImplementedError("a helper's joint mask is outside the IK hot path")
        self.name = name
        self.weight = weight
        self.base_weight = base_weight
        self.include_joints = include_joints
        self.mask = None if mask is None else np.asarray(mask, np.float32)
        self.rest_q_arg = rest_q
        self.robot = robot
        self._rest: Any = None
        self._base_rest_arg = T_world_base_rest
        self._base_rest: Any = None
        if T_world_base_rest is not None and not isinstance(T_world_base_rest, Context):
            self._base_rest = _pose_rows(T_world_base_rest)
            if isinstance(self._base_rest, N.DeviceArray):  # the reference clones it (configuration_task.py:141)
                self._base_rest = self._base_rest.clone()
        if var_key is not None:
            self.var_key = var_key

    @property
    def active(self) -> bool:
        w = np.asarray(self.weight, np.float32)
        if self.mask is not None and w.ndim <= 1:
            w = w * self.mask
        return bool(np.any(w))

    def _joint_weights(self, na: int) -> np.ndarray:
        w = super()._joint_weights(na)
        if self.mask is not None:
            w *= self.mask
        return w

    @property
    def _has_base(self) -> bool:
        return self._base_rest_arg is not None

    @property
    def residual_dim(self) -> int:
        na = self.robot.spec.num_actuated_joints
        return (na if self.include_joints or not self._has_base else 0) + (6 if self._has_base else 0)

    def _descs(self, var: Any, host: bool) -> Any:
        d = (_JointRefTask.host_desc if host else _JointRefTask.native_desc)(self, var)
        if not self._has_base:
            return d
        if isinstance(self._base_rest_arg, Context):
            raise ValueError("T_world_base_rest is a placeholder: build the term through a helper or give it")
        if not var.has_floating_base:
            raise ValueError("ConfigurationTask has a rest base pose but the state has no floating base")
        if self._base_rest is None:
            self._base_rest = _pose_rows(self._base_rest_arg)
        bw = np.ones(6, np.float32)
        if self.base_weight is not None:
            bw[:] = self.base_weight
        out = [d] if self.include_joints else []
        return out + [_base_desc(bw, self._base_rest, host)]

    def native_desc(self, var: Any) -> Any:
        return self._descs(var, False)

    def host_desc(self, var: Any) -> Any:
        return self._descs(var, True)

    def _reference(self, na: int) -> Any:
        if self._rest is not None:
            return self._rest
        r = self.rest_q_arg
        if isinstance(r, Context):
            raise ValueError("rest_q is a placeholder: build the term through a helper or give rest_q")
        if isinstance(r, str):
            spec = self.robot.spec if self.robot is not None else None
            if spec is None:
                raise ValueError('rest_q="midrange" needs a robot')
            r = spec.midrange_q
        elif r is None:
            r = np.zeros(na, np.float32)
        self._rest = _ref_rows(r, na)
        return self._rest

    def set_weight(self, weight: Union[float, Sequence[float]]) -> None:
        self.weight = weight
        self._touch()

    def bind_rest(self, rest_q: N.DeviceArray) -> None:
        """Read the rest joints from `rest_q` [rows, na] in place from now on."""
        self._rest = rest_q
        self._touch()

    def set_target(self, rest_q: Any = None, T_world_base_rest: Any = None) -> None:
        """Overwrite the rest joints in place; a new row count rebuilds (configuration_task.py:153-177)."""
        if T_world_base_rest is not None:
            new_b = _pose_rows(T_world_base_rest)
            cur_b = self._base_rest
            if isinstance(cur_b, N.DeviceArray) and cur_b.shape == new_b.shape:
                cur_b.assign(new_b)
            else:
                self._base_rest_arg = T_world_base_rest
                self._base_rest = new_b
                self._touch()
        if rest_q is None:
            return
        na = self.robot.spec.num_actuated_joints if self.robot is not None else np.asarray(rest_q).shape[-1]
        new = _ref_rows(rest_q, na)
        cur = self._rest
        if cur is not None and cur.shape == new.shape:
            if isinstance(cur, N.DeviceArray):
                cur.assign(new)
            else:
                self._rest = new.numpy() if isinstance(new, N.DeviceArray) else new
                self._touch()
            return
        self._rest = new
        self._touch()


class VelocityLimitTask(_PrevStateEval, _JointRefTask):
    """Penalise joint speeds above their limits relative to a previous state,
    w max(0, |q - q_prev| / dt - v_max) (velocity_limit_task.py:14-232).

    ``velocity_limits`` defaults to the robot's actuated joint velocity limits and
    ``weight`` to 1 per joint.  Without a previous state the term adds zero rows."""

    def __init__(self, robot: Any = None, dt: Any = 1.0, prev_state_var: Any = None, velocity_limits: Any = None,
                 weight: Optional[Union[float, Sequence[float]]] = None, name: str = ""):
        if isinstance(dt, Context):
            raise NotImplementedError("a helper-given dt is outside the IK hot path")
        if not dt > 0:
            raise ValueError("dt must be positive")
        if isinstance(velocity_limits, Context):
            raise NotImplementedError("helper-given velocity limits are outside the IK hot path")
        self.name = name
        self.dt = float(dt)
        self.weight = weight
        self.velocity_limits = None if velocity_limits is None else np.asarray(velocity_limits, np.float32)
        self.robot = robot
        self.prev_state_var = prev_state_var
        self._prev_q: Any = None
        if prev_state_var is not None and not isinstance(prev_state_var, Context):
            self._prev_q = _ref_rows(prev_state_var.q, prev_state_var.spec.num_actuated_joints)
            if isinstance(self._prev_q, N.DeviceArray):  # the reference clones the state (velocity_limit_task.py:39)
                self._prev_q = self._prev_q.clone()

    @property
    def active(self) -> bool:
        return self.weight is None or bool(np.any(self.weight))

    def _joint_weights(self, na: int) -> np.ndarray:
        w = np.ones(na, np.float32)
        if self.weight is not None:
            w[:] = self.weight
        return w if self._prev_q is not None else np.zeros_like(w)

    def _limits(self, var: Any) -> np.ndarray:
        na = var.spec.num_actuated_joints
        v = self.velocity_limits if self.velocity_limits is not None else var.spec.actuated_joint_velocity_limits
        v = np.asarray(v, np.float32).reshape(-1)
        if v.shape != (na,):
            raise ValueError(f"velocity_limits has {v.shape[0]} entries for {na} actuated joints")
        return v

    def _reference(self, na: int) -> Any:
        return self._prev_q if self._prev_q is not None else np.zeros((1, na), np.float32)

    def native_desc(self, var: Any) -> Dict[str, Any]:
        d = super().native_desc(var)
        d.update(kind=N.IK_TERM_VELOCITY_LIMIT, dt=self.dt, velocity_limits=self._limits(var))
        return d

    def host_desc(self, var: Any) -> Dict[str, Any]:
        d = super().host_desc(var)
        d.update(kind=N.IK_TERM_VELOCITY_LIMIT, dt=self.dt, velocity_limits=self._limits(var))
        return d

    def set_weight(self, weight: Union[float, Sequence[float]]) -> None:
        self.weight = weight
        self._touch()

    def bind_previous(self, prev_q: N.DeviceArray) -> None:
        """Read the previous joints from `prev_q` [rows, na] in place from now on."""
        self._prev_q = prev_q
        self._touch()

    def set_prev_state(self, prev_state: Any) -> None:
        """Copy a new previous state in place; a new row count rebuilds (velocity_limit_task.py:81-88)."""
        new = _ref_rows(prev_state.q, prev_state.spec.num_actuated_joints)
        if isinstance(self._prev_q, N.DeviceArray) and self._prev_q.shape == new.shape:
            self._prev_q.assign(new)
            return
        self._prev_q = new.clone() if isinstance(new, N.DeviceArray) else new
        self._touch()


_PENALTIES = {"smooth": N.IK_PENALTY_SMOOTH, "plain": N.IK_PENALTY_PLAIN,
              "surface_distance": N.IK_PENALTY_SURFACE_DISTANCE}


class SceneCollisionTask(ResidualTask):
    """Penalise robot collision spheres that approach scene geometry (scene_collision_task.py:276-650).

    One row per queried sphere: w * penalty(sdf(centre) - radius) with the
    reference's "smooth" (default), "plain" or "surface_distance" penalty and
    the "abs" or "sqrt_abs" residual.  The scene holds primitives (boxes,
    spheres, planes, capsules; robokit_b200.geom); `scene_indices` picks each
    problem's scene (row b // (batch // rows)).  The link bounding-sphere
    filter only skips queries whose rows are zero anyway, so it is accepted and
    changes nothing here."""

    def __init__(self, robot: Any = None, scene: Any = None, geometry: Any = None, scene_indices: Any = None,
                 use_link_bounding_sphere_filter: bool = False, weight: Union[float, Sequence[float]] = 1.0,
                 margin: Optional[float] = 0.02, sphere_indices: Optional[Sequence[int]] = None,
                 residual_mode: Literal["abs", "sqrt_abs"] = "abs", residual_eps: float = 1e-6,
                 penalty: Literal["smooth", "plain", "surface_distance"] = "smooth",
                 skip_trajectory_endpoints: bool = True, movable_only: bool = False, name: str = ""):
        if penalty not in _PENALTIES:
            raise ValueError(f"Unsupported penalty: {penalty}")
        if residual_mode not in ("abs", "sqrt_abs"):
            raise ValueError(f"Unsupported residual_mode: {residual_mode}")
        if use_link_bounding_sphere_filter and penalty == "surface_distance":
            raise NotImplementedError("the link filter with the surface-distance penalty is not supported")
        self.name = name
        self.robot = robot
        self.scene = scene
        self.geometry = geometry
        self.scene_indices = scene_indices
        self.use_link_bounding_sphere_filter = use_link_bounding_sphere_filter
        self.weight = weight
        self.margin = 0.0 if margin is None else float(margin)
        self.sphere_indices = sphere_indices
        self.residual_mode = residual_mode
        self.residual_eps = residual_eps
        self.penalty = penalty
        self.skip_trajectory_endpoints = skip_trajectory_endpoints
        self.movable_only = movable_only
        self._own_version = 0
        self._scene_idx_dev: Optional[N.DeviceArray] = None
        if robot is None or isinstance(scene, Context) or isinstance(scene_indices, Context):
            return  # configuration-time stub
        self.set_robot(robot)
        if scene_indices is not None:
            self.set_scene_indices(scene_indices)

    # -- configuration ----------------------------------------------------------------
    @property
    def _version(self) -> Any:
        rev = self.scene.revision if self.scene is not None and not isinstance(self.scene, Context) else 0
        return (self._own_version, rev)

    def _touch(self) -> None:
        self._own_version += 1

    @property
    def active(self) -> bool:
        """Nonzero weight and a scene with geometry, or a helper's scene to come."""
        if self.scene is None:
            return False
        if not isinstance(self.scene, Context) and self.scene.num_elements == 0:
            return False
        return bool(np.any(np.asarray(self.weight, np.float32)))

    def set_robot(self, robot: Any) -> None:
        self.robot = robot
        spec = robot.spec
        ns = len(spec.collision_sphere_radii)
        if ns == 0:
            raise RuntimeError("Robot has no collision spheres. Load with load_collision_spheres=True.")
        if self.sphere_indices is None and self.movable_only:
            self.sphere_indices = np.flatnonzero(np.asarray(spec.collision_spheres_link_indices) > 0)
        idx = np.arange(ns, dtype=np.int32) if self.sphere_indices is None else np.asarray(self.sphere_indices,
                                                                                           np.int32)
        if idx.ndim != 1:
            raise ValueError("sphere_indices must be 1D.")
        if np.any(idx < 0) or np.any(idx >= ns):
            raise ValueError("sphere_indices contains out-of-range indices.")
        self._sphere_idx = idx
        w = np.ones(idx.shape[0], np.float32)
        if isinstance(self.weight, (int, float)):
            w[:] = float(self.weight)
        else:
            wa = np.asarray(self.weight, np.float32)
            if wa.shape != (idx.shape[0],):
                raise ValueError(f"Expected weight shape ({idx.shape[0]},), got {wa.shape}.")
            w[:] = wa
        self._weights = w
        self._touch()

    def set_weight(self, weight: Union[float, Sequence[float]]) -> None:
        self.weight = weight
        if self.robot is not None:
            self.set_robot(self.robot)

    def set_scene_indices(self, scene_indices: Any) -> None:
        """The scene of each problem row, int32 (scene_collision_task.py:412-437); read in place when on the device."""
        if isinstance(scene_indices, N.DeviceArray) or hasattr(scene_indices, "__cuda_array_interface__"):
            try:
                d = N.as_device(scene_indices, np.int32)
            except TypeError as e:
                raise TypeError(f"scene_indices must be a 1D int32 array ({e}).") from None
        else:
            a = np.asarray(scene_indices)
            if a.dtype != np.int32:
                raise TypeError(f"scene_indices must be a 1D int32 array, got {a.dtype}.")
            d = N.DeviceArray.from_numpy(np.ascontiguousarray(a))
        if d.ndim != 1:
            raise TypeError("scene_indices must be a 1D int32 array.")
        if d.shape[0] < 1:
            raise ValueError("scene_indices must not be empty.")
        self.scene_indices = d
        self._scene_idx_dev = d
        self._touch()

    @property
    def residual_dim(self) -> int:
        return int(self._sphere_idx.shape[0])

    # -- lowering -----------------------------------------------------------------------
    def _desc(self, var: Any, scene_idx: Any) -> Dict[str, Any]:
        if self.robot is None or self.scene is None or isinstance(self.scene, Context):
            raise ValueError("SceneCollisionTask needs a robot and a scene (build it through a helper or pass both)")
        if var.spec.num_links != self.robot.spec.num_links:
            raise ValueError("term built for another robot")
        if scene_idx is not None and var.batch_size % scene_idx.shape[0]:
            raise ValueError("scene_indices must have shape (batch_size,) or divide it (one scene per candidate "
                             "group).")
        return dict(kind=N.IK_TERM_SCENE_COLLISION, weights=self._weights, query_spheres=self._sphere_idx,
                    geoms=self.scene.records(self.geometry), num_scenes=self.scene.num_scenes,
                    penalty=_PENALTIES[self.penalty], residual_sqrt=self.residual_mode == "sqrt_abs",
                    residual_eps=float(self.residual_eps), margin=self.margin, scene_indices=scene_idx)

    def native_desc(self, var: Any) -> Dict[str, Any]:
        return self._desc(var, self._scene_idx_dev)

    def host_desc(self, var: Any) -> Dict[str, Any]:
        si = None if self._scene_idx_dev is None else self._scene_idx_dev.numpy()
        return self._desc(var, si)


class SelfCollisionTask(ResidualTask):
    """Sphere self-collision hinge w * max(0, margin - surface distance) (self_collision_task.py:593-1152).

    ``pair_mode="slots"`` is the reference: at most ``max_active_pairs`` link
    pairs whose bounding spheres come within the margin, each scored by its most
    penetrating sphere pair.  ``pair_mode="all"`` scores every filtered sphere
    pair as its own residual row (no reference counterpart).
    """

    def __init__(self, robot: Any = None, weight: float = 1.0, margin: float = 0.02,
                 representation: Literal["sphere", "capsule", "link_sphere"] = "sphere",
                 residual_mode: Literal["abs", "sqrt_abs"] = "abs", residual_eps: float = 1e-6,
                 filter_adjacent_links: bool = True, max_active_pairs: int = 50, name: str = "",
                 pair_mode: Literal["slots", "all"] = "slots"):
        if representation != "sphere":
            raise NotImplementedError(f"representation={representation!r} is outside the IK hot path (spheres only)")
        if residual_mode != "abs":
            raise NotImplementedError("only residual_mode='abs' is on the IK hot path")
        if pair_mode not in ("slots", "all"):
            raise ValueError("pair_mode must be 'slots' or 'all'")
        self.name = name
        self.robot = robot
        self.weight = float(weight)
        self.margin = float(margin)
        self.representation = representation
        self.residual_mode = residual_mode
        self.filter_adjacent_links = filter_adjacent_links
        self.max_active_pairs = int(max_active_pairs)
        self.pair_mode = pair_mode
        if robot is None:
            return
        if self.max_active_pairs < 1:
            raise ValueError("max_active_pairs must be >= 1.")
        spec = robot.spec
        if not spec.has_collision_spheres:
            raise ValueError("Robot has no collision spheres.")
        if len(spec.collision_sphere_radii) < 2:
            raise ValueError("Expected at least two collision spheres.")
        self._pairs, self._link_pairs, self._offsets, self._grouped = collision_pair_tables(
            spec, filter_adjacent_links
        )

    def set_robot(self, robot: Any) -> None:
        SelfCollisionTask.__init__(self, robot, self.weight, self.margin, self.representation, self.residual_mode,
                                   1e-6, self.filter_adjacent_links, self.max_active_pairs, self.name, self.pair_mode)

    @property
    def num_pairs(self) -> int:
        return len(self._pairs)

    @property
    def residual_dim(self) -> int:
        return self.max_active_pairs if self.pair_mode == "slots" else len(self._grouped)

    def native_desc(self, var: Any) -> Dict[str, Any]:
        return dict(
            kind=N.IK_TERM_SELF_COLLISION,
            weights=np.array([self.weight], np.float32),
            margin=self.margin,
            max_active_pairs=self.max_active_pairs,
            pair_mode=N.IK_PAIRS_SLOTS if self.pair_mode == "slots" else N.IK_PAIRS_ALL,
            num_link_pairs=len(self._link_pairs),
            link_pairs=self._link_pairs.reshape(-1),
            link_pair_offsets=self._offsets,
            num_sphere_pairs=len(self._grouped),
            sphere_pairs=self._grouped.reshape(-1),
        )
