"""Dense residual terms of the IK path.

PositionTask (terms/dense/position_task.py:18-272), RotationTask
(terms/dense/rotation_task.py:25-401), PositionLimit in "abs" mode
(terms/dense/position_limit.py:185-573) and SelfCollisionTask with sphere
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
