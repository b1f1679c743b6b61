"""Scene geometry for SceneCollisionTask: primitive shapes grouped into scenes (geom/scene.py:20-400,
geom/geoms.py:60-500).

A Scene holds `num_scenes` independent scenes; each geom holds N primitives of
one shape with CSR `scene_offsets` (scene s owns primitives
[offsets[s], offsets[s+1])), optional world poses and uniform scales.  A point
queries the primitives of its scene in the order the geoms were added and, per
geom, in index order, keeping the first of strictly least signed distance.
Boxes, spheres, planes and capsules are supported; meshes and SDF volumes are
not.  The geometry is copied into each problem's device tables when a term is
lowered, so a change (update, add) makes the terms that read it rebuild.
"""

from __future__ import annotations

from typing import Any, List, Optional, Sequence, Tuple

import numpy as np

from .. import _native as N

MAX_DIST = 1e6  # distance of a point in an empty scene (geom/geoms.py:29)


def _poses_vec7(poses: Any, n: int) -> np.ndarray:
    """[n, 7] poses [x y z qw qx qy qz] from vec7 rows or 4x4 transforms (host or device)."""
    if poses is None:
        return np.tile(np.array([0, 0, 0, 1, 0, 0, 0], np.float32), (n, 1))
    a = poses.numpy() if hasattr(poses, "numpy") else np.asarray(poses)
    a = np.asarray(a, np.float64)
    if a.shape[-2:] == (4, 4):
        a = a.reshape(-1, 4, 4)
        from ..robo.robot_spec import matrix_to_quaternion

        q = np.stack([matrix_to_quaternion(m[:3, :3]) for m in a])
        out = np.concatenate([a[:, :3, 3], q], axis=1)
    else:
        out = a.reshape(-1, 7)
    if out.shape[0] < n:
        raise ValueError(f"{out.shape[0]} poses for {n} primitives")
    return np.ascontiguousarray(out[:n], np.float32)


class BaseGeom:
    """N primitives of one shape (geom/geoms.py:60-370)."""

    TYPE_ID = -1

    def __init__(self, count: int, scene_offsets: Any, poses: Any, scales: Any, capacity: Optional[int]):
        if count == 0:
            raise ValueError("Must pass at least one element.")
        self.count = count
        self.capacity = count if capacity is None else int(capacity)
        if self.capacity < count:
            raise ValueError(f"capacity {self.capacity} < element count {count}.")
        self._params = np.zeros((count, 4), np.float32)
        self._set(scene_offsets, poses, scales)
        self._scene: Optional["Scene"] = None

    def _set(self, scene_offsets: Any, poses: Any, scales: Any) -> None:
        off = np.asarray(scene_offsets, np.int64).reshape(-1)
        if off.size < 2 or off[0] != 0 or off[-1] != self.count or np.any(np.diff(off) < 0):
            raise ValueError(f"scene_offsets must run from 0 to {self.count} without decreasing, got {off}")
        self.scene_offsets = off.astype(np.int32)
        self.poses = _poses_vec7(poses, self.count)
        self.scales = np.ones(self.count, np.float32) if scales is None else np.asarray(
            scales.numpy() if hasattr(scales, "numpy") else scales, np.float32).reshape(-1)[: self.count].copy()
        if self.scales.size != self.count or np.any(~(self.scales > 0)):
            raise ValueError("scales must hold one positive value per primitive")

    @property
    def num_scenes(self) -> int:
        return self.scene_offsets.size - 1

    def _changed(self) -> None:
        if self._scene is not None:
            self._scene._revision += 1

    def _update(self, params: Optional[np.ndarray], scene_offsets: Any, poses: Any, scales: Any) -> None:
        n = self.count if scene_offsets is None else int(np.asarray(scene_offsets).reshape(-1)[-1])
        if n > self.capacity:
            raise ValueError(f"update: {n} elements exceed capacity {self.capacity}.")
        if scene_offsets is None and params is not None and params.shape[0] != self.count:
            raise ValueError(f"update: count changed ({self.count} -> {params.shape[0]}); pass scene_offsets.")
        if params is not None:
            self._params = params
        self.count = n if scene_offsets is not None else self.count
        self._set(self.scene_offsets if scene_offsets is None else scene_offsets,
                  self.poses if poses is None else poses, self.scales if scales is None else scales)
        self._changed()

    def records(self) -> np.ndarray:
        """[count, IK_GEOM_FLOATS] host records (include/b200ik.h)."""
        rec = np.zeros((self.count, N.IK_GEOM_FLOATS), np.float32)
        rec[:, 0] = self.TYPE_ID
        scene = np.repeat(np.arange(self.num_scenes), np.diff(self.scene_offsets))
        rec[:, 1] = scene
        rec[:, 2] = self.scales
        rec[:, 4:8] = self._params[: self.count]
        rec[:, 8:15] = self.poses
        return rec


def _vec4(cols: np.ndarray) -> np.ndarray:
    out = np.zeros((cols.shape[0], 4), np.float32)
    out[:, : cols.shape[1]] = cols
    return out


class BoxGeom(BaseGeom):
    """N boxes: `half_extents (N, 3)`, posed via `poses` (geom/geoms.py:372-401)."""

    TYPE_ID = N.IK_GEOM_BOX

    def __init__(self, half_extents: Any, scene_offsets: Any, poses: Any = None, scales: Any = None,
                 capacity: Optional[int] = None):
        he = np.asarray(half_extents, np.float32).reshape(-1, 3)
        super().__init__(he.shape[0], scene_offsets, poses, scales, capacity)
        self._params = _vec4(he)

    def update(self, half_extents: Any = None, scene_offsets: Any = None, poses: Any = None, scales: Any = None):
        p = None if half_extents is None else _vec4(np.asarray(half_extents, np.float32).reshape(-1, 3))
        self._update(p, scene_offsets, poses, scales)


class SphereGeom(BaseGeom):
    """N spheres: `radii (N,)`, centred via `poses` (geom/geoms.py:404-429)."""

    TYPE_ID = N.IK_GEOM_SPHERE

    def __init__(self, radii: Any, scene_offsets: Any, poses: Any = None, scales: Any = None,
                 capacity: Optional[int] = None):
        r = np.asarray(radii, np.float32).reshape(-1, 1)
        super().__init__(r.shape[0], scene_offsets, poses, scales, capacity)
        self._params = _vec4(r)

    def update(self, radii: Any = None, scene_offsets: Any = None, poses: Any = None, scales: Any = None):
        p = None if radii is None else _vec4(np.asarray(radii, np.float32).reshape(-1, 1))
        self._update(p, scene_offsets, poses, scales)


class PlaneGeom(BaseGeom):
    """Halfspaces below local z = 0 (signed distance = local z), one per `scene_offsets[-1]`
    (geom/geoms.py:432-455)."""

    TYPE_ID = N.IK_GEOM_PLANE

    def __init__(self, scene_offsets: Any, poses: Any = None, scales: Any = None, capacity: Optional[int] = None):
        count = int(np.asarray(scene_offsets).reshape(-1)[-1])
        super().__init__(count, scene_offsets, poses, scales, capacity)

    def update(self, scene_offsets: Any = None, poses: Any = None, scales: Any = None):
        n = self.count if scene_offsets is None else int(np.asarray(scene_offsets).reshape(-1)[-1])
        self._update(np.zeros((n, 4), np.float32), scene_offsets, poses, scales)


class CapsuleGeom(BaseGeom):
    """N capsules: `radii (N,)`, `half_heights (N,)`, axis local z (geom/geoms.py:458-499)."""

    TYPE_ID = N.IK_GEOM_CAPSULE

    def __init__(self, radii: Any, half_heights: Any, scene_offsets: Any, poses: Any = None, scales: Any = None,
                 capacity: Optional[int] = None):
        cols = np.stack([np.asarray(radii, np.float32).reshape(-1), np.asarray(half_heights, np.float32).reshape(-1)],
                        axis=1)
        super().__init__(cols.shape[0], scene_offsets, poses, scales, capacity)
        self._params = _vec4(cols)

    def update(self, radii: Any = None, half_heights: Any = None, scene_offsets: Any = None, poses: Any = None,
               scales: Any = None):
        if (radii is None) != (half_heights is None):
            raise ValueError("CapsuleGeom.update: pass radii and half_heights together.")
        p = None
        if radii is not None:
            p = _vec4(np.stack([np.asarray(radii, np.float32).reshape(-1),
                                np.asarray(half_heights, np.float32).reshape(-1)], axis=1))
        self._update(p, scene_offsets, poses, scales)


class Scene:
    """`num_scenes` scenes of primitive geoms (WarpScene, geom/scene.py:20-130)."""

    def __init__(self, num_scenes: int = 1, device: Any = "cuda"):
        if num_scenes < 1:
            raise ValueError("num_scenes must be >= 1")
        if device is not None and not str(device).startswith("cuda"):
            raise ValueError(f"device {device!r}: this library runs on CUDA only (no CPU fallback)")
        self._num_scenes = int(num_scenes)
        self._geoms: List[BaseGeom] = []
        self._revision = 0

    @property
    def num_scenes(self) -> int:
        return self._num_scenes

    @property
    def geoms(self) -> Tuple[BaseGeom, ...]:
        return tuple(self._geoms)

    @property
    def num_elements(self) -> int:
        return sum(g.count for g in self._geoms)

    @property
    def revision(self) -> int:
        """Advances with every change; terms reading this scene rebuild when it does."""
        return self._revision

    def add(self, geom: BaseGeom) -> "Scene":
        if not isinstance(geom, BaseGeom):
            raise TypeError(f"{type(geom).__name__} is not a primitive geom (meshes and volumes are not supported)")
        if geom.num_scenes != self._num_scenes:
            raise ValueError(f"geom has {geom.num_scenes} scenes, scene has {self._num_scenes}")
        geom._scene = self
        self._geoms.append(geom)
        self._revision += 1
        return self

    def records(self, geometry: Optional[BaseGeom] = None) -> np.ndarray:
        """All primitive records in query order (or one geom's), [n, IK_GEOM_FLOATS]."""
        geoms: Sequence[BaseGeom] = [geometry] if geometry is not None else self._geoms
        if not geoms:
            return np.zeros((0, N.IK_GEOM_FLOATS), np.float32)
        return np.concatenate([g.records() for g in geoms], axis=0)

    def __repr__(self) -> str:
        return f"Scene(num_scenes={self._num_scenes}, geoms={[type(g).__name__ for g in self._geoms]})"


__all__ = ["BaseGeom", "BoxGeom", "CapsuleGeom", "MAX_DIST", "PlaneGeom", "Scene", "SphereGeom"]
