"""Robot: the model object of the IK path (robokit robo/robot.py:29-633)."""

from __future__ import annotations

import ctypes
import weakref
from typing import Any, Optional, Sequence, Union

import numpy as np

from .. import _native as N
from .robot_spec import RobotSpec
from .robot_state import RobotState


def _destroy_robot(handle: int) -> None:
    try:
        if N._lib is not None and handle:
            N._lib.ik_robot_destroy(ctypes.c_void_p(handle))
    except Exception:
        pass


class Robot:
    """Robot model whose kinematics run on the sm_100a kernels of libb200ik.so."""

    def __init__(self, spec: RobotSpec):
        self.spec = spec
        self._handle: Optional[int] = None
        self._fin = None
        self._limits_dev: Optional[N.DeviceArray] = None

    def __repr__(self) -> str:
        return (
            f"Robot(name={self.spec.name}, num_actuated_joints={self.spec.num_actuated_joints}, "
            f"num_links={self.spec.num_links})"
        )

    @staticmethod
    def load(
        robot_description_or_path: Any,
        load_collision_spheres: bool = False,
        collision_spheres_path: Optional[str] = None,
        base_link_name: Optional[str] = None,
        ee_link_names: Optional[Union[Sequence[str], str]] = None,
        self_collision_ignore_path: Optional[str] = None,
    ) -> "Robot":
        """URDF path or text -> Robot (robo/robot.py:59-103)."""
        return Robot(
            RobotSpec.parse(
                robot_description_or_path,
                load_collision_spheres=load_collision_spheres,
                collision_spheres_path=collision_spheres_path,
                self_collision_ignore_path=self_collision_ignore_path,
                base_link_name=base_link_name,
                ee_link_names=ee_link_names,
            )
        )

    # --- sizes -----------------------------------------------------------------
    @property
    def link_names(self):
        return self.spec.link_names

    @property
    def num_actuated_joints(self) -> int:
        return self.spec.num_actuated_joints

    @property
    def zero_q(self) -> np.ndarray:
        return self.spec.zero_q

    # --- native handle ----------------------------------------------------------
    @property
    def handle(self) -> int:
        """IkRobot* of this robot (created on first use; tables are copied to the device)."""
        if self._handle is None:
            t = self.spec.native_tables()
            d = N.IkRobotDesc()
            d.num_joints = self.spec.num_joints
            d.num_links = self.spec.num_links
            d.num_actuated = self.spec.num_actuated_joints
            d.num_spheres = len(self.spec.collision_sphere_radii)
            for name, arr in t.items():
                setattr(d, name, arr.ctypes.data if arr.size else None)
            h = ctypes.c_void_p(0)
            N.check(N.lib().ik_robot_create(ctypes.byref(d), ctypes.byref(h)))
            self._handle = h.value
            self._fin = weakref.finalize(self, _destroy_robot, self._handle)
        return self._handle

    def limits_device(self) -> N.DeviceArray:
        if self._limits_dev is None:
            self._limits_dev = N.DeviceArray.from_numpy(self.spec.float32_actuated_limits().reshape(-1))
        return self._limits_dev

    # --- state and kinematics -----------------------------------------------------
    def state(self, q: Any = None, T_world_base: Any = None) -> RobotState:
        """RobotState for joint positions q (default zero_q), optional floating base (robo/robot.py:105-129)."""
        if q is None:
            q = self.spec.zero_q[None]
        return RobotState(self, q, T_world_base)

    def forward_kinematics(self, state: RobotState) -> RobotState:
        """T_world_joint, T_world_link, S_world and the collision spheres in one launch (robo/robot.py:131-271)."""
        B = state.batch_size
        spec = self.spec
        ns = len(spec.collision_sphere_radii)
        N.check(
            N.lib().ik_fk(
                self.handle,
                B,
                state.q.ptr,
                state.T_world_base.ptr if state.has_floating_base else None,
                state.T_world_joint.ptr,
                state.T_world_link.ptr,
                state.S_world.ptr,
                state.collision_sphere_centers_world.ptr if ns else None,
                state.link_bounding_sphere_centers_world.ptr if ns else None,
                None,
            )
        )
        state.is_fk_computed = True
        state.is_motion_subspace_computed = True
        state.is_collision_spheres_computed = ns > 0
        return state

    def compute_motion_subspace(self, state: RobotState) -> RobotState:
        """The FK launch writes S_world with the poses (robo/robot.py:355-397)."""
        return self.forward_kinematics(state)

    def transform_collision_spheres(self, state: RobotState) -> RobotState:
        if not self.spec.has_collision_spheres:
            return state
        return self.forward_kinematics(state)

    def sample_q(self, num_samples: int = 1, rng: Optional[np.random.Generator] = None, device: Any = None,
                 seed: Optional[int] = None) -> np.ndarray:
        """`num_samples` joint configurations, uniform within the limits, as a host float32 array
        (robo/robot.py:633-650); `rng` (a numpy Generator) or `seed` picks the stream."""
        if device is not None and not str(device).startswith("cuda"):
            raise ValueError(f"device {device!r}: this library runs on CUDA only (no CPU fallback)")
        rng = rng if rng is not None else np.random.default_rng(seed)
        lim = self.spec.float32_actuated_limits()
        return rng.uniform(lim[:, 0], lim[:, 1], size=(num_samples, lim.shape[0])).astype(np.float32)
