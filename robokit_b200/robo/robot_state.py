"""RobotState: the optimisation variable of the IK path (robokit robo/robot_state.py:41-476)."""

from __future__ import annotations

from typing import TYPE_CHECKING, Any, Literal, Optional

import numpy as np

from .. import _native as N
from ..opt.var_values import Var

if TYPE_CHECKING:
    from .robot import Robot

_IDENTITY = np.array([0, 0, 0, 1, 0, 0, 0], np.float32)
_LAZY = ("T_world_joint", "T_world_link", "S_world", "collision_sphere_centers_world",
         "link_bounding_sphere_centers_world")


class RobotState(Var):
    """Joint positions ``q [B, dofs]`` and an optional floating base ``T_world_base [B, 7]``.

    Tangent layout: [6 base twist entries if floating | actuated joints]
    (robo/robot_state.py:173-181).  Derived buffers (link poses, motion
    subspace, world spheres) are device arrays filled by
    ``Robot.forward_kinematics``.
    """

    def __init__(self, robot: "Robot", q: Any, T_world_base: Any = None):
        self.robot = robot
        self.spec = robot.spec
        na = self.spec.num_actuated_joints
        qd = N.as_device(q, np.float32)
        if qd.ndim == 1:
            qd = qd.reshape((1, qd.shape[0]))
        if qd.ndim != 2 or qd.shape[1] != na:
            raise ValueError(f"Expected q to have {na} DOFs, but got shape {qd.shape}")
        self.q = qd
        self.base_step_scale = 1e-4
        self.clamp_q_on_integrate = False
        if T_world_base is None:
            self.T_world_base = N.DeviceArray.from_numpy(np.tile(_IDENTITY, (qd.shape[0], 1)))
            self.has_floating_base = False
        else:
            b = N.as_device(T_world_base, np.float32)
            self.T_world_base = b.reshape((qd.shape[0], 7))
            self.has_floating_base = True
        self.invalidate()

    def __repr__(self) -> str:
        return f"RobotState(batch={self.batch_size}, floating={self.has_floating_base}, fk={self.is_fk_computed})"

    # --- lazily allocated derived buffers ------------------------------------------
    def __getattr__(self, name: str):
        if name in _LAZY and "_view_source" in self.__dict__:
            # a view's buffers are rows of its source's (allocated there on first use)
            off = self.__dict__["_view_offset"]
            arr = getattr(self.__dict__["_view_source"], name).row_slice(off, off + self.batch_size)
            self.__dict__[name] = arr
            return arr
        if name in _LAZY:
            B, s = self.batch_size, self.spec
            ns = len(s.collision_sphere_radii)
            shapes = {
                "T_world_joint": (B, s.num_joints, 7),
                "T_world_link": (B, s.num_links, 7),
                "S_world": (B, 6, max(s.num_joints, 1)),
                "collision_sphere_centers_world": (B, ns, 3),
                "link_bounding_sphere_centers_world": (B, s.num_links, 3),
            }
            arr = N.DeviceArray.zeros(shapes[name], np.float32)
            self.__dict__[name] = arr
            return arr
        raise AttributeError(name)

    # --- shape --------------------------------------------------------------------
    @property
    def batch_size(self) -> int:
        return self.q.shape[0]

    @property
    def shape(self):
        return self.q.shape[:-1]

    @property
    def num_elements(self) -> int:
        return self.batch_size

    @property
    def device(self) -> str:
        return "cuda:0"

    @property
    def tangent_dim(self) -> int:
        return (6 if self.has_floating_base else 0) + self.spec.num_actuated_joints

    # --- computed results --------------------------------------------------------
    def get_T_world_link(self, link_index: int) -> N.DeviceArray:
        if not self.is_fk_computed:
            raise RuntimeError("Forward kinematics has not been computed. Call robot.forward_kinematics() first.")
        B, nl = self.batch_size, self.spec.num_links
        out = N.DeviceArray.empty((B, 7), np.float32)
        N.check(N.lib().ik_copy_rows(B, 7, self.T_world_link.ptr + 4 * 7 * link_index, nl * 7, out.ptr, 7, None))
        return out

    def get_link_jacobian(self, link_index: int, reference_frame: Literal["body", "spatial"] = "body") -> N.DeviceArray:
        """[B, 6, tangent] link Jacobian (robo/robot_state.py:192-236)."""
        out = N.DeviceArray.empty((self.batch_size, 6, self.tangent_dim), np.float32)
        N.check(
            N.lib().ik_link_jacobian(
                self.robot.handle,
                self.batch_size,
                self.q.ptr,
                self.T_world_base.ptr if self.has_floating_base else None,
                int(link_index),
                1 if reference_frame == "body" else 0,
                out.ptr,
                None,
            )
        )
        return out

    # --- solver interface ----------------------------------------------------------
    def invalidate(self) -> None:
        self.is_fk_computed = False
        self.is_motion_subspace_computed = False
        self.is_collision_spheres_computed = False

    def precompute(self) -> None:
        if not self.is_fk_computed:
            self.robot.forward_kinematics(self)

    def integrate(self, velocity: Any, out: Optional["RobotState"] = None, tangent_mask: Any = None,
                  weight_decay: float = 0.0, out_velocity: Any = None) -> "RobotState":
        """q' = q + mask*v; base' = base * exp(v_base) (robo/robot_state.py:238-312)."""
        if weight_decay != 0.0 or out_velocity is not None:
            raise NotImplementedError("weight_decay / out_velocity are not on the IK path")
        v = N.as_device(velocity, np.float32)
        if v.shape != (self.batch_size, self.tangent_dim):
            raise ValueError(f"Expected velocity shape {(self.batch_size, self.tangent_dim)}, but got {v.shape}")
        if out is None:
            out = RobotState(self.robot, N.DeviceArray.empty(self.q.shape, np.float32),
                             N.DeviceArray.empty(self.T_world_base.shape, np.float32) if self.has_floating_base else None)
        m = N.as_device(tangent_mask, np.float32) if tangent_mask is not None else None
        N.check(
            N.lib().ik_integrate(
                self.batch_size,
                self.spec.num_actuated_joints,
                int(self.has_floating_base),
                self.q.ptr,
                self.T_world_base.ptr,
                v.ptr,
                N.ptr(m),
                out.q.ptr,
                out.T_world_base.ptr,
                None,
            )
        )
        if not self.has_floating_base and out.T_world_base.ptr != self.T_world_base.ptr:
            out.T_world_base.assign(self.T_world_base)
        out.invalidate()
        if self.clamp_q_on_integrate:
            out.clamp_q()
        return out

    def clamp_q(self, tangent_mask: Any = None) -> "RobotState":
        """Clamp to the float32-narrowed limits, sparing masked coordinates (robo/robot_state.py:314-333)."""
        m = None
        if tangent_mask is not None:
            mm = np.asarray(N.as_device(tangent_mask, np.float32).numpy()).reshape(-1)
            m = N.DeviceArray.from_numpy(mm[(6 if self.has_floating_base else 0):])
        N.check(N.lib().ik_clamp_q(self.batch_size, self.spec.num_actuated_joints, self.q.ptr,
                                   self.robot.limits_device().ptr, N.ptr(m), None))
        self.invalidate()
        return self

    def accept(self, accept_mask: Any, proposed: "RobotState") -> "RobotState":
        """Copy rows of `proposed` where accept_mask == 1 (robo/robot_state.py:448-476)."""
        mk = N.as_device(accept_mask, np.int32)
        B = self.batch_size
        N.check(N.lib().ik_masked_copy_rows(B, self.spec.num_actuated_joints, mk.ptr, proposed.q.ptr, self.q.ptr, None))
        if self.has_floating_base:
            N.check(N.lib().ik_masked_copy_rows(B, 7, mk.ptr, proposed.T_world_base.ptr, self.T_world_base.ptr, None))
        if self.is_fk_computed and proposed.is_fk_computed:
            s = self.spec
            N.check(N.lib().ik_masked_copy_rows(B, s.num_joints * 7, mk.ptr, proposed.T_world_joint.ptr,
                                                self.T_world_joint.ptr, None))
            N.check(N.lib().ik_masked_copy_rows(B, s.num_links * 7, mk.ptr, proposed.T_world_link.ptr,
                                                self.T_world_link.ptr, None))
        else:
            self.is_fk_computed = False
        self.is_motion_subspace_computed = False
        self.is_collision_spheres_computed = False
        return self

    def _copy_flags(self, st: "RobotState") -> None:
        st.has_floating_base = self.has_floating_base
        st.is_fk_computed = self.is_fk_computed
        st.is_motion_subspace_computed = self.is_motion_subspace_computed
        st.is_collision_spheres_computed = self.is_collision_spheres_computed
        st.base_step_scale, st.clamp_q_on_integrate = self.base_step_scale, self.clamp_q_on_integrate

    def clone(self) -> "RobotState":
        """Copies of q, the base and every derived buffer already allocated, with the same computed flags
        (robo/robot_state.py:335-354)."""
        st = RobotState.__new__(RobotState)
        st.robot, st.spec = self.robot, self.spec
        st.q, st.T_world_base = self.q.clone(), self.T_world_base.clone()
        for name in _LAZY:
            if name in self.__dict__:
                st.__dict__[name] = self.__dict__[name].clone()
        self._copy_flags(st)
        return st

    def view(self, batch_size: int, offset: int = 0) -> "RobotState":
        """Rows [offset, offset+batch_size) of every buffer, sharing storage and the computed flags
        (robo/robot_state.py:356-380)."""
        if offset < 0 or batch_size < 0 or offset + batch_size > self.batch_size:
            raise ValueError(f"view [{offset}, {offset + batch_size}) outside a batch of {self.batch_size}")
        st = RobotState.__new__(RobotState)
        st.robot, st.spec = self.robot, self.spec
        st.q = self.q.row_slice(offset, offset + batch_size)
        st.T_world_base = self.T_world_base.row_slice(offset, offset + batch_size)
        st.__dict__["_view_source"], st.__dict__["_view_offset"] = self, offset
        for name in _LAZY:
            if name in self.__dict__:
                st.__dict__[name] = self.__dict__[name].row_slice(offset, offset + batch_size)
        self._copy_flags(st)
        return st

    def gather(self, indices: Any, out: Optional["RobotState"] = None, q_only: bool = True) -> "RobotState":
        """Rows `indices` of q and the base into `out` (allocated when omitted); with q_only=False also the
        base of a fixed-base state, the link and joint poses and every other derived buffer already
        allocated, with the source's computed flags (robo/robot_state.py:410-446).  Device gathers; an
        index outside the batch raises IndexError."""
        idx = N.as_device(indices, np.int32)
        n = idx.shape[0]
        if out is None:
            out = RobotState(self.robot, N.DeviceArray.empty((n, self.spec.num_actuated_joints)),
                             N.DeviceArray.empty((n, 7)) if self.has_floating_base else None)
        elif out.batch_size != n:
            raise ValueError(f"out holds {out.batch_size} rows, {n} indices given")
        bad = N.DeviceArray.zeros(1, np.int32)
        src_rows = self.batch_size

        def rows(src: N.DeviceArray, dst: N.DeviceArray) -> None:
            width = int(np.prod(src.shape[1:]))
            N.check(N.lib().ik_gather_rows(n, width, idx.ptr, src_rows, src.ptr, dst.ptr, bad.ptr, None))

        rows(self.q, out.q)
        if self.has_floating_base or not q_only:
            rows(self.T_world_base, out.T_world_base)
        if not q_only:
            for name in _LAZY:
                if name in ("T_world_joint", "T_world_link") or name in self.__dict__:
                    rows(getattr(self, name), getattr(out, name))
        if int(bad.numpy()[0]):
            raise IndexError(f"gather index outside a batch of {src_rows}")
        self._copy_flags(out)
        if q_only:
            out.is_fk_computed = out.is_motion_subspace_computed = out.is_collision_spheres_computed = False
        return out
