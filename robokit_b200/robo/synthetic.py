"""Seeded synthetic robots and IK workloads of the benchmark configurations.

No public robot suite is named for this path, so every workload is generated
from a seed with the sizes and distributions of its configuration:

- ``serial_chain``: 7 revolute joints in series; random unit axes; parent-to-
  joint translations with components U(-0.35, 0.35) m redrawn until their norm
  is >= 0.05 m; identity origin rotations; limits +-U(2.0, 3.0) rad.
- ``add_chain_spheres``: 24 collision spheres on the 7 moving links (4 on the
  first three, 3 on the rest), centres U(-0.1, 0.1) m in the link frame, radii
  U(0.03, 0.08) m.
- ``humanoid``: pelvis base link (floating) -> two legs of 6, a waist of 3 with
  a fixed head frame, two arms of 7 from the waist top (29 revolute joints);
  link offsets with norm U(0.05, 0.40) m in random directions; limits
  +-U(1.5, 3.0) rad.
- ``hand``: floating wrist + 5 fingers of 4 revolute joints (MCP abduction about
  an axis orthogonal to the finger's shared flexion axis, then MCP, PIP, DIP
  flexion) with phalanges U(0.02, 0.05) m and a fixed tip frame; 21 keypoints
  (wrist + MCP, PIP, DIP, tip per finger).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from .robot_spec import JointRecord, RobotSpec


def _unit(rng: np.random.Generator) -> np.ndarray:
    v = rng.standard_normal(3)
    return v / np.linalg.norm(v)


def _offset(rng: np.random.Generator) -> Tuple[float, float, float]:
    while True:
        t = rng.uniform(-0.35, 0.35, 3)
        if np.linalg.norm(t) >= 0.05:
            return tuple(float(x) for x in t)


def serial_chain(seed: int = 0, dofs: int = 7) -> RobotSpec:
    rng = np.random.default_rng(seed)
    links = [f"link{i}" for i in range(dofs + 1)]
    joints: List[JointRecord] = []
    for i in range(dofs):
        lim = float(rng.uniform(2.0, 3.0))
        joints.append(
            JointRecord(
                name=f"joint{i + 1}", type="revolute", parent=links[i], child=links[i + 1], xyz=_offset(rng),
                axis=tuple(float(x) for x in _unit(rng)), lower=-lim, upper=lim,
            )
        )
    return RobotSpec.from_records(f"chain{dofs}_s{seed}", links, joints)


def add_chain_spheres(spec: RobotSpec, seed: int = 0, counts: Optional[List[int]] = None) -> RobotSpec:
    rng = np.random.default_rng(seed + 1000)
    moving = [i for i, j in enumerate(spec.link_parent_joint_indices) if j >= 0]
    counts = counts or ([4, 4, 4] + [3] * (len(moving) - 3))
    centers, radii, links = [], [], []
    for li, n in zip(moving, counts):
        for _ in range(n):
            centers.append(rng.uniform(-0.1, 0.1, 3))
            radii.append(rng.uniform(0.03, 0.08))
            links.append(li)
    spec.set_collision_spheres(np.array(centers), np.array(radii), np.array(links))
    return spec


def humanoid(seed: int = 0) -> RobotSpec:
    rng = np.random.default_rng(seed)
    links = ["pelvis"]
    joints: List[JointRecord] = []

    def off() -> Tuple[float, float, float]:
        d = _unit(rng) * rng.uniform(0.05, 0.40)
        return tuple(float(x) for x in d)

    def chain(parent: str, prefix: str, n: int) -> str:
        cur = parent
        for k in range(n):
            child = f"{prefix}_{k + 1}"
            lim = float(rng.uniform(1.5, 3.0))
            joints.append(JointRecord(name=f"{prefix}_j{k + 1}", type="revolute", parent=cur, child=child,
                                      xyz=off(), axis=tuple(float(x) for x in _unit(rng)), lower=-lim, upper=lim))
            links.append(child)
            cur = child
        return cur

    left_foot = chain("pelvis", "left_leg", 6)
    right_foot = chain("pelvis", "right_leg", 6)
    waist_top = chain("pelvis", "waist", 3)
    links.append("head")
    joints.append(JointRecord(name="head_fixed", type="fixed", parent=waist_top, child="head", xyz=off()))
    left_hand = chain(waist_top, "left_arm", 7)
    right_hand = chain(waist_top, "right_arm", 7)
    spec = RobotSpec.from_records(f"humanoid_s{seed}", links, joints)
    spec.targets = [left_hand, right_hand, left_foot, right_foot, "head"]  # type: ignore[attr-defined]
    return spec


def hand(seed: int = 0) -> RobotSpec:
    rng = np.random.default_rng(seed)
    links = ["wrist"]
    joints: List[JointRecord] = []
    keypoints = ["wrist"]
    for f in range(5):
        angle = -0.6 + 0.3 * f + rng.uniform(-0.05, 0.05)
        d = np.array([np.cos(angle), np.sin(angle), rng.uniform(-0.1, 0.1)])
        d /= np.linalg.norm(d)
        flex = np.cross(d, [0.0, 0.0, 1.0])
        flex /= np.linalg.norm(flex)
        abd = np.cross(flex, d)
        abd /= np.linalg.norm(abd)
        base = (0.07 + rng.uniform(-0.01, 0.01)) * d
        lengths = rng.uniform(0.02, 0.05, 3)
        names = [f"f{f}_abd", f"f{f}_mcp", f"f{f}_pip", f"f{f}_dip", f"f{f}_tip"]
        parent = "wrist"
        origins = [base, np.zeros(3), lengths[0] * d, lengths[1] * d, lengths[2] * d]
        axes = [abd, flex, flex, flex, None]
        for k, nm in enumerate(names):
            link = f"{nm}_link"
            if axes[k] is None:
                joints.append(JointRecord(name=nm, type="fixed", parent=parent, child=link,
                                          xyz=tuple(float(x) for x in origins[k])))
            else:
                lo, hi = (-0.5, 0.5) if k == 0 else (-0.2, 1.8)
                joints.append(JointRecord(name=nm, type="revolute", parent=parent, child=link,
                                          xyz=tuple(float(x) for x in origins[k]),
                                          axis=tuple(float(x) for x in axes[k]), lower=lo, upper=hi))
            links.append(link)
            parent = link
        keypoints += [f"f{f}_mcp_link", f"f{f}_pip_link", f"f{f}_dip_link", f"f{f}_tip_link"]
    spec = RobotSpec.from_records(f"hand_s{seed}", links, joints)
    spec.targets = keypoints  # type: ignore[attr-defined]
    return spec


@dataclass
class Workload:
    """A seeded IK batch: robot, target links, start point and targets."""

    name: str
    spec: RobotSpec
    target_links: List[int]
    q0: np.ndarray
    base0: Optional[np.ndarray]
    targets: np.ndarray  # [B, n_targets, 7]
    q_star: np.ndarray
    pose: bool  # True: Position + Rotation terms; False: positions only
    reachable: Optional[np.ndarray] = None


def _random_pose(rng: np.random.Generator, B: int, trans: float, rot: float) -> np.ndarray:
    out = np.zeros((B, 7), np.float32)
    out[:, :3] = rng.uniform(-trans, trans, (B, 3))
    ax = rng.standard_normal((B, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    ang = rng.uniform(0, rot, B)
    out[:, 3] = np.cos(ang / 2)
    out[:, 4:] = ax * np.sin(ang / 2)[:, None]
    return out


def _quat_to_mat_batch(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    s = 2.0 / (w * w + x * x + y * y + z * z)
    R = np.empty((q.shape[0], 3, 3))
    R[:, 0, 0] = 1 - s * (y * y + z * z)
    R[:, 0, 1] = s * (x * y - z * w)
    R[:, 0, 2] = s * (x * z + y * w)
    R[:, 1, 0] = s * (x * y + z * w)
    R[:, 1, 1] = 1 - s * (x * x + z * z)
    R[:, 1, 2] = s * (y * z - x * w)
    R[:, 2, 0] = s * (x * z - y * w)
    R[:, 2, 1] = s * (y * z + x * w)
    R[:, 2, 2] = 1 - s * (x * x + y * y)
    return R


def _mat_to_quat_batch(m: np.ndarray) -> np.ndarray:
    from .robot_spec import matrix_to_quaternion

    return np.stack([matrix_to_quaternion(mm) for mm in m]) if len(m) < 64 else _mat_to_quat_vec(m)


def _mat_to_quat_vec(m: np.ndarray) -> np.ndarray:
    """Batched Shepperd conversion with w >= 0 (same branch rule as matrix_to_quaternion)."""
    t = np.stack([1 + m[:, 0, 0] + m[:, 1, 1] + m[:, 2, 2], 1 + m[:, 0, 0] - m[:, 1, 1] - m[:, 2, 2],
                  1 - m[:, 0, 0] + m[:, 1, 1] - m[:, 2, 2], 1 - m[:, 0, 0] - m[:, 1, 1] + m[:, 2, 2]], axis=1)
    i = np.argmax(t, axis=1)
    s = np.sqrt(np.maximum(t[np.arange(len(m)), i], 0.0)) * 2.0
    q = np.empty((len(m), 4))
    c = [
        lambda M, s: (0.25 * s, (M[:, 2, 1] - M[:, 1, 2]) / s, (M[:, 0, 2] - M[:, 2, 0]) / s, (M[:, 1, 0] - M[:, 0, 1]) / s),
        lambda M, s: ((M[:, 2, 1] - M[:, 1, 2]) / s, 0.25 * s, (M[:, 0, 1] + M[:, 1, 0]) / s, (M[:, 0, 2] + M[:, 2, 0]) / s),
        lambda M, s: ((M[:, 0, 2] - M[:, 2, 0]) / s, (M[:, 0, 1] + M[:, 1, 0]) / s, 0.25 * s, (M[:, 1, 2] + M[:, 2, 1]) / s),
        lambda M, s: ((M[:, 1, 0] - M[:, 0, 1]) / s, (M[:, 0, 2] + M[:, 2, 0]) / s, (M[:, 1, 2] + M[:, 2, 1]) / s, 0.25 * s),
    ]
    for k in range(4):
        sel = i == k
        if np.any(sel):
            q[sel] = np.stack(c[k](m[sel], s[sel]), axis=1)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q[q[:, 0] < 0] *= -1
    return q


def fk_targets(spec: RobotSpec, q: np.ndarray, base: Optional[np.ndarray], links: List[int]) -> np.ndarray:
    """Target poses FK(q) in FP64 on the host: 4x4 products along each joint's root path."""
    B = q.shape[0]
    q = np.asarray(q, np.float64)
    ptf = spec.parent_joint_transforms
    T: List[Optional[np.ndarray]] = [None] * spec.num_joints
    for j in spec.topological_order_joint_indices:
        X0 = np.eye(4)
        X0[:3, :3] = _quat_to_mat_batch(ptf[j:j + 1, 3:])[0]
        X0[:3, 3] = ptf[j, :3]
        a = spec.actuated_joint_indices[j]
        m = spec.mimic_actuated_joint_indices[j]
        if a >= 0:
            pos = q[:, a]
        elif m >= 0:
            pos = q[:, m] * spec.mimic_multipliers[j] + spec.mimic_offsets[j]
        else:
            pos = np.zeros(B)
        M = np.tile(np.eye(4), (B, 1, 1))
        ax = spec.joint_axes[j]
        if spec.joint_types[j] == 2:
            K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
            M[:, :3, :3] = np.eye(3) + np.sin(pos)[:, None, None] * K + (1 - np.cos(pos))[:, None, None] * (K @ K)
        elif spec.joint_types[j] == 1:
            M[:, :3, 3] = ax[None, :] * pos[:, None]
        X = X0[None] @ M
        p = spec.parent_joint_indices[j]
        T[j] = X if p < 0 else T[p] @ X
    Bm = np.tile(np.eye(4), (B, 1, 1))
    if base is not None:
        Bm[:, :3, :3] = _quat_to_mat_batch(np.asarray(base[:, 3:], np.float64))
        Bm[:, :3, 3] = base[:, :3]
    out = np.zeros((B, len(links), 7))
    for k, li in enumerate(links):
        j = spec.link_parent_joint_indices[li]
        M = Bm @ T[j] if j >= 0 else Bm
        out[:, k, :3] = M[:, :3, 3]
        out[:, k, 3:] = _mat_to_quat_vec(M[:, :3, :3])
    return out.astype(np.float32)


def chain_workload(B: int, seed: int = 0, spheres: bool = False, unreachable_frac: float = 0.0) -> Workload:
    """C1 (spheres=False) / C2 (spheres=True, 10 % unreachable) start points and targets."""
    spec = serial_chain(seed)
    if spheres:
        add_chain_spheres(spec, seed)
    rng = np.random.default_rng(seed + 1)
    lim = spec.actuated_joint_limits
    q_star = rng.uniform(lim[:, 0], lim[:, 1], (B, spec.num_actuated_joints)).astype(np.float32)
    q0 = rng.uniform(lim[:, 0], lim[:, 1], (B, spec.num_actuated_joints)).astype(np.float32)
    ee = [spec.num_links - 1]
    targets = fk_targets(spec, q_star, None, ee)
    reachable = np.ones(B, bool)
    if unreachable_frac > 0:
        n = int(round(unreachable_frac * B))
        idx = rng.choice(B, n, replace=False)
        p = targets[idx, 0, :3].astype(np.float64)
        r = np.linalg.norm(p, axis=1, keepdims=True)
        targets[idx, 0, :3] = (p + 0.3 * p / np.maximum(r, 1e-9)).astype(np.float32)
        reachable[idx] = False
    return Workload("chain7" + ("_spheres" if spheres else ""), spec, ee, q0, None, targets, q_star, True, reachable)


def humanoid_workload(B: int, seed: int = 0) -> Workload:
    """C3: 5 pose targets from FK(q*, base*); start q* + N(0, 0.5) clipped, base at base*."""
    spec = humanoid(seed)
    rng = np.random.default_rng(seed + 1)
    lim = spec.actuated_joint_limits
    q_star = rng.uniform(lim[:, 0], lim[:, 1], (B, spec.num_actuated_joints)).astype(np.float32)
    base = _random_pose(rng, B, 0.5, 0.5)
    links = [spec.link_names.index(n) for n in spec.targets]  # type: ignore[attr-defined]
    targets = fk_targets(spec, q_star, base, links)
    q0 = np.clip(q_star + rng.normal(0, 0.5, q_star.shape), lim[:, 0], lim[:, 1]).astype(np.float32)
    return Workload("humanoid", spec, links, q0, base.copy(), targets, q_star, True)


def hand_workload(B: int, seed: int = 0) -> Workload:
    """C4: 21 keypoint positions FK(q*, base*) + N(0, 2 mm); start mid-range joints, base perturbed 1 cm / 0.05 rad."""
    spec = hand(seed)
    rng = np.random.default_rng(seed + 1)
    lim = spec.actuated_joint_limits
    q_star = rng.uniform(lim[:, 0], lim[:, 1], (B, spec.num_actuated_joints)).astype(np.float32)
    base = _random_pose(rng, B, 0.2, np.pi)
    links = [spec.link_names.index(n) for n in spec.targets]  # type: ignore[attr-defined]
    targets = fk_targets(spec, q_star, base, links)
    targets[:, :, :3] += rng.normal(0, 0.002, targets[:, :, :3].shape).astype(np.float32)
    q0 = np.tile(spec.midrange_q, (B, 1)).astype(np.float32)
    pert = _random_pose(rng, B, 0.01, 0.05)
    base0 = np.zeros_like(base)
    R = _quat_to_mat_batch(base[:, 3:].astype(np.float64)) @ _quat_to_mat_batch(pert[:, 3:].astype(np.float64))
    base0[:, :3] = base[:, :3] + pert[:, :3]
    base0[:, 3:] = _mat_to_quat_vec(R)
    return Workload("hand", spec, links, q0, base0.astype(np.float32), targets, q_star, False)
