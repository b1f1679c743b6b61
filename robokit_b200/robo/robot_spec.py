"""Robot specification: the kinematic tables the IK kernels run on.

Mirrors robokit's ``RobotSpec`` (robo/robot_spec.py:44-139) field for field for
the tables on the IK path, with a standard-library URDF reader in place of
yourdfpy and the derived tables of robo/robot_spec.py:1043-1142 and
:1258-1303.  Geometry meshes, capsules and MJCF are not part of this package.
"""

from __future__ import annotations

import enum
import math
import os
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from functools import cached_property
from typing import Dict, List, Optional, Sequence, Set, Tuple, Union

import numpy as np


class JointType(enum.IntEnum):
    """robo/robot_spec.py:34-41"""

    FIXED = 0
    PRISMATIC = 1
    REVOLUTE = 2


# ---------------------------------------------------------------------------
# rotations (URDF rpy convention: R = Rz(yaw) Ry(pitch) Rx(roll))
# ---------------------------------------------------------------------------
def rpy_to_matrix(rpy: Sequence[float]) -> np.ndarray:
    r, p, y = (float(v) for v in rpy)
    cr, sr, cp, sp, cy, sy = math.cos(r), math.sin(r), math.cos(p), math.sin(p), math.cos(y), math.sin(y)
    return np.array(
        [
            [cy * cp, cy * sp * sr - sy * cr, cy * sp * cr + sy * sr],
            [sy * cp, sy * sp * sr + cy * cr, sy * sp * cr - cy * sr],
            [-sp, cp * sr, cp * cr],
        ],
        dtype=np.float64,
    )


def matrix_to_quaternion(m: np.ndarray) -> np.ndarray:
    """Rotation matrix -> unit quaternion [w, x, y, z] with w >= 0.

    Shepperd's method: pick the largest of 4w^2, 4x^2, 4y^2, 4z^2 and derive
    the other components from that row (the choice robokit's
    xform/numpy/rotation_conversions.py:5-53 makes, standardised likewise).
    """
    m = np.asarray(m, dtype=np.float64)
    t = np.array(
        [
            1.0 + m[0, 0] + m[1, 1] + m[2, 2],
            1.0 + m[0, 0] - m[1, 1] - m[2, 2],
            1.0 - m[0, 0] + m[1, 1] - m[2, 2],
            1.0 - m[0, 0] - m[1, 1] + m[2, 2],
        ]
    )
    i = int(np.argmax(t))
    s = math.sqrt(max(t[i], 0.0)) * 2.0
    if i == 0:
        q = [0.25 * s, (m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s]
    elif i == 1:
        q = [(m[2, 1] - m[1, 2]) / s, 0.25 * s, (m[0, 1] + m[1, 0]) / s, (m[0, 2] + m[2, 0]) / s]
    elif i == 2:
        q = [(m[0, 2] - m[2, 0]) / s, (m[0, 1] + m[1, 0]) / s, 0.25 * s, (m[1, 2] + m[2, 1]) / s]
    else:
        q = [(m[1, 0] - m[0, 1]) / s, (m[0, 2] + m[2, 0]) / s, (m[1, 2] + m[2, 1]) / s, 0.25 * s]
    q = np.asarray(q)
    q /= np.linalg.norm(q)
    return -q if q[0] < 0 else q


def quaternion_to_matrix(q: Sequence[float]) -> np.ndarray:
    w, x, y, z = (float(v) for v in q)
    n = w * w + x * x + y * y + z * z
    s = 2.0 / n
    return np.array(
        [
            [1 - s * (y * y + z * z), s * (x * y - z * w), s * (x * z + y * w)],
            [s * (x * y + z * w), 1 - s * (x * x + z * z), s * (y * z - x * w)],
            [s * (x * z - y * w), s * (y * z + x * w), 1 - s * (x * x + y * y)],
        ]
    )


def narrow_limits_to_float32(limits: np.ndarray) -> np.ndarray:
    """Cast [lo, hi] inward to float32 (robo/robot_spec_tensors.py:17-31)."""
    limits = np.asarray(limits, dtype=np.float64).reshape(-1, 2)
    out = limits.astype(np.float32)
    if out.size == 0:
        return out
    lo, hi = out[:, 0], out[:, 1]
    np.copyto(lo, np.nextafter(lo, np.float32(np.inf)), where=lo < limits[:, 0])
    np.copyto(hi, np.nextafter(hi, np.float32(-np.inf)), where=hi > limits[:, 1])
    return out


def compute_link_bounding_spheres(
    centers: np.ndarray, radii: np.ndarray, link_indices: np.ndarray, num_links: int
) -> Tuple[np.ndarray, np.ndarray]:
    """Per-link bounding sphere of the link's collision spheres.

    Ritter's two-pass construction (farthest-point pair, then grow to cover
    every sphere), the algorithm of robo/robot_spec.py:1258-1303; links without
    spheres get a zero sphere.
    """
    bc = np.zeros((num_links, 3), dtype=np.float32)
    br = np.zeros(num_links, dtype=np.float32)
    for link in range(num_links):
        sel = link_indices == link
        if not np.any(sel):
            continue
        c = centers[sel].astype(np.float64)
        r = radii[sel].astype(np.float64)
        if len(r) == 1:
            bc[link], br[link] = c[0], r[0]
            continue
        i1 = int(np.argmax(np.linalg.norm(c - c[0], axis=1) + r))
        i2 = int(np.argmax(np.linalg.norm(c - c[i1], axis=1) + r))
        c1, r1, c2, r2 = c[i1], float(r[i1]), c[i2], float(r[i2])
        d = c2 - c1
        d12 = float(np.linalg.norm(d))
        if r1 >= d12 + r2:
            C, R = c1.copy(), r1
        elif r2 >= d12 + r1:
            C, R = c2.copy(), r2
        else:
            R = 0.5 * (d12 + r1 + r2)
            C = c1 + d * ((R - r1) / d12)
        for k in range(len(r)):
            v = c[k] - C
            dist = float(np.linalg.norm(v))
            over = dist + float(r[k]) - R
            if over > 1e-12:
                nR = R + 0.5 * over
                if dist > 1e-12:
                    C = C + v * ((nR - R) / dist)
                R = nR
        bc[link], br[link] = C, R
    return bc, br


# ---------------------------------------------------------------------------
# URDF reading (standard library)
# ---------------------------------------------------------------------------
@dataclass
class JointRecord:
    """One URDF <joint> after parsing."""

    name: str
    type: str
    parent: str
    child: str
    xyz: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rpy: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    axis: Tuple[float, float, float] = (1.0, 0.0, 0.0)
    lower: Optional[float] = None
    upper: Optional[float] = None
    velocity: Optional[float] = None
    mimic_joint: Optional[str] = None
    mimic_multiplier: float = 1.0
    mimic_offset: float = 0.0

    def to_dict(self) -> dict:
        return dict(self.__dict__)


def _floats(text: Optional[str], default: Tuple[float, ...]) -> Tuple[float, ...]:
    if text is None:
        return default
    return tuple(float(v) for v in text.split())


def read_urdf(source: Union[str, os.PathLike]) -> Tuple[str, List[str], List[JointRecord]]:
    """(robot name, link names in file order, joint records in file order)."""
    text = str(source)
    if "<robot" not in text:
        with open(source, "r") as f:
            text = f.read()
    root = ET.fromstring(text)
    if root.tag != "robot":
        raise ValueError("not a URDF: the root element is not <robot>")
    links = [el.get("name") for el in root.findall("link")]
    joints: List[JointRecord] = []
    for el in root.findall("joint"):
        origin = el.find("origin")
        axis = el.find("axis")
        limit = el.find("limit")
        mimic = el.find("mimic")
        rec = JointRecord(
            name=el.get("name"),
            type=el.get("type"),
            parent=el.find("parent").get("link"),
            child=el.find("child").get("link"),
            xyz=_floats(origin.get("xyz") if origin is not None else None, (0.0, 0.0, 0.0)),
            rpy=_floats(origin.get("rpy") if origin is not None else None, (0.0, 0.0, 0.0)),
            axis=_floats(axis.get("xyz") if axis is not None else None, (1.0, 0.0, 0.0)),
        )
        if limit is not None:
            rec.lower = float(limit.get("lower")) if limit.get("lower") is not None else None
            rec.upper = float(limit.get("upper")) if limit.get("upper") is not None else None
            rec.velocity = float(limit.get("velocity")) if limit.get("velocity") is not None else None
        if mimic is not None:
            rec.mimic_joint = mimic.get("joint")
            rec.mimic_multiplier = float(mimic.get("multiplier", 1.0))
            rec.mimic_offset = float(mimic.get("offset", 0.0))
        joints.append(rec)
    return root.get("name", ""), links, joints


def _joint_type(t: str) -> JointType:
    # robo/robot_spec.py:296-307
    if t in ("revolute", "continuous"):
        return JointType.REVOLUTE
    if t == "prismatic":
        return JointType.PRISMATIC
    return JointType.FIXED


def _joint_limits(rec: JointRecord) -> Tuple[float, float]:
    # robo/robot_spec.py:352-371
    if rec.lower is not None and rec.upper is not None:
        return rec.lower, rec.upper
    if rec.type in ("continuous", "revolute"):
        return -math.pi, math.pi
    if rec.type == "prismatic":
        return -1.0, 1.0
    return 0.0, 0.0


def _joint_velocity_limit(rec: JointRecord) -> float:
    # robo/robot_spec.py:373-384: fixed joints 0, unspecified 10
    if rec.velocity is not None:
        return rec.velocity
    return 0.0 if rec.type == "fixed" else 10.0


@dataclass
class RobotSpec:
    """Kinematic tables of one robot (robo/robot_spec.py:44-139)."""

    name: str
    joint_names: List[str]
    actuated_joint_names: List[str]
    joint_types: np.ndarray
    joint_axes: np.ndarray
    actuated_joint_indices: np.ndarray
    parent_joint_indices: np.ndarray
    parent_joint_transforms: np.ndarray
    mimic_actuated_joint_indices: np.ndarray
    mimic_multipliers: np.ndarray
    mimic_offsets: np.ndarray
    joint_limits: np.ndarray
    actuated_joint_limits: np.ndarray
    link_names: List[str]
    link_parent_joint_indices: np.ndarray
    base_link_name: str
    ee_link_names: List[str]
    local_collision_sphere_centers: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    collision_sphere_radii: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    collision_spheres_link_indices: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    self_collision_ignored_pairs: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    robot_description: str = ""
    joint_velocity_limits: Optional[np.ndarray] = None
    actuated_joint_velocity_limits: Optional[np.ndarray] = None

    def __post_init__(self):
        # tables built without velocities (synthetic robots) get the reader's default of 10 per moving joint
        if self.joint_velocity_limits is None:
            self.joint_velocity_limits = np.where(np.asarray(self.joint_types) == 0, 0.0, 10.0)
        if self.actuated_joint_velocity_limits is None:
            self.actuated_joint_velocity_limits = np.full(len(self.actuated_joint_names), 10.0)

    # --- construction ---------------------------------------------------------
    @staticmethod
    def from_records(
        name: str,
        link_names: Sequence[str],
        joints: Sequence[JointRecord],
        base_link_name: Optional[str] = None,
        ee_link_names: Optional[Union[str, Sequence[str]]] = None,
        description: str = "",
    ) -> "RobotSpec":
        """Tables from parsed URDF joints, following robo/robot_spec.py:457-617."""
        link_names = list(link_names)
        joints = list(joints)
        if isinstance(ee_link_names, str):
            ee_link_names = [ee_link_names]
        if base_link_name is not None or ee_link_names is not None:
            # keep the subtree below base_link_name and the ancestors of ee_link_names (:461-494)
            child_to_parent = {j.child: j.parent for j in joints}
            children: Dict[str, List[str]] = {}
            for j in joints:
                children.setdefault(j.parent, []).append(j.child)
            keep = set(link_names)
            if base_link_name is not None:
                desc, stack = set(), [base_link_name]
                while stack:
                    lk = stack.pop()
                    desc.add(lk)
                    stack.extend(children.get(lk, []))
                keep &= desc
            if ee_link_names is not None:
                anc = {base_link_name} if base_link_name else set()
                for ee in ee_link_names:
                    cur: Optional[str] = ee
                    while cur is not None and cur != base_link_name:
                        anc.add(cur)
                        cur = child_to_parent.get(cur)
                keep &= anc
            link_names = [lk for lk in link_names if lk in keep]
            joints = [j for j in joints if j.parent in keep and j.child in keep]
        joint_names = [j.name for j in joints]
        actuated = [j.name for j in joints if j.type != "fixed" and j.mimic_joint is None]
        jmap = {j.name: j for j in joints}
        child_to_joint = {j.child: j for j in joints}
        jidx = {n: i for i, n in enumerate(joint_names)}
        nj = len(joints)
        types = np.zeros(nj, np.int32)
        axes = np.zeros((nj, 3), np.float64)
        act = np.full(nj, -1, np.int32)
        parent = np.full(nj, -1, np.int32)
        ptf = np.zeros((nj, 7), np.float64)
        mimic = np.full(nj, -1, np.int32)
        mmul = np.ones(nj, np.float64)
        moff = np.zeros(nj, np.float64)
        limits = np.zeros((nj, 2), np.float64)
        for i, j in enumerate(joints):
            types[i] = _joint_type(j.type)
            axes[i] = j.axis if types[i] != JointType.FIXED else (0.0, 0.0, 0.0)
            if j.mimic_joint is None and j.name in actuated:
                act[i] = actuated.index(j.name)
            if j.mimic_joint is not None:
                mimic[i] = actuated.index(jmap[j.mimic_joint].name)
                mmul[i], moff[i] = j.mimic_multiplier, j.mimic_offset
            limits[i] = _joint_limits(j)
            if j.parent in child_to_joint:
                parent[i] = jidx[child_to_joint[j.parent].name]
            ptf[i, :3] = j.xyz
            ptf[i, 3:] = matrix_to_quaternion(rpy_to_matrix(j.rpy))
        act_limits = np.array([_joint_limits(jmap[n]) for n in actuated], np.float64).reshape(-1, 2)
        lpj = np.array(
            [jidx[child_to_joint[lk].name] if lk in child_to_joint else -1 for lk in link_names], np.int32
        )
        if base_link_name is None:
            child_links = {j.child for j in joints}
            base_link_name = next(n for n in link_names if n not in child_links)
        if ee_link_names is None:
            parent_links = {j.parent for j in joints}
            ee_link_names = [n for n in link_names if n not in parent_links]
        return RobotSpec(
            name=name,
            joint_names=joint_names,
            actuated_joint_names=actuated,
            joint_types=types,
            joint_axes=axes,
            actuated_joint_indices=act,
            parent_joint_indices=parent,
            parent_joint_transforms=ptf,
            mimic_actuated_joint_indices=mimic,
            mimic_multipliers=mmul,
            mimic_offsets=moff,
            joint_limits=limits,
            actuated_joint_limits=act_limits,
            link_names=link_names,
            link_parent_joint_indices=lpj,
            base_link_name=base_link_name,
            ee_link_names=list(ee_link_names),
            robot_description=description,
            joint_velocity_limits=np.array([_joint_velocity_limit(j) for j in joints], np.float64),
            actuated_joint_velocity_limits=np.array([_joint_velocity_limit(jmap[n]) for n in actuated], np.float64),
        )

    @staticmethod
    def parse(
        robot_description_or_path: Union[str, os.PathLike],
        load_collision_spheres: bool = False,
        collision_spheres_path: Optional[Union[str, os.PathLike]] = None,
        self_collision_ignore_path: Optional[Union[str, os.PathLike]] = None,
        base_link_name: Optional[str] = None,
        ee_link_names: Optional[Union[str, Sequence[str]]] = None,
    ) -> "RobotSpec":
        """URDF text or path -> RobotSpec (robo/robot_spec.py:140-208)."""
        text = str(robot_description_or_path)
        if "<robot" not in text and not os.path.exists(text):
            raise FileNotFoundError(f"Robot description file not found: {robot_description_or_path}")
        name, links, joints = read_urdf(robot_description_or_path)
        spec = RobotSpec.from_records(name, links, joints, base_link_name, ee_link_names)
        if load_collision_spheres:
            if collision_spheres_path is None:
                raise ValueError("Collision spheres path must be provided when loading collision spheres.")
            spec.load_collision_spheres(collision_spheres_path)
        if self_collision_ignore_path is not None:
            spec.load_self_collision_ignore(self_collision_ignore_path)
        return spec

    def load_collision_spheres(self, path: Union[str, os.PathLike]) -> None:
        """Per-link spheres from YAML ``collision_spheres: {link: [{center, radius}]}`` (:227-258)."""
        import yaml

        with open(path, "r") as f:
            data = yaml.safe_load(f) or {}
        centers, radii, links = [], [], []
        for link, spheres in (data.get("collision_spheres") or {}).items():
            if link not in self.link_names:
                continue
            li = self.link_names.index(link)
            for s in spheres:
                c = s["center"]
                centers.append([c[0], c[1], c[2]])
                radii.append(s["radius"])
                links.append(li)
        self.set_collision_spheres(np.array(centers).reshape(-1, 3), np.array(radii), np.array(links))

    def set_collision_spheres(self, centers: np.ndarray, radii: np.ndarray, link_indices: np.ndarray) -> None:
        self.local_collision_sphere_centers = np.asarray(centers, np.float32).reshape(-1, 3)
        self.collision_sphere_radii = np.asarray(radii, np.float32).reshape(-1)
        self.collision_spheres_link_indices = np.asarray(link_indices, np.int32).reshape(-1)
        self.__dict__.pop("_link_bounding_spheres", None)

    def load_self_collision_ignore(self, path: Union[str, os.PathLike]) -> None:
        """Link pairs to skip, YAML ``self_collision_ignore: {a: [b, ...]}`` (:210-225)."""
        import yaml

        with open(path, "r") as f:
            entries = (yaml.safe_load(f) or {}).get("self_collision_ignore") or {}
        idx = {n: i for i, n in enumerate(self.link_names)}
        pairs: Set[Tuple[int, int]] = set()
        for a, bs in entries.items():
            for b in bs:
                if a in idx and b in idx:
                    pairs.add((idx[a], idx[b]))
        self.self_collision_ignored_pairs = (
            np.array(sorted(pairs), np.int32) if pairs else np.zeros((0, 2), np.int32)
        )

    # --- sizes -----------------------------------------------------------------
    @property
    def num_joints(self) -> int:
        return len(self.joint_names)

    @property
    def num_links(self) -> int:
        return len(self.link_names)

    @property
    def num_actuated_joints(self) -> int:
        return len(self.actuated_joint_names)

    @property
    def has_collision_spheres(self) -> bool:
        return len(self.collision_sphere_radii) > 0

    @property
    def zero_q(self) -> np.ndarray:
        return np.zeros(self.num_actuated_joints, np.float32)

    @property
    def midrange_q(self) -> np.ndarray:
        lim = self.actuated_joint_limits
        return (0.5 * (lim[:, 0] + lim[:, 1])).astype(np.float32)

    # --- derived tables ----------------------------------------------------------
    @property
    def joint_twists(self) -> np.ndarray:
        """[linear; angular] twist per joint: revolute [0; axis], prismatic [axis; 0] (:320-331)."""
        tw = np.zeros((self.num_joints, 6), np.float64)
        rev = self.joint_types == JointType.REVOLUTE
        pri = self.joint_types == JointType.PRISMATIC
        tw[rev, 3:] = self.joint_axes[rev]
        tw[pri, :3] = self.joint_axes[pri]
        return tw

    @property
    def joints_to_actuated_mapping(self) -> np.ndarray:
        """(robo/robot_spec.py:1119-1131)"""
        m = np.zeros((self.num_joints, self.num_actuated_joints), np.float32)
        for j in range(self.num_joints):
            a, mi = self.actuated_joint_indices[j], self.mimic_actuated_joint_indices[j]
            if a >= 0:
                m[j, a] = 1.0
            elif mi >= 0:
                m[j, mi] = self.mimic_multipliers[j]
        return m

    @property
    def link_ancestor_joints_mask(self) -> np.ndarray:
        """(robo/robot_spec.py:1133-1142)"""
        mask = np.zeros((self.num_links, self.num_joints), bool)
        for lk in range(self.num_links):
            j = int(self.link_parent_joint_indices[lk])
            while j != -1:
                mask[lk, j] = True
                j = int(self.parent_joint_indices[j])
        return mask

    @property
    def topological_order_joint_indices(self) -> np.ndarray:
        """Parents before children (robo/robot_spec.py:1043-1068)."""
        deps: List[List[int]] = [[] for _ in range(self.num_joints)]
        indeg = [0] * self.num_joints
        for j, p in enumerate(self.parent_joint_indices):
            if p >= 0:
                deps[p].append(j)
                indeg[j] += 1
        order, queue = [], [j for j in range(self.num_joints) if indeg[j] == 0]
        while queue:
            j = queue.pop(0)
            order.append(j)
            for d in deps[j]:
                indeg[d] -= 1
                if indeg[d] == 0:
                    queue.append(d)
        if len(order) != self.num_joints:
            raise ValueError("Circular dependency detected in joint relationships")
        return np.asarray(order, np.int32)

    @cached_property
    def _link_bounding_spheres(self) -> Tuple[np.ndarray, np.ndarray]:
        return compute_link_bounding_spheres(
            self.local_collision_sphere_centers,
            self.collision_sphere_radii,
            self.collision_spheres_link_indices,
            self.num_links,
        )

    @property
    def local_link_bounding_sphere_centers(self) -> np.ndarray:
        return self._link_bounding_spheres[0]

    @property
    def link_bounding_sphere_radii(self) -> np.ndarray:
        return self._link_bounding_spheres[1]

    def float32_actuated_limits(self) -> np.ndarray:
        return narrow_limits_to_float32(self.actuated_joint_limits)

    def native_tables(self) -> dict:
        """float32 / int32 arrays in the layout of IkRobotDesc (include/b200ik.h)."""
        ptf = self.parent_joint_transforms.astype(np.float32)
        return dict(
            joint_types=np.ascontiguousarray(self.joint_types, np.int32),
            joint_axes=np.ascontiguousarray(self.joint_axes, np.float32).reshape(-1, 3),
            parent_transforms=np.ascontiguousarray(ptf).reshape(-1, 7),
            parent_joints=np.ascontiguousarray(self.parent_joint_indices, np.int32),
            actuated_indices=np.ascontiguousarray(self.actuated_joint_indices, np.int32),
            mimic_indices=np.ascontiguousarray(self.mimic_actuated_joint_indices, np.int32),
            mimic_multipliers=np.ascontiguousarray(self.mimic_multipliers, np.float32),
            mimic_offsets=np.ascontiguousarray(self.mimic_offsets, np.float32),
            link_parent_joints=np.ascontiguousarray(self.link_parent_joint_indices, np.int32),
            actuated_limits=np.ascontiguousarray(self.float32_actuated_limits()).reshape(-1, 2),
            sphere_centers=np.ascontiguousarray(self.local_collision_sphere_centers, np.float32).reshape(-1, 3),
            sphere_radii=np.ascontiguousarray(self.collision_sphere_radii, np.float32),
            sphere_links=np.ascontiguousarray(self.collision_spheres_link_indices, np.int32),
            link_bound_centers=np.ascontiguousarray(self.local_link_bounding_sphere_centers, np.float32).reshape(-1, 3),
            link_bound_radii=np.ascontiguousarray(self.link_bounding_sphere_radii, np.float32),
        )


# ---------------------------------------------------------------------------
# collision pair tables (terms/dense/self_collision_task.py:29-68, 699-737)
# ---------------------------------------------------------------------------
def compute_active_collision_pairs(
    spec: RobotSpec, ignored_link_pairs: Optional[Set[Tuple[int, int]]] = None
) -> np.ndarray:
    """Sphere pairs on links that are neither welded together nor one joint apart.

    Links are grouped into bodies by their nearest non-fixed ancestor joint;
    pairs on the same body or on bodies connected by one moving joint are
    skipped (self_collision_task.py:29-68).
    """
    sphere_link = spec.collision_spheres_link_indices
    nl = spec.num_links
    if ignored_link_pairs is not None:
        skip = np.eye(nl, dtype=bool)
        for a, b in ignored_link_pairs:
            skip[a, b] = skip[b, a] = True
    else:
        jt, pj = spec.joint_types, spec.parent_joint_indices

        def moving_ancestor(j: int) -> int:
            while j >= 0 and jt[j] == JointType.FIXED:
                j = int(pj[j])
            return j

        body = np.array([moving_ancestor(int(j)) for j in spec.link_parent_joint_indices], np.int32)
        skip = body[:, None] == body[None, :]
        for j in range(len(jt)):
            if jt[j] != JointType.FIXED:
                child = body == j
                par = body == moving_ancestor(int(pj[j]))
                skip |= np.outer(child, par) | np.outer(par, child)
    i, j = np.triu_indices(len(sphere_link), k=1)
    keep = ~skip[sphere_link[i], sphere_link[j]]
    return np.stack([i[keep], j[keep]], axis=1).astype(np.int32)


def collision_pair_tables(
    spec: RobotSpec, filter_adjacent_links: bool = True
) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(sphere pairs [P,2], link pairs [L,2], CSR offsets [L+1], sphere pairs grouped by link pair [P,2]).

    Candidate pairs after the adjacency filter and the spec's ignore list
    (self_collision_task.py:699-715), grouped by (min link, max link) in
    ascending key order (:717-737).
    """
    sl = spec.collision_spheres_link_indices
    if filter_adjacent_links:
        pairs = compute_active_collision_pairs(spec)
        ignored = {(int(a), int(b)) for a, b in spec.self_collision_ignored_pairs}
    else:
        i, j = np.triu_indices(len(sl), k=1)
        pairs = np.stack([i, j], axis=1).astype(np.int32)
        ignored = set()
    if ignored and len(pairs):
        both = ignored | {(b, a) for a, b in ignored}
        keep = [(int(sl[a]) != int(sl[b])) and ((int(sl[a]), int(sl[b])) not in both) for a, b in pairs]
        pairs = pairs[np.asarray(keep, bool)]
    nl = spec.num_links
    if len(pairs) == 0:
        z = np.zeros((0, 2), np.int32)
        return z, z, np.zeros(1, np.int32), z
    li = sl[pairs[:, 0]].astype(np.int64)
    lj = sl[pairs[:, 1]].astype(np.int64)
    key = np.minimum(li, lj) * nl + np.maximum(li, lj)
    uniq, inverse = np.unique(key, return_inverse=True)
    link_pairs = np.stack([uniq // nl, uniq % nl], axis=1).astype(np.int32)
    order = np.argsort(inverse, kind="stable")
    grouped = pairs[order].astype(np.int32)
    counts = np.bincount(inverse, minlength=len(uniq))
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return pairs.astype(np.int32), link_pairs, offsets, grouped
