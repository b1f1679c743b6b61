"""Host-side logic that needs no GPU: the C ABI's exports, URDF reading, tables, workloads."""

import ctypes
import os
import re

import numpy as np
import pytest

from robokit_b200.robo.robot_spec import (
    JointRecord,
    RobotSpec,
    collision_pair_tables,
    compute_link_bounding_spheres,
    matrix_to_quaternion,
    narrow_limits_to_float32,
    quaternion_to_matrix,
    read_urdf,
    rpy_to_matrix,
)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "b200ik.h")).read()
    return sorted(set(re.findall(r"\b(ik_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from robokit_b200 import _native as N
    from robokit_b200.build import build_library

    build_library()
    lib = ctypes.CDLL(N.LIB_PATH)
    syms = _declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(syms) == set(N._SIGNATURES), set(syms) ^ set(N._SIGNATURES)


def test_library_reports_errors_without_a_device():
    from robokit_b200 import _native as N

    lib = N.load_library()
    assert lib.ik_version() >= 10000
    # argument validation needs no device
    assert lib.ik_robot_create(None, ctypes.byref(ctypes.c_void_p())) == N.IK_E_INVALID
    assert b"NULL" in lib.ik_last_error()
    d = N.IkRobotDesc()
    d.num_joints = 100
    assert lib.ik_robot_create(ctypes.byref(d), ctypes.byref(ctypes.c_void_p())) == N.IK_E_UNSUPPORTED


URDF = """<robot name="toy">
  <link name="base"/><link name="a"/><link name="b"/><link name="c"/><link name="tip"/>
  <joint name="j1" type="revolute"><parent link="base"/><child link="a"/>
    <origin xyz="0 0 0.3" rpy="0.1 -0.2 0.3"/><axis xyz="0 0 1"/><limit lower="-2" upper="2" velocity="1"/></joint>
  <joint name="j2" type="prismatic"><parent link="a"/><child link="b"/>
    <origin xyz="0.1 0 0"/><axis xyz="1 0 0"/><limit lower="0" upper="0.2" velocity="1"/></joint>
  <joint name="j3" type="continuous"><parent link="a"/><child link="c"/><axis xyz="0 1 0"/>
    <mimic joint="j1" multiplier="-2" offset="0.5"/></joint>
  <joint name="fix" type="fixed"><parent link="b"/><child link="tip"/><origin xyz="0 0 0.05"/></joint>
</robot>"""


def test_urdf_reader_and_tables():
    spec = RobotSpec.parse(URDF)
    assert spec.joint_names == ["j1", "j2", "j3", "fix"]
    assert spec.actuated_joint_names == ["j1", "j2"]
    assert list(spec.joint_types) == [2, 1, 2, 0]
    assert list(spec.parent_joint_indices) == [-1, 0, 0, 1]
    assert list(spec.actuated_joint_indices) == [0, 1, -1, -1]
    assert list(spec.mimic_actuated_joint_indices) == [-1, -1, 0, -1]
    assert spec.mimic_multipliers[2] == -2 and spec.mimic_offsets[2] == 0.5
    assert list(spec.link_parent_joint_indices) == [-1, 0, 1, 2, 3]
    assert spec.base_link_name == "base" and set(spec.ee_link_names) == {"c", "tip"}
    np.testing.assert_allclose(spec.actuated_joint_limits, [[-2, 2], [0, 0.2]])
    m = spec.joints_to_actuated_mapping
    assert m[2, 0] == -2 and m[0, 0] == 1 and m[1, 1] == 1
    anc = spec.link_ancestor_joints_mask
    assert anc[4].tolist() == [True, True, False, True] and not anc[0].any()
    np.testing.assert_allclose(quaternion_to_matrix(spec.parent_joint_transforms[0, 3:]), rpy_to_matrix([0.1, -0.2, 0.3]),
                               atol=1e-12)
    order = list(spec.topological_order_joint_indices)
    assert order.index(0) < order.index(1) < order.index(3)
    # sub-tree filter (robot_spec.py:461-494)
    sub = RobotSpec.parse(URDF, ee_link_names=["tip"])
    assert sub.link_names == ["base", "a", "b", "tip"] and sub.joint_names == ["j1", "j2", "fix"]


def test_quaternion_conversions_roundtrip():
    rng = np.random.default_rng(0)
    for _ in range(50):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        q = q if q[0] >= 0 else -q
        np.testing.assert_allclose(matrix_to_quaternion(quaternion_to_matrix(q)), q, atol=1e-12)


def test_narrow_limits_inward():
    lim = np.array([[-0.1, 1.0471975511965976], [-np.pi, np.pi]])
    n = narrow_limits_to_float32(lim)
    assert np.all(n[:, 0] >= lim[:, 0]) and np.all(n[:, 1] <= lim[:, 1])


def test_link_bounding_spheres_cover_every_sphere():
    rng = np.random.default_rng(3)
    c = rng.uniform(-0.2, 0.2, (30, 3)).astype(np.float32)
    r = rng.uniform(0.01, 0.08, 30).astype(np.float32)
    li = rng.integers(0, 5, 30).astype(np.int32)
    bc, br = compute_link_bounding_spheres(c, r, li, 6)
    for k in range(30):
        assert np.linalg.norm(c[k] - bc[li[k]]) + r[k] <= br[li[k]] + 1e-5
    assert br[5] == 0


def test_collision_pair_tables_panda(panda_collision_spec):
    spec = panda_collision_spec
    pairs, lp, off, grouped = collision_pair_tables(spec)
    sl = spec.collision_spheres_link_indices
    ignored = {tuple(p) for p in spec.self_collision_ignored_pairs} | {tuple(p[::-1]) for p in
                                                                       spec.self_collision_ignored_pairs}
    for a, b in pairs:
        assert sl[a] != sl[b] and (sl[a], sl[b]) not in ignored
    assert off[0] == 0 and off[-1] == len(grouped) == len(pairs)
    for k, (la, lb) in enumerate(lp):
        for a, b in grouped[off[k]:off[k + 1]]:
            assert {sl[a], sl[b]} == {la, lb}
    keys = lp[:, 0] * spec.num_links + lp[:, 1]
    assert np.all(np.diff(keys) > 0)
    # filtering off keeps every pair (tests/terms/test_self_collision_task.py:57-64)
    allp, *_ = collision_pair_tables(spec, filter_adjacent_links=False)
    ns = len(sl)
    assert len(allp) == ns * (ns - 1) // 2 > len(pairs)


def test_synthetic_workloads_shapes_and_seeds():
    from robokit_b200 import configs

    a = configs.make("chain7c", 100, seed=5)
    b = configs.make("chain7c", 100, seed=5)
    np.testing.assert_array_equal(a.workload.targets, b.workload.targets)
    assert a.workload.spec.num_actuated_joints == 7 and len(a.workload.spec.collision_sphere_radii) == 24
    assert (~a.workload.reachable).sum() == 10
    _, lp, _, grouped = collision_pair_tables(a.workload.spec)
    assert len(lp) == 15 and 120 <= len(grouped) <= 240
    h = configs.make("humanoid", 8)
    assert h.workload.spec.num_actuated_joints == 29 and h.workload.base0.shape == (8, 7)
    assert len(h.workload.target_links) == 5
    k = configs.make("hand", 8)
    assert k.workload.spec.num_actuated_joints == 20 and len(k.workload.target_links) == 21
    # targets are FK(q*): the oracle's FP64 FK reproduces them
    import oracle

    rob = oracle.Robot.from_spec(h.workload.spec)
    T = oracle.fk(rob, h.workload.q_star, h.workload.base0)["T_link"][:, h.workload.target_links]
    np.testing.assert_allclose(T[..., :3], h.workload.targets[..., :3], atol=1e-5)


def test_config_lowering_descriptors():
    from robokit_b200 import configs

    cfg = configs.make("chain7c", 4, pair_mode="slots")
    descs = configs.oracle_terms(cfg)
    assert [d["kind"] for d in descs] == [1, 2, 4, 3]
    assert descs[2]["max_active_pairs"] == 50 and descs[2]["pair_mode"] == 0
    assert descs[0]["targets"].shape == (4, 1, 7)
    assert sum(t.residual_dim for t in cfg.terms) == 3 + 3 + 50 + 7
