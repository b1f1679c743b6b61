import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "panda_golden.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libb200ik.so")


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def panda_spec(golden):
    from robokit_b200.robo.robot_spec import JointRecord, RobotSpec

    g = golden["robot"]
    return RobotSpec.from_records(g["name"], g["links"], [JointRecord(**j) for j in g["joints"]])


@pytest.fixture(scope="session")
def panda_collision_spec(golden):
    """Panda with the reference's collision spheres and ignore list (tests/conftest.py:104-110)."""
    from robokit_b200.robo.robot_spec import JointRecord, RobotSpec

    g = golden["robot"]
    spec = RobotSpec.from_records(g["name"], g["links"], [JointRecord(**j) for j in g["joints"]])
    centers, radii, links = [], [], []
    for link, spheres in golden["collision_spheres"].items():
        if link not in spec.link_names:
            continue
        for s in spheres:
            centers.append(s["center"])
            radii.append(s["radius"])
            links.append(spec.link_names.index(link))
    spec.set_collision_spheres(np.array(centers), np.array(radii), np.array(links))
    idx = {n: i for i, n in enumerate(spec.link_names)}
    pairs = sorted({(idx[a], idx[b]) for a, bs in golden["self_collision_ignore"].items() for b in bs
                    if a in idx and b in idx})
    spec.self_collision_ignored_pairs = np.array(pairs, np.int32).reshape(-1, 2)
    return spec


@pytest.fixture(scope="session")
def gpu():
    """The native library on a CUDA device; a GPU test without one fails instead of skipping."""
    from robokit_b200 import _native as N
    from robokit_b200.build import build_library

    build_library()
    N.load_library()
    n = N.device_count()
    assert n > 0, "GPU test selected but no CUDA device is visible"
    return N


@pytest.fixture(scope="session")
def panda_arm_spec(golden):
    """The 7-DoF Panda of the reference's IK benchmark: finger joints fixed (scripts/benchmark/ik/helper.py:44-57)."""
    from robokit_b200.robo.robot_spec import JointRecord, RobotSpec

    g = golden["robot"]
    joints = []
    for j in g["joints"]:
        rec = dict(j)
        if rec["type"] == "prismatic":
            rec.update(type="fixed", mimic_joint=None)
        joints.append(JointRecord(**rec))
    return RobotSpec.from_records(g["name"], g["links"], joints)
