"""Regenerate tests/golden/panda_golden.json from the reference checkout.

Run from the repo root with the reference mounted (its path is the only
argument, default /root/reference):

    python tests/golden/make_golden.py /root/reference

It reads the reference's own test data — the panda URDF and collision-sphere
fixtures and the panda entries of the FK / Jacobian golden files — and writes
one small JSON: the parsed joint records (not the URDF text), the sphere and
ignore tables, and the golden poses and Jacobians.  The tests never read the
reference tree; they read this file.
"""

from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from robokit_b200.robo.robot_spec import read_urdf  # noqa: E402


def main(ref: str) -> None:
    import yaml

    fx = os.path.join(ref, "tests", "fixtures")
    name, links, joints = read_urdf(os.path.join(fx, "panda.urdf"))
    with open(os.path.join(fx, "franka_collision_spheres.yaml")) as f:
        spheres = yaml.safe_load(f)["collision_spheres"]
    with open(os.path.join(fx, "franka_self_collision_ignore.yml")) as f:
        ignore = yaml.safe_load(f)["self_collision_ignore"]
    with open(os.path.join(ref, "tests", "robo", "fk_ground_truth.json")) as f:
        fk = json.load(f)
    with open(os.path.join(ref, "tests", "robo", "jacobian_ground_truth.json")) as f:
        jac = json.load(f)
    fk_panda = next(r for r in fk["robots"] if r["robot_description_name"] == "panda_description")
    jac_panda = next(r for r in jac["robots"] if r["robot_description_name"] == "panda_description")
    out = {
        "source": "robokit tests/fixtures/panda.urdf, franka_collision_spheres.yaml, "
        "franka_self_collision_ignore.yml; tests/robo/fk_ground_truth.json and "
        "jacobian_ground_truth.json (panda_description entries)",
        "robot": {"name": name, "links": links, "joints": [j.to_dict() for j in joints]},
        "collision_spheres": {k: [{"center": s["center"], "radius": s["radius"]} for s in v] for k, v in spheres.items()},
        "self_collision_ignore": ignore,
        "fk": fk_panda,
        "jacobians": jac_panda,
    }
    dst = os.path.join(HERE, "panda_golden.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {dst} ({os.path.getsize(dst)} bytes)")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
