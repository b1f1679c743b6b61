"""The IK stack imports and loads its library without torch (tests/test_no_torch_runtime.py:1-26 checks the
same for the reference's numpy+Warp runtime): torch is plumbing for the solve_torch adapter only."""

import subprocess
import sys

_IMPORTS = """
import sys
sys.modules["torch"] = None
from robokit_b200 import _native
from robokit_b200.geom import BoxGeom, Scene
from robokit_b200.helpers.ik import IKContext, IKSolver, IKSolverConfig, presets
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
from robokit_b200.robo.robot import Robot
from robokit_b200.terms.dense import PositionTask, SceneCollisionTask
_native.load_library()
"""


def test_ik_runtime_imports_without_torch():
    subprocess.run([sys.executable, "-c", _IMPORTS], check=True, timeout=300)
