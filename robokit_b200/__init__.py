"""B200-native batched Levenberg-Marquardt inverse kinematics.

A drop-in for robokit's LM-IK path (LMOptimizer over PositionTask,
RotationTask, PositionLimit and SelfCollisionTask on a Robot): the solver runs
as hand-written sm_100a CUDA in libb200ik.so, reached through a ctypes C ABI.
The package imports no torch and has no CPU fallback.
"""

from . import _native
from .opt import LMOptimizer, LMOptimizerConfig, OptimizerConfig, VarKey, VarValues
from .robo import Robot, RobotSpec, RobotState
from .terms import PositionLimit, PositionTask, RotationTask, SelfCollisionTask

__all__ = [
    "LMOptimizer",
    "LMOptimizerConfig",
    "OptimizerConfig",
    "PositionLimit",
    "PositionTask",
    "Robot",
    "RobotSpec",
    "RobotState",
    "RotationTask",
    "SelfCollisionTask",
    "VarKey",
    "VarValues",
]
