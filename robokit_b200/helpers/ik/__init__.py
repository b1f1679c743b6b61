"""Batched IK with a candidate population (robokit helpers/ik/)."""

from . import presets
from .config import IKContext, IKSolverConfig
from .ik import IKMetrics, IKResultTorch, IKSolver

__all__ = ["IKContext", "IKMetrics", "IKResultTorch", "IKSolver", "IKSolverConfig", "presets"]
