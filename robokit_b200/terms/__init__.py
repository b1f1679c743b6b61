from .dense import PositionLimit, PositionTask, RotationTask, SelfCollisionTask
from .task import Context, NativeProblem, ResidualTask, Task

__all__ = ["Context", "NativeProblem", "PositionLimit", "PositionTask", "ResidualTask", "RotationTask",
           "SelfCollisionTask", "Task"]
