from .dense import FrameTask, PositionLimit, PositionTask, RotationTask, SelfCollisionTask
from .task import Context, NativeProblem, ResidualTask, Task

__all__ = ["Context", "FrameTask", "NativeProblem", "PositionLimit", "PositionTask", "ResidualTask", "RotationTask",
           "SelfCollisionTask", "Task"]
