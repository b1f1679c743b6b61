from .dense import (ConfigurationTask, FrameTask, PositionLimit, PositionTask, RotationTask, SelfCollisionTask,
                    SmoothnessTask, VelocityLimitTask)
from .task import Context, NativeProblem, ResidualTask, Task

__all__ = ["ConfigurationTask", "Context", "FrameTask", "NativeProblem", "PositionLimit", "PositionTask", "ResidualTask",
           "RotationTask", "SelfCollisionTask", "SmoothnessTask", "Task", "VelocityLimitTask"]
