from .dense import (ConfigurationTask, FrameTask, PositionLimit, PositionTask, RotationTask, SceneCollisionTask,
                    SelfCollisionTask, SmoothnessTask, VelocityLimitTask)
from .task import Context, NativeProblem, ResidualTask, Task

__all__ = ["ConfigurationTask", "Context", "FrameTask", "NativeProblem", "PositionLimit", "PositionTask", "ResidualTask",
           "RotationTask", "SceneCollisionTask", "SelfCollisionTask", "SmoothnessTask", "Task", "VelocityLimitTask"]
