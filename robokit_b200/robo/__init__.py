from .robot import Robot
from .robot_spec import JointType, RobotSpec, collision_pair_tables, compute_active_collision_pairs
from .robot_state import RobotState

__all__ = ["JointType", "Robot", "RobotSpec", "RobotState", "collision_pair_tables", "compute_active_collision_pairs"]
