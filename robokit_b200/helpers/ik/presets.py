"""Preset IK configurations (helpers/ik/presets.py:13-37) over the terms of this library."""

from ...opt.lm_optimizer import LMOptimizerConfig
from ...opt.population_solver import PopulationSolverConfig, Stage
from ...opt.sampler import RobertsSamplerConfig
from ...terms.dense import PositionLimit, PositionTask, RotationTask, SmoothnessTask
from .config import IKContext, IKSolverConfig

basic = (
    IKSolverConfig(sampler=RobertsSamplerConfig(keep_first=True, scale=1.0))
    .add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
    .add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
    .add(PositionLimit(weight=50.0))
)

smooth = (
    IKSolverConfig(sampler=RobertsSamplerConfig(keep_first=True, scale=1.0))
    .add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
    .add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
    .add(PositionLimit(weight=50.0))
    .add(SmoothnessTask(prev_var=IKContext.PREVIOUS_STATE, weight=0.1))
)

single_candidate = (
    IKSolverConfig(
        solver=PopulationSolverConfig(stages=[Stage(30, 1, LMOptimizerConfig(lm_lambda=1.0))], cuda_graph_mode="full"),
    )
    .add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
    .add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
    .add(PositionLimit(weight=50.0))
    .add(SmoothnessTask(prev_var=IKContext.PREVIOUS_STATE, weight=0.1))
)

__all__ = ["basic", "single_candidate", "smooth"]
