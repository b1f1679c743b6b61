"""The benchmark configurations as (workload, robot, terms, LM settings).

chain7   — 7-DoF serial chain, pose target (position + SO(3) log, unit
           weights), 1024 problems, 50 iterations, lambda0 1e-3, x10 / x0.1.
chain7c  — the chain with 24 collision spheres, sphere self-collision (margin
           0.02 m; every non-adjacent sphere pair by default, the reference's
           slot mode on request) and the joint-limit hinge; 16384 problems, 10 %
           of targets pushed 0.3 m radially outward; 100 iterations, a problem
           stops once its LM step is below 1e-6.
humanoid — floating base + 29 revolute joints, 5 pose targets (35x35 normal
           matrix), 8192 problems, start q* + N(0, 0.5) clipped with the base at
           its target value; the iteration count is not part of the
           configuration, so the 100-iteration cap with the 1e-6 step stop is used.
hand     — floating wrist + 20 finger joints, 21 keypoint positions with 2 mm
           noise, 65536 problems, 30 iterations.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List, Literal, Optional

import numpy as np

from .opt.lm_optimizer import LMOptimizerConfig
from .robo.robot import Robot
from .robo.synthetic import Workload, chain_workload, hand_workload, humanoid_workload
from .terms.dense import PositionLimit, PositionTask, RotationTask, SelfCollisionTask

DEFAULT_BATCH = {"chain7": 1024, "chain7c": 16384, "humanoid": 8192, "hand": 65536}


@dataclass
class Config:
    name: str
    workload: Workload
    robot: Robot
    terms: list
    lm: LMOptimizerConfig

    @property
    def batch(self) -> int:
        return self.workload.q0.shape[0]


def make(name: str, batch: Optional[int] = None, seed: int = 0,
         pair_mode: Literal["slots", "all"] = "all", form: Literal["plain", "persistent"] = "plain") -> Config:
    B = batch or DEFAULT_BATCH[name]
    if name == "chain7":
        wl = chain_workload(B, seed)
        robot = Robot(wl.spec)
        ee = wl.target_links[0]
        terms: List = [PositionTask(robot, ee, wl.targets, weight=1.0), RotationTask(robot, ee, wl.targets, weight=1.0)]
        lm = LMOptimizerConfig(max_iter=50, lm_lambda=1e-3, lambda_factor=10.0, early_stopping_interval=0, form=form)
    elif name == "chain7c":
        wl = chain_workload(B, seed, spheres=True, unreachable_frac=0.1)
        robot = Robot(wl.spec)
        ee = wl.target_links[0]
        terms = [
            PositionTask(robot, ee, wl.targets, weight=1.0),
            RotationTask(robot, ee, wl.targets, weight=1.0),
            SelfCollisionTask(robot, weight=1.0, margin=0.02, pair_mode=pair_mode),
            PositionLimit(robot, weight=1.0),
        ]
        lm = LMOptimizerConfig(max_iter=100, lm_lambda=1e-3, lambda_factor=10.0, early_stopping_interval=0,
                               step_tol=1e-6, form=form)
    elif name == "humanoid":
        wl = humanoid_workload(B, seed)
        robot = Robot(wl.spec)
        terms = [PositionTask(robot, wl.target_links, wl.targets, weight=1.0),
                 RotationTask(robot, wl.target_links, wl.targets, weight=1.0)]
        lm = LMOptimizerConfig(max_iter=100, lm_lambda=1e-3, lambda_factor=10.0, early_stopping_interval=0,
                               step_tol=1e-6, form=form)
    elif name == "hand":
        wl = hand_workload(B, seed)
        robot = Robot(wl.spec)
        terms = [PositionTask(robot, wl.target_links, wl.targets, weight=1.0)]
        lm = LMOptimizerConfig(max_iter=30, lm_lambda=1e-3, lambda_factor=10.0, early_stopping_interval=0, form=form)
    else:
        raise KeyError(name)
    return Config(name, wl, robot, terms, lm)


def oracle_terms(cfg: Config) -> list:
    """The same term list as plain dicts (the oracle's OrTerm fields)."""
    out = []
    for t in cfg.terms:
        d = t.host_desc(_Stub(cfg))
        out.extend(d if isinstance(d, list) else [d])
    return out


class _Stub:
    def __init__(self, cfg: Config):
        self.spec = cfg.workload.spec
        self.robot = cfg.robot
        self.batch_size = cfg.batch
        self.has_floating_base = cfg.workload.base0 is not None
