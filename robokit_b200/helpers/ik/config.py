"""Robot-free IK configuration (helpers/ik/config.py:12-80): term templates, candidate schedule, sampler."""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

from ...opt.lm_optimizer import LMOptimizerConfig
from ...opt.population_solver import PopulationSolverConfig, Stage
from ...opt.sampler import RobertsSamplerConfig
from ...terms.task import Context, ResidualTask


class IKContext(Context):
    """Values an IKSolver gives its term templates (helpers/ik/config.py:12-32)."""

    TARGET_LINKS = 0
    """Indices of the target links."""
    TARGET_LINK = 1
    """The first target link."""
    TARGET = 2
    """Target poses (batch, links, 7), which candidates share."""
    PREVIOUS_STATE = 3
    """The previous solution (batch,), from solve(prev_state=...); zeros until the first one."""
    REST_Q = 4
    """Rest configurations (batch, dofs): the zero configuration until solve(rest_state=...)."""
    REST_BASE = 5
    """Rest base poses (batch,): identity until solve(rest_state=...); None for a fixed base."""
    NUM_SOLUTIONS = 6
    """Solutions each target returns."""
    OPTIMIZATION_TERMS = 7
    """The built optimization terms (score terms are not supported here)."""
    SCENE = 8
    """The collision scene, from IKSolver(scene=...); None without one."""
    SCENE_INDICES = 9
    """Each target's scene (batch,): zeros until solve(scene_indices=...)."""


def _default_solver() -> PopulationSolverConfig:
    """64 candidates for 6 iterations, the best 4 for 10 more, then the best one (helpers/ik/config.py:37-45)."""
    return PopulationSolverConfig(
        stages=[
            Stage(6, 64, LMOptimizerConfig(lm_lambda=10.0)),
            Stage(10, 4, LMOptimizerConfig(lm_lambda=1.0)),
            Stage(0, 1),
        ],
        cuda_graph_mode="full",
    )


@dataclass
class IKSolverConfig:
    terms: List[ResidualTask] = field(default_factory=list)
    score_terms: List[ResidualTask] = field(default_factory=list)
    solver: PopulationSolverConfig = field(default_factory=_default_solver)
    sampler: RobertsSamplerConfig = field(default_factory=lambda: RobertsSamplerConfig(keep_first=True))
    base_init_sample_range: Tuple[float, float, float] = (0.1, 0.1, 0.0)
    enable_T_world_base: bool = False
    base_active_mask: Sequence[float] = (1.0, 1.0, 1.0, 1.0, 1.0, 1.0)

    def __post_init__(self):
        if len(self.base_active_mask) != 6:
            raise ValueError(f"base_active_mask length {len(self.base_active_mask)} != 6")
        if any(m != 1.0 for m in self.base_active_mask) and not self.enable_T_world_base:
            raise ValueError("base_active_mask requires enable_T_world_base=True")

    def add(self, term: ResidualTask, *, name: Optional[str] = None) -> "IKSolverConfig":
        """Append an optimization term; without `name` it is called `<cost_name>_<n>`, the first n free."""
        self._assign_name(term, name)
        self.terms.append(term)
        return self

    def add_score(self, term: ResidualTask, *, name: Optional[str] = None) -> "IKSolverConfig":
        """Append a term that ranks candidates at every select (by the sum of its squared residuals) without
        entering the optimization (helpers/ik/config.py:53-54)."""
        self._assign_name(term, name)
        self.score_terms.append(term)
        return self

    def task(self, name: str) -> ResidualTask:
        """The term added under `name` (helpers/ik/config.py:84-89)."""
        for t in (*self.terms, *self.score_terms):
            if t.name == name:
                return t
        raise KeyError(f"No IK term named {name!r}.")

    def _assign_name(self, term: ResidualTask, name: Optional[str]) -> None:
        if name is not None:
            term.name = name
            return
        taken = {t.name for t in (*self.terms, *self.score_terms)}
        n = 0
        while f"{term.cost_name}_{n}" in taken:
            n += 1
        term.name = f"{term.cost_name}_{n}"
