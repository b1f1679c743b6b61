"""Candidate schedule of a population solve (opt/population_solver.py:57-96).

A solve runs `stages` in order.  Entering a stage keeps each instance's best
`num_candidates` by cost (the first stage's width is the number of initial
candidates) and runs `iters` LM iterations on them; unset fields keep the
previous stage's.  The LM state restarts at every stage.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Literal, Optional

from .lm_optimizer import LMOptimizerConfig, OptimizerConfig


@dataclass
class Stage:
    iters: int = 0
    num_candidates: Optional[int] = None
    optimizer: Optional[OptimizerConfig] = None
    sample_every: int = 0


@dataclass
class PopulationSolverConfig:
    stages: List[Stage] = field(default_factory=lambda: [Stage(iters=10)])
    cuda_graph_mode: Literal["none", "full", "iter"] = "iter"
    use_early_stopping: bool = True
    rank_final: bool = False

    @property
    def num_candidates(self) -> List[int]:
        """Resolved width of every stage."""
        out, cur = [], 1
        for s in self.stages:
            cur = s.num_candidates if s.num_candidates is not None else cur
            out.append(int(cur))
        return out

    @property
    def optimizers(self) -> List[LMOptimizerConfig]:
        """Resolved LM configuration of every stage (default LMOptimizerConfig until one is set)."""
        out, cur = [], LMOptimizerConfig()
        for s in self.stages:
            if s.optimizer is not None:
                if not isinstance(s.optimizer, LMOptimizerConfig):
                    raise NotImplementedError("only LM stages are on the IK hot path")
                cur = s.optimizer
            out.append(cur)
        return out
