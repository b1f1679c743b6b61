"""Candidate schedule of a population solve (opt/population_solver.py:57-96).

A solve runs `stages` in order.  Entering a stage keeps each instance's best
`num_candidates` by cost (the first stage's width is the number of initial
candidates) and runs `iters` LM iterations on them; unset fields keep the
previous stage's.  The LM state restarts at every stage.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field, replace
from typing import Any, List, Literal, Optional

import numpy as np

from .lm_optimizer import LMOptimizer, LMOptimizerConfig, OptimizerConfig
from .var_values import VarKey, VarValues


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


class _Stage:
    """One stage's population (a RobotState of batch * width rows), its LM problem (None for a select-only
    stage) and launch parameters, its cost buffer and, where score terms rank it, a zero-iteration problem over
    them with a scratch copy of the population."""

    def __init__(self, width: int, iters: int, state: Any, opt: Optional[LMOptimizer], cost: Any,
                 ranker: Optional[tuple]):
        self.width, self.iters, self.state, self.opt, self.cost, self.ranker = width, iters, state, opt, cost, ranker
        self.params = None if opt is None else opt.config.native_params()


def build_stages(robot: Any, floating: bool, batch: int, config: PopulationSolverConfig, terms: List[Any],
                 score_terms: List[Any], mask: Any) -> List[_Stage]:
    """The stages of a population solve of `batch` instances (opt/population_solver.py:204-270): an LM problem
    per stage with iterations, capacity batch * width, and the score problems of the ranked stages (every stage,
    or with rank_final only the last, :179-186)."""
    from .. import _native as N

    na = robot.spec.num_actuated_joints
    ident = np.array([0, 0, 0, 1, 0, 0, 0], np.float32)

    def state(rows: int) -> Any:
        return robot.state(np.zeros((rows, na), np.float32), np.tile(ident, (rows, 1)) if floating else None)

    out, last = [], len(config.stages) - 1
    for k, (width, lm) in enumerate(zip(config.num_candidates, config.optimizers)):
        iters = config.stages[k].iters
        st = state(batch * width)
        opt = None
        if iters > 0:
            opt = LMOptimizer(terms, replace(lm, max_iter=iters, early_stopping_interval=0, form="persistent"),
                              active_dof_mask=mask)
            opt.reset(VarValues({VarKey.ROBOT: st}))
        ranker = None
        if score_terms and (not config.rank_final or k == last):
            scratch = state(batch * width)
            sc = LMOptimizer(score_terms, LMOptimizerConfig(max_iter=0, form="persistent"), active_dof_mask=mask)
            sc.reset(VarValues({VarKey.ROBOT: scratch}))
            ranker = (sc, scratch, sc.config.native_params())
        out.append(_Stage(width, iters, st, opt, N.DeviceArray.zeros(batch * width), ranker))
    if out[0].opt is None and out[0].ranker is None:
        raise NotImplementedError("a first stage without iterations needs score terms to rank it")
    return out


def run_stages(stages: List[_Stage], batch: int, floating: bool, stream: int, ranked: Any = None,
               ranked_cost: Any = None) -> None:
    """Device work of a population solve from stage 0's population (opt/population_solver.py:294-404): each
    stage's persistent LM launch, its scoring where score terms rank it, a select of every instance's best
    candidates into the next stage, and with `ranked` the final population sorted best first."""
    from .. import _native as N

    lib = N.lib()
    for k, s in enumerate(stages):
        n = batch * s.width
        base = s.state.T_world_base.ptr if floating else None
        na = s.state.q.shape[1]
        if s.opt is not None:
            s.opt._slice(n)
            N.check(lib.ik_solve_persistent(s.opt.problem.handle, n, s.state.q.ptr, base, ctypes.byref(s.params),
                                            s.cost.ptr, s.opt.lm.ptr, s.opt.iterations.ptr, s.opt.status.ptr, stream))
        if s.ranker is not None and (s.opt is not None or k == 0 or stages[k - 1].ranker is None):
            sc, scratch, prm = s.ranker  # a select from a ranked stage already carries its scores
            N.check(lib.ik_memcpy_dtod(scratch.q.ptr, s.state.q.ptr, n * na * 4, stream))
            if floating:
                N.check(lib.ik_memcpy_dtod(scratch.T_world_base.ptr, base, n * 28, stream))
            sc._slice(n)
            N.check(lib.ik_solve_persistent(sc.problem.handle, n, scratch.q.ptr,
                                            scratch.T_world_base.ptr if floating else None, ctypes.byref(prm),
                                            s.cost.ptr, sc.lm.ptr, sc.iterations.ptr, sc.status.ptr, stream))
        if k + 1 < len(stages):
            nxt = stages[k + 1]
            N.check(lib.ik_select_best(batch, s.width, nxt.width, s.cost.ptr, s.state.q.ptr, base, na,
                                       nxt.state.q.ptr, nxt.state.T_world_base.ptr if floating else None,
                                       nxt.cost.ptr, None, stream))
    if ranked is not None:
        s = stages[-1]
        N.check(lib.ik_select_best(batch, s.width, ranked.q.shape[0] // batch, s.cost.ptr, s.state.q.ptr,
                                   s.state.T_world_base.ptr if floating else None, s.state.q.shape[1], ranked.q.ptr,
                                   ranked.T_world_base.ptr if floating else None, N.ptr(ranked_cost), None,
                                   stream))
        ranked.invalidate()
    for s in stages:
        s.state.invalidate()


class PopulationSolver:
    """A population solve of `batch * num_candidates[0]` candidates (opt/population_solver.py:148-404) on the IK
    path: LM stages, each instance's best candidates kept between stages by cost (or by the score terms' cost),
    the best candidate of every instance returned.

    The population is instance-major (candidate c of instance b is row b * width + c); terms built for
    `batch` rows broadcast over the candidates.  Samplers, per-stage term lists and optimizers other than LM
    are outside this path."""

    def __init__(self, terms: Any, config: PopulationSolverConfig, device: Any = "cuda", score_terms: Any = None, *,
                 active_dof_mask: Any = None):
        if device is not None and not str(device).startswith("cuda"):
            raise ValueError(f"device {device!r}: this library runs on CUDA only (no CPU fallback)")
        if terms and isinstance(terms[0], list):
            if any(t != terms[0] for t in terms[1:]):
                raise NotImplementedError("per-stage term lists are outside the IK path")
            terms = terms[0]
        self.terms = list(terms)
        if isinstance(score_terms, (list, tuple)):
            self.score_terms = [t for t in score_terms if t is not None]
        else:
            self.score_terms = [] if score_terms is None else [score_terms]
        self.config = config
        self.device = "cuda:0"
        self._mask = active_dof_mask
        self._initialized = False
        self.final_var: Optional[VarValues] = None
        self.best_costs = None

    def setup(self, var: VarValues) -> None:
        """Build the stages for `var`'s width (opt/population_solver.py:204-270)."""
        from .. import _native as N

        state = var.get(VarKey.ROBOT)
        c0 = self.config.num_candidates[0]
        if state.batch_size % c0:
            raise ValueError(f"input batch {state.batch_size} is not a multiple of num_candidates[0]={c0}")
        mask = self._mask
        if mask is not None:
            mask = np.asarray(mask.numpy() if hasattr(mask, "numpy") else mask, np.float32).reshape(-1)
            if mask.shape != (state.tangent_dim,):
                raise ValueError("active_dof_mask must match the variable tangent dimensions")
        self.batch_size = B = state.batch_size // c0
        self._robot, self._floating = state.robot, state.has_floating_base
        self._stages = build_stages(state.robot, state.has_floating_base, B, self.config, self.terms,
                                    self.score_terms, mask)
        na = state.spec.num_actuated_joints
        ident = np.tile(np.array([0, 0, 0, 1, 0, 0, 0], np.float32), (B, 1))
        self._best = state.robot.state(np.zeros((B, na), np.float32), ident if self._floating else None)
        self.best_costs = N.DeviceArray.zeros(B)
        self._best_index = N.DeviceArray.zeros(B, np.int32)
        wf = self.config.num_candidates[-1]
        self._ranked = None
        if self.config.rank_final and wf > 1:
            self._ranked = state.robot.state(np.zeros((B * wf, na), np.float32),
                                             np.tile(ident, (wf, 1)) if self._floating else None)
            self._ranked_cost = N.DeviceArray.zeros(B * wf)
        self._stream = N.Stream()
        self._graph = None
        self._in_ptrs: Optional[tuple] = None
        self._initialized = True

    def _body(self, q_ptr: int, base_ptr: Optional[int], stream: int) -> None:
        from .. import _native as N

        s0 = self._stages[0]
        N.check(N.lib().ik_memcpy_dtod(s0.state.q.ptr, q_ptr, s0.state.q.nbytes, stream))
        if self._floating:
            N.check(N.lib().ik_memcpy_dtod(s0.state.T_world_base.ptr, base_ptr, s0.state.T_world_base.nbytes, stream))
        run_stages(self._stages, self.batch_size, self._floating, stream, self._ranked,
                   self._ranked_cost if self._ranked is not None else None)
        last = self._stages[-1]
        fb = self._floating
        N.check(N.lib().ik_select_best(self.batch_size, last.width, 1, last.cost.ptr, last.state.q.ptr,
                                       last.state.T_world_base.ptr if fb else None, last.state.q.shape[1],
                                       self._best.q.ptr, self._best.T_world_base.ptr if fb else None,
                                       self.best_costs.ptr, self._best_index.ptr, stream))

    def solve(self, var: VarValues):
        """Solve from the candidates in `var` (batch * num_candidates[0] rows); returns (best_var, best_costs):
        every instance's cheapest final candidate and its cost.  `final_var` holds the final population
        (sorted best first per instance with rank_final).  Under cuda_graph_mode "full" the device work is
        captured at the first solve and replayed while `var`'s buffers stay the same."""
        from .. import _native as N

        if not self._initialized:
            self.setup(var)
        state = var.get(VarKey.ROBOT)
        if state.batch_size != self.batch_size * self.config.num_candidates[0]:
            raise ValueError(f"Batch size mismatch: expected {self.batch_size * self.config.num_candidates[0]}, "
                             f"got {state.batch_size}")
        if state.has_floating_base != self._floating:
            raise ValueError("the floating-base layout changed since setup")
        st = self._stream.handle
        qp, bp = state.q.ptr, state.T_world_base.ptr if self._floating else None
        N.check(N.lib().ik_device_synchronize())  # the caller's writes to var precede the solve's stream
        if self.config.cuda_graph_mode == "full":
            if self._graph is None or self._in_ptrs != (qp, bp):
                self._body(qp, bp, st)
                self._graph = N.Graph(self._stream).capture(lambda: self._body(qp, bp, st))
                self._in_ptrs = (qp, bp)
            else:
                self._graph.launch()
        else:
            self._body(qp, bp, st)
        N.check(N.lib().ik_stream_synchronize(st))
        self._best.invalidate()
        final = self._ranked if self._ranked is not None else self._stages[-1].state
        self.final_var = VarValues({VarKey.ROBOT: final})
        return VarValues({VarKey.ROBOT: self._best}), self.best_costs

    def compute_costs(self, var: VarValues) -> dict:
        """|r|^2 of every term at `var`, summed by cost_name, one value per row
        (opt/population_solver.py:555-574)."""
        from .. import _native as N

        state = var.get(VarKey.ROBOT)
        n = state.batch_size
        out: dict = {}
        for t in self.terms:
            c = out.setdefault(t.cost_name, N.DeviceArray.zeros(n))
            if t.residual_dim == 0:
                continue
            r = t.compute_weighted_residual(var)
            N.check(N.lib().ik_row_sumsq(n, r.shape[1], r.ptr, r.shape[1], c.ptr, 1, None))
        N.check(N.lib().ik_device_synchronize())
        return out
