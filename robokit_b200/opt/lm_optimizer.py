"""Levenberg–Marquardt optimizer over the fused sm_100a kernel.

Drop-in for robokit's ``LMOptimizer`` / ``LMOptimizerConfig``
(opt/lm_optimizer.py:502-1005) and ``Optimizer`` / ``OptimizerConfig``
(opt/optimizer.py:159-333) on the Cholesky path: same constructor, ``solve``,
``reset``, ``step``, capacity rule and buffers (``costs``, ``delta``, ``lm``,
``pred_reduction``, ``accept_mask``).  One IK problem per lane group; the
damped normal matrix is factorised in FP64.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, replace
from typing import Any, Callable, Dict, List, Literal, Optional, Sequence, Tuple, Union

import numpy as np

from .. import _native as N
from ..terms.task import NativeProblem, ResidualTask, Task
from .var_values import VarKey, VarValues

IterationCallback = Callable[[int, VarValues, Any], None]


@dataclass(frozen=True)
class OptimizerConfig:
    """opt/optimizer.py:159-174"""

    max_iter: int = 100
    early_stopping_interval: int = 1
    cost_tol: float = 1e-9
    cuda_graph_mode: Literal["none", "iter", "full"] = "none"


@dataclass(frozen=True)
class LMOptimizerConfig(OptimizerConfig):
    """opt/lm_optimizer.py:502-530, plus the per-problem stop rules and solver form of this library."""

    lm_lambda: float = 1e-3
    lambda_factor: float = 2.0
    lambda_min: float = 1e-5
    lambda_max: float = 1e10
    rho_min: float = 1e-3
    gain_ratio_epsilon: float = 1e-8
    linear_solver: Literal["cholesky", "cg", "torch_cholesky"] = "cholesky"
    cg_max_iter: Optional[int] = None
    cg_tol: float = 1e-6
    cg_check_interval: int = 4
    # --- no reference counterpart -------------------------------------------------
    step_tol: Optional[float] = None
    """Stop a problem once its LM step norm falls below this."""
    pose_tol: Optional[Tuple[float, float]] = None
    """Stop a problem once every pose target is within (metres, radians)."""
    problem_cost_tol: Optional[float] = None
    """Stop a problem once its own cost is at most this."""
    form: Literal["plain", "persistent"] = "plain"
    """plain: one launch per iteration over the batch; persistent: a work-queue launch runs each problem to its stop."""

    def build(self, terms: Sequence[Task], device: Any = None, active_dof_mask: Any = None) -> "LMOptimizer":
        return LMOptimizer(terms, self, device, active_dof_mask)

    def native_params(self) -> N.IkLmParams:
        rules = 0
        if self.early_stopping_interval > 0 and self.form == "plain":
            rules |= N.IK_STOP_ALL_COST
        if self.step_tol is not None:
            rules |= N.IK_STOP_STEP
        if self.pose_tol is not None:
            rules |= N.IK_STOP_POSE
        if self.problem_cost_tol is not None:
            rules |= N.IK_STOP_COST
        pt = self.pose_tol if self.pose_tol is not None else (0.0, 0.0)
        cost_tol = self.problem_cost_tol if self.problem_cost_tol is not None else self.cost_tol
        return N.IkLmParams(
            int(self.max_iter),
            float(self.lm_lambda),
            float(self.lambda_factor),
            float(self.lambda_min),
            float(self.lambda_max),
            float(self.rho_min),
            float(self.gain_ratio_epsilon),
            rules,
            float(cost_tol),
            float(self.step_tol or 0.0),
            float(pt[0]),
            float(pt[1]),
            max(1, int(self.early_stopping_interval)),
        )


class LMOptimizer:
    """Batched LM over a list of residual terms (opt/lm_optimizer.py:533-1005)."""

    _config_type = LMOptimizerConfig

    def __init__(self, terms: Union[Task, Sequence[Task]], config: Optional[LMOptimizerConfig] = None,
                 device: Any = None, active_dof_mask: Any = None):
        self.terms: List[ResidualTask] = list(terms) if isinstance(terms, Sequence) else [terms]
        self.config = config if config is not None else LMOptimizerConfig()
        if self.config.linear_solver != "cholesky":
            raise NotImplementedError(
                f"linear_solver={self.config.linear_solver!r} is outside the IK hot path (Cholesky only)"
            )
        if device is not None and not str(device).startswith("cuda"):
            raise ValueError(f"device {device!r}: this library runs on CUDA only (no CPU fallback)")
        for t in self.terms:
            if not isinstance(t, ResidualTask):
                raise TypeError(f"{type(t).__name__} is not a residual term this library can lower")
        self.device = "cuda:0"
        self._mask_arg = active_dof_mask
        self._built = False
        self._problem: Optional[NativeProblem] = None
        self._versions: Tuple[int, ...] = ()
        self._iter = 0
        self.max_batch_size = 0
        self.batch_size = 0
        self._stream: Optional[N.Stream] = None
        self._graph: Optional[N.Graph] = None
        self._graph_key: Optional[tuple] = None

    # -- lifecycle ---------------------------------------------------------------------
    def _mask_np(self, D: int) -> Optional[np.ndarray]:
        if self._mask_arg is None:
            return None
        m = self._mask_arg
        m = m.numpy() if hasattr(m, "numpy") else np.asarray(m)
        m = np.asarray(m, np.float32).reshape(-1)
        if m.shape != (D,):
            raise ValueError("active_dof_mask must have shape (total_tangent_dim,).")
        return m

    def _build(self, var_values: VarValues, capacity: Optional[int] = None) -> None:
        if len(list(var_values.keys())) != 1 or VarKey.ROBOT not in var_values:
            raise TypeError("LMOptimizer here optimises one RobotState keyed VarKey.ROBOT")
        var = var_values.get(VarKey.ROBOT)
        B, D = capacity or var_values.batch_size, var_values.tangent_dim
        mask = self._mask_np(D)
        self._problem = NativeProblem(var.robot, self.terms, B, var.has_floating_base, mask)
        self._graph = None  # a recorded solve names the old problem's buffers
        self._floating = var.has_floating_base
        self._robot = var.robot
        self.total_tangent_dim = D
        self.total_residual_dim = self._problem.residual_dim
        self.max_batch_size = B
        self._versions = tuple(getattr(t, "_version", 0) for t in self.terms)
        self._full = dict(
            costs=N.DeviceArray.zeros(B),
            proposed_costs=N.DeviceArray.zeros(B),
            pred_reduction=N.DeviceArray.zeros(B),
            lm=N.DeviceArray.zeros(B),
            delta=N.DeviceArray.zeros((B, D)),
            accept_mask=N.DeviceArray.zeros(B, np.int32),
            iterations=N.DeviceArray.zeros(B, np.int32),
            status=N.DeviceArray.zeros(B, np.int32),
        )

    def _slice(self, B: int) -> None:
        """Capacity buffers as prefix views (opt/optimizer.py:313-333)."""
        if B > self.max_batch_size:
            raise ValueError(f"batch size {B} exceeds the {self.max_batch_size} this optimizer was built for")
        for k, v in self._full.items():
            setattr(self, k, v.prefix(B))
        self.batch_size = B

    def reset(self, var_values: VarValues, num_steps: Optional[int] = None) -> None:
        if not self._built:
            self._build(var_values)
            self._built = True
        elif tuple(getattr(t, "_version", 0) for t in self.terms) != self._versions:
            # weights changed: lower the terms again at the same capacity
            self._build(var_values, capacity=self.max_batch_size)
        var = var_values.get(VarKey.ROBOT)
        if var.has_floating_base != self._floating:
            raise ValueError("the floating-base layout changed since this optimizer was built")
        self._slice(var_values.batch_size)
        self.lm.copy_from_numpy(np.full(self.batch_size, self.config.lm_lambda, np.float32))
        self._num_steps = self.config.max_iter if num_steps is None else num_steps
        self._iter = 0

    def solve(self, var_values: VarValues, iteration_callback: Optional[IterationCallback] = None):
        """Optimise `var_values` in place; returns (var_values, costs) (opt/optimizer.py:216-240)."""
        self.reset(var_values)
        cfg = self.config
        var = var_values.get(VarKey.ROBOT)
        B = self.batch_size
        if iteration_callback is not None:
            self._compute_start_costs(var_values)
            iteration_callback(0, var_values, self.costs)
            for i in range(cfg.max_iter):
                self.step(var_values)
                iteration_callback(i + 1, var_values, self.costs)
                if cfg.early_stopping_interval > 0 and (i + 1) % cfg.early_stopping_interval == 0:
                    if bool(np.all(self.costs.numpy() <= cfg.cost_tol)):
                        break
            return var_values, self.costs
        prm = cfg.native_params()
        fn = N.lib().ik_solve_persistent if cfg.form == "persistent" else N.lib().ik_solve_plain
        base = var.T_world_base.ptr if var.has_floating_base else None

        def launch(stream: Optional[int]) -> None:
            N.check(fn(self._problem.handle, B, var.q.ptr, base, ctypes.byref(prm), self.costs.ptr, self.lm.ptr,
                       self.iterations.ptr, self.status.ptr, stream))

        if cfg.cuda_graph_mode == "none":
            launch(None)
        else:
            # the whole solve (one launch per iteration in the plain form) recorded once per set of buffers and
            # parameters, then replayed (opt/optimizer.py:160-174, cuda_graph_mode)
            if self._stream is None:
                self._stream = N.Stream()
            key = (B, var.q.ptr, base, self._problem.handle, self.costs.ptr, self.lm.ptr, bytes(prm))
            if self._graph is None or self._graph_key != key:
                launch(self._stream.handle)
                self._graph = N.Graph(self._stream).capture(lambda: launch(self._stream.handle))
                self._graph_key = key
            else:
                self._graph.launch()
            self._stream.synchronize()
        var.invalidate()
        return var_values, self.costs

    def _compute_start_costs(self, var_values: VarValues) -> None:
        var = var_values.get(VarKey.ROBOT)
        D = self.total_tangent_dim
        H = N.DeviceArray.empty((self.batch_size, D, D))
        g = N.DeviceArray.empty((self.batch_size, D))
        N.check(N.lib().ik_normal_equations(self._problem.handle, self.batch_size, var.q.ptr,
                                            var.T_world_base.ptr if var.has_floating_base else None,
                                            H.ptr, g.ptr, self.costs.ptr, None))

    def step(self, var_values: VarValues) -> None:
        """One LM iteration in place (LMOptimizer._step_body, lm_optimizer.py:984-1005)."""
        if not self._built or var_values.batch_size != self.batch_size:
            self.reset(var_values)
        var = var_values.get(VarKey.ROBOT)
        prm = self.config.native_params()
        N.check(
            N.lib().ik_step(self._problem.handle, self.batch_size, var.q.ptr,
                            var.T_world_base.ptr if var.has_floating_base else None, self.lm.ptr, ctypes.byref(prm),
                            self.costs.ptr, self.delta.ptr, self.pred_reduction.ptr, self.proposed_costs.ptr,
                            self.accept_mask.ptr, None)
        )
        var.invalidate()
        self._iter += 1

    # -- schedule / introspection ------------------------------------------------------
    @property
    def problem(self) -> NativeProblem:
        if self._problem is None:
            raise RuntimeError("the optimizer is built at its first solve/reset")
        return self._problem

    def set_schedule(self, group_lanes: int = 0, blocks_per_sm: int = 0) -> None:
        self.problem.set_schedule(group_lanes, blocks_per_sm)

    def autotune(self, var_values: VarValues, lanes: Sequence[int] = (1, 8, 16, 32),
                 blocks_per_sm: Sequence[int] = (0,), repeats: int = 2) -> Dict[str, Any]:
        """Time whole solves of `var_values` under each schedule that applies and keep the fastest.

        A schedule is (lanes per problem, resident blocks per SM): one lane per
        problem carries 32 problems per warp (small systems, throughput), wider
        lane groups shorten each problem's iteration (latency).  The start point
        is restored after every trial, so `var_values` is unchanged on return.
        """
        self.reset(var_values)
        var = var_values.get(VarKey.ROBOT)
        q0 = var.q.clone()
        b0 = var.T_world_base.clone() if var.has_floating_base else None

        def restore() -> None:
            var.q.assign(q0)
            if b0 is not None:
                var.T_world_base.assign(b0)
            var.invalidate()

        ev0, ev1 = N.Event(), N.Event()
        times: Dict[str, float] = {}
        best, best_ms = None, float("inf")
        for g in lanes:
            for bps in blocks_per_sm:
                try:
                    self.set_schedule(g, bps)
                except (N.NativeError, ValueError):
                    continue
                restore()
                self.solve(var_values)  # warm-up: kernel attributes, caches
                ms = 0.0
                for _ in range(max(1, repeats)):
                    restore()
                    N.synchronize()
                    ev0.record()
                    self.solve(var_values)
                    ev1.record()
                    N.synchronize()
                    ms += ev0.elapsed_ms(ev1)
                ms /= max(1, repeats)
                times[f"{g}x{bps}"] = round(ms, 4)
                if ms < best_ms:
                    best, best_ms = (g, bps), ms
        if best is None:
            raise RuntimeError("no schedule applies to this problem")
        self.set_schedule(*best)
        restore()
        return {"lanes": best[0], "blocks_per_sm": best[1], "ms": round(best_ms, 4), "times_ms": times}
