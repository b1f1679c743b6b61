"""IKSolver: batched IK over a candidate population (helpers/ik/ik.py:98-484).

For each target the solver seeds `num_candidates` joint configurations with a
Roberts spread around the joint midrange (or around `init_state`), runs the
stages of its PopulationSolverConfig — a persistent LM solve of every
candidate for the stage's iterations, then a device-side select of each
target's best candidates by cost — and returns the final stage's candidates.

Everything between the host call and the result runs on the GPU: the spread
(integrate + clamp kernels), one persistent solve launch per stage and one
select launch between stages.  The term templates of the config (PositionTask,
RotationTask with IKContext placeholders, PositionLimit) become concrete terms
that read the targets with the reference's broadcast rule (candidate c of
target b reads target row b).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, replace
from typing import Any, List, Optional, Sequence, Union

import numpy as np

from ... import _native as N
from ...opt.lm_optimizer import LMOptimizer, LMOptimizerConfig
from ...opt.sampler import RobertsSampler
from ...opt.var_values import VarKey, VarValues
from ...robo.robot_state import RobotState
from ...terms.dense import PositionLimit, PositionTask, RotationTask, SelfCollisionTask, _PoseTask
from ...terms.task import Context
from .config import IKContext, IKSolverConfig


@dataclass
class IKMetrics:
    """Per target and target link: position error [m], angle error [rad]; per target: success."""

    position_error_m: np.ndarray
    orientation_error_rad: np.ndarray
    success: np.ndarray


class IKSolver:
    def __init__(self, config: IKSolverConfig, robot: Any, target_links: Union[str, int, Sequence[Union[str, int]]],
                 device: Any = "cuda", scene: Any = None):
        if scene is not None:
            raise NotImplementedError("scene collision is outside the IK hot path")
        if config.enable_T_world_base:
            raise NotImplementedError("a floating base in IKSolver is outside this build (fixed base only)")
        if config.score_terms:
            raise NotImplementedError("score terms are outside this build (candidates rank by cost)")
        if device is not None and not str(device).startswith("cuda"):
            raise ValueError(f"device {device!r}: this library runs on CUDA only (no CPU fallback)")
        self.config = config
        self.robot = robot
        names = robot.spec.link_names
        links = [target_links] if isinstance(target_links, (str, int, np.integer)) else list(target_links)
        self.target_links = [names.index(x) if isinstance(x, str) else int(x) for x in links]
        self.num_targets = len(self.target_links)
        self.widths = config.solver.num_candidates
        self.lm_configs = config.solver.optimizers
        self._batch = None

    # --- sizes -------------------------------------------------------------------------
    @property
    def num_solutions(self) -> int:
        return self.widths[-1]

    @property
    def num_joints(self) -> int:
        return self.robot.spec.num_actuated_joints

    # --- build ---------------------------------------------------------------------------
    def _concrete_terms(self, targets: N.DeviceArray) -> list:
        out = []
        for t in self.config.terms:
            if isinstance(t, _PoseTask):
                fi, tg = t.frame_index_arg, t.T_world_target_arg
                frames = self.target_links if fi in (IKContext.TARGET_LINKS, None) else (
                    [self.target_links[0]] if fi is IKContext.TARGET_LINK else fi)
                if tg is not IKContext.TARGET and not isinstance(tg, Context):
                    raise NotImplementedError("IKSolver pose templates take T_world_target=IKContext.TARGET")
                out.append(type(t)(self.robot, frames, targets, weight=t.weight))
            elif isinstance(t, PositionLimit):
                out.append(PositionLimit(self.robot, weight=t.weight))
            elif isinstance(t, SelfCollisionTask):
                c = SelfCollisionTask(self.robot, t.weight, t.margin, max_active_pairs=t.max_active_pairs,
                                      filter_adjacent_links=t.filter_adjacent_links, pair_mode=t.pair_mode)
                out.append(c)
            else:
                raise NotImplementedError(f"{type(t).__name__} is outside the IK hot path")
        return out

    def _build(self, B: int) -> None:
        spec = self.robot.spec
        na = spec.num_actuated_joints
        self._targets = N.DeviceArray.zeros((B, self.num_targets, 7))
        self._terms = self._concrete_terms(self._targets)
        self._pose_terms = [t for t in self._terms if isinstance(t, _PoseTask)]
        self._stages = []
        for k, (width, lm) in enumerate(zip(self.widths, self.lm_configs)):
            iters = self.config.solver.stages[k].iters
            state = self.robot.state(np.zeros((B * width, na), np.float32))
            opt = None
            if iters > 0:
                cfg = replace(lm, max_iter=iters, early_stopping_interval=0, form="persistent")
                opt = LMOptimizer(self._terms, cfg)
                opt.reset(VarValues({VarKey.ROBOT: state}))
            self._stages.append((width, iters, state, opt))
        C0 = self.widths[0]
        lim = spec.float32_actuated_limits()
        self._range = (lim[:, 1] - lim[:, 0]).astype(np.float32)
        self._sampler = RobertsSampler(C0, na, self.config.sampler.seed, self.config.sampler.keep_first)
        self._mid = N.DeviceArray.from_numpy(np.tile(spec.midrange_q.astype(np.float32), (B * C0, 1)))
        self._noise_scale = None
        self._noise = None
        self._cost = [N.DeviceArray.zeros(B * w) for w in self.widths]
        self._batch = B

    def warmup(self, batch_size: int) -> None:
        """Build the buffers and run one solve on identity targets."""
        T = np.tile(np.array([0, 0, 0, 1, 0, 0, 0], np.float32), (batch_size, self.num_targets, 1))
        self.solve(T)
        N.synchronize()

    # --- solve ---------------------------------------------------------------------------
    def _seed(self, init_state: Optional[RobotState], q_range: Union[float, Sequence[float]]) -> None:
        B, C0 = self._batch, self.widths[0]
        na = self.num_joints
        state = self._stages[0][2]
        if init_state is not None:
            if init_state.batch_size != B:
                raise ValueError(f"init_state batch size {init_state.batch_size} != {B}")
            rep = np.repeat(np.arange(B, dtype=np.int32), C0)
            center = N.DeviceArray.from_numpy(init_state.q.numpy()[rep])
            scale = np.asarray(q_range, np.float32) * self._range
        else:
            center = self._mid
            scale = self._range.copy()
        if C0 == 1 and init_state is not None:
            state.q.assign(center)
            return
        if self._noise_scale is None or not np.array_equal(scale, self._noise_scale):
            self._noise = N.DeviceArray.from_numpy(self._sampler.tangent(B, scale))
            self._noise_scale = scale
        N.check(N.lib().ik_integrate(B * C0, na, 0, center.ptr, None, self._noise.ptr, None, state.q.ptr, None, None))
        state.invalidate()
        state.clamp_q()

    def solve(self, T_world_target: Any, init_state: Optional[RobotState] = None,
              out_state: Optional[RobotState] = None, init_sample_range: Optional[float] = None) -> RobotState:
        """Solutions for every target, instance-major: (batch * num_solutions, dofs) (helpers/ik/ik.py:223-304)."""
        T = N.as_device(T_world_target, np.float32)
        if T.ndim == 2:
            T = T.reshape((T.shape[0], 1, 7))
        if T.ndim != 3 or T.shape[2] != 7 or T.shape[1] != self.num_targets:
            raise ValueError(f"Target count ({T.shape[1] if T.ndim == 3 else '?'}) must match IK target count "
                             f"({self.num_targets})")
        B = T.shape[0]
        if self._batch is None:
            self._build(B)
        elif B != self._batch:
            raise ValueError(f"Batch size mismatch: expected {self._batch}, got {B}")
        self._targets.assign(T)
        for t in self._pose_terms:
            t.set_target(self._targets)
        self._seed(init_state, self.config.sampler.scale if init_sample_range is None else init_sample_range)
        na = self.num_joints
        for k, (width, iters, state, opt) in enumerate(self._stages):
            if opt is not None:
                opt.solve(VarValues({VarKey.ROBOT: state}))
                self._cost[k].assign(opt.costs)
            elif k == 0:
                self._score(state, self._cost[k])
            if k + 1 < len(self._stages):
                nxt_w, _, nxt_state, _ = self._stages[k + 1]
                N.check(N.lib().ik_select_best(B, width, nxt_w, self._cost[k].ptr, state.q.ptr, None, na,
                                               nxt_state.q.ptr, None, self._cost[k + 1].ptr, None, None))
                nxt_state.invalidate()
        final = self._stages[-1][2]
        if out_state is not None:
            out_state.q.assign(final.q)
            out_state.invalidate()
            return out_state
        return final

    @property
    def costs(self) -> N.DeviceArray:
        """Cost of each returned solution (the final stage's)."""
        return self._cost[-1]

    def _score(self, state: RobotState, out: N.DeviceArray) -> None:
        opt = LMOptimizer(self._terms, LMOptimizerConfig(max_iter=0, early_stopping_interval=0, form="persistent"))
        opt.solve(VarValues({VarKey.ROBOT: state}))
        out.assign(opt.costs)

    # --- metrics ---------------------------------------------------------------------------
    def compute_metrics(self, state: RobotState, T_world_target: Any, position_threshold: float = 0.005,
                        rotation_threshold: float = 0.05) -> IKMetrics:
        """Pose errors of every target link and success within both thresholds (helpers/ik/ik.py:60-82,387-471)."""
        T = N.as_device(T_world_target, np.float32)
        B = T.shape[0]
        nt = self.num_targets
        T = T.reshape((B, nt, 7))
        if state.batch_size != B:
            raise ValueError(f"state batch {state.batch_size} != targets {B}")
        links = N.DeviceArray.from_numpy(np.asarray(self.target_links, np.int32))
        pe, re = N.DeviceArray.empty((B, nt)), N.DeviceArray.empty((B, nt))
        ok = N.DeviceArray.empty(B, np.int32)
        N.check(N.lib().ik_metrics(self.robot.handle, B, state.q.ptr, N.ptr(state.T_world_base) if
                                   state.has_floating_base else None, nt, links.ptr, T.ptr, float(position_threshold),
                                   float(rotation_threshold), pe.ptr, re.ptr, ok.ptr, None))
        return IKMetrics(pe.numpy(), re.numpy(), ok.numpy().astype(bool))
