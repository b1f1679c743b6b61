"""IKSolver: batched IK over a candidate population (helpers/ik/ik.py:98-484).

For each target the solver seeds `num_candidates` joint configurations with a
Roberts spread around the joint midrange (or around `init_state`), runs the
stages of its PopulationSolverConfig — a persistent LM solve of every
candidate for the stage's iterations, then a device-side select of each
target's best candidates by cost — and returns the final stage's candidates.

Everything between the host call and the result runs on the GPU: the spread
(integrate + clamp kernels), one persistent solve launch per stage and one
select launch between stages.  The term templates of the config (PositionTask,
RotationTask, FrameTask with IKContext placeholders, PositionLimit,
SelfCollisionTask, SmoothnessTask and VelocityLimitTask on
IKContext.PREVIOUS_STATE, ConfigurationTask on IKContext.REST_Q,
SceneCollisionTask on IKContext.SCENE / SCENE_INDICES) become concrete terms
that read the solver's target, previous-state, rest and scene-index buffers in
place with the reference's broadcast rule (candidate c of target b reads row b).  With a previous state, each target keeps
it where it scores no worse than the solve's result (helpers/ik/ik.py:257-289).

Score terms (IKSolverConfig.add_score) rank the candidates at every select in place of the optimizer's
cost: after a stage's LM solve a zero-iteration persistent launch over the score terms prices every
candidate, and the select keeps the cheapest.  With `rank_final` only the last stage is priced that way
and its solutions come back sorted best first (opt/population_solver.py:163-202, 385-404).
"""

from __future__ import annotations

import ctypes
from typing import Any, Dict, NamedTuple, Optional, Sequence, Union

import numpy as np

from ... import _native as N
from ...opt.lm_optimizer import LMOptimizer, LMOptimizerConfig
from ...opt.population_solver import build_stages, run_stages
from ...opt.sampler import RobertsSampler
from ...opt.var_values import VarKey, VarValues
from ...robo.robot_state import RobotState
from ...terms.dense import (ConfigurationTask, FrameTask, PositionLimit, SceneCollisionTask, SelfCollisionTask,
                            SmoothnessTask, VelocityLimitTask, _PoseTask)
from ...terms.task import Context
from .config import IKContext, IKSolverConfig


_IDENTITY7 = np.array([0, 0, 0, 1, 0, 0, 0], np.float32)


class IKMetrics(NamedTuple):
    """Weight-independent accuracy (helpers/ik/ik.py:85-90): errors per target and target link, success per
    target when every link is within both thresholds.  Device arrays from compute_metrics (success as int32
    0/1), numpy from compute_metrics_numpy."""

    position_error_m: Any  # (batch, num_targets) metres
    orientation_error_rad: Any  # (batch, num_targets) radians
    success: Any  # (batch,)


class IKResultTorch(NamedTuple):
    """solve_torch's result (helpers/ik/ik.py:93-95): joints (rows, dofs) and, with a floating base, the base
    as (rows, 4, 4) homogeneous matrices."""

    q: Any
    T_world_base: Any = None


def _on_target_links(t: Any) -> bool:
    return isinstance(t, _PoseTask) and t.frame_index_arg in (IKContext.TARGET_LINKS, None)


class IKSolver:
    def __init__(self, config: IKSolverConfig, robot: Any, target_links: Union[str, int, Sequence[Union[str, int]]],
                 device: Any = "cuda", scene: Any = None):
        self.scene = scene
        if device is not None and not str(device).startswith("cuda"):
            raise ValueError(f"device {device!r}: this library runs on CUDA only (no CPU fallback)")
        self.config = config
        self.robot = robot
        names = list(robot.spec.link_names)
        links = [target_links] if isinstance(target_links, (str, int, np.integer)) else list(target_links)
        self.target_links = []
        for x in links:  # helpers/ik/ik.py:120-130
            if isinstance(x, str):
                if x not in names:
                    raise ValueError(f"link '{x}' not in robot.link_names ({len(names)} links)")
                self.target_links.append(names.index(x))
            else:
                if not 0 <= int(x) < len(names):
                    raise ValueError(f"link index {x} out of range [0, {len(names)})")
                self.target_links.append(int(x))
        self.num_targets = len(self.target_links)
        self.target_link_indices = self.target_links  # the reference's attribute name
        for t in (*config.terms, *config.score_terms):  # a term on the target links may weigh each link
            w = getattr(t, "weight", None)
            if isinstance(w, (list, tuple)) and _on_target_links(t) and len(w) != self.num_targets:
                raise ValueError(f"weight sequence length {len(w)} != {self.num_targets} (term '{t.name}' targets "
                                 f"{self.num_targets} link(s))")
        self._term_by_name = {t.name: t for t in (*config.terms, *config.score_terms)}
        self._built: Dict[int, list] = {}
        self.widths = config.solver.num_candidates
        self.lm_configs = config.solver.optimizers
        self.floating = bool(config.enable_T_world_base)
        self._joint_mask = np.ones(robot.spec.num_actuated_joints, np.float32)
        self._base_mask = np.asarray(config.base_active_mask, np.float32).copy()
        self._batch = None

    # --- active degrees of freedom (helpers/ik/ik.py:200-216) --------------------------------
    def set_active_joint_mask(self, joint_mask: Sequence[float]) -> None:
        """Which actuated joints move (1.0) or stay locked (0.0); the next solve rebuilds the stages."""
        m = np.asarray(joint_mask, np.float32).reshape(-1)
        if m.shape != self._joint_mask.shape:
            raise ValueError(f"joint_mask length {m.size} != {self._joint_mask.size}")
        self._joint_mask[:] = m
        self._rebuild()

    def set_active_base_mask(self, base_mask: Sequence[float]) -> None:
        """Active (1.0) / locked (0.0) base DOFs [x, y, z, roll, pitch, yaw]; needs enable_T_world_base=True."""
        if not self.floating:
            raise ValueError("set_active_base_mask requires enable_T_world_base=True")
        if len(base_mask) != 6:
            raise ValueError(f"base_mask length {len(base_mask)} != 6")
        self._base_mask[:] = np.asarray(base_mask, np.float32)
        self._rebuild()

    def _rebuild(self) -> None:
        if self._batch is not None:
            self._pending_batch = self._batch
            self._batch = None

    def set_weight(self, name: str, value: Union[float, Sequence[float]]) -> None:
        """A term's weight by its config name: a scalar, or one weight per target link for a term on
        IKContext.TARGET_LINKS (helpers/ik/ik.py:180-198).  The built problems are lowered again at the
        next solve's capacity; a captured solve graph is recorded again."""
        if name not in self._term_by_name:
            raise KeyError(f"No term named '{name}'. Available: {list(self._term_by_name)}")
        term = self._term_by_name[name]
        if isinstance(value, (list, tuple, np.ndarray)):
            if not _on_target_links(term):
                raise TypeError(f"per-link weights need a term on IKContext.TARGET_LINKS; '{name}' is not one")
            if len(value) != self.num_targets:
                raise ValueError(f"weight sequence length {len(value)} != {self.num_targets} (term '{name}' targets "
                                 f"{self.num_targets} link(s))")
        if isinstance(term, FrameTask):
            term.position_weight = value
        else:
            term.weight = value
        built = self._built.get(id(term), [])
        for b in built:
            b.set_weight(value)
        if built and self._batch is not None:
            self._relower()

    def _relower(self) -> None:
        """Lower every problem whose terms changed again (same capacity) and drop the captured graph."""
        for st in self._stages:
            if st.opt is not None:
                st.opt.reset(VarValues({VarKey.ROBOT: st.state}))
            if st.ranker is not None:
                st.ranker[0].reset(VarValues({VarKey.ROBOT: st.ranker[1]}))
        if self._scorer is not None:
            self._scorer.reset(VarValues({VarKey.ROBOT: self._prev_save}))
        self._cost_groups = None
        self._graph = None

    def _dof_mask(self) -> Optional[np.ndarray]:
        m = np.concatenate([self._base_mask, self._joint_mask]) if self.floating else self._joint_mask.copy()
        return None if np.all(m == 1.0) else m

    def _state(self, rows: int, q: Optional[np.ndarray] = None) -> RobotState:
        na = self.num_joints
        q = np.zeros((rows, na), np.float32) if q is None else q
        return self.robot.state(q, np.tile(_IDENTITY7, (rows, 1)) if self.floating else None)

    # --- sizes -------------------------------------------------------------------------
    @property
    def num_solutions(self) -> int:
        return self.widths[-1]

    @property
    def num_joints(self) -> int:
        return self.robot.spec.num_actuated_joints

    # --- build ---------------------------------------------------------------------------
    def _concrete_terms(self, targets: N.DeviceArray, templates: Sequence[Any]) -> list:
        out: list = []
        for t in templates:
            n0 = len(out)
            self._concrete_term(t, targets, out)
            self._built.setdefault(id(t), []).extend(out[n0:])
        return out

    def _concrete_term(self, t: Any, targets: N.DeviceArray, out: list) -> None:
        if isinstance(t, _PoseTask):
            fi, tg = t.frame_index_arg, t.T_world_target_arg
            frames = self.target_links if fi in (IKContext.TARGET_LINKS, None) else (
                [self.target_links[0]] if fi is IKContext.TARGET_LINK else fi)
            if tg is not IKContext.TARGET and not isinstance(tg, Context):
                raise NotImplementedError("IKSolver pose templates take T_world_target=IKContext.TARGET")
            if isinstance(t, FrameTask):
                out.append(FrameTask(self.robot, frames, targets, position_weight=t.position_weight,
                                     orientation_weight=t.orientation_weight))
            else:
                out.append(type(t)(self.robot, frames, targets, weight=t.weight))
        elif isinstance(t, PositionLimit):
            out.append(PositionLimit(self.robot, weight=t.weight))
        elif isinstance(t, SelfCollisionTask):
            c = SelfCollisionTask(self.robot, t.weight, t.margin, max_active_pairs=t.max_active_pairs,
                                  filter_adjacent_links=t.filter_adjacent_links, pair_mode=t.pair_mode)
            out.append(c)
        elif isinstance(t, (SmoothnessTask, ConfigurationTask, VelocityLimitTask)) and t.robot is not None:
            out.append(t)  # built with a robot: passes as is
        elif isinstance(t, SmoothnessTask):
            s = SmoothnessTask(self.robot, weight=t.weight, name=t.name)
            if t.prev_var is IKContext.PREVIOUS_STATE:
                s.bind_previous(self._prev_q, self._prev_base)
            elif t.prev_var is not None:
                raise NotImplementedError("IKSolver smoothness templates take prev_var=IKContext.PREVIOUS_STATE")
            out.append(s)
        elif isinstance(t, VelocityLimitTask):
            v = VelocityLimitTask(self.robot, dt=t.dt, velocity_limits=t.velocity_limits, weight=t.weight,
                                  name=t.name)
            if t.prev_state_var is IKContext.PREVIOUS_STATE:
                v.bind_previous(self._prev_q)
            elif t.prev_state_var is not None:
                raise NotImplementedError("IKSolver velocity templates take prev_state_var=IKContext.PREVIOUS_STATE")
            out.append(v)
        elif isinstance(t, SceneCollisionTask) and t.robot is None:
            scene = self.scene if t.scene is IKContext.SCENE else t.scene
            if scene is None or isinstance(scene, Context) or scene.num_elements == 0:
                return  # no scene: the template adds nothing (helpers/ik/ik.py:642-651)
            si = t.scene_indices
            if isinstance(si, Context) and si is not IKContext.SCENE_INDICES:
                raise NotImplementedError(f"scene_indices={si} is not an IKSolver placeholder")
            c = SceneCollisionTask(self.robot, scene, geometry=t.geometry,
                                   use_link_bounding_sphere_filter=t.use_link_bounding_sphere_filter,
                                   weight=t.weight, margin=t.margin, sphere_indices=t.sphere_indices,
                                   residual_mode=t.residual_mode, residual_eps=t.residual_eps, penalty=t.penalty,
                                   movable_only=t.movable_only, name=t.name)
            c.set_scene_indices(self._scene_idx if si is IKContext.SCENE_INDICES or si is None else si)
            out.append(c)
        elif isinstance(t, SceneCollisionTask):
            out.append(t)  # built with a robot: passes as is
        elif isinstance(t, ConfigurationTask):
            rb = t._base_rest_arg if self.floating else None  # a fixed base drops the base rows
            if rb is IKContext.REST_BASE:
                rb = self._rest_base
            elif isinstance(rb, Context):
                raise NotImplementedError(f"T_world_base_rest={rb} is not an IKSolver placeholder")
            c = ConfigurationTask(self.robot, rest_q=None if t.rest_q_arg is IKContext.REST_Q else t.rest_q_arg,
                                  T_world_base_rest=rb, weight=t.weight, base_weight=t.base_weight,
                                  include_joints=t.include_joints, name=t.name, mask=t.mask)
            if rb is self._rest_base and rb is not None:
                c._base_rest = self._rest_base  # read in place
            if t.rest_q_arg is IKContext.REST_Q:
                c.bind_rest(self._rest_q)
            elif isinstance(t.rest_q_arg, Context):
                raise NotImplementedError("IKSolver configuration templates take rest_q=IKContext.REST_Q")
            out.append(c)
        else:
            raise NotImplementedError(f"{type(t).__name__} is outside the IK hot path")

    def _build(self, B: int) -> None:
        spec = self.robot.spec
        na = spec.num_actuated_joints
        self._targets = N.DeviceArray.zeros((B, self.num_targets, 7))
        self._prev_q = N.DeviceArray.zeros((B, na))  # IKContext.PREVIOUS_STATE: zeros until a prev_state
        ident = np.tile(_IDENTITY7, (B, 1))
        self._prev_base = N.DeviceArray.from_numpy(ident) if self.floating else None
        self._rest_base = N.DeviceArray.from_numpy(ident) if self.floating else None  # IKContext.REST_BASE
        self._rest_q = N.DeviceArray.from_numpy(np.tile(spec.zero_q.astype(np.float32), (B, 1)))  # IKContext.REST_Q
        self._scene_idx = N.DeviceArray.zeros(B, np.int32)  # IKContext.SCENE_INDICES
        self._built = {}
        self._terms = self._concrete_terms(self._targets, self.config.terms)
        self._score_terms = self._concrete_terms(self._targets, self.config.score_terms)
        self._pose_terms = [t for t in (*self._terms, *self._score_terms) if isinstance(t, _PoseTask)]
        for t in self._pose_terms:  # every stage's problem (and every score problem) reads the one target buffer
            t.bind_targets(self._targets)
        self._mask = self._dof_mask()
        # LM problem per stage, score problems where score terms rank (opt/population_solver.py:179-270)
        self._stages = build_stages(self.robot, self.floating, B, self.config.solver, self._terms, self._score_terms,
                                    self._mask)
        C0 = self.widths[0]
        lim = spec.float32_actuated_limits()
        self._range = (lim[:, 1] - lim[:, 0]).astype(np.float32)
        # one Roberts spread over the whole tangent (base twist first), helpers/ik/ik.py:512-526
        Dt = (6 if self.floating else 0) + na
        self._sampler = RobertsSampler(C0, np.ones(Dt, np.float32), self.config.sampler.seed,
                                       self.config.sampler.keep_first)
        self._mid = N.DeviceArray.from_numpy(np.tile(spec.midrange_q.astype(np.float32), (B * C0, 1)))
        self._base0 = N.DeviceArray.from_numpy(np.tile(_IDENTITY7, (B * C0, 1))) if self.floating else None
        # spread around the midrange (fixed, read by the captured graph; the base stays at identity) and
        # around an init_state
        self._noise_mid = N.DeviceArray.from_numpy(self._sampler.tangent(B, self._tangent_scale(1.0, None)))
        self._noise_scale = None
        self._noise = None
        self._stream = N.Stream()
        self._graph: Optional[N.Graph] = None
        self._scorer: Optional[LMOptimizer] = None  # prices a previous state (built on the first one)
        self._ranked = None
        if self.config.solver.rank_final and self.num_solutions > 1:  # final rows sorted best first
            self._ranked = self._state(B * self.num_solutions)
            self._ranked_cost = N.DeviceArray.zeros(B * self.num_solutions)
        self._cost_groups: Optional[dict] = None
        self._batch = B

    def _tangent_scale(self, q_range: Any, base_range: Optional[Sequence[float]]) -> np.ndarray:
        """Spread of the candidate noise: base translation (only around an init_state), joints x their mask."""
        s = np.asarray(q_range, np.float32) * self._range * self._joint_mask
        if not self.floating:
            return s.astype(np.float32)
        b = np.zeros(6, np.float32)
        if base_range is not None:
            b[:3] = np.asarray(base_range, np.float32) * self._base_mask[:3]
        return np.concatenate([b, s]).astype(np.float32)

    def _score_previous(self, prev_state: RobotState, stream: int) -> None:
        """Cost of prev_state under the solve's terms (the score terms where there are some), its smoothness
        rows zero (helpers/ik/ik.py:257-270)."""
        B, na = self._batch, self.num_joints
        if self._scorer is None:
            self._prev_save = self._state(B)
            self._prev_cost = N.DeviceArray.zeros(B)
            self._scorer = LMOptimizer(self._score_terms or self._terms,
                                       LMOptimizerConfig(max_iter=0, form="persistent"),
                                       active_dof_mask=self._mask)
            self._scorer.reset(VarValues({VarKey.ROBOT: self._prev_save}))
            self._score_params = self._scorer.config.native_params()
        N.check(N.lib().ik_memcpy_dtod(self._prev_save.q.ptr, prev_state.q.ptr, self._prev_q.nbytes, stream))
        if self.floating:
            src = self._prev_base  # the previous base if one was given, else what the placeholder holds
            N.check(N.lib().ik_memcpy_dtod(self._prev_save.T_world_base.ptr, src.ptr, src.nbytes, stream))
        sc = self._scorer
        sc._slice(B)
        if self._stages[-1].iters > 0 and self._stages[-1].ranker is None:
            # The solve ends on LM iterations and reports the optimizer's 0.5 |r|^2, which the reference compares
            # with prev_state's |r|^2 (helpers/ik/ik.py:257-289, opt/population_solver.py:427-428): price prev
            # the same way.  After a select stage or with score terms both sides share one scale.
            R = sc.total_residual_dim
            if getattr(self, "_prev_r", None) is None or self._prev_r.shape != (B, R):
                self._prev_r = N.DeviceArray.empty((B, R))
            N.check(N.lib().ik_residual_jacobian(sc.problem.handle, B, self._prev_save.q.ptr,
                                                 self._prev_save.T_world_base.ptr if self.floating else None,
                                                 self._prev_r.ptr, None, stream))
            N.check(N.lib().ik_row_sumsq(B, R, self._prev_r.ptr, R, self._prev_cost.ptr, 0, stream))
            return
        N.check(N.lib().ik_solve_persistent(sc.problem.handle, B, self._prev_save.q.ptr,
                                            self._prev_save.T_world_base.ptr if self.floating else None,
                                            ctypes.byref(self._score_params), self._prev_cost.ptr, sc.lm.ptr,
                                            sc.iterations.ptr, sc.status.ptr, stream))

    def warmup(self, batch_size: int) -> None:
        """Build the buffers and run one solve on identity targets."""
        T = np.tile(np.array([0, 0, 0, 1, 0, 0, 0], np.float32), (batch_size, self.num_targets, 1))
        self.solve(T)
        N.synchronize()

    # --- solve ---------------------------------------------------------------------------
    def _seed_around(self, init_state: RobotState, q_range: Union[float, Sequence[float]], stream: int,
                     base_range: Optional[Sequence[float]] = None) -> None:
        """Candidates spread around init_state's joints and base (helpers/ik/ik.py:486-540)."""
        B, C0 = self._batch, self.widths[0]
        na = self.num_joints
        state = self._stages[0].state
        if init_state.batch_size != B:
            raise ValueError(f"init_state batch size {init_state.batch_size} != {B}")
        rep = np.repeat(np.arange(B, dtype=np.int32), C0)
        center = N.DeviceArray.from_numpy(init_state.q.numpy()[rep])
        cbase = None
        if self.floating:
            b = init_state.T_world_base.numpy() if init_state.has_floating_base else np.tile(_IDENTITY7, (B, 1))
            cbase = N.DeviceArray.from_numpy(np.ascontiguousarray(b.reshape(B, 7)[rep], np.float32))
        if C0 == 1:
            N.check(N.lib().ik_memcpy_dtod(state.q.ptr, center.ptr, center.nbytes, stream))
            if cbase is not None:
                N.check(N.lib().ik_memcpy_dtod(state.T_world_base.ptr, cbase.ptr, cbase.nbytes, stream))
        else:
            br = self.config.base_init_sample_range if base_range is None else base_range
            scale = self._tangent_scale(q_range, br)
            if self._noise_scale is None or not np.array_equal(scale, self._noise_scale):
                self._noise = N.DeviceArray.from_numpy(self._sampler.tangent(B, scale))
                self._noise_scale = scale
            N.check(N.lib().ik_integrate(B * C0, na, int(self.floating), center.ptr, N.ptr(cbase), self._noise.ptr,
                                         None, state.q.ptr, N.ptr(state.T_world_base) if self.floating else None,
                                         stream))
        N.check(N.lib().ik_clamp_q(B * C0, na, state.q.ptr, self.robot.limits_device().ptr, None, stream))
        N.check(N.lib().ik_stream_synchronize(stream))  # `center` is freed on return

    def _device_body(self, stream: int) -> None:
        """Seed from the midrange, run every stage, select between stages: device work only, on `stream`."""
        B, C0, na = self._batch, self.widths[0], self.num_joints
        q0 = self._stages[0].state
        N.check(N.lib().ik_integrate(B * C0, na, int(self.floating), self._mid.ptr, N.ptr(self._base0),
                                     self._noise_mid.ptr, None, q0.q.ptr,
                                     q0.T_world_base.ptr if self.floating else None, stream))
        N.check(N.lib().ik_clamp_q(B * C0, na, q0.q.ptr, self.robot.limits_device().ptr, None, stream))
        self._run_stages(stream)

    def _run_stages(self, stream: int) -> None:
        run_stages(self._stages, self._batch, self.floating, stream, self._ranked,
                   self._ranked_cost if self._ranked is not None else None)

    def solve(self, T_world_target: Any, prev_state: Optional[RobotState] = None,
              init_state: Optional[RobotState] = None, rest_state: Optional[RobotState] = None,
              out_state: Optional[RobotState] = None, init_sample_range: Optional[float] = None,
              base_init_sample_range: Optional[Sequence[float]] = None, scene_indices: Any = None) -> RobotState:
        """Solutions for every target, instance-major: (batch * num_solutions, dofs) (helpers/ik/ik.py:223-304).

        prev_state (batch,) fills IKContext.PREVIOUS_STATE and is kept for a target where it costs no more
        than the solve's result; rest_state fills IKContext.REST_Q.  Under cuda_graph_mode "full" the device
        work of a solve from the midrange seed is captured into one CUDA graph at the first solve and replayed
        after it; the call returns once the solutions are ready."""
        T, host = self._validate_target(T_world_target)
        B = T.shape[0]
        self._ensure_built(B)
        if prev_state is not None and self.num_solutions != 1:
            raise ValueError("prev_state requires an IK final stage with num_candidates=1.")
        st = self._stream.handle
        self._fill_inputs(T, host, prev_state, rest_state, scene_indices, st)
        if prev_state is not None:
            self._score_previous(prev_state, st)
        if init_state is not None:
            self._seed_around(init_state, self.config.sampler.scale if init_sample_range is None else init_sample_range,
                              st, base_init_sample_range)
            self._run_stages(st)
        elif self.config.solver.cuda_graph_mode == "full":
            if self._graph is None:
                self._device_body(st)  # the first solve runs directly (kernel set-up happens here)
                self._graph = N.Graph(self._stream).capture(lambda: self._device_body(st))
            else:
                self._graph.launch()
        else:
            self._device_body(st)
        final = self._stages[-1].state
        if prev_state is not None:
            fb = self.floating
            N.check(N.lib().ik_keep_previous(B, self.num_joints, self._prev_cost.ptr, self._stages[-1].cost.ptr,
                                             self._prev_save.q.ptr, self._prev_save.T_world_base.ptr if fb else None,
                                             final.q.ptr, final.T_world_base.ptr if fb else None, st))
        N.check(N.lib().ik_stream_synchronize(st))
        if out_state is not None:
            out_state.q.assign(final.q)
            if self.floating and out_state.has_floating_base:
                out_state.T_world_base.assign(final.T_world_base)
            out_state.invalidate()
            return out_state
        return final if self._ranked is None else self._ranked

    def _ensure_built(self, B: int) -> None:
        if self._batch is None and getattr(self, "_pending_batch", None) not in (None, B):
            raise ValueError(f"Batch size mismatch: expected {self._pending_batch}, got {B}")
        if self._batch is None:
            self._build(B)
        elif B != self._batch:
            raise ValueError(f"Batch size mismatch: expected {self._batch}, got {B}")

    def _validate_target(self, T_world_target: Any):
        """Targets as (batch, num_targets, 7) float32 poses [x, y, z, qw, qx, qy, qz] (helpers/ik/ik.py:473-485).

        A device array (DeviceArray, or any __cuda_array_interface__ object) must be float32; a host numpy
        array is converted to float32 and copied to the device by the solve.  (batch, 7) stands for one target
        per row.  Returns (targets, is_host)."""
        if isinstance(T_world_target, N.DeviceArray) or hasattr(T_world_target, "__cuda_array_interface__"):
            T = T_world_target if isinstance(T_world_target, N.DeviceArray) else N.DeviceArray.from_cuda_array(
                T_world_target)
            host = False
            if T.dtype != np.float32 or T.shape[-1:] != (7,):
                raise TypeError(f"T_world_target must hold float32 poses [..., 7] (x, y, z, qw, qx, qy, qz), got "
                                f"{T.dtype.name} {tuple(T.shape)}")
        elif hasattr(T_world_target, "device") and hasattr(T_world_target, "is_cuda"):
            raise ValueError(f"T_world_target must be on cuda (or a numpy array), got {T_world_target.device}")
        else:
            T = np.ascontiguousarray(T_world_target, np.float32)
            host = True
            if T.shape[-1:] != (7,):
                raise TypeError(f"T_world_target must hold poses [..., 7] (x, y, z, qw, qx, qy, qz), got {T.shape}")
        if T.ndim == 2:
            T = T.reshape((T.shape[0], 1, 7))
        if T.ndim != 3:
            raise ValueError(f"T_world_target must have logical shape [batch, targets] of 7-float poses, got "
                             f"{tuple(T.shape)}")
        if T.shape[1] != self.num_targets:
            raise ValueError(f"Target count ({T.shape[1]}) must match IK target count ({self.num_targets})")
        return T, host

    def _fill_inputs(self, T: Any, host: bool, prev_state: Optional[RobotState], rest_state: Optional[RobotState],
                     scene_indices: Any, st: int) -> None:
        """Refill the buffers the built terms read: targets, previous and rest states, scene indices
        (helpers/ik/ik.py:651-680)."""
        B = self._batch
        if prev_state is not None and prev_state.batch_size != B:
            raise ValueError(f"prev_state batch size mismatch: expected {B}, got {prev_state.batch_size}")
        if rest_state is not None and rest_state.batch_size != B:
            raise ValueError(f"rest_state batch size mismatch: expected {B}, got {rest_state.batch_size}")
        si = None
        if scene_indices is not None:
            try:
                si = N.as_device(scene_indices, np.int32)
            except TypeError:
                raise TypeError("scene_indices must be a 1D int32 array.") from None
            if si.ndim != 1:
                raise TypeError("scene_indices must be a 1D int32 array.")
            if si.shape != (B,):
                raise ValueError("scene_indices must have shape (batch_size,).")
        nbytes = self._targets.nbytes
        if host:
            N.check(N.lib().ik_memcpy_htod(self._targets.ptr, T.ctypes.data, nbytes, st))
        else:
            N.check(N.lib().ik_memcpy_dtod(self._targets.ptr, T.ptr, nbytes, st))
        if prev_state is not None:
            N.check(N.lib().ik_memcpy_dtod(self._prev_q.ptr, prev_state.q.ptr, self._prev_q.nbytes, st))
            if self.floating and prev_state.has_floating_base:
                N.check(N.lib().ik_memcpy_dtod(self._prev_base.ptr, prev_state.T_world_base.ptr,
                                               self._prev_base.nbytes, st))
        if rest_state is not None:
            N.check(N.lib().ik_memcpy_dtod(self._rest_q.ptr, rest_state.q.ptr, self._rest_q.nbytes, st))
            if self.floating and rest_state.has_floating_base:
                N.check(N.lib().ik_memcpy_dtod(self._rest_base.ptr, rest_state.T_world_base.ptr,
                                               self._rest_base.nbytes, st))
        if si is not None:
            N.check(N.lib().ik_memcpy_dtod(self._scene_idx.ptr, si.ptr, self._scene_idx.nbytes, st))

    @property
    def costs(self) -> N.DeviceArray:
        """Cost of each returned solution: 0.5 |r|^2 of the final stage's optimization terms, or of the score
        terms where they rank the final stage."""
        return self._stages[-1].cost if self._ranked is None else self._ranked_cost

    def compute_costs(self, state: RobotState, T_world_target: Any, prev_state: Optional[RobotState] = None,
                      scene_indices: Any = None) -> Dict[str, N.DeviceArray]:
        """|r|^2 of every optimization term at `state` against these targets, summed by cost_name, one value
        per row (helpers/ik/ik.py:373-385, opt/population_solver.py:555-574).  The solver's target,
        previous-state and scene-index buffers take the given values, as a solve would."""
        T, host = self._validate_target(T_world_target)
        B = T.shape[0]
        if B != state.batch_size:
            raise ValueError(f"Target batch size ({B}) must match state batch size ({state.batch_size})")
        self._ensure_built(B)
        st = self._stream.handle
        self._fill_inputs(T, host, prev_state, None, scene_indices, st)
        N.check(N.lib().ik_stream_synchronize(st))
        if self._cost_groups is None:
            groups: Dict[str, list] = {}
            for t in self._terms:
                groups.setdefault(t.cost_name, []).append(t)
            self._cost_groups = groups
        vv = VarValues({VarKey.ROBOT: state})
        out: Dict[str, N.DeviceArray] = {}
        for name, terms in self._cost_groups.items():
            c = N.DeviceArray.zeros(B)
            for i, t in enumerate(terms):
                if t.residual_dim == 0:
                    continue
                r = t.compute_weighted_residual(vv)
                N.check(N.lib().ik_row_sumsq(B, r.shape[1], r.ptr, r.shape[1], c.ptr, int(i > 0), None))
            out[name] = c
        N.check(N.lib().ik_device_synchronize())
        return out

    # --- metrics ---------------------------------------------------------------------------
    def compute_metrics(self, state: RobotState, T_world_target: Any, position_threshold_m: float = 0.005,
                        orientation_threshold_rad: float = 0.05, out: Optional[IKMetrics] = None) -> IKMetrics:
        """Pose errors of every target link and success within both thresholds, on the device
        (helpers/ik/ik.py:60-82, 387-437).  `out` (from an earlier call) is written in place and returned."""
        T, host = self._validate_target(T_world_target)
        if host:
            T = N.DeviceArray.from_numpy(T)
        B, nt = T.shape[0], self.num_targets
        if state.batch_size != B:
            raise ValueError(f"Target batch size ({B}) must match state batch size ({state.batch_size})")
        if getattr(self, "_links_dev", None) is None:
            self._links_dev = N.DeviceArray.from_numpy(np.asarray(self.target_links, np.int32))
        if out is None:
            out = IKMetrics(N.DeviceArray.empty((B, nt)), N.DeviceArray.empty((B, nt)), N.DeviceArray.empty(B, np.int32))
        elif tuple(out.position_error_m.shape) != (B, nt) or tuple(out.success.shape) != (B,):
            raise ValueError(f"out holds metrics of shape {tuple(out.position_error_m.shape)}, expected {(B, nt)}")
        N.check(N.lib().ik_metrics(self.robot.handle, B, state.q.ptr, N.ptr(state.T_world_base) if
                                   state.has_floating_base else None, nt, self._links_dev.ptr, T.ptr,
                                   float(position_threshold_m), float(orientation_threshold_rad),
                                   out.position_error_m.ptr, out.orientation_error_rad.ptr, out.success.ptr, None))
        N.check(N.lib().ik_device_synchronize())
        return out

    def compute_metrics_numpy(self, state: RobotState, T_world_target: Any, position_threshold_m: float = 0.005,
                              orientation_threshold_rad: float = 0.05) -> IKMetrics:
        """compute_metrics for host targets shaped (7,), (batch, 7) or (batch, num_targets, 7); numpy results,
        success as bool (helpers/ik/ik.py:439-471)."""
        T = T_world_target.numpy() if isinstance(T_world_target, N.DeviceArray) else T_world_target
        T = np.asarray(T, np.float32)
        if not 1 <= T.ndim <= 3 or T.shape[-1] != 7:
            raise ValueError(f"T_world_target must have shape (..., 7), got {T.shape}")
        m = self.compute_metrics(state, T.reshape(-1, self.num_targets, 7), position_threshold_m,
                                 orientation_threshold_rad)
        return IKMetrics(m.position_error_m.numpy(), m.orientation_error_rad.numpy(), m.success.numpy().astype(bool))

    # --- adapters (helpers/ik/ik.py:306-371) ------------------------------------------------------
    def solve_numpy(self, T_world_target: Any, prev_state: Optional[RobotState] = None,
                    init_state: Optional[RobotState] = None, rest_state: Optional[RobotState] = None,
                    out_state: Optional[RobotState] = None, init_sample_range: Optional[float] = None,
                    base_init_sample_range: Optional[Sequence[float]] = None) -> RobotState:
        """solve() for host poses shaped (7,), (batch, 7) or (batch, num_targets, 7)."""
        T = np.asarray(T_world_target, np.float32)
        if not 1 <= T.ndim <= 3 or T.shape[-1] != 7:
            raise ValueError(f"T_world_target must have shape (..., 7), got {T.shape}")
        return self.solve(T.reshape(-1, self.num_targets, 7), prev_state=prev_state, init_state=init_state,
                          rest_state=rest_state, out_state=out_state, init_sample_range=init_sample_range,
                          base_init_sample_range=base_init_sample_range)

    def _poses_from_matrices(self, mats: Any) -> N.DeviceArray:
        m = N.as_device(mats, np.float32)
        n = m.size // 16
        out = N.DeviceArray.empty(tuple(m.shape[:-2]) + (7,))
        N.check(N.lib().ik_pose_from_matrix(n, m.ptr, out.ptr, None))
        return out

    def solve_torch(self, T_world_target: Any, prev_state: Optional[RobotState] = None, init_q: Any = None,
                    init_T_world_base: Any = None, rest_q: Any = None, rest_T_world_base: Any = None,
                    init_sample_range: Optional[float] = None,
                    base_init_sample_range: Optional[Sequence[float]] = None) -> IKResultTorch:
        """solve() for CUDA torch tensors: targets and bases as (..., 4, 4) homogeneous matrices; returns torch
        copies of the joints and, with a floating base, the base matrices."""
        import torch

        if not 2 <= T_world_target.ndim <= 4 or tuple(T_world_target.shape[-2:]) != (4, 4):
            raise ValueError(f"T_world_target must have shape (..., 4, 4), got {tuple(T_world_target.shape)}")
        if not T_world_target.is_cuda:
            raise ValueError(f"T_world_target must be on cuda, got {T_world_target.device}")
        mats = T_world_target.reshape(-1, self.num_targets, 4, 4).to(torch.float32).contiguous()
        held = [mats]  # tensors whose memory the device arrays below wrap

        def to_state(q: Any, T_base: Any) -> Optional[RobotState]:
            if q is None:
                return None
            qt = q.to(device=mats.device, dtype=torch.float32).contiguous()
            held.append(qt)
            base = None
            if T_base is not None and self.floating:
                bt = T_base.to(device=mats.device, dtype=torch.float32).reshape(-1, 4, 4).contiguous()
                held.append(bt)
                base = self._poses_from_matrices(bt)
            return self.robot.state(qt, base)

        torch.cuda.current_stream().synchronize()  # the tensors are written before the library reads them
        poses = self._poses_from_matrices(mats)
        init_state, rest_state = to_state(init_q, init_T_world_base), to_state(rest_q, rest_T_world_base)
        N.check(N.lib().ik_device_synchronize())
        state = self.solve(poses, prev_state=prev_state, init_state=init_state, rest_state=rest_state,
                           init_sample_range=init_sample_range, base_init_sample_range=base_init_sample_range)
        q = torch.as_tensor(state.q, device=mats.device).clone()
        T_base = None
        if self.floating:
            rows = state.q.shape[0]
            m = N.DeviceArray.empty((rows, 4, 4))
            N.check(N.lib().ik_matrix_from_pose(rows, state.T_world_base.ptr, m.ptr, None))
            N.check(N.lib().ik_device_synchronize())
            T_base = torch.as_tensor(m, device=mats.device).clone()
        torch.cuda.current_stream().synchronize()
        return IKResultTorch(q=q, T_world_base=T_base)
