"""Host logic of the population solver, the IK helper and the serving stream (no GPU)."""

import ctypes

import numpy as np
import pytest

from robokit_b200 import _native as N
from robokit_b200.helpers.ik import IKContext, IKSolverConfig, presets
from robokit_b200.opt import LMOptimizerConfig
from robokit_b200.opt.population_solver import PopulationSolverConfig, Stage
from robokit_b200.opt.sampler import RobertsSampler, roberts_samples
from robokit_b200.terms.task import Context


def test_roberts_sequence():
    """R_d: alpha_i = 1 - phi_d^-(i+1) with phi_d the root of x^(d+1) = x + 1 (d = 1: the golden ratio)."""
    s = roberts_samples(6, 1)
    phi = (1 + 5 ** 0.5) / 2
    np.testing.assert_allclose(s[:, 0], np.modf(np.arange(6) * (1 - 1 / phi))[0], atol=1e-12)
    s3 = roberts_samples(64, 3)
    assert s3.shape == (64, 3) and s3.min() >= 0 and s3.max() < 1
    phi3 = 1.0
    for _ in range(60):
        phi3 -= (phi3 ** 4 - phi3 - 1) / (4 * phi3 ** 3 - 1)
    np.testing.assert_allclose(s3[1], 1 - phi3 ** -np.arange(1.0, 4.0), atol=1e-9)
    # low discrepancy: every tenth of [0, 1) gets 4 to 8 of 64 points per axis (i.i.d. uniform draws spread wider)
    counts = np.stack([np.histogram(s3[:, k], bins=10, range=(0, 1))[0] for k in range(3)])
    assert counts.min() >= 4 and counts.max() <= 8


def test_roberts_sampler_keep_first_and_tiling():
    s = RobertsSampler(4, [1.0, 1.0], keep_first=True)
    assert np.all(s.offsets[0] == 0) and np.all(s.offsets[1] == -0.5)
    t = s.tangent(3, np.array([2.0, 1.0], np.float32))
    assert t.shape == (12, 2)
    np.testing.assert_array_equal(t[4:8], t[0:4])
    np.testing.assert_allclose(t[:4], s.offsets * [2.0, 1.0])
    assert np.abs(t).max() <= 1.0


def test_stage_resolution():
    cfg = PopulationSolverConfig(stages=[Stage(6, 64, LMOptimizerConfig(lm_lambda=10.0)), Stage(10, 4), Stage(0, 1)])
    assert cfg.num_candidates == [64, 4, 1]
    assert [o.lm_lambda for o in cfg.optimizers] == [10.0, 10.0, 10.0]
    assert presets.basic.solver.num_candidates == [64, 4, 1]
    assert [o.lm_lambda for o in presets.basic.solver.optimizers] == [10.0, 1.0, 1.0]
    assert presets.single_candidate.solver.num_candidates == [1]


def test_ik_config_templates_and_validation():
    assert isinstance(IKContext.TARGET, Context) and isinstance(IKContext.TARGET_LINKS, Context)
    t = presets.basic.terms[0]
    assert t.frame_index_arg is IKContext.TARGET_LINKS and t.weight == 20.0
    with pytest.raises(ValueError, match="base_active_mask"):
        IKSolverConfig(base_active_mask=(1, 1, 1, 0, 1, 1))
    with pytest.raises(ValueError, match="length"):
        IKSolverConfig(base_active_mask=(1, 1))


def test_mixed_stream_shape():
    from robokit_b200 import serve

    class _Cfg:  # a stand-in pool: only the size is read
        batch = 4096

    types = [serve.StreamType(str(k), _Cfg(), None) for k in range(4)]
    reqs = serve.make_stream(types, rate=100000.0, duration=2.0, seed=3)
    assert reqs == serve.make_stream(types, rate=100000.0, duration=2.0, seed=3)  # seeded
    t = np.array([r.t_arrive for r in reqs])
    b = np.array([r.batch for r in reqs])
    assert np.all(np.diff(t) > 0) and t[-1] < 2.0
    assert b.min() >= 1 and b.max() <= 4096
    assert all(0 <= r.start and r.start + r.batch <= 4096 for r in reqs)
    # the problem rate is the requested one within sampling noise
    assert 0.7 < b.sum() / 2.0 / 100000.0 < 1.4
    assert {r.type_id for r in reqs} == {0, 1, 2, 3}


def test_select_and_graph_argument_checks_need_no_device():
    lib = N.load_library()
    assert lib.ik_select_best(4, 8, 9, None, None, None, 3, None, None, None, None, None) == N.IK_E_INVALID
    assert lib.ik_select_best(4, 8, 2, None, None, None, 3, None, None, None, None, None) == N.IK_E_INVALID
    assert lib.ik_graph_begin(None) == N.IK_E_INVALID
    assert lib.ik_graph_launch(None, None) == N.IK_E_INVALID
    assert lib.ik_graph_destroy(None) == N.IK_OK
    assert lib.ik_server_poll(None, None, 0, None) == N.IK_E_INVALID


def test_joint_reference_terms_host_side(panda_spec):
    """SmoothnessTask / ConfigurationTask lower to joint-reference rows; unsupported reference options raise."""
    from robokit_b200.terms.dense import ConfigurationTask, SmoothnessTask

    class _Robot:
        spec = panda_spec

    class _V:
        spec, batch_size, has_floating_base = panda_spec, 4, False

    na = panda_spec.num_actuated_joints
    c = ConfigurationTask(_Robot(), rest_q="midrange", weight=0.5, mask=np.arange(na) % 2)
    d = c.host_desc(_V)
    assert d["kind"] == N.IK_TERM_JOINT_REF and d["target_rows"] == 1 and c.residual_dim == na
    np.testing.assert_array_equal(d["targets"][0], panda_spec.midrange_q)
    np.testing.assert_array_equal(d["weights"], 0.5 * (np.arange(na) % 2))
    z = ConfigurationTask(_Robot(), weight=[1.0] * na).host_desc(_V)
    assert not np.any(z["targets"])
    s = SmoothnessTask(_Robot(), weight=0.1)
    assert not np.any(s.host_desc(_V)["weights"])  # no previous state: zero rows
    tmpl = SmoothnessTask(prev_var=IKContext.PREVIOUS_STATE, weight=0.1)
    assert tmpl.active and tmpl.robot is None
    with pytest.raises(NotImplementedError):
        SmoothnessTask(_Robot(), warmup_frames=5, frame=IKContext.TARGET)
    # base blocks: six more rows on a floating base, refused on a fixed one
    class _VF:
        spec, batch_size, has_floating_base = panda_spec, 4, True

    sb = SmoothnessTask(_Robot(), base_weight=2.0, weight=0.5)
    assert sb.residual_dim == na + 6
    with pytest.raises(ValueError, match="no floating base"):
        sb.host_desc(_V)
    jd, bd = sb.host_desc(_VF)
    assert bd["kind"] == N.IK_TERM_BASE_REF and not np.any(bd["weights"])  # no previous state yet
    cb = ConfigurationTask(_Robot(), T_world_base_rest=[[0.1, 0, 0, 1, 0, 0, 0]], base_weight=3.0)
    assert cb.residual_dim == na + 6
    jd, bd = cb.host_desc(_VF)
    assert jd["kind"] == N.IK_TERM_JOINT_REF and np.all(bd["weights"] == 3.0) and bd["targets"].shape == (1, 7)
    only = ConfigurationTask(_Robot(), T_world_base_rest=np.eye(4), include_joints=False)
    (bd,) = only.host_desc(_VF)
    assert only.residual_dim == 6 and np.all(bd["weights"] == 1.0)
    np.testing.assert_allclose(bd["targets"], [[0, 0, 0, 1, 0, 0, 0]], atol=1e-7)
    with pytest.raises(ValueError):
        cb.host_desc(_V)
    with pytest.raises(ValueError):
        ConfigurationTask(_Robot(), rest_q="zero")
    assert [type(t).__name__ for t in presets.smooth.terms] == ["PositionTask", "RotationTask", "PositionLimit",
                                                                "SmoothnessTask"]
    assert type(presets.single_candidate.terms[-1]).__name__ == "SmoothnessTask"


def test_velocity_limit_term_host_side(panda_spec):
    from robokit_b200.terms.dense import VelocityLimitTask

    class _Robot:
        spec = panda_spec

    class _V:
        spec, batch_size, has_floating_base = panda_spec, 4, False

    na = panda_spec.num_actuated_joints
    v = VelocityLimitTask(_Robot(), dt=0.02)
    d = v.host_desc(_V)
    assert d["kind"] == N.IK_TERM_VELOCITY_LIMIT and d["dt"] == 0.02 and v.residual_dim == na
    np.testing.assert_allclose(d["velocity_limits"], panda_spec.actuated_joint_velocity_limits)
    assert not np.any(d["weights"])  # no previous state: zero rows
    with pytest.raises(ValueError):
        VelocityLimitTask(_Robot(), dt=0.0)
    with pytest.raises(ValueError):
        VelocityLimitTask(_Robot(), velocity_limits=[1.0, 2.0]).host_desc(_V)
    # the URDF reader's velocity limits: the file's value, 0 for fixed joints without one, else 10
    from robokit_b200.robo.robot_spec import JointRecord, RobotSpec

    recs = [JointRecord("a", "revolute", "l0", "l1", velocity=3.0), JointRecord("b", "continuous", "l1", "l2"),
            JointRecord("c", "fixed", "l2", "l3")]
    s = RobotSpec.from_records("r", ["l0", "l1", "l2", "l3"], recs)
    np.testing.assert_array_equal(s.joint_velocity_limits, [3.0, 10.0, 0.0])
    np.testing.assert_array_equal(s.actuated_joint_velocity_limits, [3.0, 10.0])


def test_scene_geometry_and_term_host_side(panda_collision_spec):
    """Primitive records in query order, CSR validation, and the scene term's lowering and argument checks."""
    from robokit_b200.geom import BoxGeom, CapsuleGeom, PlaneGeom, Scene, SphereGeom
    from robokit_b200.terms.dense import SceneCollisionTask

    s = Scene(num_scenes=2)
    box = BoxGeom([[0.1, 0.2, 0.3], [1, 1, 1]], [0, 1, 2], poses=np.eye(4)[None].repeat(2, 0))
    s.add(box).add(SphereGeom([0.5], [0, 0, 1])).add(PlaneGeom([0, 1, 1])).add(CapsuleGeom([0.1], [0.4], [0, 1, 1]))
    rec = s.records()
    assert rec.shape == (5, N.IK_GEOM_FLOATS)
    np.testing.assert_array_equal(rec[:, 0], [N.IK_GEOM_BOX, N.IK_GEOM_BOX, N.IK_GEOM_SPHERE, N.IK_GEOM_PLANE,
                                              N.IK_GEOM_CAPSULE])
    np.testing.assert_array_equal(rec[:, 1], [0, 1, 1, 0, 0])
    np.testing.assert_allclose(rec[0, 4:8], [0.1, 0.2, 0.3, 0])
    np.testing.assert_allclose(rec[0, 8:15], [0, 0, 0, 1, 0, 0, 0])
    np.testing.assert_allclose(rec[4, 4:6], [0.1, 0.4])
    rev = s.revision
    box.update(poses=[[0, 0, 1, 1, 0, 0, 0], [0, 0, 2, 1, 0, 0, 0]])
    assert s.revision > rev and s.records()[1, 10] == 2.0
    with pytest.raises(ValueError):
        BoxGeom([[1, 1, 1]], [0, 2])
    with pytest.raises(ValueError):
        s.add(SphereGeom([1.0], [0, 1]))  # one scene in a two-scene scene
    with pytest.raises(ValueError):
        Scene(1, device="cpu")

    class _Robot:
        spec = panda_collision_spec

    class _V:
        spec, batch_size, has_floating_base = panda_collision_spec, 8, False

    ns = len(panda_collision_spec.collision_sphere_radii)
    t = SceneCollisionTask(_Robot(), s, weight=2.0, margin=0.05, penalty="plain", residual_mode="sqrt_abs")
    d = t.host_desc(_V)
    assert d["kind"] == N.IK_TERM_SCENE_COLLISION and t.residual_dim == ns and d["num_scenes"] == 2
    assert d["penalty"] == N.IK_PENALTY_PLAIN and d["residual_sqrt"] and np.all(d["weights"] == 2.0)
    mov = SceneCollisionTask(_Robot(), s, movable_only=True)
    assert mov.residual_dim == int(np.sum(panda_collision_spec.collision_spheres_link_indices > 0))
    v0 = t._version
    s.add(PlaneGeom([0, 1, 1]))
    assert t._version != v0  # a changed scene rebuilds the terms that read it
    with pytest.raises(ValueError, match="Unsupported penalty"):
        SceneCollisionTask(_Robot(), s, penalty="hard")
    with pytest.raises(ValueError, match="out-of-range"):
        SceneCollisionTask(_Robot(), s, sphere_indices=[ns])
    with pytest.raises(ValueError, match="weight shape"):
        SceneCollisionTask(_Robot(), s, weight=[1.0, 2.0])
    assert not SceneCollisionTask(_Robot(), Scene(1)).active


class TestRobertsSamplerReference:
    """tests/opt/test_sampler.py:17-70 (TestRobertsSampler), on the host spread that fill() uploads."""

    @staticmethod
    def _fill(num_candidates=4, batch=2, scale=(0.5, 0.5), **kw):
        return RobertsSampler(num_candidates=num_candidates, scale=scale, **kw).tangent(batch)

    def test_shape_and_bounds(self):
        noise = self._fill()
        assert noise.shape == (8, 2) and np.abs(noise).max() <= 0.25

    def test_scale_is_per_column(self):
        noise = self._fill(scale=(1.0, 0.0))
        assert np.abs(noise[:, 1]).max() == 0.0 and np.abs(noise[:, 0]).max() > 0.0

    def test_every_instance_gets_the_same_seed_offsets(self):
        noise = self._fill(num_candidates=4, batch=3)
        np.testing.assert_array_equal(noise[0:4], noise[4:8])
        np.testing.assert_array_equal(noise[0:4], noise[8:12])

    def test_keep_first_leaves_candidate_zero_untouched(self):
        noise = self._fill(keep_first=True)
        np.testing.assert_array_equal(noise[0], np.zeros(2))
        assert np.abs(noise[1:4]).max() > 0.0

    def test_seed_shifts_the_sequence(self):
        assert not np.array_equal(self._fill(seed=0), self._fill(seed=7))

    def test_covers_more_evenly_than_random(self):
        cells = lambda pts: len({(int(x * 8), int(y * 8)) for x, y in pts})  # noqa: E731
        assert cells(roberts_samples(64, 2)) > cells(np.random.default_rng(0).random((64, 2)))

    def test_scale_assign_and_config_build(self):
        s = RobertsSampler(4, (1.0, 1.0))
        s.scale.assign(np.array([0.0, 2.0], np.float32))
        assert np.abs(s.tangent(1)[:, 0]).max() == 0.0
        with pytest.raises(ValueError):
            s.scale.assign([1.0])
