"""SceneCollisionTask over primitive geometry on the GPU against the FP64 oracle."""

import numpy as np
import pytest

import oracle
from robokit_b200 import _native as N
from robokit_b200.geom import BoxGeom, CapsuleGeom, PlaneGeom, Scene, SphereGeom
from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues
from robokit_b200.terms.dense import PositionLimit, PositionTask, RotationTask, SceneCollisionTask

pytestmark = pytest.mark.gpu

ROT = np.array([0.9, 0.2, -0.3, 0.25]) / np.linalg.norm([0.9, 0.2, -0.3, 0.25])


def _view(spec, B, floating):
    class _V:
        pass

    v = _V()
    v.spec, v.batch_size, v.has_floating_base = spec, B, floating
    return v


def _scene():
    """Scene 0: one primitive of each shape against the arm; scene 1: a tilted plane only."""
    s = Scene(num_scenes=2)
    s.add(BoxGeom([[0.12, 0.08, 0.08]], [0, 1, 1], poses=[[0.4, 0.15, 0.55, *ROT]], scales=[1.3]))
    s.add(SphereGeom([0.1], [0, 1, 1], poses=[[0.35, -0.15, 0.6, 1, 0, 0, 0]]))
    s.add(CapsuleGeom([0.05], [0.12], [0, 1, 1], poses=[[0.45, 0.15, 0.3, *ROT]]))
    s.add(PlaneGeom([0, 1, 2], poses=[[0, 0, 0.1, 1, 0, 0, 0], [0, 0, 0.6, 0.99, 0.05, -0.05, 0.0]]))
    return s


@pytest.mark.parametrize("penalty", ["smooth", "plain", "surface_distance"])
@pytest.mark.parametrize("floating", [False, True])
def test_scene_rows_match_the_oracle(gpu, panda_collision_spec, penalty, floating):
    from robokit_b200.robo.robot import Robot

    spec = panda_collision_spec
    robot = Robot(spec)
    rng = np.random.default_rng(7)
    B = 64
    na = spec.num_actuated_joints
    q = (spec.midrange_q + rng.normal(0, 0.3, (B, na))).astype(np.float32)
    base = None
    if floating:
        base = rng.normal(size=(B, 7)).astype(np.float32)
        base[:, :3] *= 0.05
        base[:, 3] = 8.0
        base[:, 3:] /= np.linalg.norm(base[:, 3:], axis=1, keepdims=True)
    scene = _scene()
    sidx = N.DeviceArray.from_numpy(np.array([0, 1, 0, 1], np.int32))  # 16 problems per row
    ns = len(spec.collision_sphere_radii)
    w = np.linspace(0.5, 2.0, ns).astype(np.float32)
    terms = [SceneCollisionTask(robot, scene, scene_indices=sidx, weight=w, margin=0.15, penalty=penalty),
             SceneCollisionTask(robot, scene, sphere_indices=np.arange(0, ns, 3), margin=0.1,
                                residual_mode="sqrt_abs", residual_eps=1e-4)]
    st = robot.state(q, base)
    vv = VarValues({VarKey.ROBOT: st})
    D = st.tangent_dim
    R = sum(t.residual_dim for t in terms)
    r = N.DeviceArray.zeros((B, R))
    J = N.DeviceArray.zeros((B, R, D))
    off = 0
    for t in terms:
        t.compute_weighted_residual(vv, out_residual=r, row_offset=off)
        t.compute_weighted_jacobian(vv, out_jacobian=J, row_offset=off)
        off += t.residual_dim
    ro, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(spec),
                                      oracle.Terms([t.host_desc(_view(spec, B, floating)) for t in terms]), q, base)
    rg, Jg = r.numpy(), J.numpy()
    if penalty != "surface_distance":
        assert (ro[:, :ns] > 0).mean() > 0.05 and (ro[:, :ns] == 0).mean() > 0.05
    np.testing.assert_allclose(rg, ro, rtol=1e-4, atol=5e-5)
    np.testing.assert_allclose(Jg, Jo, rtol=1e-3, atol=2e-4)


def test_empty_and_changed_scenes(gpu, panda_collision_spec):
    from robokit_b200.robo.robot import Robot

    spec = panda_collision_spec
    robot = Robot(spec)
    q = np.tile(spec.midrange_q, (4, 1)).astype(np.float32)
    vv = VarValues({VarKey.ROBOT: robot.state(q)})
    scene = Scene(num_scenes=1)
    plane = PlaneGeom([0, 1], poses=[[0, 0, -5.0, 1, 0, 0, 0]])
    scene.add(plane)
    task = SceneCollisionTask(robot, scene, margin=0.05)
    assert not np.any(task.compute_weighted_residual(vv).numpy())  # far below the arm
    plane.update(poses=[[0, 0, 0.5, 1, 0, 0, 0]])  # the term sees the change
    r = task.compute_weighted_residual(vv).numpy()
    c = oracle.fk(oracle.Robot.from_spec(spec), q[:1])["spheres"][0]
    sd = c[:, 2] - 0.5 - spec.collision_sphere_radii
    expect = np.where(sd < 0, 0.025 - sd, np.where(sd <= 0.05, 0.5 / (0.05 + 1e-6) * (sd - 0.05) ** 2, 0.0))
    np.testing.assert_allclose(r[0], expect, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("form", ["persistent", "plain"])
def test_lm_with_scene_collision_matches_the_oracle(gpu, panda_collision_spec, form):
    """Reach FK targets while a box and a table plane push the arm: per-problem costs agree with the oracle."""
    from robokit_b200.robo.robot import Robot

    spec = panda_collision_spec
    robot = Robot(spec)
    hand = spec.link_names.index("panda_hand")
    B = 128
    qs = robot.sample_q(B, seed=31)
    T = robot.forward_kinematics(robot.state(qs)).get_T_world_link(hand).numpy().reshape(B, 1, 7)
    rng = np.random.default_rng(3)
    lo, hi = spec.float32_actuated_limits().T
    q0 = np.clip(qs + rng.normal(0, 0.2, qs.shape), lo, hi).astype(np.float32)
    scene = Scene(1)
    scene.add(BoxGeom([[0.1, 0.1, 0.1]], [0, 1], poses=[[0.5, 0.0, 0.3, 1, 0, 0, 0]]))
    scene.add(PlaneGeom([0, 1], poses=[[0, 0, -0.05, 1, 0, 0, 0]]))
    terms = [PositionTask(robot, hand, T, weight=10.0), RotationTask(robot, hand, T, weight=5.0),
             PositionLimit(robot, 10.0), SceneCollisionTask(robot, scene, weight=2.0, margin=0.03,
                                                            movable_only=True)]
    opt = LMOptimizer(terms, LMOptimizerConfig(max_iter=30, lm_lambda=1e-2, lambda_factor=2.0,
                                               early_stopping_interval=0, form=form))
    st = robot.state(q0)
    opt.solve(VarValues({VarKey.ROBOT: st}))
    rob = oracle.Robot.from_spec(spec)
    ot = oracle.Terms([t.host_desc(_view(spec, B, False)) for t in terms])
    o = oracle.solve(rob, ot, oracle.params(max_iter=30, lambda_init=1e-2, lambda_factor=2.0), q0, None, threads=8)
    cost_g = 0.5 * (oracle.residual_jacobian(rob, ot, st.q.numpy(), None)[0] ** 2).sum(axis=1)
    cost_o = 0.5 * (oracle.residual_jacobian(rob, ot, o["q"], None)[0] ** 2).sum(axis=1)
    close = np.abs(cost_g - cost_o) <= 1e-3 * np.maximum(1e-3, cost_o)
    assert close.mean() >= 0.85, close.mean()
    c0 = 0.5 * (oracle.residual_jacobian(rob, ot, q0, None)[0] ** 2).sum(axis=1)
    assert np.median(cost_g) < 0.1 * np.median(c0)


def test_iksolver_with_a_scene(gpu, panda_collision_spec):
    """IKSolver(scene=...) with a SceneCollisionTask template: targets reached, and an obstacle in one scene
    pushes the arm out of it while the other scene (empty of it) does not; scene_indices select per target."""
    from robokit_b200.helpers.ik import IKContext, IKSolver, IKSolverConfig
    from robokit_b200.opt.sampler import RobertsSamplerConfig
    from robokit_b200.robo.robot import Robot

    spec = panda_collision_spec
    robot = Robot(spec)
    hand = spec.link_names.index("panda_hand")
    B = 64
    qs = robot.sample_q(B, seed=12)
    T = robot.forward_kinematics(robot.state(qs)).get_T_world_link(hand).numpy().reshape(B, 1, 7)
    scene = Scene(num_scenes=2)
    # a wide slab through the workspace in scene 1 only; both scenes share a floor far below
    scene.add(BoxGeom([[0.05, 1.0, 1.0]], [0, 0, 1], poses=[[0.25, 0.0, 0.5, 1, 0, 0, 0]]))
    scene.add(PlaneGeom([0, 1, 2], poses=[[0, 0, -1.0, 1, 0, 0, 0]] * 2))
    cfg = IKSolverConfig(sampler=RobertsSamplerConfig(keep_first=True, scale=1.0))
    cfg.add(PositionTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=20.0))
    cfg.add(RotationTask(frame_index=IKContext.TARGET_LINKS, T_world_target=IKContext.TARGET, weight=10.0))
    cfg.add(PositionLimit(weight=50.0))
    cfg.add(SceneCollisionTask(scene=IKContext.SCENE, scene_indices=IKContext.SCENE_INDICES, weight=20.0,
                               margin=0.01, movable_only=True))
    ik = IKSolver(cfg, robot, "panda_hand", scene=scene)
    free = ik.solve(T).q.numpy().copy()  # scene indices default to 0: no slab
    assert ik.compute_metrics_numpy(robot.state(free), T).success.mean() >= 0.9
    blocked = ik.solve(T, scene_indices=np.ones(B, np.int32)).q.numpy()
    with pytest.raises(ValueError):
        ik.solve(T, scene_indices=np.ones(B // 2, np.int32))
    rob = oracle.Robot.from_spec(spec)
    mov = np.flatnonzero(spec.collision_spheres_link_indices > 0)

    def pen(q):  # deepest penetration of the slab by a movable sphere
        c = oracle.fk(rob, q)["spheres"][:, mov]
        d = np.max(np.abs(c - [0.25, 0.0, 0.5]) - [0.05, 1.0, 1.0], axis=2)
        return np.maximum(0, spec.collision_sphere_radii[mov][None] - d).max(axis=1)

    assert np.mean(pen(blocked) < 0.02) > np.mean(pen(free) < 0.02)


# tests/terms/test_scene_collision_task.py:524-640 (TestWarpSceneCollisionTaskMultiScene), with primitive planes
# and boxes in place of the meshes: a multi-scene task with a batch partition equals the concatenation of
# single-scene tasks, and bad scene indices are refused.
_QY90 = [0.7071067811865476, 0.0, 0.7071067811865476, 0.0]  # local z onto world x


def _plane_x(x, offsets):
    return PlaneGeom(offsets, poses=[[x, 0.0, 0.0, *_QY90]] * int(offsets[-1]))


def _scene_single(k):
    s = Scene(1)
    if k == 0:
        s.add(_plane_x(0.3, [0, 1])).add(BoxGeom([[0.2, 0.2, 0.2]], [0, 1], poses=[[0.6, 0, 0.4, 1, 0, 0, 0]]))
        s.add(SphereGeom([0.1], [0, 1]))
    elif k == 1:
        s.add(_plane_x(0.5, [0, 1])).add(BoxGeom([[0.1, 0.1, 0.1]], [0, 1]))
    else:
        s.add(BoxGeom([[0.15, 0.15, 0.15]], [0, 1], poses=[[0.3, 0.1, 0.5, 1, 0, 0, 0]]))
    return s


def _scene_multi(n):
    s = Scene(n)
    planes = [0.3, 0.5][: min(n, 2)]
    off_p = [0, 1, 2] + [2] * (n - 2)
    s.add(PlaneGeom(off_p[: n + 1], poses=[[x, 0.0, 0.0, *_QY90] for x in planes]))
    boxes, off_b = [[0.6, 0, 0.4, 1, 0, 0, 0], [0, 0, 0, 1, 0, 0, 0]], [0, 1, 2]
    he = [[0.2, 0.2, 0.2], [0.1, 0.1, 0.1]]
    if n == 3:
        boxes.append([0.3, 0.1, 0.5, 1, 0, 0, 0])
        he.append([0.15, 0.15, 0.15])
        off_b = [0, 1, 2, 3]
    s.add(BoxGeom(he, off_b, poses=boxes))
    s.add(SphereGeom([0.1], [0, 1] + [1] * (n - 1)))
    return s


def _run_scene_task(robot, q, scene, scene_indices=None):
    st = robot.state(q=q)
    task = SceneCollisionTask(robot=robot, scene=scene, scene_indices=scene_indices, weight=1.0, margin=0.02,
                              residual_mode="abs")
    vv = VarValues({VarKey.ROBOT: st})
    return task.compute_weighted_residual(vv).numpy(), task.compute_weighted_jacobian_analytic(vv).numpy()


@pytest.mark.parametrize("partition", [[0, 2], [0, 1, 5]])
def test_multi_scene_matches_per_scene_tasks(gpu, panda_collision_spec, partition):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_collision_spec)
    rng = np.random.RandomState(len(partition))
    B = 4 if len(partition) == 2 else 6
    q = (rng.randn(B, robot.num_actuated_joints) * 0.1 + robot.spec.midrange_q).astype(np.float32)
    bounds = np.r_[partition, B]
    idx = np.repeat(np.arange(len(partition), dtype=np.int32), np.diff(bounds))
    r_multi, j_multi = _run_scene_task(robot, q, _scene_multi(len(partition)), N.DeviceArray.from_numpy(idx))
    parts = [_run_scene_task(robot, q[lo:hi], _scene_single(k)) for k, (lo, hi) in
             enumerate(zip(bounds[:-1], bounds[1:])) if hi > lo]
    r_ref = np.concatenate([p[0] for p in parts])
    j_ref = np.concatenate([p[1] for p in parts])
    assert r_multi.shape == r_ref.shape and j_multi.shape == j_ref.shape
    assert np.allclose(r_multi, r_ref, atol=1e-5, rtol=1e-5)
    assert np.allclose(j_multi, j_ref, atol=1e-5, rtol=1e-5)


def test_rejects_bad_scene_indices(gpu, panda_collision_spec):
    from robokit_b200.robo.robot import Robot

    robot = Robot(panda_collision_spec)
    scene = _scene_multi(2)
    q = np.zeros((4, robot.num_actuated_joints), np.float32)
    with pytest.raises(TypeError, match="int32"):
        _run_scene_task(robot, q, scene, N.DeviceArray.zeros(4, np.float32))
    with pytest.raises(TypeError, match="1D"):
        _run_scene_task(robot, q, scene, N.DeviceArray.zeros((4, 1), np.int32))
    with pytest.raises(ValueError, match="batch_size"):
        _run_scene_task(robot, q, scene, N.DeviceArray.zeros(3, np.int32))
