"""The continuous-batching server (ik_server_*): results alone vs in the mix, admission, relaunch, errors."""

import time
from dataclasses import replace

import numpy as np
import pytest

from robokit_b200 import _native as N
from robokit_b200 import serve
from robokit_b200.opt import LMOptimizer, VarKey, VarValues

pytestmark = pytest.mark.gpu


def _pool_solution(st):
    """Every problem of the type's pool solved in one persistent launch (problems are independent)."""
    wl = st.cfg.workload
    opt = LMOptimizer(st.cfg.terms, st.lm)
    state = st.cfg.robot.state(wl.q0, wl.base0)
    opt.solve(VarValues({VarKey.ROBOT: state}))
    base = state.T_world_base.numpy() if state.has_floating_base else None
    return {"q": state.q.numpy(), "base": base, "cost": opt.costs.numpy(), "iterations": opt.iterations.numpy()}


def _submit(srv, types, r):
    q0, base0, tg = serve._inputs(types[r.type_id], r)
    return srv.submit(r.type_id, q0, tg, base0)


def _close_to_pool(res, ref, r):
    sl = slice(r.start, r.start + r.batch)
    # the server kernel and the batch kernel are compiled separately; the
    # tolerance covers a different FMA contraction choice, nothing else
    np.testing.assert_allclose(res["q"], ref["q"][sl], rtol=0, atol=1e-4)
    np.testing.assert_allclose(res["cost"], ref["cost"][sl], rtol=1e-4, atol=1e-9)
    if ref["base"] is not None:
        np.testing.assert_allclose(res["base"], ref["base"][sl], rtol=0, atol=1e-4)
    assert np.mean(res["iterations"] == ref["iterations"][sl]) > 0.95


def test_results_alone_equal_results_in_the_mix(gpu):
    """Requests of four robots submitted back to back overlap on the GPU; each result equals the same
    request served alone (bitwise) and the batch solve of the same problems (within tolerance)."""
    types = serve.mixed_types(pool=512, seed=5)
    refs = [_pool_solution(st) for st in types]
    rng = np.random.default_rng(0)
    reqs = []
    for i in range(16):
        k = i % 4
        b = int(rng.integers(1, 160))
        reqs.append(serve.RequestSpec(0.0, k, int(rng.integers(0, 512 - b)), b))
    srv = serve.make_server(types)
    ids = [_submit(srv, types, r) for r in reqs]
    mixed = srv.wait(ids, timeout_s=120)
    for r, i in zip(reqs, ids):
        _close_to_pool(mixed[i], refs[r.type_id], r)
    # the same requests one at a time through the same server
    for r, i in list(zip(reqs, ids))[:6]:
        j = _submit(srv, types, r)
        alone = srv.wait([j], timeout_s=60)[j]
        for key in ("q", "cost", "iterations", "status"):
            np.testing.assert_array_equal(alone[key], mixed[i][key])
    srv.close()


def test_requests_wait_for_free_slots(gpu):
    types = serve.mixed_types(pool=256, seed=9)[:2]
    refs = [_pool_solution(st) for st in types]
    srv = serve.make_server(types, slots=64)
    reqs = [serve.RequestSpec(0.0, 1, 40 * i, 40) for i in range(5)] + [serve.RequestSpec(0.0, 0, 7, 64)]
    ids = [_submit(srv, types, r) for r in reqs]
    assert srv.info(1)["pending"] >= 3
    out = srv.wait(ids, timeout_s=120)
    for r, i in zip(reqs, ids):
        _close_to_pool(out[i], refs[r.type_id], r)
    info = srv.info(1)
    assert info["free_slots"] == 64 and info["pending"] == 0 and info["inflight"] == 0
    srv.close()


def test_kernel_relaunches_after_idle_exit(gpu):
    types = serve.mixed_types(pool=128, seed=3)[:1]
    ref = _pool_solution(types[0])
    srv = serve.make_server(types)
    for start in (0, 50, 90):
        r = serve.RequestSpec(0.0, 0, start, 30)
        i = _submit(srv, types, r)
        _close_to_pool(srv.wait([i], timeout_s=60)[i], ref, r)
        time.sleep(0.05)  # far longer than the idle limit: the kernel exits
    assert srv.info(0)["launches"] >= 2
    srv.close()


def test_server_errors(gpu):
    types = serve.mixed_types(pool=64, seed=1)[:1]
    srv = serve.make_server(types, slots=32)
    q0, base0, tg = serve._inputs(types[0], serve.RequestSpec(0.0, 0, 0, 40))
    with pytest.raises(N.NativeError, match="exceeds"):
        srv.submit(0, q0, tg, base0)
    with pytest.raises(ValueError, match="not registered"):
        srv.submit(3, q0[:2], [t[:2] for t in tg], base0)
    with pytest.raises(ValueError):
        srv.submit(0, q0[:2], [t[:3] for t in tg], base0)
    small = serve.IKServer(budget_bytes=1024)
    with pytest.raises(N.NativeError, match="budget"):
        small.add_type(types[0].cfg.robot, types[0].cfg.terms, types[0].lm, 4096)
    small.close()
    srv.close()


def test_server_serves_shared_references_and_refuses_per_problem_ones(gpu, panda_collision_spec):
    """A request carries only seeds and pose targets, so a served type may hold joint-reference, velocity,
    base-reference and scene terms whose reference is one shared row (a rest pose, one scene); its results equal
    the batch solve of the same problems.  A per-problem reference or scene index is refused at registration."""
    from robokit_b200.geom import BoxGeom, Scene, SphereGeom
    from robokit_b200.opt import LMOptimizerConfig
    from robokit_b200.robo.robot import Robot
    from robokit_b200.terms.dense import ConfigurationTask, PositionTask, SceneCollisionTask, SmoothnessTask

    robot = Robot(panda_collision_spec)
    hand = robot.link_names.index("panda_hand")
    n = 48
    q0 = robot.sample_q(n, seed=3)
    T = robot.forward_kinematics(robot.state(robot.sample_q(n, seed=4))).get_T_world_link(hand).numpy()
    rest = panda_collision_spec.midrange_q.astype(np.float32)
    scene = Scene(1).add(BoxGeom([[0.1, 0.1, 0.1]], [0, 1], poses=[[0.5, 0.0, 0.3, 1, 0, 0, 0]]))
    lm = LMOptimizerConfig(max_iter=20, early_stopping_interval=0)

    def extra():
        return [ConfigurationTask(robot=robot, rest_q=rest, weight=0.1),
                SceneCollisionTask(robot, scene, weight=5.0, margin=0.05)]

    placeholder = PositionTask(robot, hand, T[:1].reshape(1, 1, 7), weight=10.0)
    srv = serve.IKServer(budget_bytes=64 << 20)
    try:
        tid = srv.add_type(robot, [placeholder, *extra()], lm, 64)
        rid = srv.submit(tid, q0, [T.reshape(n, 1, 7)])
        got = srv.wait([rid], timeout_s=60)[rid]
        opt = LMOptimizer([PositionTask(robot, hand, T.reshape(n, 1, 7), weight=10.0), *extra()],
                          replace(lm, form="persistent"))
        state = robot.state(q0.copy())
        opt.solve(VarValues({VarKey.ROBOT: state}))
        np.testing.assert_allclose(got["q"], state.q.numpy(), rtol=0, atol=1e-4)
        np.testing.assert_allclose(got["cost"], opt.costs.numpy(), rtol=1e-4, atol=1e-9)
        prev4 = robot.state(np.zeros((4, robot.num_actuated_joints), np.float32))
        with pytest.raises(N.NativeError, match="one shared reference row"):
            srv.add_type(robot, [placeholder, SmoothnessTask(robot=robot, prev_var=prev4, weight=1.0)], lm, 16)
        two = Scene(2).add(SphereGeom([0.1, 0.1], [0, 1, 2]))
        with pytest.raises(ValueError, match="scene_indices"):  # per-problem scenes do not lower to one row
            srv.add_type(robot, [placeholder, SceneCollisionTask(robot, two, scene_indices=N.DeviceArray.from_numpy(
                np.array([0, 1], np.int32)), weight=1.0)], lm, 16)
    finally:
        srv.close()


def test_server_serves_velocity_and_base_references(gpu, panda_collision_spec):
    """The remaining shared-reference kinds: a velocity limit against a fixed previous state, and the base rows
    of a ConfigurationTask on a floating base; served results equal the batch solve."""
    from robokit_b200.opt import LMOptimizerConfig
    from robokit_b200.robo.robot import Robot
    from robokit_b200.terms.dense import ConfigurationTask, PositionTask, VelocityLimitTask

    robot = Robot(panda_collision_spec)
    hand = robot.link_names.index("panda_hand")
    n = 32
    q0 = robot.sample_q(n, seed=8)
    base0 = np.tile(np.array([0.05, -0.02, 0.0, 1, 0, 0, 0], np.float32), (n, 1))
    T = robot.forward_kinematics(robot.state(robot.sample_q(n, seed=9))).get_T_world_link(hand).numpy()
    T[:, 0] += 0.2
    prev = robot.state(panda_collision_spec.midrange_q[None].astype(np.float32))
    rest_base = np.array([[0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0]], np.float32)
    lm = LMOptimizerConfig(max_iter=20, early_stopping_interval=0)

    def extra():
        return [VelocityLimitTask(robot=robot, dt=0.5, prev_state_var=prev, weight=1.0),
                ConfigurationTask(robot=robot, rest_q=panda_collision_spec.zero_q.astype(np.float32),
                                  T_world_base_rest=rest_base, weight=0.01, base_weight=[1, 1, 10, 10, 10, 1])]

    srv = serve.IKServer(budget_bytes=64 << 20)
    try:
        tid = srv.add_type(robot, [PositionTask(robot, hand, T[:1].reshape(1, 1, 7), weight=10.0), *extra()], lm, 64,
                           floating=True)
        rid = srv.submit(tid, q0, [T.reshape(n, 1, 7)], base0)
        got = srv.wait([rid], timeout_s=60)[rid]
        opt = LMOptimizer([PositionTask(robot, hand, T.reshape(n, 1, 7), weight=10.0), *extra()],
                          replace(lm, form="persistent"))
        state = robot.state(q0.copy(), base0.copy())
        opt.solve(VarValues({VarKey.ROBOT: state}))
        np.testing.assert_allclose(got["q"], state.q.numpy(), rtol=0, atol=1e-4)
        np.testing.assert_allclose(got["base"], state.T_world_base.numpy(), rtol=0, atol=1e-4)
        np.testing.assert_allclose(got["cost"], opt.costs.numpy(), rtol=1e-4, atol=1e-9)
    finally:
        srv.close()
