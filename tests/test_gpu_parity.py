"""CUDA path vs the FP64 oracle, stage by stage, through the C ABI.

Tolerances (FP32 kinematics vs FP64 oracle): poses, twists, residuals and
Jacobian entries within 1e-5 relative (+1e-5 absolute); normal equations within
1e-5 of their scale; the FP64 damped solve on identical inputs within 1e-9.
"""

import ctypes

import numpy as np
import pytest

import oracle
from robokit_b200 import configs
from robokit_b200.robo.robot import Robot

pytestmark = pytest.mark.gpu

CASES = [("chain7", 64), ("chain7c", 64), ("humanoid", 32), ("hand", 32)]


def _cfg(name, B, seed=0, pair_mode="all"):
    return configs.make(name, B, seed=seed, pair_mode=pair_mode)


def _dev(N, a, dt=np.float32):
    return None if a is None else N.DeviceArray.from_numpy(np.ascontiguousarray(a, dt))


def _problem(cfg):
    from robokit_b200.terms.task import NativeProblem

    return NativeProblem(cfg.robot, cfg.terms, cfg.batch, cfg.workload.base0 is not None, None)


def test_fk_golden_on_gpu(gpu, panda_spec, golden):
    N = gpu
    robot = Robot(panda_spec)
    from robokit_b200.robo.robot_spec import quaternion_to_matrix

    for c in golden["fk"]["configurations"]:
        q = np.array(c["qpos"], np.float32)[None]
        base = None if c["T_world_base"] is None else np.array(c["T_world_base"], np.float32)[None]
        st = robot.forward_kinematics(robot.state(q, base))
        T = st.T_world_link.numpy()[0]
        for lp in c["link_poses"]:
            if lp["link_name"] not in panda_spec.link_names:
                continue
            li = panda_spec.link_names.index(lp["link_name"])
            e = np.array(lp["xyz_wxyz"])
            np.testing.assert_allclose(T[li, :3], e[:3], atol=1e-5)
            np.testing.assert_allclose(quaternion_to_matrix(T[li, 3:]), quaternion_to_matrix(e[3:]), atol=1e-5)


def test_link_jacobian_golden_on_gpu(gpu, panda_spec, golden):
    robot = Robot(panda_spec)
    for c in golden["jacobians"]["configurations"]:
        q = np.array(c["qpos"], np.float32)[None]
        base = None if c["T_world_base"] is None else np.array(c["T_world_base"], np.float32)[None]
        st = robot.state(q, base)
        for lj in c["link_jacobians"]:
            if lj["link_name"] not in panda_spec.link_names:
                continue
            li = panda_spec.link_names.index(lj["link_name"])
            for frame in ("body", "spatial"):
                J = st.get_link_jacobian(li, frame).numpy()[0]
                e = np.array(lj[f"{frame}_J_joints"])
                if base is not None:
                    e = np.concatenate([np.array(lj[f"{frame}_J_base"]), e], axis=1)
                np.testing.assert_allclose(J, e, atol=2e-5, err_msg=f"{c['name']} {lj['link_name']} {frame}")


@pytest.mark.parametrize("name,B", CASES)
def test_fk_vs_oracle(gpu, name, B):
    cfg = _cfg(name, B)
    wl = cfg.workload
    st = cfg.robot.forward_kinematics(cfg.robot.state(wl.q0, wl.base0))
    o = oracle.fk(oracle.Robot.from_spec(wl.spec), wl.q0, wl.base0)
    Tl = st.T_world_link.numpy()
    Tg = Tl.copy()
    To = o["T_link"]
    # quaternion sign is standardised (w >= 0) on both sides
    np.testing.assert_allclose(Tg, To, rtol=1e-5, atol=2e-5)
    np.testing.assert_allclose(st.S_world.numpy(), o["S_world"], rtol=1e-5, atol=2e-5)
    if wl.spec.has_collision_spheres:
        np.testing.assert_allclose(st.collision_sphere_centers_world.numpy(), o["spheres"], rtol=1e-5, atol=2e-5)
        np.testing.assert_allclose(st.link_bounding_sphere_centers_world.numpy(), o["link_bounds"], rtol=1e-5,
                                   atol=2e-5)


@pytest.mark.parametrize("pair_mode", ["all", "slots"])
@pytest.mark.parametrize("name,B", CASES)
def test_residual_jacobian_vs_oracle(gpu, name, B, pair_mode):
    if pair_mode == "slots" and name != "chain7c":
        pytest.skip("slot mode only differs with a collision term")
    N = gpu
    cfg = _cfg(name, B, pair_mode=pair_mode)
    wl = cfg.workload
    prob = _problem(cfg)
    R, D = prob.residual_dim, prob.tangent_dim
    q, base = _dev(N, wl.q0), _dev(N, wl.base0)
    r = N.DeviceArray.empty((B, R))
    J = N.DeviceArray.empty((B, R, D))
    N.check(N.lib().ik_residual_jacobian(prob.handle, B, q.ptr, N.ptr(base), r.ptr, J.ptr, None))
    ro, Jo = oracle.residual_jacobian(oracle.Robot.from_spec(wl.spec), oracle.Terms(configs.oracle_terms(cfg)),
                                      wl.q0, wl.base0)
    scale = max(1.0, float(np.abs(Jo).max()))
    np.testing.assert_allclose(r.numpy(), ro, rtol=1e-5, atol=2e-5)
    np.testing.assert_allclose(J.numpy(), Jo, rtol=1e-5, atol=2e-5 * scale)


@pytest.mark.parametrize("name,B", CASES)
def test_normal_equations_vs_oracle(gpu, name, B):
    N = gpu
    cfg = _cfg(name, B)
    wl = cfg.workload
    prob = _problem(cfg)
    D = prob.tangent_dim
    q, base = _dev(N, wl.q0), _dev(N, wl.base0)
    H = N.DeviceArray.empty((B, D, D))
    g = N.DeviceArray.empty((B, D))
    c = N.DeviceArray.empty(B)
    N.check(N.lib().ik_normal_equations(prob.handle, B, q.ptr, N.ptr(base), H.ptr, g.ptr, c.ptr, None))
    Ho, go, co = oracle.normal_equations(oracle.Robot.from_spec(wl.spec), oracle.Terms(configs.oracle_terms(cfg)),
                                         wl.q0, wl.base0)
    for b in range(B):
        sH = max(1e-6, np.abs(Ho[b]).max())
        np.testing.assert_allclose(H.numpy()[b], Ho[b], atol=1e-5 * sH, rtol=1e-5)
        sg = max(1e-6, np.abs(go[b]).max())
        np.testing.assert_allclose(g.numpy()[b], go[b], atol=1e-5 * sg + 1e-7, rtol=1e-4)
    np.testing.assert_allclose(c.numpy(), co, rtol=1e-5, atol=1e-9)


def test_damped_solve_vs_oracle(gpu):
    N = gpu
    rng = np.random.default_rng(1)
    for D in (1, 6, 7, 13, 26, 35, 64):
        B = 33
        A = rng.normal(size=(B, D, D)).astype(np.float32)
        H = (A @ A.transpose(0, 2, 1)).astype(np.float32)
        g = rng.normal(size=(B, D)).astype(np.float32)
        lam = np.exp(rng.uniform(np.log(1e-5), np.log(1e5), B)).astype(np.float32)
        dH, dg, dl = _dev(N, H), _dev(N, g), _dev(N, lam)
        delta = N.DeviceArray.empty((B, D))
        pred = N.DeviceArray.empty(B)
        spd = N.DeviceArray.empty(B, np.int32)
        N.check(N.lib().ik_damped_solve(B, D, dH.ptr, dg.ptr, dl.ptr, delta.ptr, pred.ptr, spd.ptr, None))
        do, po, so = oracle.damped_solve(H.astype(np.float64), g.astype(np.float64), lam.astype(np.float64))
        assert spd.numpy().all() and so.all()
        # identical FP64 arithmetic on identical inputs; the step is rounded to float32 at the output
        np.testing.assert_allclose(delta.numpy(), do, rtol=2e-6, atol=1e-30)
        np.testing.assert_allclose(pred.numpy(), po, rtol=2e-6)
    # a non-SPD damped matrix is reported and gives a zero step
    H = -np.eye(4, dtype=np.float32)[None]
    dH, dg, dl = _dev(N, H), _dev(N, np.ones((1, 4))), _dev(N, np.array([1e-5]))
    delta = N.DeviceArray.empty((1, 4))
    pred = N.DeviceArray.empty(1)
    spd = N.DeviceArray.empty(1, np.int32)
    N.check(N.lib().ik_damped_solve(1, 4, dH.ptr, dg.ptr, dl.ptr, delta.ptr, pred.ptr, spd.ptr, None))
    assert spd.numpy()[0] == 0 and np.all(delta.numpy() == 0) and pred.numpy()[0] == 0


def test_accept_reject_kats_on_gpu(gpu):
    """tests/opt/test_optimizer_acceptance.py:41-69."""
    N = gpu
    prm = N.IkLmParams(1, 1.0, 2.0, 1e-6, 1e6, 1e-3, 1e-8, 0, 0.0, 0.0, 0.0, 0.0, 1)
    cost = _dev(N, [1.0, 1.0, 1.0])
    cnew = _dev(N, [1.1, 0.8, 0.8])
    pred = _dev(N, [-0.05, -0.05, 0.2])
    lam = _dev(N, [1.0, 1.0, 1.0])
    acc = N.DeviceArray.zeros(3, np.int32)
    N.check(N.lib().ik_accept_reject(3, cost.ptr, cnew.ptr, pred.ptr, lam.ptr, acc.ptr, ctypes.byref(prm), None))
    assert list(acc.numpy()) == [0, 0, 1]
    np.testing.assert_allclose(cost.numpy(), [1.0, 1.0, 0.8], atol=1e-6)
    np.testing.assert_allclose(lam.numpy(), [2.0, 2.0, 0.5])


@pytest.mark.parametrize("name,B", CASES)
def test_single_step_vs_oracle(gpu, name, B):
    """One LM iteration: cost, step, predicted reduction, proposal cost and the accept decision."""
    N = gpu
    cfg = _cfg(name, B)
    wl = cfg.workload
    prob = _problem(cfg)
    D = prob.tangent_dim
    lam0 = 0.1  # conditioning of the FP32 normal matrix bounds step parity; see DESIGN
    q, base = _dev(N, wl.q0), _dev(N, wl.base0)
    lam = _dev(N, np.full(B, lam0, np.float32))
    prm = N.IkLmParams(1, lam0, 10.0, 1e-5, 1e10, 1e-3, 1e-8, 0, 0.0, 0.0, 0.0, 0.0, 1)
    cost, delta = N.DeviceArray.empty(B), N.DeviceArray.empty((B, D))
    pred, cnew, acc = N.DeviceArray.empty(B), N.DeviceArray.empty(B), N.DeviceArray.empty(B, np.int32)
    N.check(N.lib().ik_step(prob.handle, B, q.ptr, N.ptr(base), lam.ptr, ctypes.byref(prm), cost.ptr, delta.ptr,
                            pred.ptr, cnew.ptr, acc.ptr, None))
    rob, terms = oracle.Robot.from_spec(wl.spec), oracle.Terms(configs.oracle_terms(cfg))
    Ho, go, co = oracle.normal_equations(rob, terms, wl.q0, wl.base0)
    do, po, _ = oracle.damped_solve(Ho, go, np.full(B, lam0))
    dn = delta.numpy()
    for b in range(B):
        np.testing.assert_allclose(dn[b], do[b], rtol=1e-4, atol=1e-4 * np.abs(do[b]).max() + 1e-7)
    np.testing.assert_allclose(pred.numpy(), po, rtol=1e-3, atol=1e-7)
    # the proposal's cost, evaluated by the oracle at the GPU's own proposal
    qp = (wl.q0 + dn[:, (6 if wl.base0 is not None else 0):]).astype(np.float32)
    bp = None
    if wl.base0 is not None:
        out = N.DeviceArray.empty((B, 7))
        qo = N.DeviceArray.empty(wl.q0.shape)
        N.check(N.lib().ik_integrate(B, wl.q0.shape[1], 1, _dev(N, wl.q0).ptr, _dev(N, wl.base0).ptr, delta.ptr,
                                     None, qo.ptr, out.ptr, None))
        bp = out.numpy()
    r_new, _ = oracle.residual_jacobian(rob, terms, qp, bp)
    c_new_o = 0.5 * np.sum(r_new ** 2, axis=1)
    np.testing.assert_allclose(cnew.numpy(), c_new_o, rtol=1e-4, atol=1e-9)
    # the accept rule applied by the oracle to the GPU's scalars reproduces the GPU's decision
    op = oracle.params(lambda_factor=10.0, lambda_min=1e-5, lambda_max=1e10)
    c_start = np.where(acc.numpy() == 1, co, cost.numpy())
    _, _, acc_o = oracle.accept_reject(co, cnew.numpy(), pred.numpy(), np.full(B, lam0), op)
    agree = np.mean(acc_o == acc.numpy())
    assert agree >= 0.95, agree
    np.testing.assert_allclose(c_start, co, rtol=1e-5, atol=1e-9)
