"""Pin the FP64 oracle against the reference's own golden vectors and unit-test recipes."""

import numpy as np
import pytest

import oracle
from robokit_b200.robo.robot_spec import quaternion_to_matrix


def _pose_close(a, e, atol):
    """Compare poses as rotation matrices + translations (quaternion sign is not unique)."""
    return np.abs(np.asarray(a[:3]) - e[:3]).max() <= atol and np.abs(
        quaternion_to_matrix(a[3:]) - quaternion_to_matrix(e[3:])
    ).max() <= atol


def test_fk_golden(panda_spec, golden):
    """tests/robo/test_forward_kinematics.py:40-65, atol 1e-5."""
    rob = oracle.Robot.from_spec(panda_spec)
    checked = 0
    for c in golden["fk"]["configurations"]:
        q = np.array(c["qpos"], np.float32)[None]
        base = None if c["T_world_base"] is None else np.array(c["T_world_base"], np.float32)[None]
        out = oracle.fk(rob, q, base)
        for lp in c["link_poses"]:
            if lp["link_name"] not in panda_spec.link_names:
                continue
            li = panda_spec.link_names.index(lp["link_name"])
            assert _pose_close(out["T_link"][0, li], np.array(lp["xyz_wxyz"]), 1e-5), (c["name"], lp["link_name"])
            checked += 1
    assert checked >= 40


def test_jacobian_golden(panda_spec, golden):
    """tests/robo/test_jacobians.py:13-66, atol 1e-5 (body and spatial, with and without a base)."""
    rob = oracle.Robot.from_spec(panda_spec)
    for c in golden["jacobians"]["configurations"]:
        q = np.array(c["qpos"], np.float32)[None]
        base = None if c["T_world_base"] is None else np.array(c["T_world_base"], np.float32)[None]
        for lj in c["link_jacobians"]:
            if lj["link_name"] not in panda_spec.link_names:
                continue
            li = panda_spec.link_names.index(lj["link_name"])
            for frame in ("body", "spatial"):
                J = oracle.link_jacobian(rob, q, base, li, frame == "body")[0]
                e = np.array(lj[f"{frame}_J_joints"])
                if base is not None:
                    e = np.concatenate([np.array(lj[f"{frame}_J_base"]), e], axis=1)
                np.testing.assert_allclose(J, e, atol=1e-5, err_msg=f"{c['name']} {lj['link_name']} {frame}")


def test_fk_doctest_panda_hand(panda_spec):
    """robo/robot.py:41-44 and :147-154 known answers (atol 1e-4)."""
    rob = oracle.Robot.from_spec(panda_spec)
    q = np.array([[0.0, -1.2, 0.0, -2.0, 0.0, 1.0, 0.0, 0.0]], np.float32)
    hand = panda_spec.link_names.index("panda_hand")
    out = oracle.fk(rob, q)
    assert _pose_close(out["T_link"][0, hand], np.array([6.0860e-02, -4.7547e-12, 7.6373e-01, 0.0382, 0.9193,
                                                          0.3808, 0.0922]), 1e-4)
    base = np.array([[1.0, 2.0, 3.0, 0.7071, 0.0, 0.7071, 0.0]], np.float32)
    out = oracle.fk(rob, q, base)
    assert _pose_close(out["T_link"][0, hand], np.array([1.76371783, 2.0, 2.93915576, -0.24222432, 0.71524162,
                                                          0.29626278, -0.58478125]), 1e-3)


def test_accept_reject_kats():
    """tests/opt/test_optimizer_acceptance.py:41-69 (rho_min 1e-3, eps 1e-8, factor 2, lambda in [1e-6, 1e6])."""
    prm = oracle.params(lambda_factor=2.0, lambda_min=1e-6, lambda_max=1e6, rho_min=1e-3, gain_ratio_epsilon=1e-8)
    cost, lam, acc = oracle.accept_reject([1.0, 1.0, 1.0], [1.1, 0.8, 0.8], [-0.05, -0.05, 0.2], [1.0, 1.0, 1.0], prm)
    assert list(acc) == [0, 0, 1]
    np.testing.assert_allclose(cost, [1.0, 1.0, 0.8])
    np.testing.assert_allclose(lam, [2.0, 2.0, 0.5])


def test_damped_solve_matches_numpy():
    """lm_optimizer.py:56-79 vs np.linalg.solve (tests/opt/test_optimizer.py:574-597 recipe)."""
    rng = np.random.default_rng(0)
    for D in (7, 26, 35, 64):
        A = rng.normal(size=(4, D, D))
        H = A @ A.transpose(0, 2, 1) + 0.3 * np.eye(D)
        g = rng.normal(size=(4, D))
        lam = np.array([0.01, 1.0, 1000.0, 1e5])
        delta, pred, spd = oracle.damped_solve(H, g, lam)
        exp = np.linalg.solve(H + lam[:, None, None] * np.eye(D), -g[..., None])[..., 0]
        np.testing.assert_allclose(delta, exp, rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(pred, 0.5 * np.sum(exp * (lam[:, None] * exp - g), 1), rtol=1e-9)
        assert spd.all()
    # an indefinite matrix is reported, with a zero step
    H = -np.eye(3)[None]
    delta, pred, spd = oracle.damped_solve(H, np.ones((1, 3)), np.array([1e-5]))
    assert spd[0] == 0 and np.all(delta == 0) and pred[0] == 0


def test_masked_step_matches_reduced_problem(panda_spec):
    """tests/opt/test_optimizer.py:366-429: the mask zeroes J columns before forming J^T J."""
    rob = oracle.Robot.from_spec(panda_spec)
    hand = panda_spec.link_names.index("panda_hand")
    q = panda_spec.midrange_q[None].astype(np.float32)
    tgt = np.array([[[0.4, 0.1, 0.5, 1.0, 0.0, 0.0, 0.0]]], np.float32)
    terms = oracle.Terms([
        dict(kind=1, num_frames=1, frame_links=[hand], weights=[10.0] * 3, targets=tgt, target_rows=1),
        dict(kind=2, num_frames=1, frame_links=[hand], weights=[2.0] * 3, targets=tgt, target_rows=1),
    ])
    D = panda_spec.num_actuated_joints
    mask = np.ones(D, np.float32)
    mask[1] = 0.0
    r, J = oracle.residual_jacobian(rob, terms, q)
    Jm = J[0] * mask[None]
    lam = 1e-2
    exp = np.linalg.solve(Jm.T @ Jm + lam * np.eye(D), -(Jm.T @ r[0]))
    H, g, cost = oracle.normal_equations(rob, terms, q, None, mask)
    delta, pred, spd = oracle.damped_solve(H, g, np.array([lam]))
    assert abs(delta[0, 1]) < 1e-12
    np.testing.assert_allclose(delta[0], exp, rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(cost[0], 0.5 * r[0] @ r[0])


def test_oracle_jacobian_matches_finite_differences(panda_collision_spec):
    """The analytic Jacobian of every term kind vs central differences of the residuals."""
    from robokit_b200.robo.robot_spec import collision_pair_tables

    spec = panda_collision_spec
    rob = oracle.Robot.from_spec(spec)
    hand = spec.link_names.index("panda_hand")
    pairs, lp, off, grouped = collision_pair_tables(spec)
    tgt = np.array([[[0.3, -0.2, 0.6, 0.9, 0.1, 0.3, 0.2]]], np.float32)
    tgt[..., 3:] /= np.linalg.norm(tgt[..., 3:])
    for mode in (0, 1):
        terms = oracle.Terms([
            dict(kind=1, num_frames=1, frame_links=[hand], weights=[2.0, 3.0, 4.0], targets=tgt, target_rows=1),
            dict(kind=2, num_frames=1, frame_links=[hand], weights=[1.0, 1.5, 0.5], targets=tgt, target_rows=1),
            dict(kind=3, weights=np.full(spec.num_actuated_joints, 2.0)),
            dict(kind=4, weights=[1.5], margin=0.5, max_active_pairs=50, pair_mode=mode,
                 num_link_pairs=len(lp), link_pairs=lp.ravel(), link_pair_offsets=off,
                 num_sphere_pairs=len(grouped), sphere_pairs=grouped.ravel()),
        ])
        rng = np.random.default_rng(7)
        q = (spec.midrange_q + rng.normal(0, 0.15, spec.num_actuated_joints)).astype(np.float64)
        base = np.array([[0.1, -0.2, 0.3, 0.9, 0.1, -0.3, 0.2]])
        base[:, 3:] /= np.linalg.norm(base[:, 3:])
        _, J = oracle.residual_jacobian(rob, terms, q[None].astype(np.float32), base.astype(np.float32))
        # joint columns: float32 inputs limit the difference step
        eps = 1e-3
        fd = np.zeros_like(J[0])
        kink = np.zeros(J.shape[1], bool)  # hinge rows whose activity changes inside the stencil
        nlim = spec.num_actuated_joints
        stable = np.ones(J.shape[2], bool)  # columns whose slot selection is the same on both sides
        for a in range(spec.num_actuated_joints):
            qp, qm = q.copy(), q.copy()
            qp[a] += eps
            qm[a] -= eps
            rp, _ = oracle.residual_jacobian(rob, terms, qp[None].astype(np.float32), base.astype(np.float32))
            rm, _ = oracle.residual_jacobian(rob, terms, qm[None].astype(np.float32), base.astype(np.float32))
            fd[:, 6 + a] = (rp[0] - rm[0]) / (2 * eps)
            kink |= (rp[0] == 0) != (rm[0] == 0)
            if mode == 0:
                sp, sm = rp[0][6 + nlim:], rm[0][6 + nlim:]
                stable[6 + a] = np.count_nonzero(sp) == np.count_nonzero(sm) and np.max(np.abs(sp - sm)) < 0.05
        if mode == 1:
            fd[kink] = J[0][kink]
        # rotation rows use the reference's approximate Jacobian (no SO(3) J_l^-1 factor,
        # rotation_task.py:374-390); compare position, limit and collision rows exactly
        rows = np.r_[0:3, 6:J.shape[1]]
        if mode == 0:
            # slot rows follow the selection order: compare column sums where the selection is stable
            # (tests/terms/test_self_collision_task.py:124-157 compares sums likewise)
            rows = np.r_[0:3, 6:6 + nlim]
            cols = np.nonzero(stable[6:])[0] + 6
            assert len(cols) >= 4
            np.testing.assert_allclose(J[0][6 + nlim:, cols].sum(0), fd[6 + nlim:, cols].sum(0), atol=2e-2)
        np.testing.assert_allclose(J[0][rows][:, 6:], fd[rows][:, 6:], atol=2e-2)


def test_oracle_lm_reaches_reachable_targets():
    """A small C1 batch: LM from random starts reaches most FK targets."""
    from robokit_b200 import configs

    cfg = configs.make("chain7", 128, seed=3)
    rob = oracle.Robot.from_spec(cfg.workload.spec)
    terms = oracle.Terms(configs.oracle_terms(cfg))
    prm = oracle.params(max_iter=50, lambda_init=1e-3, lambda_factor=10.0)
    out = oracle.solve(rob, terms, prm, cfg.workload.q0, threads=4)
    pe, re, ok = oracle.metrics(rob, out["q"], None, cfg.workload.target_links, cfg.workload.targets, 1e-3, 0.01)
    assert ok.mean() > 0.6
    # start cost never increases (accepted steps only decrease the cost)
    H, g, c0 = oracle.normal_equations(rob, terms, cfg.workload.q0)
    assert np.all(out["cost"] <= c0 + 1e-12)
    # multithreaded and single-threaded solves agree exactly
    out1 = oracle.solve(rob, terms, prm, cfg.workload.q0, threads=1)
    np.testing.assert_array_equal(out1["q"], out["q"])


def test_oracle_frame_term_matches_finite_differences(panda_spec):
    """FrameTask ("log") residual and Jacobian of the oracle vs central differences (joint columns),
    with and without a floating base; the residual is zero at the frame's own pose."""
    spec = panda_spec
    rob = oracle.Robot.from_spec(spec)
    hand = spec.link_names.index("panda_hand")
    link4 = spec.link_names.index("panda_link4")
    rng = np.random.default_rng(3)
    q = (spec.midrange_q + rng.normal(0, 0.3, spec.num_actuated_joints)).astype(np.float64)
    tgt = np.array([[[0.3, -0.2, 0.6, 0.7, 0.2, -0.5, 0.4], [0.1, 0.3, 0.4, 0.2, 0.9, 0.1, -0.3]]], np.float32)
    tgt[..., 3:] /= np.linalg.norm(tgt[..., 3:], axis=-1, keepdims=True)
    terms = oracle.Terms([dict(kind=5, num_frames=2, frame_links=[hand, link4], weights=[2.0, 0.7, 1.0, 3.0],
                               targets=tgt, target_rows=1)])
    for base in (None, np.array([[0.1, -0.2, 0.3, 0.9, 0.1, -0.3, 0.2]])):
        if base is not None:
            base[:, 3:] /= np.linalg.norm(base[:, 3:])
            base = base.astype(np.float32)
        boff = 0 if base is None else 6
        r, J = oracle.residual_jacobian(rob, terms, q[None].astype(np.float32), base)
        assert r.shape == (1, 12)
        eps = 1e-3
        for a in range(spec.num_actuated_joints):
            qp, qm = q.copy(), q.copy()
            qp[a] += eps
            qm[a] -= eps
            rp, _ = oracle.residual_jacobian(rob, terms, qp[None].astype(np.float32), base)
            rm, _ = oracle.residual_jacobian(rob, terms, qm[None].astype(np.float32), base)
            np.testing.assert_allclose(J[0][:, boff + a], (rp[0] - rm[0]) / (2 * eps), atol=5e-3)
    # at the frame's own pose the residual vanishes
    T_link = oracle.fk(rob, q[None].astype(np.float32))["T_link"]
    own = np.stack([T_link[0, hand], T_link[0, link4]])[None].astype(np.float32)
    r0, _ = oracle.residual_jacobian(rob, oracle.Terms([dict(kind=5, num_frames=2, frame_links=[hand, link4],
                                                             weights=[1.0] * 4, targets=own, target_rows=1)]),
                                     q[None].astype(np.float32))
    assert np.abs(r0).max() < 1e-6


def test_oracle_joint_reference_term(panda_spec):
    """Joint-reference rows (smoothness / rest): r = w (q - ref[b // (B // rows)]), J = diag(w) on the joint
    columns, after the six base columns of a floating base."""
    spec = panda_spec
    rob = oracle.Robot.from_spec(spec)
    na = spec.num_actuated_joints
    rng = np.random.default_rng(7)
    B = 6
    q = rng.normal(0, 0.5, (B, na)).astype(np.float32)
    ref = rng.normal(0, 0.5, (2, na)).astype(np.float32)  # 2 rows, 3 problems each
    w = np.linspace(0.2, 1.5, na).astype(np.float32)
    terms = oracle.Terms([dict(kind=6, weights=w, targets=ref, target_rows=2)])
    assert oracle.residual_dim(rob, terms) == na
    for base in (None, np.tile(np.array([[0.1, 0, 0, 1, 0, 0, 0]], np.float32), (B, 1))):
        boff = 0 if base is None else 6
        r, J = oracle.residual_jacobian(rob, terms, q, base)
        rows = np.arange(B) // 3
        np.testing.assert_allclose(r, w * (q.astype(np.float64) - ref[rows]), rtol=1e-12, atol=1e-12)
        expect = np.zeros((B, na, boff + na))
        expect[:, np.arange(na), boff + np.arange(na)] = w
        np.testing.assert_array_equal(J, expect)


def test_oracle_velocity_limit_term(panda_spec):
    """Velocity rows: qd = (q - prev) / dt, r = w max(0, |qd| - vmax), J = w sign(qd) / dt where active."""
    spec = panda_spec
    rob = oracle.Robot.from_spec(spec)
    na = spec.num_actuated_joints
    rng = np.random.default_rng(9)
    B = 5
    prev = rng.normal(0, 0.5, (1, na)).astype(np.float32)  # one row for every problem
    q = (prev + rng.normal(0, 0.3, (B, na))).astype(np.float32)
    dt = 0.1
    vmax = np.full(na, 2.0, np.float32)
    w = np.linspace(0.5, 1.5, na).astype(np.float32)
    terms = oracle.Terms([dict(kind=7, weights=w, targets=prev, target_rows=1, dt=dt, velocity_limits=vmax)])
    assert oracle.residual_dim(rob, terms) == na
    r, J = oracle.residual_jacobian(rob, terms, q)
    qd = (q.astype(np.float64) - prev) / np.float32(dt)
    act = np.abs(qd) > vmax
    assert act.any() and (~act).any()
    np.testing.assert_allclose(r, np.where(act, w * (np.abs(qd) - vmax), 0.0), rtol=1e-12, atol=1e-12)
    expect = np.zeros((B, na, na))
    expect[:, np.arange(na), np.arange(na)] = np.where(act, w * np.sign(qd) / np.float32(dt), 0.0)
    np.testing.assert_allclose(J, expect, rtol=1e-12, atol=0)


def _scene_records(rows):
    """[n, 16] primitive records: (type, scene, scale, params, pose vec7)."""
    out = np.zeros((len(rows), 16), np.float32)
    for i, (typ, scene, scale, prm, pose) in enumerate(rows):
        out[i, 0], out[i, 1], out[i, 2] = typ, scene, scale
        out[i, 4:4 + len(prm)] = prm
        p = np.asarray(pose, np.float64)
        p[3:] /= np.linalg.norm(p[3:])
        out[i, 8:15] = p
    return out


@pytest.mark.parametrize("prim", ["box", "sphere", "plane", "capsule"])
@pytest.mark.parametrize("penalty", [0, 1, 2])
def test_oracle_scene_term_matches_finite_differences(panda_collision_spec, prim, penalty):
    """Scene-collision rows of the oracle: the Jacobian agrees with central differences of the residual for each
    primitive type and penalty, with and without a floating base; rows beyond the margin are zero."""
    spec = panda_collision_spec
    rob = oracle.Robot.from_spec(spec)
    rng = np.random.default_rng(4)
    rot = [0.9, 0.2, -0.3, 0.25]
    # placed against the arm at this configuration (sphere centres span x 0-0.65 m, z 0.08-0.9 m)
    geo = {"box": (0, [0.12, 0.08, 0.08], [0.4, 0.15, 0.55] + rot),
           "sphere": (1, [0.1], [0.35, 0.15, 0.55] + rot),
           "plane": (2, [], [0.0, 0.0, 0.6] + [0.99, 0.05, -0.05, 0.0]),
           "capsule": (3, [0.05, 0.12], [0.45, 0.15, 0.58] + rot)}[prim]
    rec = _scene_records([(geo[0], 0, 1.3, geo[1], geo[2])])
    ns = len(spec.collision_sphere_radii)
    term = dict(kind=8, weights=np.linspace(0.5, 2.0, ns), query_spheres=np.arange(ns), geoms=rec, num_scenes=1,
                penalty=penalty, margin=0.15, residual_sqrt=0, residual_eps=1e-6)
    terms = oracle.Terms([term])
    assert oracle.residual_dim(rob, terms) == ns
    q = (spec.midrange_q + rng.normal(0, 0.3, spec.num_actuated_joints)).astype(np.float64)
    for base in (None, np.array([[0.05, -0.02, 0.03, 0.98, 0.05, -0.1, 0.1]])):
        if base is not None:
            base[:, 3:] /= np.linalg.norm(base[:, 3:])
            base = base.astype(np.float32)
        boff = 0 if base is None else 6
        r, J = oracle.residual_jacobian(rob, terms, q[None].astype(np.float32), base)
        if penalty != 2:
            assert (r[0] > 0).any() and (r[0] == 0).any()
        eps = 1e-4
        for a in range(spec.num_actuated_joints):
            qp, qm = q.copy(), q.copy()
            qp[a] += eps
            qm[a] -= eps
            rp, _ = oracle.residual_jacobian(rob, terms, qp[None], base)
            rm, _ = oracle.residual_jacobian(rob, terms, qm[None], base)
            fd = (rp[0] - rm[0]) / (2 * eps)
            # the hinge's kink and the box's face switches are the only places where the two may differ
            smooth = (np.abs(r[0]) > 1e-3) | (J[0][:, boff + a] == 0)
            np.testing.assert_allclose(J[0][smooth, boff + a], fd[smooth], atol=2e-3, rtol=1e-3)


def test_oracle_scene_selection_and_query_order(panda_collision_spec):
    """Each problem reads its scene (row b // (B // rows)); a point keeps the first primitive of least distance;
    an empty scene leaves every sphere at 1e6."""
    spec = panda_collision_spec
    rob = oracle.Robot.from_spec(spec)
    ns = len(spec.collision_sphere_radii)
    rec = _scene_records([(2, 0, 1.0, [], [0, 0, 0.2, 1, 0, 0, 0]),     # scene 0: plane z = 0.2
                          (2, 1, 1.0, [], [0, 0, 0.6, 1, 0, 0, 0]),     # scene 1: plane z = 0.6 ...
                          (2, 1, 1.0, [], [0, 0, 0.6, 1, 0, 0, 0])])    # ... twice (ties keep the first)
    q = np.tile(spec.midrange_q, (4, 1)).astype(np.float32)
    term = dict(kind=8, weights=np.ones(ns), query_spheres=np.arange(ns), geoms=rec, num_scenes=3, penalty=2,
                margin=0.02, residual_sqrt=0, residual_eps=1e-6, scene_indices=np.array([1, 2], np.int32))
    r, _ = oracle.residual_jacobian(rob, oracle.Terms([term]), q)
    c = oracle.fk(rob, q[:1])["spheres"][0]
    expect = np.abs(c[:, 2] - 0.6 - spec.collision_sphere_radii)  # problems 0, 1: scene 1
    np.testing.assert_allclose(r[0], expect, rtol=1e-9, atol=1e-7)  # radii are stored as float32
    np.testing.assert_allclose(r[1], expect, rtol=1e-9, atol=1e-7)
    np.testing.assert_allclose(r[2:], np.broadcast_to(1e6 - spec.collision_sphere_radii.astype(np.float32), (2, ns)),
                               rtol=1e-6)


def _qmul(a, b):
    w1, x1, y1, z1 = a
    w2, x2, y2, z2 = b
    return np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2])


def _qrot(q, v):
    return _qmul(_qmul(q, np.r_[0.0, v]), q * [1, -1, -1, -1])[1:]


def test_oracle_base_reference_term_matches_finite_differences(panda_spec):
    """Floating-base reference rows w (.) log(T_base T_ref^-1): the base block of the Jacobian agrees with
    central differences under the right-multiplied base update, the joint columns are zero, and the rows
    vanish at the reference."""
    spec = panda_spec
    rob = oracle.Robot.from_spec(spec)
    na = spec.num_actuated_joints
    q = spec.midrange_q[None].astype(np.float32)
    ref = np.array([[0.2, -0.1, 0.3, 0.8, 0.3, -0.4, 0.2]])
    ref[:, 3:] /= np.linalg.norm(ref[:, 3:])
    w = np.array([1.0, 2.0, 0.5, 1.5, 0.7, 3.0])
    terms = oracle.Terms([dict(kind=9, weights=w, targets=ref.astype(np.float32), target_rows=1)])
    assert oracle.residual_dim(rob, terms) == 6
    base = np.array([0.5, 0.3, -0.2, 0.6, -0.2, 0.5, 0.4])
    base[3:] /= np.linalg.norm(base[3:])
    r, J = oracle.residual_jacobian(rob, terms, q, base[None].astype(np.float32))
    assert J.shape == (1, 6, 6 + na) and not np.any(J[0][:, 6:])
    eps = 1e-4

    def moved(c, s):
        t, qb = base[:3].copy(), base[3:].copy()
        if c < 3:
            e = np.zeros(3)
            e[c] = s * eps
            t = t + _qrot(qb, e)
        else:
            e = np.zeros(3)
            e[c - 3] = 1.0
            qb = _qmul(qb, np.r_[np.cos(s * eps / 2), np.sin(s * eps / 2) * e])
        return np.r_[t, qb][None].astype(np.float64)

    for c in range(6):
        rp, _ = oracle.residual_jacobian(rob, terms, q, moved(c, 1))
        rm, _ = oracle.residual_jacobian(rob, terms, q, moved(c, -1))
        np.testing.assert_allclose(J[0][:, c], (rp[0] - rm[0]) / (2 * eps), atol=2e-3)
    r0, _ = oracle.residual_jacobian(rob, terms, q, ref.astype(np.float32))
    assert np.abs(r0).max() < 1e-6
