"""Algorithmic work model of one LM-IK problem, for the roofline.

Counts are floating-point operations of the algorithm as the fused kernel runs
it (idle lanes and integer index work excluded); sin, cos, atan2, asin, sqrt
and divide count one each.  One problem-iteration costs

    solve (FP64)  + integrate + eval(proposal)        every iteration
    linearise                                          after every accepted step (+1 at the start)

so a solve costs  iters * (F64_solve + F32_integrate + F32_eval)
                + (accepts + 1) * F32_lin  + F32_eval(start).

Per-operation counts: quaternion product 28, quaternion rotation of a vector
30, pose composition 61; revolute local transform 67, prismatic 64; world
sphere 33; position residual 12, rotation residual 77, each squared row into
the compensated cost 5; joint-limit row 11; sphere-pair distance test 12;
motion-subspace column 39; Jacobian entry 12 per contributing joint + 15
(position) or 3 (rotation); collision Jacobian entry 34 per contributing joint
+ 12 for the normal; J^T J + J^T r 2 (T + D) per row plus a 4-flop compensated
merge of every entry per 32-row chunk; FP64 Cholesky sum_k [2 + (D-k-1) +
(D-k-1)(D-k)] plus 2 D^2 for the triangular solves and 5 D for the predicted
reduction and step norm.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, List, Sequence

import numpy as np

QMUL, QROT = 28, 30
COMPOSE = QMUL + QROT + 3
LOCAL = {0: 0, 1: 3 + COMPOSE, 2: 6 + COMPOSE}
SPHERE = QROT + 3
POS_RES, ROT_RES, COST_ROW = 12, 77, 5
LIMIT_ROW = 11
PAIR_TEST = 12
SUBSPACE = QROT + 9
CHUNK = 32


@dataclass
class WorkModel:
    eval32: float      # one residual evaluation (FK, spheres, residuals, cost)
    lin32: float       # one linearisation (subspace, Jacobian, J^T J / J^T r)
    solve64: float     # one damped FP64 solve
    integrate32: float

    def solve_flops(self, iters: np.ndarray, accepts: np.ndarray) -> tuple:
        """(FP32 flops, FP64 flops) of solves that ran `iters` iterations with `accepts` accepted steps."""
        it = np.asarray(iters, np.float64)
        ac = np.asarray(accepts, np.float64)
        f32 = float(np.sum(it * (self.integrate32 + self.eval32) + (ac + 1) * self.lin32 + self.eval32))
        f64 = float(np.sum(it * self.solve64))
        return f32, f64


def _fk_composes(spec: Any, floating: bool) -> int:
    parent = list(spec.parent_joint_indices)
    anc = list(parent)
    n = 0
    while any(a >= 0 for a in anc):
        n += sum(1 for a in anc if a >= 0)
        anc = [anc[a] if a >= 0 else -1 for a in anc]
    return n + (len(parent) if floating else 0)


def work_model(spec: Any, term_descs: Sequence[dict], floating: bool, active_collision_rows: float = 0.0) -> WorkModel:
    """Work of one problem of robot `spec` under the lowered terms (the IkTermDesc fields)."""
    nj = spec.num_joints
    D = (6 if floating else 0) + spec.num_actuated_joints
    T = D * (D + 1) // 2
    E = T + D
    types = list(spec.joint_types)
    fk = sum(LOCAL[int(t)] for t in types) + COMPOSE * _fk_composes(spec, floating)
    anc = spec.link_ancestor_joints_mask
    contrib = spec.joints_to_actuated_mapping != 0  # [nj, na]
    ev = fk
    lin = SUBSPACE * sum(1 for t in types if t != 0)
    has_coll = any(d["kind"] == 4 for d in term_descs)
    if has_coll:
        ev += SPHERE * len(spec.collision_sphere_radii)
    rows = 0
    for d in term_descs:
        k = d["kind"]
        if k in (1, 2):
            links = list(d["frame_links"])
            ev += len(links) * ((POS_RES if k == 1 else ROT_RES) + 3 * COST_ROW)
            for li in links:
                # columns: base (QROT each, +cross for angular) + actuated (12 per contributing ancestor joint)
                per = 0
                if floating:
                    per += 3 * QROT + 3 * (QROT + 9)
                for a in range(spec.num_actuated_joints):
                    per += 12 * int(np.sum(contrib[:, a] & anc[li]))
                per += D * (15 if k == 1 else 3)
                lin += per
            rows += 3 * len(links)
        elif k == 3:
            ev += LIMIT_ROW * spec.num_actuated_joints
            lin += 6 * spec.num_actuated_joints
        elif k == 4:
            nsp = d["num_sphere_pairs"]
            if d["pair_mode"] == 1:
                ev += PAIR_TEST * nsp
            else:
                nlp = d["num_link_pairs"]
                ev += PAIR_TEST * nlp + SPHERE * spec.num_links
                ev += PAIR_TEST * nsp  # narrow phase: at most every pair of the kept link pairs
            # active rows: normal + per-joint terms over the two links' ancestors
            lin += active_collision_rows * (12 + 34 * max(1, int(np.mean(np.sum(anc, axis=1)))) * 2)
    rows_lin = rows + active_collision_rows
    lin += 2 * (T + D) * rows_lin + 4 * E * max(1, int(np.ceil(rows_lin / CHUNK)))
    chol = sum(2 + (D - k - 1) + (D - k - 1) * (D - k) for k in range(D))
    solve64 = chol + 2 * D * D + 5 * D
    integ = spec.num_actuated_joints + (110 if floating else 0)
    return WorkModel(eval32=float(ev), lin32=float(lin), solve64=float(solve64), integrate32=float(integ))
