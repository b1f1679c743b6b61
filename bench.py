#!/usr/bin/env python
"""Converged IK solves/s of the batched LM-IK path on B200.

Workload (default): the 7-DoF serial chain with 24 collision spheres — 16384
independent problems, pose target + sphere self-collision (every non-adjacent
sphere pair, margin 0.02 m) + joint-limit hinge, 10 % of targets pushed 0.3 m
beyond the workspace, 100 LM iterations with a per-problem stop once the step
norm falls below 1e-6.  A *step* is one full batched solve.  A problem counts
as converged when its final pose error is <= 1 mm and <= 0.01 rad.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU is replicas only (problems are independent; no collective on the
data path): each rank solves its own batch and rank 0 reports the aggregate.
"""

from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged IK solves/s on 1 B200 at <=1 mm/0.01 rad"
UNIT = "solves/s"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--config", default="chain7c")
    p.add_argument("--batch", type=int, default=0)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--pair-mode", choices=["all", "slots"], default="all")
    p.add_argument("--form", choices=["persistent", "plain"], default="persistent")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--lanes", type=int, default=0, help="lanes per problem (0 = automatic, 1, 8, 16 or 32)")
    p.add_argument("--no-plain", action="store_true", help="skip the plain-form comparison run")
    p.add_argument("--no-serve", action="store_true", help="skip the mixed-stream serving comparison")
    p.add_argument("--no-ik", action="store_true", help="skip the IKSolver preset benchmark")
    p.add_argument("--serve-rate", type=float, default=100000.0, help="mixed stream arrival rate, problems/s")
    p.add_argument("--serve-seconds", type=float, default=1.0, help="mixed stream duration")
    p.add_argument("--serve-sweep", default="", help="comma-separated rates: print one serving line per rate")
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU work of the baseline sample")
    return p.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (host side only: barrier + max/sum over ranks)
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def reduce(self, values, op):
        if self.world == 1:
            return values
        import torch

        t = torch.tensor(values, dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.SUM)
        return t.tolist()

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi samples (every 50 ms) kept for the wall-clock windows of the timed regions."""

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None
        self.windows = []

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            t_end = time.time() + 5.0
            while time.time() < t_end and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def mark(self, t0: float, t1: float) -> None:
        """Record one timed window [t0, t1] in host wall-clock seconds."""
        self.windows.append((t0, t1))

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(f[2]), float(f[3]), [n for n, v in zip(names, f[6:10])
                                                              if v.lower() == "active"]))
            except ValueError:
                continue
        os.unlink(self.path)
        inside = [r for r in rows if any(a - 0.06 <= r[0] <= b + 0.06 for a, b in self.windows)]
        scope = "timed region"
        if not inside:  # windows shorter than the sampling period: the whole loaded span
            inside, scope = rows, "warm-up + timed region (timed windows shorter than the 50 ms sampling)"
        sm = [r[1] for r in inside]
        reasons = sorted({n for r in inside for n in r[3]})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(r[2] for r in inside)) if inside else None,
                "reasons": reasons, "samples": len(sm), "scope": scope}


# ---------------------------------------------------------------------------
# the B200 arm
# ---------------------------------------------------------------------------
def converged_mask(N, cfg, q, base, pos=1e-3, rot=0.01):
    """ik_metrics on the GPU: every target within pos [m] and rot [rad]."""
    wl = cfg.workload
    B = cfg.batch
    nt = len(wl.target_links)
    links = N.DeviceArray.from_numpy(np.asarray(wl.target_links, np.int32))
    tg = N.DeviceArray.from_numpy(wl.targets.reshape(B, nt, 7))
    pe = N.DeviceArray.empty((B, nt))
    re = N.DeviceArray.empty((B, nt))
    ok = N.DeviceArray.empty(B, np.int32)
    N.check(N.lib().ik_metrics(cfg.robot.handle, B, q.ptr, N.ptr(base), nt, links.ptr, tg.ptr, pos, rot, pe.ptr,
                               re.ptr, ok.ptr, None))
    return ok.numpy().astype(bool), pe.numpy(), re.numpy()


def _measured_hbm_gbs():
    """HBM copy bandwidth measured on this pool (driver-written file), else the recipe's fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


def _profiled_traffic(args, B):
    """DRAM bytes per launch from the committed ncu summary, for the workload it was captured on."""
    if args.config != "chain7c" or args.form != "persistent" or args.pair_mode != "all":
        return None
    try:
        with open(os.path.join(ROOT, "profiles", "lm_persistent_kernel_chain7c.md")) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    v = int(line.split(":")[1].split()[0])
                    return v if B == 16384 else None
    except OSError:
        pass
    return None


def time_solves(N, opt, vv, q_work, q0_dev, steps, warmup, flush, clocks=None):
    """Device-resident timing, L2 flushed between steps, CUDA events on the launching stream.

    Returns (ms per step, ms per solve launch, library kernel launches in the timed region): a step is the
    on-device reset of q to the start point plus one whole solve."""
    ev0, ev1, ev2 = N.Event(), N.Event(), N.Event()
    for _ in range(warmup):
        q_work.assign(q0_dev)
        opt.solve(vv)
    N.synchronize()
    launches0 = N.launch_count()
    total = solve = 0.0
    t0 = time.time()
    for _ in range(steps):
        flush.zero_()
        N.synchronize()
        ev0.record()
        q_work.assign(q0_dev)
        ev1.record()
        opt.solve(vv)
        ev2.record()
        N.synchronize()
        total += ev0.elapsed_ms(ev2)
        solve += ev1.elapsed_ms(ev2)
    if clocks is not None:
        clocks.mark(t0, time.time())
    launches = N.launch_count() - launches0
    return total / steps, solve / steps, launches


def run_b200(args, dist: Dist) -> dict:
    from robokit_b200 import _native as N
    from robokit_b200 import configs
    from robokit_b200.flops import work_model
    from robokit_b200.opt import LMOptimizer, LMOptimizerConfig, VarKey, VarValues

    N.load_library()
    ndev = N.device_count()
    if ndev < 1:
        raise SystemExit("no CUDA device")
    N.check(N.lib().ik_set_device(dist.local_rank % ndev))
    import ctypes

    p32, p64 = ctypes.c_float(), ctypes.c_float()
    N.check(N.lib().ik_measure_fma_peak(0, ctypes.byref(p32)))
    N.check(N.lib().ik_measure_fma_peak(1, ctypes.byref(p64)))

    cfg = configs.make(args.config, args.batch or None, seed=args.seed + dist.rank, pair_mode=args.pair_mode,
                       form=args.form)
    wl = cfg.workload
    B = cfg.batch
    floating = wl.base0 is not None
    state = cfg.robot.state(wl.q0, wl.base0)
    q0_dev = state.q.clone()
    vv = VarValues({VarKey.ROBOT: state})
    opt = LMOptimizer(cfg.terms, cfg.lm)
    if args.lanes:
        opt.reset(vv)
        opt.set_schedule(args.lanes)
    flush = N.DeviceArray.empty(256 * 1024 * 1024 // 4)  # 256 MiB > 126 MB L2

    clocks = Clocks(dist.local_rank % ndev)
    dist.barrier()
    clocks.start()
    ms, ms_kernel, launches = time_solves(N, opt, vv, state.q, q0_dev, args.steps, args.warmup, flush, clocks)
    ms_max = dist.reduce([ms], "max")[0]

    ok, pe, re = converged_mask(N, cfg, state.q, state.T_world_base if floating else None)
    iters = opt.iterations.numpy()
    status = opt.status.numpy()
    accepts = status >> 8
    n_conv = int(ok.sum())
    conv_total, batch_total = dist.reduce([float(n_conv), float(B)], "sum")
    value = conv_total / (ms_max * 1e-3)

    # roofline: FP32 + FP64 CUDA-core work of this solve against the measured FMA peaks
    descs = configs.oracle_terms(cfg)
    # active collision rows per linearisation, estimated at the solution
    act_rows = 0.0
    coll = [t for t in cfg.terms if t.__class__.__name__ == "SelfCollisionTask"]
    if coll:
        from robokit_b200.terms.task import NativeProblem

        prob = NativeProblem(cfg.robot, coll, B, floating, None)
        r = N.DeviceArray.empty((B, prob.residual_dim))
        N.check(N.lib().ik_residual_jacobian(prob.handle, B, state.q.ptr,
                                             state.T_world_base.ptr if floating else None, r.ptr, None, None))
        act_rows = float(np.mean(np.sum(r.numpy() > 0, axis=1)))
    wm = work_model(wl.spec, descs, floating, act_rows)
    f32, f64 = wm.solve_flops(iters, accepts)
    t_s = ms_kernel * 1e-3
    peak_eff = (f32 + f64) / (f32 / (p32.value * 1e12) + f64 / (p64.value * 1e12)) / 1e12
    achieved = (f32 + f64) / t_s / 1e12
    # HBM side: bytes the solve must move (start point and targets in, solution and scalars out)
    n_pose = sum(1 for t in cfg.terms if hasattr(t, "T_world_target"))
    state_floats = wl.q0.shape[1] + (7 if floating else 0)
    alg_bytes = B * (4 * 2 * state_floats + 4 * 7 * len(wl.target_links) * n_pose + 4 * 4)
    hbm_peak = _measured_hbm_gbs()
    roofline = {
        "bound": "fp32",
        "achieved": round(achieved, 3),
        "peak": round(peak_eff, 3),
        "unit": "TFLOP/s",
        "frac": round(achieved / peak_eff, 4),
        "traffic": _profiled_traffic(args, B),
        "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of this launch "
                          "(profiles/lm_persistent_kernel_chain7c.md)",
        "hbm": {"algorithmic_bytes": int(alg_bytes), "achieved_gbs": round(alg_bytes / t_s / 1e9, 2),
                "peak_gbs": hbm_peak, "frac": round(alg_bytes / t_s / 1e9 / hbm_peak, 6) if hbm_peak else None},
        "peak_source": "measured FMA-chain FP32 %.1f / FP64 %.1f TFLOP/s (ik_measure_fma_peak), "
                       "weighted by this solve's FP32/FP64 work" % (p32.value, p64.value),
        "flops_fp32": f32,
        "flops_fp64": f64,
    }

    # end to end through the public API with host buffers: pinned q0 + targets in, q + cost out
    pin_q0 = N.PinnedBuffer(wl.q0.shape)
    pin_q0.array[:] = wl.q0
    pose_terms = [t for t in cfg.terms if hasattr(t, "T_world_target")]
    pin_t = N.PinnedBuffer(wl.targets.shape)
    pin_t.array[:] = wl.targets
    pin_q = N.PinnedBuffer(wl.q0.shape)
    pin_c = N.PinnedBuffer((B,))
    ev0, ev1 = N.Event(), N.Event()
    e2e_ms = 0.0
    bi = pin_q0.array.nbytes + len(pose_terms) * pin_t.array.nbytes
    bo = pin_q.array.nbytes + pin_c.array.nbytes
    for k in range(args.warmup + args.steps):
        if k == args.warmup:
            t_e2e = time.time()
        flush.zero_()
        N.synchronize()
        ev0.record()
        N.check(N.lib().ik_memcpy_htod(state.q.ptr, pin_q0.ptr, pin_q0.array.nbytes, None))
        for t in pose_terms:
            N.check(N.lib().ik_memcpy_htod(t.T_world_target.ptr, pin_t.ptr, pin_t.array.nbytes, None))
        opt.solve(vv)
        N.check(N.lib().ik_memcpy_dtoh(pin_q.ptr, state.q.ptr, pin_q.array.nbytes, None))
        N.check(N.lib().ik_memcpy_dtoh(pin_c.ptr, opt.costs.ptr, pin_c.array.nbytes, None))
        ev1.record()
        N.synchronize()
        if k >= args.warmup:
            e2e_ms += ev0.elapsed_ms(ev1)
    clocks.mark(t_e2e, time.time())
    clk = clocks.stop()
    e2e_ms /= args.steps
    e2e_max = dist.reduce([e2e_ms], "max")[0]
    e2e = {"value": round(conv_total / (e2e_max * 1e-3), 1), "unit": UNIT, "h2d_bytes_per_step": int(bi),
           "d2h_bytes_per_step": int(bo), "ms_per_step": round(e2e_max, 4)}

    # the plain form (one launch per iteration over the fixed batch) on the same workload
    plain = None
    if not args.no_plain and args.form != "plain":
        lm_plain = LMOptimizerConfig(**{**cfg.lm.__dict__, "form": "plain"})
        opt_p = LMOptimizer(cfg.terms, lm_plain)
        st_p = cfg.robot.state(wl.q0, wl.base0)
        vvp = VarValues({VarKey.ROBOT: st_p})
        if args.lanes:
            opt_p.reset(vvp)
            opt_p.set_schedule(args.lanes)
        ms_p, _, launches_p = time_solves(N, opt_p, vvp, st_p.q, q0_dev, max(3, args.steps // 2), 3, flush)
        ms_p = dist.reduce([ms_p], "max")[0]
        okp, _, _ = converged_mask(N, cfg, st_p.q, st_p.T_world_base if floating else None)
        convp = dist.reduce([float(okp.sum())], "sum")[0]
        plain = {"value": round(convp / (ms_p * 1e-3), 1), "ms_per_step": round(ms_p, 4),
                 "launches_per_step": launches_p // max(3, args.steps // 2),
                 "speedup_persistent_over_plain": round(ms_p / ms_max, 3)}
        # the same plain solve recorded once as a CUDA graph and replayed (cuda_graph_mode "full")
        lm_pg = LMOptimizerConfig(**{**cfg.lm.__dict__, "form": "plain", "cuda_graph_mode": "full"})
        opt_pg = LMOptimizer(cfg.terms, lm_pg)
        st_pg = cfg.robot.state(wl.q0, wl.base0)
        vvg = VarValues({VarKey.ROBOT: st_pg})
        if args.lanes:
            opt_pg.reset(vvg)
            opt_pg.set_schedule(args.lanes)
        ms_g, _, _ = time_solves(N, opt_pg, vvg, st_pg.q, q0_dev, max(3, args.steps // 2), 3, flush)
        ms_g = dist.reduce([ms_g], "max")[0]
        plain["graph_ms_per_step"] = round(ms_g, 4)

    g, bps = opt.problem.schedule()
    out = {
        "metric": METRIC,
        "value": round(value, 1),
        "unit": UNIT,
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_max, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32+fp64",
        "data": "synthetic (seeded generator of the configuration's distributions)",
        "config": {
            "workload": f"{args.config}: {B} problems/rank, 7-DoF chain + 24 spheres, pose + self-collision "
                        f"({args.pair_mode} pairs) + joint limits, 100 it, step stop 1e-6"
            if args.config == "chain7c" else f"{args.config}: {B} problems/rank",
            "problems": int(batch_total),
            "form": args.form,
            "group_lanes": g,
            "l2": "flushed between steps (256 MiB write)",
            "parallelism": f"replicas x{dist.world}",
        },
        "converged": int(conv_total),
        "converged_frac": round(conv_total / batch_total, 4),
        "mean_iterations": round(float(iters.mean()), 2),
        "e2e": e2e,
        "roofline": roofline,
        "gpu_launches": int(launches),
        "gpu_launches_per_step": int(launches // args.steps),
        "clocks": clk,
    }
    if plain is not None:
        out["plain"] = plain
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(cfg, args.cpu_seconds, samples_only=False)
    if dist.world == 1 and not args.no_serve:
        out["serving"] = serve_compare(args.serve_rate, args.serve_seconds, args.seed)
    if dist.world == 1 and not args.no_ik:
        out["ik_solver"] = ik_solver_bench()
    return out


# the reference's published IKSolver(presets.basic) times on an RTX 4090 (scripts/benchmark/ik/results.csv)
REFERENCE_IK_MS = {1: 0.646, 10: 0.610, 100: 0.813, 1000: 3.410, 2000: 7.124}


def _panda_arm():
    """The 7-DoF Panda of the reference's IK benchmark (finger joints fixed), from the committed fixture."""
    from robokit_b200.robo.robot_spec import JointRecord, RobotSpec

    with open(os.path.join(ROOT, "tests", "golden", "panda_golden.json")) as f:
        g = json.load(f)["robot"]
    joints = [JointRecord(**({**j, "type": "fixed", "mimic_joint": None} if j["type"] == "prismatic" else j))
              for j in g["joints"]]
    return RobotSpec.from_records(g["name"], g["links"], joints)


def ik_solver_bench(batches=(1, 10, 100, 1000, 2000), runs: int = 5) -> dict:
    """IKSolver(presets.basic) on FK-sampled Panda targets, the protocol of scripts/benchmark/ik/helper.py:124-160:
    fresh targets per run, wall time of one batched solve (synchronised), success at 5 mm / 0.05 rad, 98th
    percentile errors of the successful instances."""
    from robokit_b200 import _native as N
    from robokit_b200.helpers.ik import IKSolver, presets
    from robokit_b200.robo.robot import Robot

    spec = _panda_arm()
    robot = Robot(spec)
    link = spec.link_names.index("panda_hand")
    rows = []
    for B in batches:
        ik = IKSolver(presets.basic, robot, "panda_hand")
        targets = []
        for r in range(runs):
            q = robot.sample_q(B, seed=42 + r)
            st = robot.forward_kinematics(robot.state(q))
            targets.append(np.ascontiguousarray(st.get_T_world_link(link).numpy().reshape(B, 1, 7)))
        ik.solve(targets[0])
        N.synchronize()
        times, succ, pos, rot = [], [], [], []
        for T in targets:
            t0 = time.perf_counter()
            sol = ik.solve(T)
            N.synchronize()
            times.append((time.perf_counter() - t0) * 1e3)
            m = ik.compute_metrics_numpy(sol, T)
            ok = m.success
            succ.append(100.0 * ok.mean())
            if ok.any():
                pos.append(float(np.percentile(m.position_error_m[ok, 0], 98)) * 1e3)
                rot.append(float(np.percentile(m.orientation_error_rad[ok, 0], 98)))
        ms = float(np.mean(times))
        rows.append({"batch": B, "time_ms": round(ms, 4), "time_ms_std": round(float(np.std(times)), 4),
                     "solves_per_s": round(B / (ms * 1e-3), 1), "success_pct": round(float(np.mean(succ)), 3),
                     "pos_err_mm_p98": round(float(np.mean(pos)), 6) if pos else None,
                     "ori_err_rad_p98": round(float(np.mean(rot)), 7) if rot else None,
                     "reference_rtx4090_time_ms": REFERENCE_IK_MS.get(B)})
    return {"workload": "IKSolver(presets.basic: 64 -> 4 -> 1 candidates, 6 + 10 LM iterations) on the 7-DoF Panda, "
                        "one FK-sampled pose target per instance (target link panda_hand; the reference's benchmark "
                        "uses panda_hand_tcp, 0.1034 m further along the hand axis), 5 runs per batch",
            "rows": rows}


def serve_compare(rate: float, seconds: float, seed: int) -> dict:
    """The mixed stream: four robots, log-uniform batch sizes in [1, 4096], Poisson arrivals of `rate`
    problems/s, stop at 1e-4 m / 1e-3 rad or 100 iterations; served persistent form vs plain batches."""
    from robokit_b200 import serve

    types = serve.mixed_types(pool=4096, seed=seed)
    srv = serve.make_server(types, slots=16384)
    serve.run_served(srv, types, serve.make_stream(types, max(rate, 50000.0), 0.2, seed=seed + 1000))  # warm-up
    # at low rates, stretch the stream (up to 10 s) so that it holds about 50 requests
    seconds = max(seconds, min(10.0, 50 * 4095 / np.log(4096) / rate))
    reqs = serve.make_stream(types, rate, seconds, seed=seed)
    served = serve.run_served(srv, types, reqs)
    srv.close()
    plain = serve.run_plain(types, reqs)
    return {
        "stream": f"4 robots (chain7, chain7c, humanoid, hand), Poisson {rate:.0f} problems/s for {seconds} s, "
                  "batch log-uniform [1, 4096], stop 1e-4 m / 1e-3 rad, cap 100 iterations",
        "rate": rate,
        "served": served,
        "plain": plain,
        "converged_per_s_served_over_plain": round(served["converged_per_s"] / max(plain["converged_per_s"], 1e-9),
                                                   3),
    }


# ---------------------------------------------------------------------------
# CPU: the FP64 oracle port of the reference algorithm (all host threads)
# ---------------------------------------------------------------------------
def _oracle_solve(cfg, idx, threads):
    import oracle
    from robokit_b200 import configs

    wl = cfg.workload
    lm = cfg.lm
    rob = oracle.Robot.from_spec(wl.spec)
    descs = configs.oracle_terms(cfg)
    for d in descs:
        if "targets" in d:
            d["targets"] = d["targets"][idx]
            d["target_rows"] = len(idx)
    rules = (2 if lm.step_tol else 0) | (4 if lm.pose_tol else 0)
    prm = oracle.params(max_iter=lm.max_iter, lambda_init=lm.lm_lambda, lambda_factor=lm.lambda_factor,
                        lambda_min=lm.lambda_min, lambda_max=lm.lambda_max, rho_min=lm.rho_min,
                        gain_ratio_epsilon=lm.gain_ratio_epsilon, stop_rules=rules, step_tol=lm.step_tol or 0.0)
    terms = oracle.Terms(descs)
    base0 = None if wl.base0 is None else wl.base0[idx]
    t0 = time.perf_counter()
    out = oracle.solve(rob, terms, prm, wl.q0[idx], base0, threads=threads)
    dt = time.perf_counter() - t0
    pe, re, ok = oracle.metrics(rob, out["q"], out["base"], wl.target_links, wl.targets[idx], 1e-3, 0.01)
    return dt, int(ok.sum())


def _sample_size(cfg, seconds, threads):
    B = cfg.batch
    n = min(B, max(64, threads * 16))
    dt, _ = _oracle_solve(cfg, np.arange(n), threads)
    per = dt / n
    return int(min(B, max(n, seconds / max(per, 1e-9))))


def cpu_baseline(cfg, seconds, samples_only=False) -> dict:
    import oracle

    oracle.build()
    threads = os.cpu_count() or 1
    n = _sample_size(cfg, seconds, threads)
    idx = np.arange(n)
    dt, conv = _oracle_solve(cfg, idx, threads)
    return {"value": round(conv / dt, 1), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {n} of the {cfg.batch} problems, FP64 C port of the reference LM (oracle/), "
                      f"{threads} threads, {dt:.1f} s"}


def run_reference(args, dist: Dist) -> dict:
    from robokit_b200 import configs

    if dist.rank != 0:
        return {}
    import oracle

    oracle.build()
    cfg = configs.make(args.config, args.batch or None, seed=args.seed, pair_mode=args.pair_mode)
    threads = os.cpu_count() or 1
    per_step = max(5.0, min(args.cpu_seconds, 150.0 / max(1, args.steps + args.warmup)))
    n = _sample_size(cfg, per_step, threads)
    idx = np.arange(n)
    for _ in range(args.warmup):
        _oracle_solve(cfg, idx, threads)
    tot, conv = 0.0, 0
    for _ in range(args.steps):
        dt, conv = _oracle_solve(cfg, idx, threads)
        tot += dt
    ms = tot / args.steps * 1e3
    value = conv / (ms * 1e-3)
    sample = (f"first {n} of the {cfg.batch} problems per step, FP64 C port of the reference LM (oracle/): "
              f"the reference itself needs warp-lang, absent here")
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 1),
        "unit": UNIT,
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp64",
        "data": "synthetic (seeded generator of the configuration's distributions)",
        "config": {"workload": f"{args.config}: {n} problems per step (bounded CPU sample)", "problems": n},
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    dist = Dist()
    try:
        if args.serve_sweep and args.impl == "b200":
            from robokit_b200 import _native as N

            N.load_library()
            N.check(N.lib().ik_set_device(dist.local_rank))
            for rate in [float(x) for x in args.serve_sweep.split(",") if x]:
                line = serve_compare(rate, args.serve_seconds, args.seed)
                if dist.rank == 0:
                    print(json.dumps({"serving_sweep": line}), flush=True)
            return
        out = run_reference(args, dist) if args.impl == "reference" else run_b200(args, dist)
        if dist.rank == 0 and out:
            print(json.dumps(out), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
