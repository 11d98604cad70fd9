#!/usr/bin/env python
"""RK4 time-step throughput of the kielflow hot path on B200.

Workload (default ``fp32bulk256``): one RK4 step of the full right-hand side
(R2C/C2R 3-D FFTs, 2/3 dealiasing, advection, continuity, E-force, pressure,
friction, spectral viscosity beyond 0.6 k_max, Laplacian diffusion,
penalization) and four FP64 nonlinear Poisson solves (FAS V-cycles, 4 levels,
2+2 red-black point-Newton sweeps, residual <= 1e-10) on a 256^3 periodic box,
FFTs / products / RK4 stages in FP32.  Metric: RK4 steps/s, with the plain
FP64 path on the same workload and the relative phi error between the two.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs under torchrun, one independent replica (seed = rank) per GPU
("replicas only": a single grid does not shard here); timing is the max over
ranks of CUDA-event time on each rank's stream.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK4 steps/s at 256^3 FP32-bulk vs plain FP64 on B200 at stated phi error; adj/fwd"
UNIT = "steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kf", choices=["kf", "reference"])
    ap.add_argument("--workload", default="fp32bulk256")
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison arm")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default kernel variants (no kf_autotune; profiling runs)")
    ap.add_argument("--cpu-ref", default="", help=argparse.SUPPRESS)
    ap.add_argument("--rbgs-rows", type=int, default=-1,
                    help="force the smoother variant (kf_set_tuning rbgs_rows: 4, 8, 16, or 0 for the "
                         "streaming sweep) after the autotuner; -1 keeps the autotuner's choice")
    ap.add_argument("--coarse-block", type=int, default=1, choices=[0, 1],
                    help="kf_set_coarse_block: 1 (the default) runs the V-cycle's levels of at most "
                         "16^3 points in one shared-memory block, 0 level by level")
    ap.add_argument("--overlap", type=int, default=1, choices=[0, 1],
                    help="kf_set_overlap: 1 (the default) runs the u', s transforms of each stage beside "
                         "its Poisson solve, 0 after it")
    ap.add_argument("--profile-range", action="store_true",
                    help="bracket the first arm's profile steps (launched kernel by kernel, the same "
                         "kernels as the timed graph replays) with cudaProfilerStart/Stop, for "
                         "ncu --profile-from-start off; changes no work")
    ap.add_argument("--marks", default="100,500,2000", help="steps at which --workload precision compares")
    ap.add_argument("--sweep-steps", type=int, default=10,
                    help="RK4 steps per instance of the 48-instance sweep leg; 0 skips it")
    ap.add_argument("--adjoint-steps", type=int, default=200,
                    help="RK4 steps of the adjoint leg (128^3 FP64, checkpoints every 15); 0 skips it")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(gpu_index), "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [ln.strip().split(",") for ln in open(self.f.name) if ln.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        loaded = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str, workload: str, alg_bytes_per_launch: float):
    """DRAM bytes per launch of `kernel`: the ratio DRAM bytes / algorithmic
    bytes of one ncu capture of that kernel on this workload (profiles/
    ncu_traffic.json), applied to the average algorithmic bytes of its launches
    here (the capture is one launch of the finest level; the ratio carries to
    the others).  None when no capture exists."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p)).get(workload, {})
    v = d.get(kernel.split("(")[0].split("/")[0])
    if not v or not v.get("traffic_over_alg"):
        return None
    return float(v["traffic_over_alg"]) * alg_bytes_per_launch


# --------------------------------------------------------------------- CPU leg
class _QuietStdout:
    """Silence C-level stdout (the reference prints progress from its
    constructors, e.g. rhs_standard.cpp:32) so rank 0 prints one JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def workload_config(w, name, ws):
    """The config dict of a workload, shared by both arms of the bench."""
    from kielflow_b200 import configs as C
    cfg = C.config_for(w)
    st, nd, mask, dt = C.make_inputs(w)
    return {"workload": f"{name}: {w['n']}^3 box 2*pi*4, M {w['M']}, nu {w['tau']}, Q {w['Q']}, sigma {w['sigma']}, "
                        f"FAS {cfg.mg_levels} levels 2+2 to residual {cfg.res_tol:.3g} (FP32 bulk: 2^-23 max|n_d|; "
                        f"FP64: 1e-10; at most {cfg.max_cycles} V-cycles per solve), penalization, diffusion 1e-3, "
                        f"SV > 0.6 k_max",
            "n": w["n"], "dt": dt, "l2": "inputs larger than L2 (state + work buffers > 2 GB)",
            "axes": (f"axis_CoSiSt m {w['stretch']:.6g} (sine-stretched, chain-rule derivatives)"
                     if w.get("stretch") else "axis_CoEqSt"),
            "parallelism": f"replicas x{ws}"}


def oracle_rk4_seconds(w, n, steps, warmup, budget_s):
    """The CPU restatement of the path (oracle/, pinned to the reference's own
    sources) on the workload's physics at n^3 in FP64: seconds of each timed
    RK4 step, after `warmup` untimed steps, stopping once budget_s is spent
    (at least one timed step).  Runs on all host cores (KF_ORACLE_THREADS)."""
    from kielflow_b200 import configs as C
    from oracle import bind  # CPU baseline / reference arm only
    st, nd, mask, dt = C.make_inputs(w, n=n)
    from kielflow_b200._lib import KF_FP64
    cfg = C.config_for(w, n=n, precision=KF_FP64)  # the CPU path computes in double
    o = bind.Oracle(bind.KfoConfig(*[getattr(cfg, f) for f, _ in bind.KfoConfig._fields_]))
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rk4(dt, warmup)
    times, t_start = [], time.perf_counter()
    while len(times) < steps:
        t0 = time.perf_counter()
        o.rk4(dt, 1)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s:
            break
    return times, bind.lib().kfs_nthreads()


def cpu_baseline_entry(w, name):
    """Bounded CPU sample for the GPU arm's line: two RK4 steps of the oracle
    at 128^3 (after one untimed step), scaled to 256^3 by N log N."""
    n_s, n_f = 128, w["n"]
    times, cores = oracle_rk4_seconds(w, n_s, 2, 1, 60.0)
    t = statistics.mean(times)
    scale = (n_f / n_s) ** 3 * (math.log(n_f) / math.log(n_s))
    return {"value": 1.0 / (scale * t), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"{len(times)} RK4 steps of the CPU restatement (oracle/kf_oracle.cpp, pinned to the "
                       f"reference's own rhs_standard/RKO4/solver sources) on the {name} physics at "
                       f"{n_s}^3 in FP64, mean {t:.2f} s on {cores} threads, scaled by N log N "
                       f"({scale:.2f}x) to {n_f}^3")}


def run_reference(args):
    """The reference arm: the CPU path on the GPU arm's own workload (the
    FP32-bulk workload's physics, computed in FP64 as the reference's FFTW path
    does), real RK4 steps at full size on all host cores."""
    from kielflow_b200 import configs as C
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import bind
    try:
        bind.lib()
    except OSError as e:
        print(json.dumps({"impl": "reference", "unavailable": f"oracle not built: {e}"}))
        return 0
    name = args.workload
    w = C.WORKLOADS[name]
    warm = min(args.warmup, 1)
    times, cores = oracle_rk4_seconds(w, w["n"], args.steps, warm, budget_s=150.0)
    tot = sum(times)
    v = len(times) / tot
    cb = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
          "sample": (f"{len(times)} full {w['n']}^3 RK4 steps (of {args.steps} requested; the timed region "
                     f"stops after 150 s) of the CPU restatement (oracle/kf_oracle.cpp, pinned to the "
                     f"reference's own sources: rhs_standard, RKO4, Poisson solvers, effect_penalization, "
                     f"effect_diffusion) on {cores} threads, FP64, after {warm} untimed step")}
    out = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": len(times),
           "steps_requested": args.steps, "warmup": warm, "ms_per_step": 1000.0 * tot / len(times),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(w, name, 1), "impl": "reference", "cpu_baseline": cb,
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


# --------------------------------------------------------------------- GPU arm
def adjoint_leg(nsteps: int, stream, ckpt_every: int = 15):
    """Cost of the discrete adjoint against its forward pass on the
    differentiation workload (128^3 FP64, M 0.9, nu 0.1, Q -20): device time
    of nsteps RK4 steps + J alone, and of the full gradient run (checkpointed
    forward pass, recomputation, reverse sweep), with and without the stored
    stage potentials."""
    import kielflow_b200 as kf
    from kielflow_b200 import configs as C

    w = C.WORKLOADS["adj128"]
    st, nd, mask, dt = C.make_inputs(w)
    win = C.wake_window(w["n"])
    with kf.Context(C.config_for(w)) as ctx:
        ctx.set_stream(stream.cuda_stream)
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.adjoint(win, 0, dt, 1, kf.KF_ADJ_J_ONLY, want_dn0=False)  # converged phi of the initial state
        phi0 = ctx.get_phi()

        def run(flags, steps):
            ctx.set_state(*st)
            ctx.set_phi(phi0)
            return ctx.adjoint(win, steps, dt, ckpt_every, flags, want_dn0=False)

        run(0, min(nsteps, 2 * ckpt_every))  # warm-up: buffers, graph capture
        f = run(kf.KF_ADJ_J_ONLY, nsteps)
        a = run(0, nsteps)
        b = run(kf.KF_ADJ_STORE_PHI, nsteps)
    tot_a, tot_b = a["fwd_ms"] + a["bwd_ms"], b["fwd_ms"] + b["bwd_ms"]
    return {"workload": f"adj128: {w['n']}^3 FP64, M {w['M']}, nu {w['tau']}, Q {w['Q']}, {nsteps} RK4 steps, "
                        f"checkpoints every {ckpt_every}; J = h^3 sum w phi_T, Gaussian window width 2 at (4,0,0)",
            "J": a["J"], "dJ_dM": a["dJ_dM"], "dJ_dtau": a["dJ_dtau"], "dJ_dQ": a["dJ_dnd"] / w["Q"],
            "forward_ms": f["fwd_ms"], "gradient_ms": tot_a, "adj_over_fwd": tot_a / f["fwd_ms"],
            "gradient_ms_store_phi": tot_b, "adj_over_fwd_store_phi": tot_b / f["fwd_ms"],
            "adjoint_poisson_solves": a["adj_solves"], "adjoint_v_cycles": a["adj_cycles"],
            "timing": "CUDA events on the context's stream (kf_grad_out fwd_ms/bwd_ms)"}


def run_kf(args):
    import numpy as np
    import torch

    import kielflow_b200 as kf
    from kielflow_b200 import configs as C

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    w = C.WORKLOADS[args.workload]
    st, nd, mask, dt = C.make_inputs(w, seed=rank)
    stream = torch.cuda.Stream()

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def timed_arm(precision, profile=False, clocks=False, prange=False):
        cfg = C.config_for(w, precision=precision)
        ctx = kf.Context(cfg)
        ctx.set_stream(stream.cuda_stream)
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        # radix plan and smoother shape, timed on this context
        tune = ctx.autotune() if not args.no_tune else {"fft_plan": 0, "rbgs_rows": 8,
                                                         "fft_radices": [[], []]}
        if args.rbgs_rows >= 0:
            ctx.set_tuning(tune["fft_plan"], args.rbgs_rows)
            tune = dict(tune, rbgs_rows=args.rbgs_rows)
        ctx.set_coarse_block(args.coarse_block == 1)
        ctx.set_overlap(args.overlap == 1)
        ctx.rk4(dt, args.warmup)
        ctx.synchronize()
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(torch.cuda.current_device()) if clocks else None
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.launch_count()
        with torch.cuda.stream(stream):
            e0.record(stream)
            ctx.rk4(dt, args.steps)
            e1.record(stream)
        stream.synchronize()
        torch.cuda.synchronize()
        barrier()
        launches = ctx.launch_count() - l0
        clk = sampler.stop() if sampler else None
        ms = max_over_ranks(e0.elapsed_time(e1))
        d = ctx.diag()
        phi = ctx.get_phi()  # after warm-up + timed steps in both precisions
        state = ctx.get_state()
        prof = None
        if profile:
            # per-kernel CUDA-event profile of further steps of the same run
            # (kernels launched one by one, each bracketed by events)
            ctx.profile(True)
            if prange:
                torch.cuda.synchronize()
                torch.cuda.profiler.start()
            ctx.rk4(dt, max(1, min(args.steps, 3)))
            if prange:
                torch.cuda.synchronize()
                torch.cuda.profiler.stop()
            prof = ctx.profile_read()
            ctx.profile(False)
        ctx.tune = tune
        return ctx, ms, launches, prof, clk, d, phi, state

    ctx32, ms32, launches, prof, clk, d32, phi32, st32 = timed_arm(w["precision"], profile=True, clocks=True,
                                                                      prange=args.profile_range)
    value = ws * args.steps / (ms32 / 1000.0)

    # end-to-end through the C ABI with host (pinned) buffers: H2D state, one
    # RK4 step, D2H state, every step (interface_ode_solver::solve semantics)
    shape_c = ctx32.shape_c
    host = [torch.empty(shape_c, dtype=torch.complex128, pin_memory=True).numpy() for _ in range(4)]
    for h, s in zip(host, st):
        h[...] = s
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.e2e_steps):
            ctx32.step_host(host, dt, 1)  # interface_ode_solver::solve on host arrays
        e1.record(stream)
    stream.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1))
    bytes_io = 4 * int(np.prod(shape_c)) * 16
    e2e = None
    if args.e2e_steps > 0:
        # this box's page-locked copy bandwidth, for reading the number
        hb = torch.empty(bytes_io // 8, dtype=torch.float64, pin_memory=True)
        db = torch.empty(bytes_io // 8, dtype=torch.float64, device="cuda")
        c0, c1, c2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        with torch.cuda.stream(stream):
            c0.record(stream)
            db.copy_(hb, non_blocking=True)
            c1.record(stream)
            hb.copy_(db, non_blocking=True)
            c2.record(stream)
        stream.synchronize()
        e2e = {"value": ws * args.e2e_steps / (ms_e2e / 1000.0), "unit": UNIT, "h2d_bytes_per_step": bytes_io,
               "d2h_bytes_per_step": bytes_io, "steps": args.e2e_steps,
               "call": "kf_step_host (interface_ode_solver::solve on page-locked host arrays)",
               "link_h2d_GBps": bytes_io / (c0.elapsed_time(c1) * 1e6),
               "link_d2h_GBps": bytes_io / (c1.elapsed_time(c2) * 1e6)}
        del hb, db
    tune32 = ctx32.tune
    ctx32.close()
    del ctx32

    fp64 = None
    if not args.no_fp64 and w["precision"] != kf.KF_FP64:
        ctx64, ms64, _, _, _, d64, phi64, st64 = timed_arm(kf.KF_FP64)
        tune64 = ctx64.tune
        ctx64.close()
        n_ = w["n"]

        def real(F):
            return np.fft.irfftn(F, s=(n_, n_, n_), axes=(0, 1, 2))

        def rel_linf(a, b):
            return float(np.abs(a - b).max() / np.abs(b).max())

        err = rel_linf(phi32, phi64)
        u32 = np.stack([real(x) for x in st32[:3]])
        u64 = np.stack([real(x) for x in st64[:3]])
        u32[0] += w["M"]
        u64[0] += w["M"]
        errs = {"phi": err, "n": rel_linf(np.exp(real(st32[3])), np.exp(real(st64[3]))), "u_total": rel_linf(u32, u64),
                "at_step": args.warmup + args.steps, "norm": "relative max-norm over the grid"}
        del u32, u64
        fp64 = {"value": ws * args.steps / (ms64 / 1000.0), "ms_per_step": ms64 / args.steps,
                "phi_rel_err_fp32_vs_fp64": max_over_ranks(err),
                "fp32_vs_fp64_errors": {k: (max_over_ranks(v) if isinstance(v, float) else v) for k, v in errs.items()},
                "charge_fp32": d32.charge, "charge_fp64": d64.charge,
                "kinetic_fp32": d32.kinetic, "kinetic_fp64": d64.kinetic,
                "tuning": {"fft_radices": tune64["fft_radices"][tune64["fft_plan"]],
                           "rbgs_rows": tune64["rbgs_rows"]}}

    adj = adjoint_leg(args.adjoint_steps, stream) if args.adjoint_steps > 0 else None
    sweep = sweep_leg(args, args.sweep_steps) if args.sweep_steps > 0 else None

    if rank != 0:
        if ws > 1:
            torch.distributed.destroy_process_group()
        return 0

    # roofline of the dominant kernel (largest share of profiled GPU time)
    peak, peak_kind = measured_peaks()
    total_ms = sum(v[0] for v in prof.values())
    dom, (dms, dn, dbytes) = max(prof.items(), key=lambda kv: kv[1][0])
    avg_ms = dms / dn
    achieved = (dbytes / dn) / (avg_ms / 1000.0) / 1e9
    traffic = ncu_traffic(dom, args.workload, dbytes / dn)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": traffic, "alg_bytes_per_launch": dbytes / dn, "avg_launch_ms": avg_ms,
                "share_of_gpu_time": dms / total_ms,
                "kernels": {k: {"ms": v[0], "launches": v[1], "GB/s": (v[2] / v[0] / 1e6 if v[0] else 0.0),
                                "share": v[0] / total_ms} for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}}

    cpu = None
    if not args.no_cpu and ws == 1:
        try:
            cpu = cpu_baseline_entry(w, args.workload)
        except OSError as e:
            cpu = {"unavailable": f"oracle not built: {e}"}

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 bulk + fp64 Poisson"
        if w["precision"] == kf.KF_FP32_BULK else "f64",
        "data": "synthetic (seeded noise, Gaussian dust; seed = rank)",
        "config": workload_config(w, args.workload, ws),
        "tuning": {"fft_radices": tune32["fft_radices"][tune32["fft_plan"]], "rbgs_rows": tune32["rbgs_rows"],
                   "rbgs_rows_meaning": "0: streaming TMA-staged sweep (k_rbgs_march)",
                   "coarse_block": args.coarse_block, "overlap": args.overlap},
        "gpu_launches": launches,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clk,
        "poisson": {"solves": d32.solves, "v_cycles": d32.total_iterations,
                    "last_residual": d32.last_residual, "not_converged": d32.not_converged},
        "fp64": fp64,
        "adjoint": adj,
        "sweep48": sweep,
    }
    print(json.dumps(out))
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def sweep_leg(args, steps: int):
    """The 48-instance sweep (16 each at 64^3, 96^3, 128^3): instance-steps/s
    with all of a rank's instances driven concurrently (kf_batch_rk4_steps),
    and the same instances one after another.  Instances are partitioned
    across ranks by cost; wall time is the max over ranks."""
    import torch

    from kielflow_b200 import dist as kdist
    from kielflow_b200.sweep import run_sweep, sweep_instances

    ws, rank, _ = dist_env()
    inst = sweep_instances(seed=0)
    mine = [inst[i] for i in kdist.partition([x.n for x in inst], ws)[rank]]
    if ws > 1:
        torch.distributed.barrier()
    tunings = {}
    wall_c, _, dg = run_sweep(mine, steps=steps, mode="batched", warmup=args.warmup, tunings=tunings)
    wall_c = kdist.max_over_ranks(wall_c, device="cuda")
    wall_s, _, _ = run_sweep(mine, steps=steps, mode="sequential", warmup=args.warmup, tune=tunings)
    wall_s = kdist.max_over_ranks(wall_s, device="cuda")
    total = len(inst) * steps
    return {"metric": "sweep instance-steps/s (48 instances, 64^3/96^3/128^3, FP32 bulk)",
            "value": total / wall_c, "unit": "instance-steps/s", "steps": steps, "warmup": args.warmup,
            "sequential_value": total / wall_s, "batched_over_sequential": wall_s / wall_c,
            "v_cycles_per_solve": (sum(d.total_iterations for d in dg) / max(1, sum(d.solves for d in dg))),
            "config": {"workload": "sweep48: 16 x 64^3, 16 x 96^3, 16 x 128^3; M ~ U[0.3,1.5], nu ~ U[0.01,0.3], "
                                   "Q ~ U[-50,-5], sigma 0.5 (seed 0); FP32 bulk, FP64 FAS Poisson to 2^-23 max|n_d|",
                       "timing": "host wall clock around fully synchronised runs, max over ranks; warm-up steps "
                                 "(graph capture) outside", "batched": "kf_batch_rk4_steps",
                       "sequential": "kf_rk4_steps per instance, one after another",
                       "tuning": {str(n): {"fft_radices": t["fft_radices"][t["fft_plan"]],
                                           "rbgs_rows": t["rbgs_rows"]} for n, t in sorted(tunings.items())}}}


def run_sweep_bench(args):
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    torch.cuda.set_device(local)
    out = sweep_leg(args, args.steps)
    if rank == 0:
        out.update({"n_gpus": ws, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                    "dtype": "fp32 bulk + fp64 Poisson", "data": "synthetic"})
        print(json.dumps(out))
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def cpu_reference_run(n: int, steps: int, workload: str):
    """The reference's own Runge_kutta_O4 + rhs_standard + cascadic multigrid
    (its sources compiled into oracle/_ref) for `steps` RK4 steps of the
    workload's initial state at n^3, one thread; prints seconds as JSON.  Run
    in a subprocess: the reference keeps one grid size per process."""
    from kielflow_b200 import configs as C
    from oracle import bind  # CPU baseline leg only
    if not bind.ref_available():
        print(json.dumps({"unavailable": "oracle/_ref not built"}))
        return 0
    w = C.WORKLOADS[workload]
    st, nd, mask, dt = C.make_inputs(w, n)
    with _QuietStdout():
        R = bind.Reference(n, C.L_BOX, w["M"], w["tau"], C.THETA, poisson_mode=1)
        R.set_real(0, nd)
        R.set_real(1, mask)
        R.set_state(st)
        t0 = time.perf_counter()
        R.rk4(dt, steps)
        sec = time.perf_counter() - t0
    print(json.dumps({"n": n, "steps": steps, "seconds": sec, "s_per_step": sec / steps}))
    return 0


def run_small(args):
    """The smaller configurations: plain FP64 GPU steps/s at 32^3 (Jacobi to
    1e-10) and 128^3 (FAS 4 levels 2+2), and the reference's CPU path on the
    same inputs (subprocesses, one core), for the baseline table."""
    import subprocess

    import kielflow_b200 as kf
    from kielflow_b200 import configs as C

    out = {"workload": "small", "gpu": {}, "cpu_reference": {}}
    for name, steps in (("jacobi32", 100), ("fas128", 20)):
        w = C.WORKLOADS[name]
        st, nd, mask, dt = C.make_inputs(w)
        with kf.Context(C.config_for(w)) as ctx:
            ctx.set_state(*st)
            ctx.set_sources(nd, mask)
            ctx.rk4(dt, 3)
            ctx.synchronize()
            t0 = time.perf_counter()
            ctx.rk4(dt, steps)
            ctx.synchronize()
            sec = time.perf_counter() - t0
        out["gpu"][name] = {"steps": steps, "seconds": sec, "steps_per_s": steps / sec,
                            "timing": "host wall clock around a synchronised run"}
    if not args.no_cpu:
        for name, n, steps in (("jacobi32", 32, 100), ("fas128", 128, 2)):
            r = subprocess.run([sys.executable, __file__, "--cpu-ref", f"{n},{steps},{name}"],
                               capture_output=True, text=True, timeout=900)
            line = [x for x in r.stdout.splitlines() if x.startswith("{")]
            out["cpu_reference"][name] = json.loads(line[-1]) if line else {"unavailable": r.stderr[-300:]}
        out["cpu_reference"]["note"] = ("the reference's own RK4 + rhs_standard + cascadic multigrid "
                                        "(kielflow.cpp's solver plan), single thread")
    print(json.dumps(out))
    return 0


def run_precision(args):
    """FP32 bulk against plain FP64 on the 256^3 precision workload: relative
    L2 and max-norm errors of n = exp(s), u' and phi after 100, 500 and 2000
    steps of the same seeded run."""
    import numpy as np

    import kielflow_b200 as kf
    from kielflow_b200 import configs as C

    w = C.WORKLOADS["fp32bulk256"]
    st, nd, mask, dt = C.make_inputs(w)
    n = w["n"]
    ctxs = {}
    for p in (kf.KF_FP32_BULK, kf.KF_FP64):
        c = kf.Context(C.config_for(w, precision=p))
        c.set_state(*st)
        c.set_sources(nd, mask)
        ctxs[p] = c
    marks = [int(x) for x in args.marks.split(",")]
    done, rows = 0, []

    def real(F):
        return np.fft.irfftn(F, s=(n, n, n), axes=(0, 1, 2))

    def errs(a, b):
        d = a - b
        return {"l2": float(np.sqrt((d * d).sum() / (b * b).sum())), "linf": float(np.abs(d).max() / np.abs(b).max())}

    for m in marks:
        for c in ctxs.values():
            c.rk4(dt, m - done)
        done = m
        s32, s64 = ctxs[kf.KF_FP32_BULK].get_state(), ctxs[kf.KF_FP64].get_state()
        row = {"step": m,
               "n": errs(np.exp(real(s32[3])), np.exp(real(s64[3]))),
               "u": errs(np.stack([real(x) for x in s32[:3]]), np.stack([real(x) for x in s64[:3]])),
               "phi": errs(ctxs[kf.KF_FP32_BULK].get_phi(), ctxs[kf.KF_FP64].get_phi())}
        rows.append(row)
        print(json.dumps(row), file=sys.stderr, flush=True)
    for c in ctxs.values():
        c.close()
    print(json.dumps({"workload": "precision: fp32bulk256 vs fp64_256, same seed", "dt": dt, "errors": rows,
                      "note": "u is the perturbation u' (relative to its own size)"}))
    return 0


def main():
    args = parse()
    if args.cpu_ref:
        n, steps, name = args.cpu_ref.split(",")
        return cpu_reference_run(int(n), int(steps), name)
    if args.workload == "small":
        return run_small(args)
    if args.workload == "precision":
        return run_precision(args)
    if args.workload == "adjoint":  # the adjoint leg alone (profiling runs)
        import torch
        print(json.dumps({"workload": "adjoint", "adjoint": adjoint_leg(args.adjoint_steps, torch.cuda.Stream())}))
        return 0
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "sweep48":
        return run_sweep_bench(args)
    return run_kf(args)


if __name__ == "__main__":
    sys.exit(main())
