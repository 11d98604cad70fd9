"""Parameter sweep of independent instances with uneven grids.

The sweep workload: 48 instances, 16 each at 64^3, 96^3 and 128^3, with Mach
number ~ U[0.3, 1.5], friction ~ U[0.01, 0.3] and dust charge ~ U[-50, -5]
drawn from one seed (SplitMix64), the initial noise recipe of inputs.py, FP32
bulk with the FP64 Poisson solve.  Instances are independent: across GPUs they
are partitioned by cost (dist.partition), with no collective on the data path.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import configs as C
from .inputs import SplitMix64


@dataclass
class Instance:
    index: int
    n: int
    M: float
    tau: float
    Q: float
    seed: int


def sweep_instances(seed: int = 0, sizes=(64, 96, 128), per_size: int = 16):
    rng = SplitMix64(seed, 1000)
    out = []
    for n in sizes:
        for _ in range(per_size):
            M = 0.3 + 1.2 * rng.uniform()
            tau = 0.01 + 0.29 * rng.uniform()
            Q = -50.0 + 45.0 * rng.uniform()
            out.append(Instance(len(out), n, M, tau, Q, seed * 1000 + len(out)))
    return out


def workload_of(inst: Instance) -> dict:
    w = dict(C.WORKLOADS["fp32bulk256"])
    w.update(n=inst.n, M=inst.M, tau=inst.tau, Q=inst.Q, sigma=0.5)
    return w


def run_sweep(instances, steps: int, mode: str = "batched", precision=None, warmup: int = 1,
              max_threads: int = 64, tune=True, tunings: dict | None = None):
    """Advance every instance `steps` RK4 steps on the current GPU.

    Each instance is its own context (device memory, tables, CUDA stream,
    captured step graph).  Modes:
      "batched"    -- one kf_batch_rk4_steps call: this thread queues every
                      instance's step graph on its own stream, step by step,
                      so the instances' kernels overlap on the GPU;
      "threads"    -- a pool of host threads, one kf_rk4_steps call each
                      (the C calls release the GIL);
      "sequential" -- one instance after another (the baseline).
    With `tune`, the first instance of each grid size is autotuned
    (kf_autotune: transform radix plan, smoother block shape) and its choice
    is given to every instance of that size; `tune` may instead be such a
    result per size ({n: {"fft_plan": p, "rbgs_rows": r}}, e.g. the `tunings`
    of an earlier run) to apply without timing.  `tunings`, when a dict,
    receives {n: the choice used}.  `warmup` steps per instance run first, outside
    the timed region (graph capture, first-touch of the buffers).  Returns (wall seconds of the timed
    steps, [final state per instance], [diag per instance]).
    """
    import threading
    import time

    from ._lib import Context, batch_rk4

    ctxs, dts = [], []
    for inst in instances:
        w = workload_of(inst)
        st, nd, mask, dt = C.make_inputs(w, seed=inst.seed)
        ctx = Context(C.config_for(w, precision=precision))
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctxs.append(ctx)
        dts.append(dt)
    if tune:
        chosen = dict(tune) if isinstance(tune, dict) else {}
        for inst, ctx in zip(instances, ctxs):
            if inst.n not in chosen:
                chosen[inst.n] = ctx.autotune()
            else:
                ctx.set_tuning(chosen[inst.n]["fft_plan"], chosen[inst.n]["rbgs_rows"])
        if tunings is not None:
            tunings.update(chosen)
    if warmup > 0:
        for ctx, dt in zip(ctxs, dts):
            ctx.rk4(dt, warmup)
    for ctx in ctxs:
        ctx.synchronize()
    errors = []

    def work(i):
        try:
            ctxs[i].rk4(dts[i], steps)
            ctxs[i].synchronize()
        except Exception as e:  # surfaced after the join
            errors.append((i, e))

    t0 = time.perf_counter()
    if mode == "batched":
        batch_rk4(ctxs, dts, steps)
    elif mode == "threads":
        nthreads = min(max_threads, len(ctxs))
        pending = list(range(len(ctxs)))
        lock = threading.Lock()

        def runner():
            while True:
                with lock:
                    if not pending:
                        return
                    i = pending.pop(0)
                work(i)

        threads = [threading.Thread(target=runner) for _ in range(nthreads)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    elif mode == "sequential":
        for i in range(len(ctxs)):
            work(i)
    else:
        raise ValueError(f"unknown mode {mode!r}")
    wall = time.perf_counter() - t0
    if errors:
        raise errors[0][1]
    states = [ctx.get_state() for ctx in ctxs]
    diags = [ctx.diag() for ctx in ctxs]
    for ctx in ctxs:
        ctx.close()
    return wall, states, diags
