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
