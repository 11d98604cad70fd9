"""Parameter sweep of independent instances with uneven grids (sweep.py):
batched and threaded execution give the same per-instance results as
sequential execution, bit for bit, with the variants the sequential run's
autotuning chose."""
import numpy as np
import pytest

from kielflow_b200 import KF_FP32_BULK
from kielflow_b200.sweep import Instance, run_sweep

pytestmark = pytest.mark.gpu


def test_concurrent_sweep_matches_sequential():
    inst = [Instance(0, 32, 0.5, 0.1, -10.0, 1), Instance(1, 64, 1.3, 0.02, -40.0, 2),
            Instance(2, 32, 1.0, 0.2, -5.0, 3), Instance(3, 64, 0.4, 0.3, -25.0, 4)]
    tunings = {}
    _, seq, dseq = run_sweep(inst, steps=2, mode="sequential", precision=KF_FP32_BULK, tunings=tunings)
    assert sorted(tunings) == [32, 64]
    for mode in ("batched", "threads"):
        _, con, dcon = run_sweep(inst, steps=2, mode=mode, precision=KF_FP32_BULK, tune=tunings)
        for a, b in zip(seq, con):
            for x, y in zip(a, b):
                assert np.array_equal(x, y)
        for a, b in zip(dseq, dcon):
            assert a.total_iterations == b.total_iterations and a.not_converged == 0


def test_batched_sweep_instances_vs_oracle():
    """One instance of each sweep grid size (64^3, 96^3, 128^3, drawn by the
    sweep's own generator), advanced together by kf_batch_rk4_steps in FP32
    bulk, against the FP64 oracle of the same instance: n = e^s, the total
    velocity and phi within 1e-5 relative after 2 steps."""
    from kielflow_b200 import KF_FP64
    from kielflow_b200 import configs as C
    from kielflow_b200.sweep import sweep_instances, workload_of
    from oracle import bind
    from test_gpu_parity import TOL32, oracle_for, rel

    pick = []
    for n in (64, 96, 128):
        pick.append(next(i for i in sweep_instances(seed=0) if i.n == n))
    steps = 2
    _, states, diags = run_sweep(pick, steps=steps, mode="batched", precision=KF_FP32_BULK, warmup=0)
    for inst, g, d in zip(pick, states, diags):
        assert d.not_converged == 0
        w = workload_of(inst)
        st, nd, mask, dt = C.make_inputs(w, seed=inst.seed)
        o = oracle_for(C.config_for(w, precision=KF_FP64))
        o.set_state(st)
        o.set_sources(nd, mask)
        o.rk4(dt, steps)
        r = o.get_state()
        ug = np.stack([bind.c2r(x) for x in g[:3]])
        ur = np.stack([bind.c2r(x) for x in r[:3]])
        ug[0] += inst.M
        ur[0] += inst.M
        assert rel(ug, ur) < TOL32, (inst.n, "u")
        assert rel(np.exp(bind.c2r(g[3])), np.exp(bind.c2r(r[3]))) < TOL32, (inst.n, "n")
