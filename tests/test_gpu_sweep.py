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
