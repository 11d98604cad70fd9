"""The reference's own time loop with the GPU adapters dropped in.

oracle/_ref/drop_in_driver (built from oracle/drop_in_driver.cpp against the
reference's sources and include/kf_adapters.hpp) advances one seeded state
with the reference's rhs_standard + Runge_kutta_O4 + cascadic multigrid, then
with kf_gpu_rhs + kf_gpu_rk4 in their place; the two final states must agree.
"""
import os
import subprocess

import numpy as np
import pytest

from kielflow_b200 import inputs as I

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "drop_in_driver")


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="drop-in driver not built (needs the reference sources)")
@pytest.mark.parametrize("n,steps,stretched", [(16, 3, False), (32, 2, False), (16, 3, True)])
def test_reference_loop_with_gpu_adapters(tmp_path, n, steps, stretched):
    """stretched: the frontend's axis_CoSiSt grid, read by the adapter from the
    reference's own grid object."""
    L = I.L_DEFAULT
    m = I.frontend_stretch(L) if stretched else 0.0
    M, tau, theta, dt = 0.8, 0.1, 30.0, 0.05 if not stretched else 0.02
    st = I.initial_state(n, seed=21)
    nd = I.gauss_charge(n, L, -10.0, 0.5, m)
    mask = I.sphere_mask(n, L, 0.5, m)
    np.concatenate([np.ascontiguousarray(a).view(np.float64).ravel() for a in st]).tofile(tmp_path / "state.bin")
    nd.tofile(tmp_path / "nd.bin")
    mask.tofile(tmp_path / "mask.bin")
    args = [DRIVER, str(tmp_path), str(n), str(M), str(tau), str(theta), str(dt), str(steps)]
    if stretched:
        args.append(repr(m))
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    nc = n * n * (n // 2 + 1)
    ref = np.fromfile(tmp_path / "ref_state.bin").view(np.complex128).reshape(4, nc)
    gpu = np.fromfile(tmp_path / "gpu_state.bin").view(np.complex128).reshape(4, nc)
    scale = np.abs(ref).max()
    err = np.abs(gpu - ref).max() / scale
    assert err < 1e-10, err
