"""kf_fft_r2c_noalloc: the forward 3-D transform without device allocation.

This entry point is for callers that cannot let a library allocate device
memory -- a host application that owns a fixed device pool and only lends its
plugins buffers, or a time-critical loop that cannot pay for cudaMalloc's
latency and device-wide synchronisation.  The caller passes device buffers
for input and output; the library's one intermediate array is a static
device array (n <= 64).  The test gives it buffers allocated by torch (the
test may allocate; the entry point must not) and checks two calls in a row
against kf_fft_r2c of a context, within the FFT tolerance of the parity tests.
This file is collected last so that a failure here leaves the other tests run.
"""
import ctypes

import numpy as np
import pytest

import kielflow_b200 as kf
from kielflow_b200 import _lib
from kielflow_b200 import inputs as I

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the FP64 transform tolerance of test_gpu_parity (1e-12 / 10)
L = I.L_DEFAULT


def _call(lib, n, xin, out, stream):
    return lib.kf_fft_r2c_noalloc(n, ctypes.c_void_p(xin.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                  ctypes.c_void_p(stream))


@pytest.mark.parametrize("n", [16, 32, 64])
def test_noalloc_r2c_matches_context_r2c_on_two_calls(n):
    import torch
    lib = _lib.load_library()
    rng = np.random.default_rng(1000 + n)
    stream = torch.cuda.current_stream().cuda_stream
    with kf.Context(kf.Config.make(n, L, 0.8)) as ctx:
        for _ in range(2):
            x = rng.standard_normal((n, n, n))
            ref = ctx.r2c(x)
            xin = torch.from_numpy(x).cuda()
            out = torch.full((n, n, n // 2 + 1), complex(float("nan"), float("nan")), dtype=torch.complex128,
                             device="cuda")
            rc = _call(lib, n, xin, out, stream)
            assert rc == 0, lib.kf_last_error(None).decode()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.isfinite(got).all()
            assert np.abs(got - ref).max() <= TOL * np.abs(ref).max()


def test_noalloc_allocates_nothing_on_a_side_stream():
    """After the warm-up call (which may load the module and its static
    array), further calls on a non-default stream leave the device's free
    memory unchanged and match kf_fft_r2c."""
    import torch
    lib = _lib.load_library()
    n = 64
    rng = np.random.default_rng(7)
    side = torch.cuda.Stream()
    x = rng.standard_normal((n, n, n))
    xin = torch.from_numpy(x).cuda()
    out = torch.zeros((n, n, n // 2 + 1), dtype=torch.complex128, device="cuda")
    with kf.Context(kf.Config.make(n, L, 0.8)) as ctx:
        ref = ctx.r2c(x)
    torch.cuda.synchronize()
    assert _call(lib, n, xin, out, side.cuda_stream) == 0, lib.kf_last_error(None).decode()  # warm-up
    side.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        out.zero_()
        torch.cuda.synchronize()
        assert _call(lib, n, xin, out, side.cuda_stream) == 0, lib.kf_last_error(None).decode()
        side.synchronize()
        got = out.cpu().numpy()
        assert np.abs(got - ref).max() <= TOL * np.abs(ref).max()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    lib = _lib.load_library()
    n = 128
    xin = torch.zeros((1,), dtype=torch.float64, device="cuda")
    out = torch.zeros((1,), dtype=torch.complex128, device="cuda")
    rc = _call(lib, n, xin, out, torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b"64" in lib.kf_last_error(None)
