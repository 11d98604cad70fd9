"""Kernel variants (kf_set_tuning, kf_autotune) through the C ABI.

Every transform plan reproduces the oracle within the path's tolerance
(FP64 1e-12 relative, FP32-bulk 1e-5, max-norm per field); the smoother's rows
per block change only the launch shape, so its potentials are bit-identical.
"""
import numpy as np
import pytest

import kielflow_b200 as kf
from kielflow_b200 import configs as C
from kielflow_b200 import inputs as I
from oracle import bind

from test_gpu_parity import RHS_CASES, TOL32, TOL64, oracle_for, rel, state_rel

pytestmark = pytest.mark.gpu

L = I.L_DEFAULT


@pytest.mark.parametrize("n", [16, 32, 64, 96, 128, 256])
@pytest.mark.parametrize("prec", [kf.KF_FP64, kf.KF_FP32_BULK])
def test_fft_plan1_vs_oracle(n, prec):
    rng = np.random.default_rng(n + 1)
    x = rng.standard_normal((n, n, n))
    with kf.Context(kf.Config.make(n, L, 0.8, precision=prec)) as ctx:
        ctx.set_tuning(1, 8)
        F = ctx.r2c(x)
        Fo = bind.r2c(x)
        tol = TOL64 if prec == kf.KF_FP64 else TOL32
        assert rel(F, Fo) < tol / 10
        xb = ctx.c2r(Fo)
        assert rel(xb, bind.c2r(Fo)) < tol / 10


@pytest.mark.parametrize("case", ["all_jacobi", "penalized"])
@pytest.mark.parametrize("n", [32, 64])
def test_rhs_plan1_vs_oracle(case, n):
    w = C.WORKLOADS["jacobi32"]
    st, nd, mask, dt = C.make_inputs(w, n=n, seed=2)
    cfg = C.config_for(w, n=n, terms=RHS_CASES[case], sv_cut=0.6)
    with kf.Context(cfg) as ctx:
        ctx.set_tuning(1, 8)
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rhs()
        g = ctx.get_state()
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rhs()
    assert max(state_rel(g, o.get_state())) < TOL64


@pytest.mark.parametrize("rows", [4, 16])
def test_rk4_fas_variants_vs_oracle(rows):
    """fas128 physics at 64^3 (FP64, captured step): plan 1 and another
    smoother shape, three steps, against the oracle."""
    n, steps = 64, 3
    w = C.WORKLOADS["fas128"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg = C.config_for(w, n=n)
    with kf.Context(cfg) as ctx:
        ctx.set_tuning(1, rows)
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rk4(dt, steps)
        g = ctx.get_state()
        gphi = ctx.get_phi()
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rk4(dt, steps)
    assert max(state_rel(g, o.get_state())) < TOL64
    assert rel(gphi, o.get_phi()) < TOL64


@pytest.mark.parametrize("n,levels", [(64, 3), (128, 4), (256, 6)])
def test_rbgs_variants_bit_identical(n, levels):
    """The half-sweep kernels (4, 8, 16 rows) and the streaming TMA-staged
    sweep (rows 0; levels n >= 64, residual fused into the last pre-smoothing
    sweep) give the same potential bit for bit, with the same cycle count."""
    st = I.initial_state(n, seed=5)
    nd = I.gauss_charge(n, L, -10.0, 0.5)
    rho = np.exp(np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2))) + nd
    cfg = kf.Config.make(n, L, 0.8, poisson_mode=kf.KF_PS_FAS, mg_levels=levels, res_tol=1e-11, mg_omega=1.25)
    out, cyc = {}, {}
    with kf.Context(cfg) as ctx:
        for rows in ((4, 8, 16, 0) if n == 64 else (8, 0)):
            ctx.set_tuning(0, rows)
            out[rows] = ctx.poisson(np.zeros((n, n, n)), rho)
            cyc[rows] = ctx.diag().last_iterations
    for rows in out:
        assert np.array_equal(out[rows], out[8]), rows
        assert cyc[rows] == cyc[8]


@pytest.mark.parametrize("prec", [kf.KF_FP64, kf.KF_FP32_BULK])
def test_rk4_streaming_smoother_bit_identical(prec):
    """Captured FAS steps at 128^3 (levels 128 and 64 streamed): state,
    potential and V-cycle counts equal to the half-sweep kernels'."""
    n, steps = 128, 2
    w = C.WORKLOADS["fas128"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg = C.config_for(w, n=n, precision=prec)
    res = {}
    for rows in (8, 0):
        with kf.Context(cfg) as ctx:
            ctx.set_tuning(0, rows)
            ctx.set_state(*st)
            ctx.set_sources(nd, mask)
            ctx.rk4(dt, steps)
            res[rows] = (ctx.get_state(), ctx.get_phi(), ctx.diag().total_iterations)
    (s8, p8, c8), (s0, p0, c0) = res[8], res[0]
    assert all(np.array_equal(a, b) for a, b in zip(s8, s0))
    assert np.array_equal(p8, p0) and c8 == c0


@pytest.mark.parametrize("n,levels,prec", [(64, 4, kf.KF_FP64), (256, 6, kf.KF_FP32_BULK)])
def test_coarse_block_bit_identical(n, levels, prec):
    """Captured FAS steps whose cycle reaches 8^3 (64-32-16-8, and the 6-level
    256^3 cycle): the 16^3 and 8^3 levels in one shared-memory block give the
    state, potential and V-cycle counts of the level-by-level kernels."""
    steps = 2 if n == 64 else 1
    w = C.WORKLOADS["fas128"] if n == 64 else C.WORKLOADS["fp32bulk256"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg = C.config_for(w, n=n, precision=prec, mg_levels=levels)
    res = {}
    for on in (False, True):
        with kf.Context(cfg) as ctx:
            ctx.set_coarse_block(on)
            ctx.set_state(*st)
            ctx.set_sources(nd, mask)
            ctx.rk4(dt, steps)
            d = ctx.diag()
            res[on] = (ctx.get_state(), ctx.get_phi(), d.total_iterations, d.not_converged)
    (sa, pa, ca, na), (sb, pb, cb, nb) = res[False], res[True]
    assert all(np.array_equal(a, b) for a, b in zip(sa, sb))
    assert np.array_equal(pa, pb) and ca == cb and na == nb == 0


def test_coarse_block_vs_oracle():
    """The 4-level cycle at 64^3 (coarsest 8^3, levels 16 and 8 in the
    block) against the oracle: 3 FP64 steps at 1e-12, equal V-cycle count."""
    n, steps = 64, 3
    w = C.WORKLOADS["fas128"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg = C.config_for(w, n=n, mg_levels=4)
    with kf.Context(cfg) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rk4(dt, steps)
        g, gphi, it = ctx.get_state(), ctx.get_phi(), ctx.diag().total_iterations
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rk4(dt, steps)
    assert max(state_rel(g, o.get_state())) < TOL64
    assert rel(gphi, o.get_phi()) < TOL64
    assert it == o.stats().total_iterations


def test_autotune_keeps_state_and_steps():
    """kf_autotune on a 64^3 FP32-bulk context between captured steps: state,
    potential and time unchanged; the following steps equal those of a context
    given the same variants by kf_set_tuning."""
    n = 64
    w = C.WORKLOADS["fp32bulk256"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg = C.config_for(w, n=n)
    with kf.Context(cfg) as a, kf.Context(cfg) as b:
        for c in (a, b):
            c.set_state(*st)
            c.set_sources(nd, mask)
            c.rk4(dt, 2)
        s0, p0 = a.get_state(), a.get_phi()
        t = a.autotune(3)
        assert t["fft_plan"] in (0, 1) and t["rbgs_rows"] in (0, 4, 8, 16)
        for rad, thr in zip(t["fft_radices"], t["fft_threads"]):
            assert int(np.prod(rad)) == n and thr > 0
        timed = [x for x in t["rbgs_ms"] if x > 0]
        assert min(t["fft_ms"]) > 0 and len(timed) == 4  # 64^3: the streaming sweep is a candidate
        assert t["fft_ms"][t["fft_plan"]] == min(t["fft_ms"])
        assert t["rbgs_ms"][(4, 8, 16, 0).index(t["rbgs_rows"])] == min(timed)
        s1, p1 = a.get_state(), a.get_phi()
        assert all(np.array_equal(x, y) for x, y in zip(s0, s1)) and np.array_equal(p0, p1)
        b.set_tuning(t["fft_plan"], t["rbgs_rows"])
        a.rk4(dt, 2)
        b.rk4(dt, 2)
        ga, gb = a.get_state(), b.get_state()
        assert all(np.array_equal(x, y) for x, y in zip(ga, gb))
        assert np.array_equal(a.get_phi(), b.get_phi())


def test_set_tuning_rejects_other_values():
    with kf.Context(kf.Config.make(32, L, 0.8)) as ctx:
        for args in ((2, 8), (0, 6), (-1, 16)):
            with pytest.raises(kf.KfError):
                ctx.set_tuning(*args)
        assert ctx.L.kf_set_coarse_block(ctx.h, 2) == -1  # KF_ERR_ARG
