"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances: FP64 path 1e-12 relative (max-norm, per field) unless a test
states otherwise; FP32-bulk path against the FP64 oracle 1e-5 relative.
"""
import numpy as np
import pytest

import kielflow_b200 as kf
from kielflow_b200 import configs as C
from kielflow_b200 import inputs as I
from oracle import bind

pytestmark = pytest.mark.gpu

L = I.L_DEFAULT
TOL64 = 1e-12
TOL32 = 1e-5


def rel(a, b, scale=0.0):
    """max|a-b| / max(max|b|, scale).  `scale` is the largest field of the same
    output: the z transforms pack two real fields into one complex line, so a
    field that is exactly zero picks up rounding noise of its partner's size."""
    return float(np.abs(a - b).max() / max(np.abs(b).max(), scale, 1e-300))


def state_rel(g, r):
    scale = max(np.abs(x).max() for x in r)
    return [rel(a, b, scale) for a, b in zip(g, r)]


def oracle_for(cfg):
    return bind.Oracle(bind.KfoConfig(*[getattr(cfg, f) for f, _ in bind.KfoConfig._fields_]))


@pytest.mark.parametrize("n", [16, 32, 64, 96, 128, 256])
@pytest.mark.parametrize("prec", [kf.KF_FP64, kf.KF_FP32_BULK])
def test_fft_r2c_c2r_vs_oracle(n, prec):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n))
    with kf.Context(kf.Config.make(n, L, 0.8, precision=prec)) as ctx:
        F = ctx.r2c(x)
        Fo = bind.r2c(x)
        tol = TOL64 if prec == kf.KF_FP64 else TOL32
        assert rel(F, Fo) < tol / 10
        xb = ctx.c2r(Fo)
        assert rel(xb, bind.c2r(Fo)) < tol / 10
        assert rel(xb, x) < tol / 10


RHS_CASES = {
    "linear": kf.KF_T_DISSIPATION | kf.KF_T_SVISCOSITY | kf.KF_T_PRESSURE | kf.KF_T_E_EXT | kf.KF_T_DIFFUSION,
    "advection": kf.KF_T_ADVECTION,
    "continuity": kf.KF_T_CONTINUITY,
    "penalized": kf.KF_T_ADVECTION | kf.KF_T_CONTINUITY | kf.KF_T_E_EXT | kf.KF_T_PENALIZATION,
    "shipped_jacobi": kf.KF_T_SHIPPED,
    "all_jacobi": kf.KF_T_ALL,
}


@pytest.mark.parametrize("case", list(RHS_CASES))
@pytest.mark.parametrize("n", [32, 64])
def test_rhs_vs_oracle(case, n):
    w = C.WORKLOADS["jacobi32"]
    st, nd, mask, dt = C.make_inputs(w, n=n, seed=2)
    cfg = C.config_for(w, n=n, terms=RHS_CASES[case], sv_cut=0.6)
    with kf.Context(cfg) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rhs()
        g = ctx.get_state()
        gphi = ctx.get_phi()
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rhs()
    r = o.get_state()
    errs = state_rel(g, r)
    assert max(errs) < TOL64, (case, errs)
    if RHS_CASES[case] & kf.KF_T_POISSON:
        assert rel(gphi, o.get_phi()) < TOL64


@pytest.mark.parametrize("mode", [kf.KF_PS_JACOBI_RES, kf.KF_PS_FAS, kf.KF_PS_CASCADIC, kf.KF_PS_JACOBI_REF])
def test_poisson_vs_oracle(mode):
    n = 32
    st = I.initial_state(n, seed=5)
    nd = I.gauss_charge(n, L, -10.0, 0.5)
    rho = np.exp(np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2))) + nd
    cfg = kf.Config.make(n, L, 0.8, poisson_mode=mode, nlj_max_it=100000 if mode == 1 else 200,
                         nlj_limit=1e-9, mg_levels=2, res_tol=1e-11)
    with kf.Context(cfg) as ctx:
        pg = ctx.poisson(np.zeros((n, n, n)), rho)
        dg = ctx.diag()
    o = oracle_for(cfg)
    po = o.poisson(np.zeros((n, n, n)), rho)
    so = o.stats()
    assert rel(pg, po) < TOL64
    if mode in (kf.KF_PS_JACOBI_RES, kf.KF_PS_FAS):
        assert dg.last_residual <= 1e-11
        assert dg.last_iterations == so.last_iterations


def test_rk4_jacobi32_config0_100_steps():
    """Configuration 0 as specified: 32^3, FP64, nonlinear Jacobi to residual
    1e-10, 100 RK4 steps (RKO4.cpp:50-241, kielflow.cpp:277-331)."""
    w = C.WORKLOADS["jacobi32"]
    st, nd, mask, dt = C.make_inputs(w)
    cfg = C.config_for(w)
    steps = w["steps"]
    assert steps == 100
    with kf.Context(cfg) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rk4(dt, steps)
        g = ctx.get_state()
        gphi = ctx.get_phi()
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rk4(dt, steps)
    r = o.get_state()
    errs = state_rel(g, r)
    assert max(errs) < TOL64, errs
    assert rel(gphi, o.get_phi()) < TOL64
    # the same window in FP32 bulk against this FP64 oracle run
    e = fp32_vs_fp64_errors(w, 32, steps, ref=(r, o.get_phi()))
    assert max(e.values()) < TOL32, e


def test_rk4_fas128_config1_20_steps():
    """Configuration 1's parity window: 128^3, FP64, FAS V-cycles (4 levels,
    2 + 2 sweeps) to residual 1e-10, spectral viscosity beyond 0.6 k_max,
    the first 20 RK4 steps, 1e-12 relative in n, u and phi."""
    n, steps = 128, 20
    w = C.WORKLOADS["fas128"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg = C.config_for(w, n=n)
    assert cfg.mg_levels == 4 and cfg.mg_pre == 2 and cfg.mg_post == 2 and cfg.res_tol == 1e-10
    with kf.Context(cfg) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rk4(dt, steps)
        g = ctx.get_state()
        gphi = ctx.get_phi()
        gd = ctx.diag()
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rk4(dt, steps)
    r = o.get_state()
    errs = state_rel(g, r)
    assert max(errs) < TOL64, errs
    # n = e^s and u in physical space, relative max-norm
    assert rel(np.exp(bind.c2r(g[3])), np.exp(bind.c2r(r[3]))) < TOL64
    assert rel(gphi, o.get_phi()) < TOL64
    assert gd.total_iterations == o.stats().total_iterations
    # the same window in FP32 bulk against this FP64 oracle run
    e = fp32_vs_fp64_errors(w, n, steps, ref=(r, o.get_phi()))
    assert max(e.values()) < TOL32, e


@pytest.mark.parametrize("n,steps", [(64, 3), (128, 1)])
def test_rk4_fas_vs_oracle(n, steps):
    """Workload fas128 physics (FP64, FAS V-cycles, SV beyond 0.6 k_max)."""
    w = C.WORKLOADS["fas128"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg = C.config_for(w, n=n)
    with kf.Context(cfg) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rk4(dt, steps)
        g = ctx.get_state()
        gphi = ctx.get_phi()
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rk4(dt, steps)
    r = o.get_state()
    errs = state_rel(g, r)
    assert max(errs) < TOL64, errs
    assert rel(gphi, o.get_phi()) < TOL64


def fp32_vs_fp64_errors(w, n, steps, ref=None):
    """FP32-bulk GPU run against the FP64 oracle (residual 1e-10) of the same
    inputs: relative max-norm errors of n = e^s, of the total velocity
    M e_x + u' (three components together) and of phi.  `ref` = (state, phi)
    of an FP64 oracle run of these inputs already made."""
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg32 = C.config_for(w, n=n, precision=kf.KF_FP32_BULK)
    cfg64 = C.config_for(w, n=n, precision=kf.KF_FP64)
    assert cfg64.res_tol == 1e-10 and cfg32.res_tol == C.fp32_res_tol(w["Q"], w["sigma"])
    with kf.Context(cfg32) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rk4(dt, steps)
        g = ctx.get_state()
        gphi = ctx.get_phi()
        assert ctx.diag().not_converged == 0
    if ref is None:
        o = oracle_for(cfg64)
        o.set_state(st)
        o.set_sources(nd, mask)
        o.rk4(dt, steps)
        ref = (o.get_state(), o.get_phi())
    r, ophi = ref
    ug = np.stack([bind.c2r(x) for x in g[:3]])
    ur = np.stack([bind.c2r(x) for x in r[:3]])
    ug[0] += w["M"]
    ur[0] += w["M"]
    return {"n": rel(np.exp(bind.c2r(g[3])), np.exp(bind.c2r(r[3]))), "u": rel(ug, ur),
            "phi": rel(gphi, ophi)}


def test_fp32_bulk_vs_fp64_oracle():
    """FP32 bulk (FFTs, products, RK4 stages) with the FP64 Poisson solve at
    its FP32-matched residual target, against the FP64 oracle: n, the total
    velocity and phi within 1e-5 relative after 3 steps at 64^3."""
    e = fp32_vs_fp64_errors(C.WORKLOADS["fp32bulk256"], 64, 3)
    assert max(e.values()) < TOL32, e


# 96^3: the radix-3 plans (96 = 6 * 4 * 4 and 4 * 4 * 6) in the right-hand side
# and RK4, in both precisions
@pytest.mark.parametrize("case", ["all_fas", "penalized", "linear"])
@pytest.mark.parametrize("plan", [0, 1])
def test_rhs96_vs_oracle(case, plan):
    """At 96^3 the Poisson solve of the full set is the sweep's FAS cycle (the
    Jacobi solver of configuration 0 runs only at 32^3: its Carre factor comes
    from a sum whose order differs between the GPU tree and the reference's
    loop, which over the thousands of sweeps at 96^3 reaches 1e-11)."""
    n = 96
    w = C.WORKLOADS["fas128" if case == "all_fas" else "jacobi32"]
    st, nd, mask, dt = C.make_inputs(w, n=n, seed=3)
    terms = kf.KF_T_ALL if case == "all_fas" else RHS_CASES[case]
    cfg = C.config_for(w, n=n, terms=terms, sv_cut=0.6)
    with kf.Context(cfg) as ctx:
        ctx.set_tuning(plan, 0)
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rhs()
        g = ctx.get_state()
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rhs()
    assert max(state_rel(g, o.get_state())) < TOL64


@pytest.mark.parametrize("plan", [0, 1])
def test_rk4_fas96_vs_oracle(plan):
    """The sweep's 96^3 instances (FAS levels 96, 48, 24, 12): FP64 3 steps at
    1e-12, and FP32 bulk against the FP64 oracle at 1e-5."""
    n, steps = 96, 3
    w = C.WORKLOADS["fas128"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg = C.config_for(w, n=n)
    with kf.Context(cfg) as ctx:
        ctx.set_tuning(plan, 0)
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
    e = fp32_vs_fp64_errors(dict(w, precision=kf.KF_FP32_BULK), n, steps)
    assert max(e.values()) < TOL32, e
