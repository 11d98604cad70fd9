"""Sine-stretched axes (axis_CoSiSt, the reference frontend's grid) through the
C ABI against the oracle, which reproduces the reference on this grid bit for
bit (tests/test_oracle_cpu.py).  Tolerances as the equidistant parity tests:
FP64 1e-12 relative (max-norm per field), FP32 bulk 1e-5 on n and phi.
"""
import os

import numpy as np
import pytest

import kielflow_b200 as kf
from kielflow_b200 import configs as C
from kielflow_b200 import inputs as I
from oracle import bind

from test_gpu_parity import RHS_CASES, TOL32, TOL64, oracle_for, rel, state_rel

pytestmark = pytest.mark.gpu

L = I.L_DEFAULT
M_ST = I.frontend_stretch(L)


def stretched_inputs(n, seed=2, Q=-10.0, sigma=0.5):
    st = I.initial_state(n, seed=seed)
    nd = I.gauss_charge(n, L, Q, sigma, M_ST)
    mask = I.sphere_mask(n, L, 0.5, M_ST)
    return st, nd, mask


@pytest.mark.parametrize("case", ["linear", "advection", "continuity", "penalized", "all_jacobi"])
@pytest.mark.parametrize("n", [32, 64])
def test_stretched_rhs_vs_oracle(case, n):
    w = C.WORKLOADS["jacobi32"]
    st, nd, mask = stretched_inputs(n)
    cfg = C.config_for(w, n=n, terms=RHS_CASES[case], sv_cut=0.6, stretch_m=M_ST)
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
    errs = state_rel(g, o.get_state())
    assert max(errs) < TOL64, (case, errs)
    if RHS_CASES[case] & kf.KF_T_POISSON:
        assert rel(gphi, o.get_phi()) < TOL64


def test_stretched_shipped_cascadic_vs_oracle():
    """The reference's own configuration on its frontend grid: shipped terms,
    cascadic multigrid, two RK4 steps (host-driven path)."""
    n = 32
    st, nd, mask = stretched_inputs(n, seed=4, Q=-5.0, sigma=0.7)
    cfg = kf.Config.make(n, L, 1.1, tau=0.2, poisson_mode=kf.KF_PS_CASCADIC, stretch_m=M_ST)
    with kf.Context(cfg) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rk4(0.01, 2)
        g = ctx.get_state()
        gphi = ctx.get_phi()
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rk4(0.01, 2)
    assert max(state_rel(g, o.get_state())) < TOL64
    assert rel(gphi, o.get_phi()) < TOL64


@pytest.mark.parametrize("mode", [kf.KF_PS_FAS, kf.KF_PS_CASCADIC, kf.KF_PS_JACOBI_RES])
def test_stretched_poisson_vs_oracle(mode):
    n = 32
    st, nd, _ = stretched_inputs(n, seed=5)
    rho = np.exp(np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2))) + nd
    cfg = kf.Config.make(n, L, 0.8, poisson_mode=mode, nlj_max_it=200000, mg_levels=2, res_tol=1e-11,
                         stretch_m=M_ST)
    with kf.Context(cfg) as ctx:
        pg = ctx.poisson(np.zeros((n, n, n)), rho)
        dg = ctx.diag()
    o = oracle_for(cfg)
    po = o.poisson(np.zeros((n, n, n)), rho)
    assert rel(pg, po) < TOL64
    if mode == kf.KF_PS_FAS:
        assert dg.last_residual <= 1e-11 and dg.last_iterations == o.stats().last_iterations


def test_stretched_rk4_fas_vs_oracle():
    """stretch256 physics at 64^3 in FP64 (FAS, captured step): three steps."""
    n, steps = 64, 3
    w = C.WORKLOADS["stretch256"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg = C.config_for(w, n=n, precision=kf.KF_FP64)
    assert cfg.stretch_m == M_ST
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
    assert max(state_rel(g, o.get_state())) < TOL64
    assert rel(gphi, o.get_phi()) < TOL64


def test_stretched_fp32_bulk_vs_fp64_oracle():
    n, steps = 64, 3
    w = C.WORKLOADS["stretch256"]
    st, nd, mask, dt = C.make_inputs(w, n=n)
    cfg32 = C.config_for(w, n=n)
    with kf.Context(cfg32) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.rk4(dt, steps)
        g = ctx.get_state()
        gphi = ctx.get_phi()
    o = oracle_for(C.config_for(w, n=n, precision=kf.KF_FP64))
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rk4(dt, steps)
    r = o.get_state()
    for q in range(3):
        assert rel(bind.c2r(g[q]), bind.c2r(r[q])) < 1e-3  # u' is a 1e-3 perturbation
    assert rel(np.exp(bind.c2r(g[3])), np.exp(bind.c2r(r[3]))) < TOL32
    assert rel(gphi, o.get_phi()) < TOL32


def test_stretched_diag_uses_cell_volumes():
    """kf_diag sums with the stretched cell volumes h^3 dS(x) dS(y) dS(z)."""
    n = 32
    st, nd, mask = stretched_inputs(n)
    cfg = kf.Config.make(n, L, 0.8, poisson_mode=kf.KF_PS_FAS, mg_levels=2, res_tol=1e-11, stretch_m=M_ST)
    with kf.Context(cfg) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        d = ctx.diag()
        phi = ctx.get_phi()
    h = L / n
    x = -0.5 * L + h * np.arange(n)
    dS = 1.0 - (2.0 * np.pi * M_ST / L) * np.cos(2.0 * np.pi * x / L)
    wv = dS[:, None, None] * dS[None, :, None] * dS[None, None, :] * h ** 3
    s = np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2))
    charge = float((wv * (np.exp(s) - np.exp(phi) + nd)).sum())
    assert abs(d.charge - charge) <= 1e-10 * max(1.0, abs(charge))
    assert abs(wv.sum() - L ** 3) < 1e-9 * L ** 3  # the cells tile the box


def test_stretched_files_and_guards(tmp_path):
    n = 32
    st, nd, mask = stretched_inputs(n)
    cfg = kf.Config.make(n, L, 0.8, poisson_mode=kf.KF_PS_FAS, mg_levels=2, stretch_m=M_ST)
    path = os.path.join(str(tmp_path), "b.kfh")
    with kf.Context(cfg) as ctx:
        ctx.set_state(*st)
        ctx.save(path, kf.KF_FILE_BACKUP, 0.5)
        with pytest.raises(kf.KfError):
            ctx.adjoint(np.zeros((n, n, n)), 1, 0.01)
    info = kf.file_info(path)
    assert info["type"] == 3 and info["m"] == M_ST
    with kf.Context(kf.Config.make(n, L, 0.8, poisson_mode=kf.KF_PS_FAS, mg_levels=2)) as flat:
        with pytest.raises(kf.KfError):
            flat.load(path)
    with kf.Context(cfg) as ctx:
        assert ctx.load(path) == 0.5
    with pytest.raises(kf.KfError):
        kf.Context(kf.Config.make(n, L, 0.8, stretch_m=L / (2.0 * np.pi)))  # not monotone
