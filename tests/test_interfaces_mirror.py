"""The host mirror of the reference's interfaces (kielflow_b200/interfaces.py)
drives the GPU the way the reference's own objects are driven: in-place
interface_rhs::solve, interface_ode_solver::solve and
interface_poisson_solver::solve, each against the oracle (FP64, max-norm over
the four fields: 1e-12 relative for the FAS solve, 1e-10 where the reference's
cascadic plan decides its sweeps on relative-update tests, as in
tests/test_gpu_dropin.py).  Collected last: the paths underneath are tested
earlier, this file adds the mirror's plumbing."""
import numpy as np
import pytest

import kielflow_b200 as kf
from kielflow_b200 import inputs as I

from test_gpu_parity import TOL64, oracle_for, rel, state_rel

TOL_CASCADIC = 1e-10

pytestmark = pytest.mark.gpu

L = I.L_DEFAULT


def shipped_case(n=16, seed=21):
    st = I.initial_state(n, seed=seed)
    nd = I.gauss_charge(n, L, -10.0, 0.5)
    mask = I.sphere_mask(n, L, 0.5)
    return st, nd, mask


def test_rhs_and_rk4_through_the_interfaces():
    n, M, tau, theta, dt = 16, 0.8, 0.1, 30.0, 0.05
    st, nd, mask = shipped_case(n)
    grid = kf.Grid(n, L)
    params = kf.Parameters(M=M, tau=tau, theta=theta)
    cfg = kf.Config.make(n, L, M, tau=tau, theta=theta, terms=kf.KF_T_SHIPPED, poisson_mode=kf.KF_PS_CASCADIC)
    # interface_rhs::solve: the four fields replaced by their time derivative
    rhs = kf.RhsStandard(params, grid, nd, mask, terms=kf.KF_T_SHIPPED, poisson_mode=kf.KF_PS_CASCADIC)
    F = [np.ascontiguousarray(a, np.complex128).copy() for a in st]
    rhs.solve(0.0, *F)
    o = oracle_for(cfg)
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rhs()
    assert max(state_rel(F, o.get_state())) < TOL_CASCADIC
    assert rel(rhs.Phi, o.get_phi()) < TOL_CASCADIC
    # interface_ode_solver::solve: one RK4 step of dt, in place
    rhs2 = kf.RhsStandard(params, grid, nd, mask, terms=kf.KF_T_SHIPPED, poisson_mode=kf.KF_PS_CASCADIC)
    rk = kf.RungeKuttaO4(rhs2, dt)
    G = [np.ascontiguousarray(a, np.complex128).copy() for a in st]
    rk.solve(*G)
    o2 = oracle_for(cfg)
    o2.set_state(st)
    o2.set_sources(nd, mask)
    o2.rk4(dt, 1)
    assert max(state_rel(G, o2.get_state())) < TOL_CASCADIC
    assert rk.t == dt


def test_poisson_through_the_interface():
    n = 32
    st = I.initial_state(n, seed=5)
    nd = I.gauss_charge(n, L, -10.0, 0.5)
    rho = np.exp(np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2))) + nd
    ps = kf.PoissonSolver(kf.Grid(n, L), mode=kf.KF_PS_FAS, mg_levels=2, res_tol=1e-11)
    phi = np.zeros((n, n, n))
    ps.solve(phi, rho)  # Phi_IO: initial guess in, solution out
    assert ps.converged()
    o = oracle_for(kf.Config.make(n, L, 0.0, poisson_mode=kf.KF_PS_FAS, mg_levels=2, res_tol=1e-11))
    assert rel(phi, o.poisson(np.zeros((n, n, n)), rho)) < TOL64
    with pytest.raises(ValueError):
        ps.solve(np.zeros((n, n, n - 1)), rho)  # field size not matching
