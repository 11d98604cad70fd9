"""Generate the golden vectors of the reference's own hot-path code.

Runs the reference's sources compiled here (oracle/_ref/libkfref.so: the
reference's RKO4.cpp, rhs_standard.cpp, OP_*.cpp, solver_poisson_*.cpp,
field_interpolation.cpp ... with the FFT shim) on seeded inputs and stores
inputs and outputs as .npz fixtures next to this script.  The reference
publishes no test vectors of its own; these pin the oracle restatement.

    python tests/golden/make_golden.py [name ...]   (needs the reference sources)

names: ops transfer poisson shipped stretch (default: all)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from kielflow_b200 import inputs as I  # noqa: E402
from oracle import bind  # noqa: E402

L = I.L_DEFAULT


def shipped_case(n, M, tau, theta, Q, sigma, seed, nsteps, dt, m=0.0):
    st = I.initial_state(n, seed=seed)
    nd = I.gauss_charge(n, L, Q, sigma, m)
    mask = I.sphere_mask(n, L, 0.5, m)
    R = bind.Reference(n, L, M, tau, theta, poisson_mode=1, m=m)
    R.set_state(st)
    R.set_real(0, nd)
    R.set_real(1, mask)
    R.rhs()
    rhs = R.get_state()
    phi_rhs = R.get_real(2)
    R2 = bind.Reference(n, L, M, tau, theta, poisson_mode=1, m=m)
    R2.set_state(st)
    R2.set_real(0, nd)
    R2.set_real(1, mask)
    R2.rk4(dt, nsteps)
    rk = R2.get_state()
    return dict(n=n, M=M, tau=tau, theta=theta, dt=dt, nsteps=nsteps, nd=nd, mask=mask,
                s0_ux=st[0], s0_uy=st[1], s0_uz=st[2], s0_s=st[3],
                rhs_ux=rhs[0], rhs_uy=rhs[1], rhs_uz=rhs[2], rhs_s=rhs[3], rhs_phi=phi_rhs,
                rk_ux=rk[0], rk_uy=rk[1], rk_uz=rk[2], rk_s=rk[3])


def stretch_case(Rl, D):
    """The sine-stretched grid of the reference's frontend (axis_CoSiSt,
    m = L (1 - 0.3) / (2 pi), frontend.cpp:285-287): positions, the sampled
    Gaussian, the chain-rule derivatives, the cascadic multigrid solve and the
    shipped right-hand side with three RK4 steps."""
    m = L * (1.0 - 0.3) / (2.0 * np.pi)
    rng = np.random.default_rng(4321)
    n = 16
    pos = np.zeros(n + 2)
    Rl.kfref_positions(n, L, m, pos.ctypes.data_as(D))
    gauss = np.zeros((n, n, n))
    Rl.kfref_gauss_m(n, L, m, -5.0, 0.7, gauss.ctypes.data_as(D))
    x = rng.standard_normal((n, n, n))
    F = np.zeros((n, n, n // 2 + 1), np.complex128)
    Rl.kfref_fft_r2c(n, L, x.ctypes.data_as(D), F.ctypes.data_as(D))
    dF = []
    for d in range(3):
        o = np.zeros_like(F)
        Rl.kfref_deriv_m(n, L, m, d, F.ctypes.data_as(D), o.ctypes.data_as(D))
        dF.append(o)
    n2 = 32
    st = I.initial_state(n2, seed=9)
    s = np.fft.irfftn(st[3], s=(n2, n2, n2), axes=(0, 1, 2))
    rho = np.exp(s) + I.gauss_charge(n2, L, -10.0, 0.5, m)
    phi_m = np.zeros((n2, n2, n2))
    Rl.kfref_mg_solve_m(n2, L, m, phi_m.ctypes.data_as(D), rho.ctypes.data_as(D))
    case = shipped_case(n, 1.1, 0.2, 30.0, -5.0, 0.7, seed=11, nsteps=3, dt=0.01, m=m)
    return dict(m=m, positions=pos, gauss=gauss, F=F, dx=dF[0], dy=dF[1], dz=dF[2], rho32=rho,
                phi_cascadic32=phi_m, **case)


def main(names):
    if not bind.ref_available():
        bind.build(with_ref=True)
    Rl = bind.ref()
    rng = np.random.default_rng(1234)
    D = bind._D
    if "stretch" in names:
        np.savez_compressed(os.path.join(HERE, "stretch16.npz"), **stretch_case(Rl, D))
    if not {"ops", "transfer", "poisson", "shipped"} & set(names):
        print("golden vectors written to", HERE)
        return
    # spectral operators at 16^3
    n = 16
    x = rng.standard_normal((n, n, n))
    F = np.zeros((n, n, n // 2 + 1), np.complex128)
    Rl.kfref_fft_r2c(n, L, x.ctypes.data_as(D), F.ctypes.data_as(D))
    xb = np.zeros((n, n, n))
    Rl.kfref_fft_c2r(n, L, F.ctypes.data_as(D), xb.ctypes.data_as(D))
    Fd = F.copy()
    Rl.kfref_dealias(n, L, Fd.ctypes.data_as(D))
    Fp = F.copy()
    Rl.kfref_phi_filter(n, L, Fp.ctypes.data_as(D))
    dF = []
    for d in range(3):
        o = np.zeros_like(F)
        Rl.kfref_deriv(n, L, d, F.ctypes.data_as(D), o.ctypes.data_as(D))
        dF.append(o)
    np.savez_compressed(os.path.join(HERE, "ops16.npz"), x=x, F=F, xb=xb, dealiased=Fd, phifilt=Fp,
                        dx=dF[0], dy=dF[1], dz=dF[2])
    # inter-grid transfer
    a8 = rng.standard_normal((8, 8, 8))
    up = np.zeros((16, 16, 16))
    Rl.kfref_transfer(0, 8, L, a8.ctypes.data_as(D), up.ctypes.data_as(D))
    a16 = rng.standard_normal((16, 16, 16))
    dn = np.zeros((8, 8, 8))
    Rl.kfref_transfer(1, 16, L, a16.ctypes.data_as(D), dn.ctypes.data_as(D))
    np.savez_compressed(os.path.join(HERE, "transfer.npz"), a8=a8, up=up, a16=a16, dn=dn)
    # nonlinear Jacobi and the cascadic multigrid plan at 32^3
    n = 32
    st = I.initial_state(n, seed=3)
    nd = I.gauss_charge(n, L, -10.0, 0.5)
    s = np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2))
    rho = np.exp(s) + nd
    phi_j = np.zeros((n, n, n))
    Rl.kfref_nlj_solve(n, L, phi_j.ctypes.data_as(D), rho.ctypes.data_as(D), 60, 1e-9)
    phi_m = np.zeros((n, n, n))
    Rl.kfref_mg_solve(n, L, phi_m.ctypes.data_as(D), rho.ctypes.data_as(D))
    np.savez_compressed(os.path.join(HERE, "poisson32.npz"), rho=rho, phi_jacobi60=phi_j, phi_cascadic=phi_m)
    # the shipped right-hand side and two RK4 steps at 16^3
    case = shipped_case(16, 0.8, 0.1, 30.0, -10.0, 0.5, seed=7, nsteps=2, dt=0.05)
    np.savez_compressed(os.path.join(HERE, "shipped16.npz"), **case)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1:] or ["ops", "transfer", "poisson", "shipped", "stretch"])
