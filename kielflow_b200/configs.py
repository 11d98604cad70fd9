"""The standard workloads of the kielflow time step, with their sizes.

Physics shared by all workloads: box side L = 2*pi*4 Debye lengths, theta =
Te/Ti = 30 (the reference frontend's default, frontend.cpp:70), Laplacian
diffusion D = 1e-3 on s and u', dust grain = Gaussian charge at the box
centre, penalization sphere of radius 0.5 with eta_d = -1e-3 (masking form of
effect_penalization.cpp:35; targets u'_x = -M, u'_y = u'_z = 0, s = -10 as in
rhs_standard.cpp:486-526), the phi filter and the grad(s)/theta pressure term
of rhs_standard.cpp:218-248, 2/3 dealiasing, initial noise amplitude 1e-3 on
|m| <= 4, dt = 0.2 h / max|u| from the initial state.
"""
from __future__ import annotations

import math

from ._lib import (KF_FP32_BULK, KF_FP64, KF_PS_FAS, KF_PS_JACOBI_RES, KF_T_ALL, KF_T_SVISCOSITY, Config)

L_BOX = 2.0 * math.pi * 4.0
THETA = 30.0
DIFF_D = 1e-3
PEN_ETA = -1e-3
MASK_RADIUS = 0.5
CFL = 0.2
STRETCH_FRONTEND = L_BOX * (1.0 - 0.3) / (2.0 * math.pi)  # frontend.cpp:285-287
# over-relaxation of the FAS smoother's point Newton step: 4.9 V-cycles per
# solve at 256^3 against 7.7 with the plain step (measured over 1.0 ... 1.3)
MG_OMEGA = 1.25

WORKLOADS = {
    # plain FP64, nonlinear Jacobi to residual 1e-10, no spectral viscosity
    "jacobi32": dict(n=32, M=0.8, tau=0.1, Q=-10.0, sigma=0.5, steps=100, sv=False,
                     poisson_mode=KF_PS_JACOBI_RES, precision=KF_FP64),
    # plain FP64, FAS V-cycles (4 levels, 2+2), spectral viscosity beyond 0.6 k_max
    "fas128": dict(n=128, M=1.2, tau=0.1, Q=-10.0, sigma=0.5, steps=1000, sv=True,
                   poisson_mode=KF_PS_FAS, precision=KF_FP64),
    # FP32 bulk (FFTs, products, RK4) with the FP64 Poisson solve, 256^3
    "fp32bulk256": dict(n=256, M=1.0, tau=0.05, Q=-50.0, sigma=0.3, steps=2000, sv=True,
                        poisson_mode=KF_PS_FAS, precision=KF_FP32_BULK),
    # the same 256^3 problem in plain FP64 (the comparison arm)
    "fp64_256": dict(n=256, M=1.0, tau=0.05, Q=-50.0, sigma=0.3, steps=2000, sv=True,
                     poisson_mode=KF_PS_FAS, precision=KF_FP64),
    # adjoint workload geometry (forward part)
    "adj128": dict(n=128, M=0.9, tau=0.1, Q=-20.0, sigma=0.5, steps=200, sv=True,
                   poisson_mode=KF_PS_FAS, precision=KF_FP64),
    # the fp32bulk256 physics on the reference frontend's sine-stretched grid
    # (axis_CoSiSt, m = L (1 - 0.3) / (2 pi): 0.3 h cells at the grain).  The
    # cells' aspect ratios reach 1.7/0.3, so the point smoother of the FAS
    # cycle converges slowly there (about 0.75 per plain V-cycle against 0.07
    # on the equidistant grid): stronger over-relaxation (62 -> 19 cycles per
    # solve at 64^3 for 1.0 -> 1.5) and a higher cycle cap
    "stretch256": dict(n=256, M=1.0, tau=0.05, Q=-50.0, sigma=0.3, steps=2000, sv=True,
                       poisson_mode=KF_PS_FAS, precision=KF_FP32_BULK, stretch=STRETCH_FRONTEND,
                       max_cycles=600, omega=1.5),
}


def fp32_res_tol(Q: float, sigma: float) -> float:
    """Residual target of the FP64 Poisson solve when its source comes from an
    FP32 state (KF_FP32_BULK): the FP32 unit roundoff 2^-23 times the largest
    magnitude of the source rho = e^s + n_d, which the grain's peak density
    |Q| / (pi^1.5 sigma^3) sets (fkt3d_Gauss, masks.hpp:351-366).  Below that the
    solve only resolves the rounding of its own input; the FP64 residual, Newton
    update and coarsest solve are unchanged.  The FP64 path keeps 1e-10."""
    return 2.0 ** -23 * abs(Q) / (math.pi ** 1.5 * sigma ** 3)


def config_for(w: dict, n: int | None = None, precision: int | None = None, **over) -> Config:
    """kf_config of a workload dict (optionally on another grid size)."""
    n = n or w["n"]
    terms = KF_T_ALL if w["sv"] else (KF_T_ALL & ~KF_T_SVISCOSITY)
    # multigrid levels: 4 at 128^3 (the stated plan), coarsest 8^3 at 256^3,
    # otherwise halve while even until the coarsest level is at most 16^3
    if n == 128:
        levels = 4
    elif n == 256:
        levels = 6
    else:
        levels, m = 1, n
        while m > 16 and m % 2 == 0:
            m //= 2
            levels += 1
    prec = w["precision"] if precision is None else precision
    res_tol = fp32_res_tol(w["Q"], w["sigma"]) if prec == KF_FP32_BULK else 1e-10
    kw = dict(tau=w["tau"], theta=THETA, diff_D=DIFF_D, sv_eps=0.5, sv_cut=0.6 if w["sv"] else 0.0,
              pen_eta=PEN_ETA, terms=terms, poisson_mode=w["poisson_mode"], nlj_max_it=100000,
              nlj_limit=0.5e-5, res_tol=res_tol, mg_levels=levels, mg_pre=2, mg_post=2, coarse_tol=1e-13,
              max_cycles=w.get("max_cycles", 100), phi_extrap=1, mg_omega=w.get("omega", MG_OMEGA),
              precision=prec, stretch_m=w.get("stretch", 0.0))
    kw.update(over)
    return Config.make(n, L_BOX, w["M"], **kw)


# objective of the adjoint workload: J = h^3 sum w phi_T with a Gaussian window
# exp(-|x - x0|^2 / width^2) of width 2 centred 4 Debye lengths downstream
# (+x, the direction of the mean flow M e_x) of the grain at the origin
WAKE_X0 = (4.0, 0.0, 0.0)
WAKE_WIDTH = 2.0


def wake_window(n: int, L: float = L_BOX, x0=WAKE_X0, width: float = WAKE_WIDTH):
    from . import inputs as I
    x = I.axis_values(n, L)
    r2 = ((x[:, None, None] - x0[0]) ** 2 + (x[None, :, None] - x0[1]) ** 2
          + (x[None, None, :] - x0[2]) ** 2)
    return __import__("numpy").exp(-r2 / (width * width))


def make_inputs(w: dict, n: int | None = None, seed: int = 0):
    """(state, n_d, mask, dt) of a workload, from the seeded generator."""
    from . import inputs as I
    n = n or w["n"]
    m = w.get("stretch", 0.0)
    st = I.initial_state(n, seed=seed)
    nd = I.gauss_charge(n, L_BOX, w["Q"], w["sigma"], m)
    mask = I.sphere_mask(n, L_BOX, MASK_RADIUS, m)
    dt = I.cfl_dt(st, n, L_BOX, w["M"], CFL, m)
    return st, nd, mask, dt
