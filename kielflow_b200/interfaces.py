"""Host mirror of the reference's operator interfaces for the time step.

Each class keeps the reference's name (in Python spelling), its argument
meaning and its in-place behaviour, and raises where the reference throws:

* :class:`RhsStandard` -- ``interface_rhs::solve(t, FUx, FUy, FUz, Fni)``
  (include/interface_rhs.hpp:11-12; src/kielflow/rhs_standard.cpp:89-566):
  replaces the four spectral fields by their time derivative.
* :class:`RungeKuttaO4` -- ``interface_ode_solver::solve(FUx, FUy, FUz, Fni)``
  (include/interface_ODE_solver.hpp:11-12; src/kielflow/RKO4.cpp:50-241):
  advances the fields by one dt.
* :class:`PoissonSolver` -- ``interface_poisson_solver::solve(Phi_IO, rho)``
  (include/interface_poisson_solver.hpp:18) and the relaxation-solver setters
  ``set_max_iterations``, ``set_tolerance``, ``converged`` (:29-31).

The state stays resident on the GPU between calls; numpy arrays passed in are
copied to the device and results copied back, as the reference's field
objects are host memory.
"""
from __future__ import annotations

import math

import numpy as np

from ._lib import (KF_FP64, KF_PS_FAS, KF_PS_JACOBI_REF, KF_T_SHIPPED, Config, Context, KfError)
from .inputs import axis_values, k_values
from .inputs import val_at as _val_at


class Grid:
    """``grid`` of three alike axes (grid_base.cpp:9-17), cubic, l0 = -L/2:
    ``axis_CoEqSt(l0, L, n)`` (axis_EqSt.cpp:6-61, type_id 1) or, with m > 0,
    the sine-stretched ``axis_CoSiSt(l0, L, n, m)`` (axis_SiSt.cpp, type_id 3;
    the reference frontend's grid uses m = L (1 - 0.3) / (2 pi))."""

    def __init__(self, n: int, L: float, m: float = 0.0):
        if not (0.0 <= m and 2.0 * math.acos(-1.0) * m < L):
            raise ValueError("axis_CoSiSt needs 0 <= 2 pi m < L")
        self.Nx = self.Ny = self.Nz = int(n)
        self.n = int(n)
        self.L = float(L)
        self.l0 = -0.5 * L
        self.m = float(m)
        self.type_id = 3 if m else 1

    def val_at(self, i: int) -> float:
        return _val_at(i, self.n, self.L, self.m)

    def dS(self, i: int) -> float:
        """Derivative of the axis map at index i (axis_SiSt.cpp:158-164; 1 for axis_CoEqSt)."""
        pi = math.acos(-1.0)
        x = self.l0 + (self.L / self.n) * i
        return 1.0 - (2.0 * pi * self.m / self.L) * math.cos(2.0 * pi * x / self.L)

    def k_val_at(self, i: int) -> float:
        pi = math.acos(-1.0)
        n = self.n
        return (2.0 * pi * i / self.L) if i <= n // 2 else (2.0 * pi * (i - n) / self.L)

    def x(self) -> np.ndarray:
        return axis_values(self.n, self.L, self.m)

    def k(self) -> np.ndarray:
        return k_values(self.n, self.L)

    @property
    def shape_real(self):
        return (self.n, self.n, self.n)

    @property
    def shape_spectral(self):
        return (self.n, self.n, self.n // 2 + 1)


class Parameters:
    """``parameters`` (include/parameters.hpp:7-21)."""

    def __init__(self, M=0.0, tau=0.0, theta=0.0, mu=0.0, beta=0.0):
        self.pi = math.acos(-1.0)
        self.M, self.tau, self.theta, self.mu, self.beta = M, tau, theta, mu, beta


def _check_spectral(grid: Grid, *fields):
    for f in fields:
        if f.shape != grid.shape_spectral or f.dtype != np.complex128:
            raise ValueError("field size not matching")  # field_real.cpp:164-169


class RhsStandard:
    """``rhs_standard`` on the GPU.

    ``params``, ``potential`` (Phi, kept as the warm start of the next solve,
    as rhs_standard.hpp:45 holds a reference to it), ``density_dust`` (n_d)
    and ``solid_mask`` (H) mirror the reference constructor
    (rhs_standard.cpp:7-8); ``terms``/``poisson``/``precision`` select the
    runtime options of :class:`Config`.
    """

    def __init__(self, params: Parameters, grid: Grid, density_dust, solid_mask, potential=None,
                 terms=KF_T_SHIPPED, diff_D=0.0, sv_eps=0.5, sv_cut=0.0, pen_eta=0.0,
                 poisson_mode=KF_PS_JACOBI_REF, precision=KF_FP64, **poisson_kw):
        self.grid = grid
        self.params = params
        cfg = Config.make(grid.n, grid.L, params.M, tau=params.tau, theta=params.theta, diff_D=diff_D,
                          sv_eps=sv_eps, sv_cut=sv_cut, pen_eta=pen_eta, terms=terms,
                          poisson_mode=poisson_mode, precision=precision, stretch_m=grid.m, **poisson_kw)
        self.ctx = Context(cfg)
        self.ctx.set_sources(density_dust, solid_mask)
        if potential is not None:
            self.ctx.set_phi(potential)

    @property
    def Phi(self) -> np.ndarray:
        return self.ctx.get_phi()

    def solve(self, t: float, FUx, FUy, FUz, Fni) -> None:
        _check_spectral(self.grid, FUx, FUy, FUz, Fni)
        self.ctx.set_state(FUx, FUy, FUz, Fni)
        self.ctx.rhs(t)
        self.ctx.get_state([FUx, FUy, FUz, Fni])


class RungeKuttaO4:
    """``Runge_kutta_O4(rhs, dt)`` (RKO4.hpp:26-38): fixed dt, classic RK4."""

    def __init__(self, rhs: RhsStandard, dt: float = 0.01):
        self.rhs = rhs
        self.dt = float(dt)
        self.t = 0.0

    def solve(self, FUx, FUy, FUz, Fni) -> None:
        _check_spectral(self.rhs.grid, FUx, FUy, FUz, Fni)
        ctx = self.rhs.ctx
        ctx.set_state(FUx, FUy, FUz, Fni)
        ctx.rk4(self.dt, 1)
        ctx.get_state([FUx, FUy, FUz, Fni])
        self.t += self.dt

    def steps(self, nsteps: int) -> None:
        """nsteps steps on the device-resident state (no host copies)."""
        self.rhs.ctx.rk4(self.dt, nsteps)
        self.t += nsteps * self.dt


class PoissonSolver:
    """The nonlinear Poisson solver ``lap phi = exp(phi) - rho`` as an
    ``interface_relaxation_solver``: Jacobi (solver_poisson_jacobi_nlin) or
    multigrid (cascadic plan of kielflow.cpp:207-217, or FAS V-cycles)."""

    def __init__(self, grid: Grid, mode=KF_PS_FAS, **kw):
        self.grid = grid
        self.kw = dict(kw)
        self.mode = mode
        self._converged = False
        self._ctx = None

    def _context(self):
        if self._ctx is None:
            cfg = Config.make(self.grid.n, self.grid.L, 0.0, poisson_mode=self.mode, stretch_m=self.grid.m,
                              **self.kw)
            self._ctx = Context(cfg)
        return self._ctx

    def set_max_iterations(self, it: int):
        self.kw["nlj_max_it" if self.mode in (0, 1) else "max_cycles"] = int(it)
        self._ctx = None

    def set_tolerance(self, tol: float):
        self.kw["nlj_limit" if self.mode == KF_PS_JACOBI_REF else "res_tol"] = float(tol)
        self._ctx = None

    def converged(self) -> bool:
        return self._converged

    def solve(self, Phi_IO: np.ndarray, rho: np.ndarray) -> None:
        if Phi_IO.shape != self.grid.shape_real or rho.shape != self.grid.shape_real:
            raise ValueError("field size not matching")
        ctx = self._context()
        try:
            out = ctx.poisson(Phi_IO, rho)
            self._converged = True
        except KfError as e:
            if e.code != -4:
                raise
            self._converged = False
            out = ctx.get_phi()
        Phi_IO[...] = out

    def stats(self):
        return self._context().diag()
