"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE).

Loads ``oracle/liboracle.so`` (the restatement, kf_oracle.cpp) and, when it was
built, ``oracle/_ref/libkfref.so`` (the reference's own sources compiled with
ref_capi.cpp).  Only tests/, bench.py's CPU-baseline leg and
__graft_entry__.smoke() import this module; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libkfref.so")
# directory of the kielflow sources that `make ref` compiles; taken from the
# environment only (a machine without them uses the prebuilt _ref files)
REF_SRC = os.environ.get("KF_REFERENCE_SRC", "")

KFO_POISSON = 1 << 0
KFO_DISSIPATION = 1 << 1
KFO_SVISCOSITY = 1 << 2
KFO_E_INT = 1 << 3
KFO_PRESSURE = 1 << 4
KFO_E_EXT = 1 << 5
KFO_CONTINUITY = 1 << 6
KFO_ADVECTION = 1 << 7
KFO_PENALIZATION = 1 << 8
KFO_DIFFUSION = 1 << 9
KFO_SHIPPED = 0xFF
KFO_ALL = 0x3FF

PS_JACOBI_REF, PS_JACOBI_RES, PS_CASCADIC, PS_FAS = 0, 1, 2, 3

_D = ctypes.POINTER(ctypes.c_double)


class KfoConfig(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("L", ctypes.c_double), ("M", ctypes.c_double),
        ("tau", ctypes.c_double), ("theta", ctypes.c_double), ("diff_D", ctypes.c_double),
        ("sv_eps", ctypes.c_double), ("sv_cut", ctypes.c_double), ("pen_eta", ctypes.c_double),
        ("terms", ctypes.c_int), ("poisson_mode", ctypes.c_int), ("nlj_max_it", ctypes.c_int),
        ("nlj_limit", ctypes.c_double), ("res_tol", ctypes.c_double), ("mg_levels", ctypes.c_int),
        ("mg_pre", ctypes.c_int), ("mg_post", ctypes.c_int), ("coarse_tol", ctypes.c_double),
        ("max_cycles", ctypes.c_int), ("phi_extrap", ctypes.c_int), ("stretch_m", ctypes.c_double),
        ("mg_omega", ctypes.c_double),
    ]


class KfoStats(ctypes.Structure):
    _fields_ = [("last_iterations", ctypes.c_int), ("total_iterations", ctypes.c_int),
                ("solves", ctypes.c_int), ("last_residual", ctypes.c_double),
                ("not_converged", ctypes.c_int)]


def build(with_ref: bool = True) -> None:
    """Compile liboracle.so and, when the reference sources are present,
    _ref/libkfref.so (a machine without the reference sources uses the prebuilt files)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if with_ref and REF_SRC and os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)
    elif with_ref and not ref_available():
        print("oracle: KF_REFERENCE_SRC is not set to the kielflow sources and _ref/libkfref.so is "
              "not built; the tests that compare against the reference itself will be skipped")


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        L = ctypes.CDLL(ORACLE_SO)
        L.kfo_create.restype = ctypes.c_void_p
        L.kfo_create.argtypes = [ctypes.POINTER(KfoConfig)]
        for name in ("kfo_destroy",):
            getattr(L, name).argtypes = [ctypes.c_void_p]
        for name in ("kfo_set_state", "kfo_get_state"):
            getattr(L, name).argtypes = [ctypes.c_void_p, _D, _D, _D, _D]
        L.kfo_set_sources.argtypes = [ctypes.c_void_p, _D, _D]
        L.kfo_set_phi.argtypes = [ctypes.c_void_p, _D]
        L.kfo_get_phi.argtypes = [ctypes.c_void_p, _D]
        L.kfo_rhs.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.kfo_positions.argtypes = [ctypes.c_void_p, _D]
        L.kfo_metric.argtypes = [ctypes.c_void_p, _D]
        L.kfo_deriv.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D]
        L.kfo_penalize.argtypes = [ctypes.c_void_p, ctypes.c_double, _D, _D]
        L.kfo_rk4.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.kfo_poisson.argtypes = [ctypes.c_void_p, _D, _D]
        L.kfo_poisson_stats_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(KfoStats)]
        L.kfo_residual.argtypes = [ctypes.c_void_p, _D, _D]
        L.kfo_residual.restype = ctypes.c_double
        L.kfo_tables.argtypes = [ctypes.c_void_p, _D, _D, _D]
        L.kfo_r2c.argtypes = [ctypes.c_int, _D, _D]
        L.kfo_c2r.argtypes = [ctypes.c_int, _D, _D]
        L.kfo_transfer.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _D, _D]
        L.kfs_r2c_3d.argtypes = [ctypes.c_int] * 3 + [_D, _D]
        L.kfs_c2r_3d.argtypes = [ctypes.c_int] * 3 + [_D, _D]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_SO)
        R.kfref_create.restype = ctypes.c_void_p
        R.kfref_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double]
        R.kfref_positions.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _D]
        R.kfref_deriv_m.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _D, _D]
        R.kfref_mg_solve_m.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _D, _D]
        R.kfref_gauss_m.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, _D]
        R.kfref_destroy.argtypes = [ctypes.c_void_p]
        R.kfref_last_error.restype = ctypes.c_char_p
        R.kfref_set_state.argtypes = [ctypes.c_void_p, _D, _D, _D, _D]
        R.kfref_get_state.argtypes = [ctypes.c_void_p, _D, _D, _D, _D]
        R.kfref_set_real.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        R.kfref_get_real.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        R.kfref_get_sv.argtypes = [ctypes.c_void_p, _D]
        R.kfref_rhs.argtypes = [ctypes.c_void_p, ctypes.c_double]
        R.kfref_rk4.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        R.kfref_fft_r2c.argtypes = [ctypes.c_int, ctypes.c_double, _D, _D]
        R.kfref_fft_c2r.argtypes = [ctypes.c_int, ctypes.c_double, _D, _D]
        R.kfref_dealias.argtypes = [ctypes.c_int, ctypes.c_double, _D]
        R.kfref_phi_filter.argtypes = [ctypes.c_int, ctypes.c_double, _D]
        R.kfref_deriv.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, _D, _D]
        R.kfref_nlj_solve.argtypes = [ctypes.c_int, ctypes.c_double, _D, _D, ctypes.c_int,
                                      ctypes.c_double]
        R.kfref_mg_solve.argtypes = [ctypes.c_int, ctypes.c_double, _D, _D]
        R.kfref_transfer.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _D, _D]
        R.kfref_gauss.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]
        R.kfref_penalize.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, _D, _D, _D]
        R.kfref_diffuse.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _D, _D]
        _ref = R
    return _ref


def config(n, L, M, tau=0.1, theta=30.0, diff_D=0.0, sv_eps=0.5, sv_cut=0.0, pen_eta=0.0,
           terms=KFO_SHIPPED, poisson_mode=PS_JACOBI_REF, nlj_max_it=80, nlj_limit=0.5e-5,
           res_tol=1e-10, mg_levels=4, mg_pre=2, mg_post=2, coarse_tol=1e-13, max_cycles=50,
           phi_extrap=0, stretch_m=0.0, mg_omega=0.0):
    return KfoConfig(n, L, M, tau, theta, diff_D, sv_eps, sv_cut, pen_eta, terms, poisson_mode,
                     nlj_max_it, nlj_limit, res_tol, mg_levels, mg_pre, mg_post, coarse_tol,
                     max_cycles, phi_extrap, stretch_m, mg_omega)


class Oracle:
    """The restatement on one grid: state, sources, RHS, RK4, Poisson."""

    def __init__(self, cfg: KfoConfig):
        self.cfg = cfg
        self.n = cfg.n
        self.L = lib()
        self.h = self.L.kfo_create(ctypes.byref(cfg))
        self.shape_c = (cfg.n, cfg.n, cfg.n // 2 + 1)
        self.shape_r = (cfg.n, cfg.n, cfg.n)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.kfo_destroy(self.h)
            self.h = None

    def set_state(self, st):
        arrs = [np.ascontiguousarray(a, dtype=np.complex128) for a in st]
        self.L.kfo_set_state(self.h, *[a.ctypes.data_as(_D) for a in arrs])

    def get_state(self):
        out = [np.zeros(self.shape_c, np.complex128) for _ in range(4)]
        self.L.kfo_get_state(self.h, *[a.ctypes.data_as(_D) for a in out])
        return out

    def set_sources(self, nd, mask):
        nd = np.ascontiguousarray(nd, np.float64)
        mask = np.ascontiguousarray(mask, np.float64)
        self.L.kfo_set_sources(self.h, _p(nd), _p(mask))

    def set_phi(self, phi):
        phi = np.ascontiguousarray(phi, np.float64)
        self.L.kfo_set_phi(self.h, _p(phi))

    def get_phi(self):
        out = np.zeros(self.shape_r)
        self.L.kfo_get_phi(self.h, _p(out))
        return out

    def rhs(self, t=0.0):
        rc = self.L.kfo_rhs(self.h, t)
        if rc:
            raise RuntimeError(f"oracle rhs failed: {rc}")

    def rk4(self, dt, nsteps=1):
        rc = self.L.kfo_rk4(self.h, dt, nsteps)
        if rc:
            raise RuntimeError(f"oracle rk4 failed: {rc}")

    def poisson(self, phi, rho):
        phi = np.array(phi, dtype=np.float64, order="C")
        rho = np.ascontiguousarray(rho, np.float64)
        rc = self.L.kfo_poisson(self.h, _p(phi), _p(rho))
        if rc:
            raise RuntimeError(f"oracle poisson failed: {rc}")
        return phi

    def stats(self):
        s = KfoStats()
        self.L.kfo_poisson_stats_get(self.h, ctypes.byref(s))
        return s

    def residual(self, phi, rho):
        phi = np.ascontiguousarray(phi, np.float64)
        rho = np.ascontiguousarray(rho, np.float64)
        return self.L.kfo_residual(self.h, _p(phi), _p(rho))

    def tables(self):
        P = np.zeros(self.shape_c, np.float64)
        SV = np.zeros(self.shape_c, np.float64)
        PF = np.zeros(self.shape_c, np.float64)
        self.L.kfo_tables(self.h, _p(P), _p(SV), _p(PF))
        return P, SV, PF

    def positions(self):
        """val_at(i) for i = -1 .. n."""
        out = np.zeros(self.n + 2)
        self.L.kfo_positions(self.h, _p(out))
        return out

    def deriv(self, d, F):
        """OP_partial_derivative along axis d of a half spectrum."""
        F = np.ascontiguousarray(F, np.complex128)
        out = np.zeros(self.shape_c, np.complex128)
        self.L.kfo_deriv(self.h, d, F.ctypes.data_as(_D), out.ctypes.data_as(_D))
        return out

    def penalize(self, fix, F_in, F_out):
        """The right-hand side's masking penalization of one field: returns
        r2c((1 - H) c2r(F_out) + H pen_eta (c2r(F_in) - fix))."""
        F_in = np.ascontiguousarray(F_in, np.complex128)
        out = np.array(F_out, np.complex128, order="C", copy=True)
        self.L.kfo_penalize(self.h, fix, F_in.ctypes.data_as(_D), out.ctypes.data_as(_D))
        return out

    def metric(self):
        """The filtered 1/dS of the derivative along one axis (n values)."""
        out = np.zeros(self.n)
        self.L.kfo_metric(self.h, _p(out))
        return out


def ref_penalize(n, L, eta, fix, H, F_in, F_out):
    """effect_penalization(eta, H, fix).execute(F_in, F_out) of the reference
    (effect_penalization.cpp:21-44); returns the new F_out."""
    H = np.ascontiguousarray(H, np.float64)
    F_in = np.ascontiguousarray(F_in, np.complex128)
    out = np.array(F_out, np.complex128, order="C", copy=True)
    R = ref()
    if R.kfref_penalize(n, L, eta, fix, _p(H), F_in.ctypes.data_as(_D), out.ctypes.data_as(_D)):
        raise RuntimeError(R.kfref_last_error().decode())
    return out


def ref_diffuse(n, L, nu, F_in, F_out):
    """effect_diffusion(nu).execute(F_in, F_out) of the reference as written
    (effect_diffusion.cpp:16-44); one grid size per process."""
    F_in = np.ascontiguousarray(F_in, np.complex128)
    out = np.array(F_out, np.complex128, order="C", copy=True)
    R = ref()
    if R.kfref_diffuse(n, L, nu, F_in.ctypes.data_as(_D), out.ctypes.data_as(_D)):
        raise RuntimeError(R.kfref_last_error().decode())
    return out


def r2c(x: np.ndarray) -> np.ndarray:
    n = x.shape[0]
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros((n, n, n // 2 + 1), np.complex128)
    lib().kfo_r2c(n, _p(x), out.ctypes.data_as(_D))
    return out


def c2r(F: np.ndarray) -> np.ndarray:
    """Inverse transform with the reference's 1/N scaling (OP_iFFT.cpp:59-61)."""
    n = F.shape[0]
    F = np.ascontiguousarray(F, np.complex128)
    out = np.zeros((n, n, n), np.float64)
    lib().kfo_c2r(n, F.ctypes.data_as(_D), _p(out))
    return out


def transfer(kind: int, x: np.ndarray, L: float) -> np.ndarray:
    n = x.shape[0]
    m = 2 * n if kind == 0 else n // 2
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros((m, m, m))
    lib().kfo_transfer(kind, n, L, _p(x), _p(out))
    return out


class Reference:
    """The reference's own rhs_standard / Runge_kutta_O4 / Poisson objects
    (compiled from its sources) on one grid."""

    def __init__(self, n, L, M, tau=0.1, theta=30.0, poisson_mode=1, nlj_max_it=80,
                 nlj_limit=0.5e-5, m=0.0):
        self.R = ref()
        self.n = n
        self.h = self.R.kfref_create(n, L, M, tau, theta, poisson_mode, nlj_max_it, nlj_limit, m)
        if not self.h:
            raise RuntimeError(self.R.kfref_last_error().decode())
        self.shape_c = (n, n, n // 2 + 1)
        self.shape_r = (n, n, n)

    def __del__(self):
        if getattr(self, "h", None):
            self.R.kfref_destroy(self.h)
            self.h = None

    def set_state(self, st):
        arrs = [np.ascontiguousarray(a, dtype=np.complex128) for a in st]
        self.R.kfref_set_state(self.h, *[a.ctypes.data_as(_D) for a in arrs])

    def get_state(self):
        out = [np.zeros(self.shape_c, np.complex128) for _ in range(4)]
        self.R.kfref_get_state(self.h, *[a.ctypes.data_as(_D) for a in out])
        return out

    def set_real(self, which, x):
        x = np.ascontiguousarray(x, np.float64)
        self.R.kfref_set_real(self.h, which, _p(x))

    def get_real(self, which):
        out = np.zeros(self.shape_r)
        self.R.kfref_get_real(self.h, which, _p(out))
        return out

    def sv(self):
        out = np.zeros(self.shape_c)
        self.R.kfref_get_sv(self.h, _p(out))
        return out

    def rhs(self, t=0.0):
        if self.R.kfref_rhs(self.h, t):
            raise RuntimeError(self.R.kfref_last_error().decode())

    def rk4(self, dt, nsteps=1):
        if self.R.kfref_rk4(self.h, dt, nsteps):
            raise RuntimeError(self.R.kfref_last_error().decode())
