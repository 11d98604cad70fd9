"""ctypes binding of libkf.so (include/kielflow_b200.h)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))

KF_OK = 0
KF_ERRORS = {-1: "KF_ERR_ARG", -2: "KF_ERR_CUDA", -3: "KF_ERR_NAN", -4: "KF_ERR_NOT_CONVERGED",
             -5: "KF_ERR_NO_DEVICE"}

KF_T_POISSON = 1 << 0
KF_T_DISSIPATION = 1 << 1
KF_T_SVISCOSITY = 1 << 2
KF_T_E_INT = 1 << 3
KF_T_PRESSURE = 1 << 4
KF_T_E_EXT = 1 << 5
KF_T_CONTINUITY = 1 << 6
KF_T_ADVECTION = 1 << 7
KF_T_PENALIZATION = 1 << 8
KF_T_DIFFUSION = 1 << 9
KF_T_SHIPPED = 0xFF
KF_T_ALL = 0x3FF

KF_PS_JACOBI_REF, KF_PS_JACOBI_RES, KF_PS_CASCADIC, KF_PS_FAS = 0, 1, 2, 3
KF_FP64, KF_FP32_BULK = 0, 1

_D = ctypes.POINTER(ctypes.c_double)


class KfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{KF_ERRORS.get(code, code)}: {msg}")
        self.code = code


class Config(ctypes.Structure):
    """kf_config (include/kielflow_b200.h)."""
    _fields_ = [
        ("n", ctypes.c_int), ("L", ctypes.c_double), ("M", ctypes.c_double), ("tau", ctypes.c_double),
        ("theta", ctypes.c_double), ("diff_D", ctypes.c_double), ("sv_eps", ctypes.c_double),
        ("sv_cut", ctypes.c_double), ("pen_eta", ctypes.c_double), ("terms", ctypes.c_int),
        ("poisson_mode", ctypes.c_int), ("nlj_max_it", ctypes.c_int), ("nlj_limit", ctypes.c_double),
        ("res_tol", ctypes.c_double), ("mg_levels", ctypes.c_int), ("mg_pre", ctypes.c_int),
        ("mg_post", ctypes.c_int), ("coarse_tol", ctypes.c_double), ("max_cycles", ctypes.c_int),
        ("phi_extrap", ctypes.c_int), ("precision", ctypes.c_int), ("stretch_m", ctypes.c_double),
        ("mg_omega", ctypes.c_double),
    ]

    @classmethod
    def make(cls, n, L, M, tau=0.1, theta=30.0, diff_D=0.0, sv_eps=0.5, sv_cut=0.0, pen_eta=0.0,
             terms=KF_T_SHIPPED, poisson_mode=KF_PS_JACOBI_REF, nlj_max_it=80, nlj_limit=0.5e-5,
             res_tol=1e-10, mg_levels=4, mg_pre=2, mg_post=2, coarse_tol=1e-13, max_cycles=50,
             phi_extrap=0, precision=KF_FP64, stretch_m=0.0, mg_omega=0.0):
        return cls(n, L, M, tau, theta, diff_D, sv_eps, sv_cut, pen_eta, terms, poisson_mode, nlj_max_it,
                   nlj_limit, res_tol, mg_levels, mg_pre, mg_post, coarse_tol, max_cycles, phi_extrap, precision,
                   stretch_m, mg_omega)

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class DiagOut(ctypes.Structure):
    _fields_ = [("solves", ctypes.c_int), ("last_iterations", ctypes.c_int),
                ("total_iterations", ctypes.c_longlong), ("last_residual", ctypes.c_double),
                ("not_converged", ctypes.c_int), ("charge", ctypes.c_double), ("kinetic", ctypes.c_double),
                ("stage_cycles", ctypes.c_longlong * 4)]


class GradOut(ctypes.Structure):
    """kf_grad_out (include/kielflow_b200.h)."""
    _fields_ = [("J", ctypes.c_double), ("dJ_dM", ctypes.c_double), ("dJ_dtau", ctypes.c_double),
                ("dJ_dnd", ctypes.c_double), ("fwd_ms", ctypes.c_double), ("bwd_ms", ctypes.c_double),
                ("adj_cycles", ctypes.c_longlong), ("adj_solves", ctypes.c_int), ("checkpoints", ctypes.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class TuneOut(ctypes.Structure):
    """kf_tune_out (include/kielflow_b200.h)."""
    _fields_ = [("fft_plan", ctypes.c_int), ("rbgs_rows", ctypes.c_int), ("fft_radices", (ctypes.c_int * 4) * 2),
                ("fft_threads", ctypes.c_int * 2), ("fft_ms", ctypes.c_double * 2), ("rbgs_ms", ctypes.c_double * 4)]

    def as_dict(self):
        return {"fft_plan": self.fft_plan, "rbgs_rows": self.rbgs_rows,
                "fft_radices": [[r for r in row if r] for row in self.fft_radices],
                "fft_threads": list(self.fft_threads), "fft_ms": list(self.fft_ms), "rbgs_ms": list(self.rbgs_ms)}


class Output(ctypes.Structure):
    """kf_output (include/kielflow_b200.h)."""
    _fields_ = [("step", ctypes.c_int), ("t", ctypes.c_double), ("kind", ctypes.c_int),
                ("FUx", _D), ("FUy", _D), ("FUz", _D), ("Fn", _D), ("FPh", _D)]


OUTPUT_FN = ctypes.CFUNCTYPE(None, ctypes.POINTER(Output), ctypes.c_void_p)
KF_OUT_SLICE, KF_OUT_BACKUP = 1, 2
KF_FILE_SLICE, KF_FILE_BACKUP = 1, 2


class FileInfo(ctypes.Structure):
    """kf_file_info (include/kielflow_b200.h)."""
    _fields_ = [("n", ctypes.c_int), ("kind", ctypes.c_int), ("L", ctypes.c_double), ("l0", ctypes.c_double),
                ("time", ctypes.c_double), ("M", ctypes.c_double), ("tau", ctypes.c_double),
                ("theta", ctypes.c_double), ("mu", ctypes.c_double), ("beta", ctypes.c_double),
                ("type", ctypes.c_int), ("m", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def file_info(path: str) -> dict:
    """kf_file_info_read: grid, time and parameters of a .kfh file (no GPU needed)."""
    L = load_library()
    info = FileInfo()
    rc = L.kf_file_info_read(path.encode(), ctypes.byref(info))
    if rc:
        raise KfError(rc, L.kf_last_error(None).decode())
    return info.as_dict()

KF_ADJ_STORE_PHI = 1
KF_ADJ_J_ONLY = 2


def library_path() -> str:
    return os.environ.get("KIELFLOW_B200_LIB", os.path.join(PKG, "libkf.so"))


EXPORTS = [
    "kf_ctx_create", "kf_ctx_destroy", "kf_last_error", "kf_set_stream", "kf_synchronize", "kf_set_state",
    "kf_get_state", "kf_set_sources", "kf_set_phi", "kf_get_phi", "kf_rhs_eval", "kf_rk4_steps",
    "kf_poisson_solve", "kf_diag", "kf_fft_r2c", "kf_fft_c2r", "kf_state_device_ptrs", "kf_launch_count",
    "kf_profile_enable", "kf_profile_read", "kf_profile_class_name", "kf_fft_r2c_noalloc", "kf_adjoint_run",
    "kf_batch_rk4_steps", "kf_set_state_linear", "kf_get_output", "kf_run", "kf_save", "kf_load",
    "kf_file_info_read", "kf_frontend_state", "kf_step_host", "kf_autotune", "kf_set_tuning",
    "kf_set_coarse_block", "kf_set_overlap",
]
KCLASSES = 19

_lib = None


def load_library():
    """Load libkf.so; raises if it is missing (there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise KfError(-5, f"CUDA library not built: {path} (run python -m kielflow_b200.build)")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.kf_ctx_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(vp)]
    L.kf_ctx_destroy.argtypes = [vp]
    L.kf_last_error.argtypes = [vp]
    L.kf_last_error.restype = ctypes.c_char_p
    L.kf_set_stream.argtypes = [vp, vp]
    L.kf_synchronize.argtypes = [vp]
    L.kf_set_state.argtypes = [vp, _D, _D, _D, _D]
    L.kf_get_state.argtypes = [vp, _D, _D, _D, _D]
    L.kf_set_sources.argtypes = [vp, _D, _D]
    L.kf_set_phi.argtypes = [vp, _D]
    L.kf_get_phi.argtypes = [vp, _D]
    L.kf_rhs_eval.argtypes = [vp, ctypes.c_double]
    L.kf_rk4_steps.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    L.kf_poisson_solve.argtypes = [vp, _D, _D]
    L.kf_diag.argtypes = [vp, ctypes.POINTER(DiagOut)]
    L.kf_fft_r2c.argtypes = [vp, _D, _D]
    L.kf_fft_c2r.argtypes = [vp, _D, _D]
    L.kf_state_device_ptrs.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                       ctypes.POINTER(vp)]
    L.kf_launch_count.argtypes = [vp]
    L.kf_launch_count.restype = ctypes.c_longlong
    L.kf_profile_enable.argtypes = [vp, ctypes.c_int]
    L.kf_profile_read.argtypes = [vp, ctypes.c_int, _D, ctypes.POINTER(ctypes.c_longlong), _D]
    L.kf_profile_class_name.argtypes = [ctypes.c_int]
    L.kf_profile_class_name.restype = ctypes.c_char_p
    L.kf_fft_r2c_noalloc.argtypes = [ctypes.c_int, vp, vp, vp]
    L.kf_set_state_linear.argtypes = [vp, _D, _D, _D, _D]
    L.kf_get_output.argtypes = [vp, _D, _D, _D, _D, _D]
    L.kf_run.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                         ctypes.c_char_p, OUTPUT_FN, ctypes.c_void_p]
    L.kf_frontend_state.argtypes = [vp, ctypes.c_double]
    L.kf_step_host.argtypes = [vp, ctypes.c_int, ctypes.c_double, _D, _D, _D, _D]
    L.kf_save.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_double]
    L.kf_load.argtypes = [vp, ctypes.c_char_p, _D]
    L.kf_file_info_read.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    L.kf_batch_rk4_steps.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, _D]
    L.kf_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(TuneOut)]
    L.kf_set_tuning.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.kf_set_coarse_block.argtypes = [vp, ctypes.c_int]
    L.kf_set_overlap.argtypes = [vp, ctypes.c_int]
    L.kf_adjoint_run.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D,
                                 ctypes.POINTER(GradOut), _D, _D]
    _lib = L
    return L


def _ptr(a: np.ndarray):
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data_as(_D)


def batch_rk4(contexts, dts, nsteps: int):
    """kf_batch_rk4_steps: nsteps RK4 steps of every context (its own dt),
    queued from this thread on the contexts' streams; returns when all are done."""
    L = load_library()
    n = len(contexts)
    arr = (ctypes.c_void_p * n)(*[c.h.value for c in contexts])
    d = np.ascontiguousarray(dts, np.float64)
    if d.shape != (n,):
        raise ValueError("one dt per context")
    rc = L.kf_batch_rk4_steps(arr, n, nsteps, _ptr(d))
    if rc:
        raise KfError(rc, L.kf_last_error(None).decode())


class Context:
    """One grid resident on the GPU (kf_ctx)."""

    def __init__(self, cfg: Config):
        self.L = load_library()
        self.cfg = cfg
        h = ctypes.c_void_p()
        rc = self.L.kf_ctx_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc:
            raise KfError(rc, self.L.kf_last_error(None).decode())
        self.h = h
        n = cfg.n
        self.shape_c = (n, n, n // 2 + 1)
        self.shape_r = (n, n, n)

    def _check(self, rc):
        if rc:
            raise KfError(rc, self.L.kf_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.kf_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- data movement -------------------------------------------------
    def set_state(self, FUx, FUy, FUz, Fni):
        arrs = [np.ascontiguousarray(a, np.complex128) for a in (FUx, FUy, FUz, Fni)]
        for a in arrs:
            if a.shape != self.shape_c:
                raise ValueError(f"spectral field must have shape {self.shape_c}")
        self._check(self.L.kf_set_state(self.h, *[a.ctypes.data_as(_D) for a in arrs]))

    def set_state_linear(self, FUx, FUy, FUz, Fn):
        """kf_set_state_linear: u' spectra and the spectrum of n (linear scale)."""
        arrs = [np.ascontiguousarray(a, np.complex128) for a in (FUx, FUy, FUz, Fn)]
        for a in arrs:
            if a.shape != self.shape_c:
                raise ValueError(f"spectral field must have shape {self.shape_c}")
        self._check(self.L.kf_set_state_linear(self.h, *[a.ctypes.data_as(_D) for a in arrs]))

    def get_output(self):
        """kf_get_output: (FUx, FUy, FUz, Fn, FPh) as save_slice receives them."""
        out = [np.empty(self.shape_c, np.complex128) for _ in range(5)]
        self._check(self.L.kf_get_output(self.h, *[a.ctypes.data_as(_D) for a in out]))
        return out

    def run(self, iterations: int, dt: float, t0: float = 0.0, slice_every: int = 10, backup_every: int = 50,
            callback=None, out_dir: str | None = None):
        """kf_run: the reference's time loop; callback(step, t, kind, fields) gets
        copies of (FUx, FUy, FUz, Fn, FPh) at each output step; with out_dir the
        slice / backup .kfh files are written there."""
        nc = int(np.prod(self.shape_c))
        shape = self.shape_c

        def fn(p, _user):
            o = p.contents
            fields = [np.ctypeslib.as_array(getattr(o, k), shape=(2 * nc,)).view(np.complex128).reshape(shape).copy()
                      for k in ("FUx", "FUy", "FUz", "Fn", "FPh")]
            if callback is not None:
                callback(o.step, o.t, o.kind, fields)

        cfn = OUTPUT_FN(fn)
        self._check(self.L.kf_run(self.h, iterations, dt, t0, slice_every, backup_every,
                                  None if out_dir is None else out_dir.encode(), cfn, None))

    def frontend_state(self, n_background: float = 1.0):
        """kf_frontend_state: the frontend's initial state from the context's n_d."""
        self._check(self.L.kf_frontend_state(self.h, n_background))

    def save(self, path: str, kind: int = KF_FILE_BACKUP, t: float = 0.0):
        """kf_save: the current state as a slice or backup .kfh file."""
        self._check(self.L.kf_save(self.h, path.encode(), kind, t))

    def load(self, path: str) -> float:
        """kf_load: a backup .kfh file into the state and phi; returns its time."""
        t = ctypes.c_double()
        self._check(self.L.kf_load(self.h, path.encode(), ctypes.byref(t)))
        return t.value

    def get_state(self, out=None):
        out = out or [np.empty(self.shape_c, np.complex128) for _ in range(4)]
        self._check(self.L.kf_get_state(self.h, *[a.ctypes.data_as(_D) for a in out]))
        return out

    def set_sources(self, nd=None, mask=None):
        nd = None if nd is None else np.ascontiguousarray(nd, np.float64)
        mask = None if mask is None else np.ascontiguousarray(mask, np.float64)
        self._check(self.L.kf_set_sources(self.h, None if nd is None else _ptr(nd),
                                          None if mask is None else _ptr(mask)))

    def set_phi(self, phi):
        phi = np.ascontiguousarray(phi, np.float64)
        self._check(self.L.kf_set_phi(self.h, _ptr(phi)))

    def get_phi(self):
        out = np.empty(self.shape_r, np.float64)
        self._check(self.L.kf_get_phi(self.h, _ptr(out)))
        return out

    # ---- the hot path --------------------------------------------------
    def rhs(self, t: float = 0.0):
        self._check(self.L.kf_rhs_eval(self.h, t))

    def step_host(self, arrays, dt: float, nsteps: int = 1):
        """kf_step_host: advance the state held in four host arrays (complex128,
        C-contiguous, updated in place)."""
        for a in arrays:
            if a.shape != self.shape_c or a.dtype != np.complex128 or not a.flags["C_CONTIGUOUS"]:
                raise ValueError(f"state arrays must be C-contiguous complex128 {self.shape_c}")
        self._check(self.L.kf_step_host(self.h, nsteps, dt, *[a.ctypes.data_as(_D) for a in arrays]))

    def autotune(self, reps: int = 5) -> dict:
        """kf_autotune: time the transform plans and smoother shapes on this
        context's buffers, keep the fastest; returns the choices and timings."""
        o = TuneOut()
        self._check(self.L.kf_autotune(self.h, reps, ctypes.byref(o)))
        return o.as_dict()

    def set_tuning(self, fft_plan: int, rbgs_rows: int):
        """kf_set_tuning: select the transform plan (0, 1) and the smoother: 4, 8
        (the default) or 16 rows per block of the half-sweep kernel, or 0 for the
        streaming TMA-staged sweep."""
        self._check(self.L.kf_set_tuning(self.h, fft_plan, rbgs_rows))

    def set_coarse_block(self, on: bool):
        """kf_set_coarse_block: run the V-cycle's levels of at most 16^3 points
        (when a level lies below them) as one shared-memory block (True, the
        default) or level by level (False); bit-identical potentials."""
        self._check(self.L.kf_set_coarse_block(self.h, 1 if on else 0))

    def set_overlap(self, on: bool):
        """kf_set_overlap: in the captured step, run the u' and s transforms
        beside the Poisson solve on a second stream (True, the default) or
        after it (False); bit-identical results."""
        self._check(self.L.kf_set_overlap(self.h, 1 if on else 0))

    def rk4(self, dt: float, nsteps: int = 1):
        self._check(self.L.kf_rk4_steps(self.h, nsteps, dt))

    def poisson(self, phi, rho):
        phi = np.array(phi, dtype=np.float64, order="C", copy=True)
        rho = np.ascontiguousarray(rho, np.float64)
        self._check(self.L.kf_poisson_solve(self.h, _ptr(phi), _ptr(rho)))
        return phi

    def adjoint(self, w, nsteps: int, dt: float, ckpt_every: int = 15, flags: int = 0,
                want_dn0: bool = True, want_lam0: bool = False):
        """kf_adjoint_run: J = h^3 sum w phi_T and its gradients (a dict; 'dn0' is
        dJ/dn0 as an (n, n, n) array, 'lam0' the four spectral cotangents)."""
        w = np.ascontiguousarray(w, np.float64)
        if w.shape != self.shape_r:
            raise ValueError(f"w must have shape {self.shape_r}")
        g = GradOut()
        dn0 = np.empty(self.shape_r, np.float64) if want_dn0 else None
        lam0 = np.empty((4,) + self.shape_c, np.complex128) if want_lam0 else None
        self._check(self.L.kf_adjoint_run(self.h, nsteps, dt, ckpt_every, flags, _ptr(w), ctypes.byref(g),
                                          None if dn0 is None else _ptr(dn0),
                                          None if lam0 is None else lam0.ctypes.data_as(_D)))
        out = g.as_dict()
        out["dn0"] = dn0
        out["lam0"] = lam0
        return out

    def diag(self) -> DiagOut:
        d = DiagOut()
        self._check(self.L.kf_diag(self.h, ctypes.byref(d)))
        return d

    def r2c(self, x):
        x = np.ascontiguousarray(x, np.float64)
        out = np.empty(self.shape_c, np.complex128)
        self._check(self.L.kf_fft_r2c(self.h, _ptr(x), out.ctypes.data_as(_D)))
        return out

    def c2r(self, F):
        F = np.ascontiguousarray(F, np.complex128)
        out = np.empty(self.shape_r, np.float64)
        self._check(self.L.kf_fft_c2r(self.h, F.ctypes.data_as(_D), _ptr(out)))
        return out

    def synchronize(self):
        self._check(self.L.kf_synchronize(self.h))

    def set_stream(self, stream_handle):
        self._check(self.L.kf_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def device_state_ptrs(self):
        p = [ctypes.c_void_p() for _ in range(4)]
        self._check(self.L.kf_state_device_ptrs(self.h, *[ctypes.byref(x) for x in p]))
        return [x.value for x in p]

    def launch_count(self) -> int:
        return int(self.L.kf_launch_count(self.h))

    def profile(self, on: bool):
        self._check(self.L.kf_profile_enable(self.h, 1 if on else 0))

    def profile_read(self):
        """{kernel class name: (ms, launches, algorithmic bytes)} since profile(True)."""
        out = {}
        for k in range(KCLASSES):
            ms, n, b = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double()
            self._check(self.L.kf_profile_read(self.h, k, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(b)))
            if n.value:
                out[self.L.kf_profile_class_name(k).decode()] = (ms.value, n.value, b.value)
        return out
