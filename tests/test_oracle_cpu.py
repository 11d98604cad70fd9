"""The CPU oracle: FFT shim vs numpy, restatement vs the reference's own code.

The reference ships no tests or golden vectors (it has no test directory), so
the oracle is pinned two ways: against the reference compiled here from its
own sources (oracle/_ref, bit for bit) and against the committed fixtures in
tests/golden/ that make_golden.py wrote from that build.
"""
import os

import numpy as np
import pytest

from kielflow_b200 import configs as C
from kielflow_b200 import inputs as I
from oracle import bind

GOLD = os.path.join(os.path.dirname(__file__), "golden")
L = I.L_DEFAULT


def _gold(name):
    return np.load(os.path.join(GOLD, name))


@pytest.mark.parametrize("shape", [(4, 4, 4), (8, 6, 10), (16, 16, 16), (12, 24, 96), (32, 32, 32), (96, 8, 8)])
def test_shim_fft_matches_numpy(shape):
    rng = np.random.default_rng(sum(shape))
    x = rng.standard_normal(shape)
    Lb = bind.lib()
    out = np.zeros(shape[:2] + (shape[2] // 2 + 1,), np.complex128)
    Lb.kfs_r2c_3d(*shape, x.ctypes.data_as(bind._D), out.ctypes.data_as(bind._D))
    ref = np.fft.rfftn(x)
    assert np.abs(out - ref).max() <= 1e-15 * np.abs(ref).max() * 8
    back = np.zeros(shape)
    Lb.kfs_c2r_3d(*shape, ref.ctypes.data_as(bind._D), back.ctypes.data_as(bind._D))
    assert np.abs(back / np.prod(shape) - x).max() <= 1e-15 * np.abs(x).max() * 8


def test_oracle_ops_match_golden():
    g = _gold("ops16.npz")
    F = bind.r2c(g["x"])
    assert np.array_equal(F, g["F"])
    assert np.array_equal(bind.c2r(g["F"]), g["xb"])
    o = bind.Oracle(bind.config(16, L, 0.8))
    P, SV, PF = o.tables()
    assert np.array_equal(g["F"] * P, g["dealiased"])
    assert np.array_equal(g["F"] * PF, g["phifilt"])


def test_oracle_transfer_matches_golden():
    g = _gold("transfer.npz")
    assert np.array_equal(bind.transfer(0, g["a8"], L), g["up"])
    assert np.array_equal(bind.transfer(1, g["a16"], L), g["dn"])


def test_oracle_jacobi_and_cascadic_match_golden():
    g = _gold("poisson32.npz")
    o = bind.Oracle(bind.config(32, L, 0.8, poisson_mode=bind.PS_JACOBI_REF, nlj_max_it=60, nlj_limit=1e-9))
    phi = o.poisson(np.zeros((32, 32, 32)), g["rho"])
    assert np.array_equal(phi, g["phi_jacobi60"])
    o2 = bind.Oracle(bind.config(32, L, 0.8, poisson_mode=bind.PS_CASCADIC))
    phi2 = o2.poisson(np.zeros((32, 32, 32)), g["rho"])
    assert np.array_equal(phi2, g["phi_cascadic"])


def test_oracle_shipped_rhs_and_rk4_match_golden():
    g = _gold("shipped16.npz")
    st = [g["s0_ux"], g["s0_uy"], g["s0_uz"], g["s0_s"]]
    cfg = bind.config(int(g["n"]), L, float(g["M"]), tau=float(g["tau"]), theta=float(g["theta"]),
                      terms=bind.KFO_SHIPPED, poisson_mode=bind.PS_CASCADIC)
    o = bind.Oracle(cfg)
    o.set_state(st)
    o.set_sources(g["nd"], g["mask"])
    o.rhs()
    out = o.get_state()
    for a, k in zip(out, ("rhs_ux", "rhs_uy", "rhs_uz", "rhs_s")):
        assert np.array_equal(a, g[k]), k
    assert np.array_equal(o.get_phi(), g["rhs_phi"])
    o2 = bind.Oracle(cfg)
    o2.set_state(st)
    o2.set_sources(g["nd"], g["mask"])
    o2.rk4(float(g["dt"]), int(g["nsteps"]))
    for a, k in zip(o2.get_state(), ("rk_ux", "rk_uy", "rk_uz", "rk_s")):
        assert np.array_equal(a, g[k]), k


@pytest.mark.skipif(not bind.ref_available(), reason="reference not compiled here")
def test_oracle_matches_reference_build_live():
    """Same as the golden check, on a second seed, against the live reference build."""
    n, M = 16, 1.1
    st = I.initial_state(n, seed=11)
    nd = I.gauss_charge(n, L, -5.0, 0.7)
    mask = I.sphere_mask(n, L, 0.5)
    R = bind.Reference(n, L, M, 0.2, 30.0, poisson_mode=1)
    R.set_state(st)
    R.set_real(0, nd)
    R.set_real(1, mask)
    R.rhs()
    o = bind.Oracle(bind.config(n, L, M, tau=0.2, terms=bind.KFO_SHIPPED, poisson_mode=bind.PS_CASCADIC))
    o.set_state(st)
    o.set_sources(nd, mask)
    o.rhs()
    for a, b in zip(R.get_state(), o.get_state()):
        assert np.array_equal(a, b)
    assert np.array_equal(R.sv(), o.tables()[1])


def test_oracle_fas_and_jacobi_agree_on_converged_phi():
    """Both residual-stopped solvers reach the same discrete solution."""
    n = 32
    st = I.initial_state(n, seed=5)
    nd = I.gauss_charge(n, L, -10.0, 0.5)
    rho = np.exp(np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2))) + nd
    oj = bind.Oracle(bind.config(n, L, 0.8, poisson_mode=bind.PS_JACOBI_RES, nlj_max_it=100000, res_tol=1e-11))
    of = bind.Oracle(bind.config(n, L, 0.8, poisson_mode=bind.PS_FAS, mg_levels=2, res_tol=1e-11))
    pj = oj.poisson(np.zeros((n, n, n)), rho)
    pf = of.poisson(np.zeros((n, n, n)), rho)
    assert oj.residual(pj, rho) <= 1e-11 and of.residual(pf, rho) <= 1e-11
    assert np.abs(pj - pf).max() < 1e-10


def test_workload_inputs_are_deterministic():
    w = C.WORKLOADS["jacobi32"]
    a = C.make_inputs(w, n=16, seed=3)
    b = C.make_inputs(w, n=16, seed=3)
    for x, y in zip(a[0], b[0]):
        assert np.array_equal(x, y)
    assert a[3] == b[3]
    u = np.fft.irfftn(a[0][0], s=(16, 16, 16), axes=(0, 1, 2))
    assert 1e-4 < np.abs(u).max() < 1e-1


def test_oracle_stretched_grid_matches_golden():
    """axis_CoSiSt (the frontend's sine-stretched grid): positions, the sampled
    dust, the chain-rule derivatives, the cascadic multigrid solve, the shipped
    right-hand side and three RK4 steps of the reference, bit for bit."""
    g = _gold("stretch16.npz")
    m, n = float(g["m"]), int(g["n"])
    assert m == pytest.approx(I.frontend_stretch(L), rel=1e-15)
    cfg = bind.config(n, L, float(g["M"]), tau=float(g["tau"]), theta=float(g["theta"]),
                      terms=bind.KFO_SHIPPED, poisson_mode=bind.PS_CASCADIC, stretch_m=m)
    o = bind.Oracle(cfg)
    assert np.array_equal(o.positions(), g["positions"])
    assert np.array_equal(np.array([I.val_at(i, n, L, m) for i in range(-1, n + 1)]), g["positions"])
    assert np.allclose(I.gauss_charge(n, L, -5.0, 0.7, m), g["gauss"], rtol=1e-14, atol=0)
    for d, k in enumerate(("dx", "dy", "dz")):
        assert np.array_equal(o.deriv(d, g["F"]), g[k]), k
    st = [g["s0_ux"], g["s0_uy"], g["s0_uz"], g["s0_s"]]
    o.set_state(st)
    o.set_sources(g["nd"], g["mask"])
    o.rhs()
    for a, k in zip(o.get_state(), ("rhs_ux", "rhs_uy", "rhs_uz", "rhs_s")):
        assert np.array_equal(a, g[k]), k
    assert np.array_equal(o.get_phi(), g["rhs_phi"])
    o2 = bind.Oracle(cfg)
    o2.set_state(st)
    o2.set_sources(g["nd"], g["mask"])
    o2.rk4(float(g["dt"]), int(g["nsteps"]))
    for a, k in zip(o2.get_state(), ("rk_ux", "rk_uy", "rk_uz", "rk_s")):
        assert np.array_equal(a, g[k]), k
    o3 = bind.Oracle(bind.config(32, L, 0.8, poisson_mode=bind.PS_CASCADIC, stretch_m=m))
    assert np.array_equal(o3.poisson(np.zeros((32, 32, 32)), g["rho32"]), g["phi_cascadic32"])


def test_oracle_stretched_fas_reaches_jacobi_solution():
    """The FAS cycle on stretched spacings converges to the discrete solution
    the point-Jacobi solver reaches (same stencil, same tolerance)."""
    n = 32
    m = I.frontend_stretch(L)
    st = I.initial_state(n, seed=5)
    nd = I.gauss_charge(n, L, -10.0, 0.5, m)
    rho = np.exp(np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2))) + nd
    oj = bind.Oracle(bind.config(n, L, 0.8, poisson_mode=bind.PS_JACOBI_RES, nlj_max_it=200000, res_tol=1e-11,
                                 stretch_m=m))
    of = bind.Oracle(bind.config(n, L, 0.8, poisson_mode=bind.PS_FAS, mg_levels=2, res_tol=1e-11, stretch_m=m))
    pj = oj.poisson(np.zeros((n, n, n)), rho)
    pf = of.poisson(np.zeros((n, n, n)), rho)
    # the Jacobi stop tests the iterate before its last sweep
    assert oj.residual(pj, rho) <= 2e-11 and of.residual(pf, rho) <= 1e-11
    assert np.abs(pj - pf).max() < 1e-9
    assert of.stats().not_converged == 0


def test_known_answers_single_mode_mask_and_constant_source():
    """Analytic checks of the restatement (no reference run needed):
    - the spectral derivative of cos(2 pi m x / L) along each axis is
      -(2 pi m / L) sin(2 pi m x / L) (OP_partial_derivative, uniform grid);
    - the 2/3 mask keeps exactly the modes with |k~| < 2/3 (an independent count);
    - with a constant source rho = c every solver's fixed point is phi = ln c."""
    n, m = 32, 3
    o = bind.Oracle(bind.config(n, L, 0.8, poisson_mode=bind.PS_JACOBI_RES, nlj_max_it=100000, res_tol=1e-13))
    x = I.axis_values(n, L)
    kx = 2.0 * np.pi * m / L
    for d in range(3):
        shape = [1, 1, 1]
        shape[d] = n
        f = np.broadcast_to(np.cos(kx * x).reshape(shape), (n, n, n)).copy()
        df = bind.c2r(o.deriv(d, bind.r2c(f)))
        want = np.broadcast_to((-kx * np.sin(kx * x)).reshape(shape), (n, n, n))
        assert np.abs(df - want).max() < 1e-12 * kx
    P = o.tables()[0]
    k = I.k_values(n, L) / I.k_values(n, L)[n // 2]
    kk = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, : n // 2 + 1] ** 2)
    assert int(P.sum()) == int((kk < 2.0 / 3.0).sum())
    assert set(np.unique(P)) <= {0.0, 1.0}
    for mode in (bind.PS_JACOBI_RES, bind.PS_FAS, bind.PS_CASCADIC):
        oc = bind.Oracle(bind.config(n, L, 0.8, poisson_mode=mode, nlj_max_it=100000, res_tol=1e-13, mg_levels=2,
                                     mg_omega=1.25))
        c = 1.7
        phi = oc.poisson(np.zeros((n, n, n)), np.full((n, n, n), c))
        assert np.abs(phi - np.log(c)).max() < 1e-9, mode


def test_oracle_fas_over_relaxed_reaches_the_same_solution():
    """The over-relaxed smoother (mg_omega 1.25) and the plain Newton step
    reach the same discrete solution (its cycle savings show on the deeper
    hierarchies and warm-started solves of the time step, not on this
    two-level solve from zero)."""
    n = 32
    st = I.initial_state(n, seed=5)
    nd = I.gauss_charge(n, L, -10.0, 0.5)
    rho = np.exp(np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2))) + nd
    out = {}
    for om in (0.0, 1.25):
        o = bind.Oracle(bind.config(n, L, 0.8, poisson_mode=bind.PS_FAS, mg_levels=2, res_tol=1e-11, mg_omega=om))
        phi = o.poisson(np.zeros((n, n, n)), rho)
        s = o.stats()
        assert o.residual(phi, rho) <= 1e-11 and s.not_converged == 0
        out[om] = (phi, s.last_iterations)
    assert np.abs(out[0.0][0] - out[1.25][0]).max() < 1e-10


def test_oracle_config_layout_matches_its_header(tmp_path):
    """kfo_config (oracle/kf_oracle.h) against bind.KfoConfig, compiled with the
    host C compiler: size and every field offset."""
    import ctypes
    import os
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    hdr = os.path.join(os.path.dirname(bind.__file__), "kf_oracle.h")
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{hdr}"', "int main(void) {",
             'printf("sizeof %zu\\n", sizeof(kfo_config));']
    for f, _ in bind.KfoConfig._fields_:
        lines.append(f'printf("{f} %zu\\n", offsetof(kfo_config, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "kfo.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "kfo"
    subprocess.run([cc, "-std=c99", "-o", str(exe), str(src)], check=True)
    got = dict(line.split() for line in
               subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines())
    assert int(got["sizeof"]) == ctypes.sizeof(bind.KfoConfig)
    for f, _ in bind.KfoConfig._fields_:
        assert int(got[f]) == getattr(bind.KfoConfig, f).offset, f


# ------------------------------------------------- the terms the shipped RHS lacks
# Diffusion, masking penalization and the spectral-viscosity cut are not called by
# the reference's rhs_standard.cpp; their formula sources are effect_penalization.cpp
# and effect_diffusion.cpp, compiled into oracle/_ref from the reference's sources.

needs_ref = pytest.mark.skipif(not bind.ref_available(), reason="reference not compiled here")


def _seeded_spectra(n, seed, count):
    rng = np.random.default_rng(seed)
    return [bind.r2c(rng.standard_normal((n, n, n))) for _ in range(count)]


@needs_ref
@pytest.mark.parametrize("fix", [0.0, -1.0, -10.0])
def test_oracle_penalization_matches_reference_effect(fix):
    """The restatement's masking penalization is effect_penalization::execute
    (effect_penalization.cpp:21-44) bit for bit, on a ragged mask."""
    n = 16
    rng = np.random.default_rng(7)
    H = (rng.random((n, n, n)) < 0.3).astype(np.float64)
    H[0, 0, :] = 0.5  # a partial cell value, not only 0/1
    F_in, F_out = _seeded_spectra(n, 11, 2)
    o = bind.Oracle(bind.config(n, L, 1.0, pen_eta=C.PEN_ETA))
    o.set_sources(np.zeros((n, n, n)), H)
    assert np.array_equal(o.penalize(fix, F_in, F_out), bind.ref_penalize(n, L, C.PEN_ETA, fix, H, F_in, F_out))


@needs_ref
def test_reference_penalization_guard():
    """effect_penalization's constructor refuses a positive damping (:7-12)
    (the library's context refuses pen_eta > 0 the same way: GPU tests)."""
    n = 8
    F = _seeded_spectra(n, 3, 1)[0]
    with pytest.raises(RuntimeError, match="damping"):
        bind.ref_penalize(n, L, 1e-3, 0.0, np.zeros((n, n, n)), F, F)


def test_oracle_diffusion_single_mode_known_answer():
    """Laplacian diffusion alone: d/dt q^ = -D |k|^2 q^ for a single Fourier
    mode of every field (k from the axis's k_val_at, the Nyquist +pi n/L of
    axis_EqSt.cpp:57-61 included), to the last bit or two."""
    n = 16
    D = C.DIFF_D
    kv = [2 * np.pi / L * (i if i <= n // 2 else i - n) for i in range(n)]
    o = bind.Oracle(bind.config(n, L, 1.0, diff_D=D, terms=bind.KFO_DIFFUSION))
    o.set_sources(np.zeros((n, n, n)), np.zeros((n, n, n)))
    for m in [(1, 0, 1), (1, 2, 3), (0, 0, 5), (4, 4, 4), (8, 15, 7)]:
        F = np.zeros((n, n, n // 2 + 1), np.complex128)
        F[m] = 0.3 - 0.7j
        o.set_state([F, 2 * F, -F, 0.5 * F])
        o.rhs()
        k2 = kv[m[0]] ** 2 + kv[m[1]] ** 2 + kv[m[2]] ** 2
        for got, a in zip(o.get_state(), (1.0, 2.0, -1.0, 0.5)):
            want = -D * k2 * a * F
            assert np.abs(got - want).max() <= 4.5e-16 * np.abs(want).max()


@needs_ref
def test_oracle_diffusion_matches_reference_effect_imaginary_part():
    """effect_diffusion::execute (effect_diffusion.cpp:16-44) subtracts nu times
    the sum of the three second derivatives (OP_partial_derivative twice, the
    Nyquist k of axis_EqSt.cpp:57-61 included) from the accumulator that the
    right-hand side negates.  Its imaginary part agrees with the restatement to
    rounding; its real part uses the imaginary parts again (:39-40), which the
    restatement does not copy: there it is D |k|^2 Re q^."""
    import subprocess
    import sys
    # effect_diffusion keeps function-static derivative operators: its own process
    code = (
        "import numpy as np, sys; sys.path.insert(0, %r)\n"
        "from oracle import bind\n"
        "from kielflow_b200 import inputs as I\n"
        "n, L, D = 16, I.L_DEFAULT, 1e-3\n"
        "rng = np.random.default_rng(5)\n"
        "F = bind.r2c(rng.standard_normal((n, n, n)))\n"
        "o = bind.Oracle(bind.config(n, L, 1.0, diff_D=D, terms=bind.KFO_DIFFUSION))\n"
        "o.set_sources(np.zeros((n, n, n)), np.zeros((n, n, n)))\n"
        "o.set_state([F, F, F, F]); o.rhs(); fb = -o.get_state()[3]\n"
        "r = bind.ref_diffuse(n, L, D, F, np.zeros_like(F))\n"
        "print(float(np.abs(r.imag - fb.imag).max() / np.abs(fb.imag).max()),"
        " bool(np.array_equal(r.real, r.imag)),"
        " float(np.abs(fb.real - fb.imag).max() / np.abs(fb.real).max()))\n"
    ) % os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    e_im, slip, re_vs_im = out.stdout.split()
    assert float(e_im) <= 1e-15
    assert slip == "True"           # the reference's real part repeats the imaginary sum
    assert float(re_vs_im) > 1e-3   # the restatement's real part does not
