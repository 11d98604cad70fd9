"""Discrete adjoint of the FP64 time step (kf_adjoint_run) against central
finite differences of the same forward map, through the test-only
torch.autograd.Function of adjoint_harness.

The finite-difference runs solve every Poisson problem with a fixed number of
V-cycles (res_tol <= 0) from a shared, converged initial guess, so that J is a
smooth function of the inputs; the step is 1e-6 (absolute for M and tau,
relative for Q, and along a unit-amplitude low-mode direction for n0).
Tolerance: 1e-6 relative.
"""
import numpy as np
import pytest
import torch

import kielflow_b200 as kf
from kielflow_b200 import inputs as I

from adjoint_harness import WakePotential, WakeProblem

pytestmark = pytest.mark.gpu

FD_STEP = 1e-6
TOL = 1e-6


def low_mode_direction(n, seed=7):
    """Unit max-amplitude real field on the integer modes 0 < |m| <= 3."""
    H = I.noise_spectrum(n, seed, 11, amp=1.0, kmax=3)
    d = np.fft.irfftn(H, s=(n, n, n), axes=(0, 1, 2))
    return d / np.abs(d).max()


def fd_check(prob, M, tau, Q):
    n0 = prob.n0
    Mt = torch.tensor(M, dtype=torch.float64, requires_grad=True)
    taut = torch.tensor(tau, dtype=torch.float64, requires_grad=True)
    Qt = torch.tensor(Q, dtype=torch.float64, requires_grad=True)
    n0t = torch.tensor(n0, requires_grad=True)
    J = WakePotential.apply(Mt, taut, Qt, n0t, prob)
    gM, gtau, gQ, gn0 = torch.autograd.grad(J, (Mt, taut, Qt, n0t))
    d = low_mode_direction(prob.n)
    Jf = lambda **kw: prob.run(kw.get("M", M), kw.get("tau", tau), kw.get("Q", Q), kw.get("n0", n0),
                               grad=False)["J"]
    hQ = FD_STEP * abs(Q)
    fd = {
        "M": (Jf(M=M + FD_STEP) - Jf(M=M - FD_STEP)) / (2 * FD_STEP),
        "tau": (Jf(tau=tau + FD_STEP) - Jf(tau=tau - FD_STEP)) / (2 * FD_STEP),
        "Q": (Jf(Q=Q + hQ) - Jf(Q=Q - hQ)) / (2 * hQ),
        "n0.d": (Jf(n0=n0 + FD_STEP * d) - Jf(n0=n0 - FD_STEP * d)) / (2 * FD_STEP),
    }
    adj = {"M": float(gM), "tau": float(gtau), "Q": float(gQ), "n0.d": float((gn0.numpy() * d).sum())}
    err = {k: abs(adj[k] - fd[k]) / max(abs(fd[k]), 1e-300) for k in fd}
    print(f"\nJ = {float(J.detach()):.15e}")
    for k in fd:
        print(f"  dJ/d{k:5s} adjoint {adj[k]: .12e}  FD {fd[k]: .12e}  rel {err[k]:.2e}")
    return err


def test_adjoint_vs_fd_small():
    """32^3, all terms (penalization included), 6 steps with checkpoints every
    4 (a full and a ragged segment)."""
    prob = WakeProblem(32, steps=6, ckpt_every=4)
    err = fd_check(prob, 0.9, 0.1, -20.0)
    assert max(err.values()) < TOL, err


def test_adjoint_vs_fd_no_penalization():
    """The penalization-free form of the right-hand side (K = -(lin + r2c(products)))."""
    prob = WakeProblem(32, steps=5, ckpt_every=2, terms=kf.KF_T_ALL & ~kf.KF_T_PENALIZATION)
    err = fd_check(prob, 0.9, 0.1, -20.0)
    assert max(err.values()) < TOL, err


def test_adjoint_store_phi_identical():
    """KF_ADJ_STORE_PHI recomputes the same stage inputs without solving
    Poisson problems: the gradients agree to rounding."""
    prob = WakeProblem(32, steps=6, ckpt_every=4)
    a = prob.run(0.9, 0.1, -20.0, prob.n0)
    b = prob.run(0.9, 0.1, -20.0, prob.n0, flags=kf.KF_ADJ_STORE_PHI)
    for k in ("J", "dJ_dM", "dJ_dtau", "dJ_dQ"):
        assert abs(a[k] - b[k]) <= 1e-12 * abs(a[k]), (k, a[k], b[k])
    assert np.abs(a["dn0"] - b["dn0"]).max() <= 1e-12 * np.abs(a["dn0"]).max()


def test_adjoint_vs_fd_128():
    """The differentiation workload: 128^3, M 0.9, nu 0.1, Q -20, 200 RK4
    steps, checkpoints every 15 steps."""
    prob = WakeProblem(128, steps=200, ckpt_every=15)
    err = fd_check(prob, 0.9, 0.1, -20.0)
    assert max(err.values()) < TOL, err
