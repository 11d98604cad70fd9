"""Test-only harness: the wake-potential functional of the FP64 time step as a
torch.autograd.Function whose backward is the discrete adjoint of the C ABI
(kf_adjoint_run).

    J(M, tau, Q, n0) = h^3 sum_x w(x) phi_T(x)

phi_T is the Poisson solution after `steps` RK4 steps from the state
(u'_x, u'_y, u'_z, s^ = r2c(ln n0)) with the dust charge Q * g(x) (g the unit
Gaussian grain) and the window w of kielflow_b200.configs.wake_window.
"""
from __future__ import annotations

import numpy as np
import torch

import kielflow_b200 as kf
from kielflow_b200 import configs as C
from kielflow_b200 import inputs as I


class WakeProblem:
    """Everything but the four differentiated inputs, fixed across runs."""

    def __init__(self, n, steps, ckpt_every=15, M=0.9, tau=0.1, Q=-20.0, sigma=0.5, terms=None,
                 fixed_cycles=14, seed=0):
        w = dict(C.WORKLOADS["adj128"])
        w.update(M=M, tau=tau, Q=Q, sigma=sigma)
        self.w = w
        self.n, self.steps, self.ckpt_every = n, steps, ckpt_every
        self.terms = terms
        self.fixed_cycles = fixed_cycles
        st, _, mask, dt = C.make_inputs(w, n, seed=seed)
        self.u = st[:3]
        self.n0 = np.exp(np.fft.irfftn(st[3], s=(n, n, n), axes=(0, 1, 2)))
        self.g = I.gauss_charge(n, C.L_BOX, 1.0, sigma)  # unit charge shape
        self.mask = mask
        self.dt = dt  # held fixed for every parameter value
        self.window = C.wake_window(n)
        # the first solve's initial guess, shared by all runs: a converged
        # solution at the base parameters
        with kf.Context(self.config(M, tau, tolerance=True)) as ctx:
            self._load(ctx, Q, self.n0)
            ctx.set_phi(np.zeros((n, n, n)))
            ctx.adjoint(self.window, 0, self.dt, 1, kf.KF_ADJ_J_ONLY, want_dn0=False)
            self.phi0 = ctx.get_phi()

    def config(self, M, tau, tolerance=False):
        over = {} if tolerance else dict(res_tol=-1.0, max_cycles=self.fixed_cycles)
        if self.terms is not None:
            over["terms"] = self.terms
        return C.config_for(dict(self.w, M=M, tau=tau), self.n, **over)

    def _load(self, ctx, Q, n0):
        s_hat = np.fft.rfftn(np.log(n0), axes=(0, 1, 2))
        ctx.set_state(self.u[0], self.u[1], self.u[2], s_hat)
        ctx.set_sources(Q * self.g, self.mask)

    def run(self, M, tau, Q, n0, grad=True, flags=0):
        with kf.Context(self.config(M, tau)) as ctx:
            self._load(ctx, Q, n0)
            ctx.set_phi(self.phi0)
            fl = flags | (0 if grad else kf.KF_ADJ_J_ONLY)
            r = ctx.adjoint(self.window, self.steps, self.dt, self.ckpt_every, fl, want_dn0=grad)
            r["residual"] = ctx.diag().last_residual
            if grad:
                r["dJ_dQ"] = r["dJ_dnd"] / Q
            return r


class WakePotential(torch.autograd.Function):
    """J(M, tau, Q, n0) with the discrete adjoint as its backward."""

    @staticmethod
    def forward(ctx, M, tau, Q, n0, problem):
        r = problem.run(float(M), float(tau), float(Q), n0.detach().cpu().numpy())
        ctx.save_for_backward(torch.tensor(r["dJ_dM"], dtype=torch.float64),
                              torch.tensor(r["dJ_dtau"], dtype=torch.float64),
                              torch.tensor(r["dJ_dQ"], dtype=torch.float64),
                              torch.from_numpy(r["dn0"]))
        ctx.run_info = r
        return torch.tensor(r["J"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        dM, dtau, dQ, dn0 = ctx.saved_tensors
        return gJ * dM, gJ * dtau, gJ * dQ, gJ * dn0, None
