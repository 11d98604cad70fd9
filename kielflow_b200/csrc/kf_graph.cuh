// kf_graph.cuh -- device-side control of one RK4 step replayed as a CUDA graph.
//
// The host driver decides three things per stage that depend on run-time
// values: the stage time, the start of the Poisson solve (linear extrapolation
// of the last two solutions at distinct times) and whether the FAS V-cycles
// have converged.  For a captured step these decisions are taken by the
// one-thread kernels below on a small device-resident record, with the same
// arithmetic as the host path (so both paths give identical results), and the
// convergence loop is a conditional WHILE node driven by k_fas_check.
#pragma once

#include <cuda_runtime.h>

namespace kf {

struct DevTime {
    double t, t_stage, tau_a, tau_b;
    int nhist, newtime, pad0, pad1;
};

struct DevPois {
    double r;                // max residual of the current solve
    double last_residual;    // at exit of the last finished solve
    long long total_cycles;  // over all finished solves
    int cyc;                 // V-cycles of the current solve
    int last_cycles;
    int solves, not_converged, nans, pad;
    long long stage_cycles[4];  // per RK stage
};

// mode 0: t_stage = t + x;  mode 1: t = t + x
__global__ void k_time(DevTime *d, double x, int mode) {
    if (threadIdx.x || blockIdx.x) return;
    if (mode == 0)
        d->t_stage = d->t + x;
    else
        d->t = d->t + x;
}

// Start of a solve at t_stage (the host's phi_guess): extrapolate phi when
// t_stage is a new time and two earlier solutions exist, or record phi.
__global__ void k_guess(double *__restrict__ phi, double *__restrict__ phi_a, const DevTime *__restrict__ d,
                        long N) {
    const double t = d->t_stage, ta = d->tau_a, tb = d->tau_b;
    const int nh = d->nhist;
    const bool newtime = nh == 0 || t != tb;
    if (!newtime || nh == 0) return;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double b = phi[i];
    if (nh >= 2) {
        const double w = (t - tb) / (tb - ta);
        phi[i] = __dadd_rn(b, __dmul_rn(w, __dsub_rn(b, phi_a[i])));
    }
    phi_a[i] = b;
}

// after k_guess: remember whether this solve is at a new time; shift tau_a
__global__ void k_guess_post(DevTime *d) {
    if (threadIdx.x || blockIdx.x) return;
    const int nh = d->nhist;
    const bool newtime = nh == 0 || d->t_stage != d->tau_b;
    d->newtime = newtime;
    if (newtime && nh != 0) d->tau_a = d->tau_b;
}

// after the solve: a solve at a new time enters the history
__global__ void k_hist_post(DevTime *d) {
    if (threadIdx.x || blockIdx.x) return;
    if (d->newtime) {
        d->nhist = d->nhist < 2 ? d->nhist + 1 : 2;
        d->tau_b = d->t_stage;
    }
}

// Convergence test of the FAS loop from the 64 max slots of k_resmax:
// continue while r > tol and cyc < max_cycles (fixed: while cyc < max_cycles).
// The loop is bounded by max_cycles whatever r is (NaN included).
__global__ void k_fas_check(const unsigned long long *__restrict__ slots, DevPois *p, double tol, int max_cycles,
                            int first, int fixed, int stage, cudaGraphConditionalHandle h) {
    if (threadIdx.x || blockIdx.x) return;
    unsigned long long m = 0;
    for (int s = 0; s < 64; ++s) m = slots[s] > m ? slots[s] : m;
    const double r = __longlong_as_double((long long)m);
    const int cyc = first ? 0 : p->cyc + 1;
    p->cyc = cyc;
    p->r = r;
    const bool cont = fixed ? cyc < max_cycles : (r > tol && cyc < max_cycles);
    if (!cont) {
        p->solves += 1;
        p->total_cycles += cyc;
        p->last_cycles = cyc;
        p->last_residual = r;
        p->stage_cycles[stage & 3] += cyc;
        if (r != r)
            p->nans += 1;
        else if (!fixed && r > tol)
            p->not_converged += 1;
    }
    cudaGraphSetConditional(h, cont ? 1u : 0u);
}

// Adaptive FAS solve, one WHILE iteration = pre-smoothing and residual of the
// finest level, this test, then (IF node) the rest of the V-cycle.  The test
// uses the residual of the pre-smoothed iterate: the solve ends there when its
// max |f| <= tol (or max_cycles cycles are done), so the returned phi carries
// the measured residual and no cycle ends with a residual pass of its own.
__global__ void k_fas_begin(DevPois *p, cudaGraphConditionalHandle hw) {
    if (threadIdx.x || blockIdx.x) return;
    p->cyc = 0;
    cudaGraphSetConditional(hw, 1u);
}

__global__ void k_fas_check_mid(const unsigned long long *__restrict__ slots, DevPois *p, double tol, int max_cycles,
                                int stage, cudaGraphConditionalHandle hw, cudaGraphConditionalHandle hi) {
    if (threadIdx.x || blockIdx.x) return;
    unsigned long long m = 0;
    for (int s = 0; s < 64; ++s) m = slots[s] > m ? slots[s] : m;
    const double r = __longlong_as_double((long long)m);
    const int cyc = p->cyc;
    p->r = r;
    const bool cont = r > tol && cyc < max_cycles;
    if (cont) {
        p->cyc = cyc + 1;
    } else {
        p->solves += 1;
        p->total_cycles += cyc;
        p->last_cycles = cyc;
        p->last_residual = r;
        p->stage_cycles[stage & 3] += cyc;
        if (r != r)
            p->nans += 1;
        else if (r > tol)
            p->not_converged += 1;
    }
    cudaGraphSetConditional(hw, cont ? 1u : 0u);
    cudaGraphSetConditional(hi, cont ? 1u : 0u);
}

}  // namespace kf
