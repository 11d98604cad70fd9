/*
 * kf_oracle.h -- C API of the CPU oracle (TEST INFRASTRUCTURE).
 *
 * A plain C++ restatement of the reference's RK4 time-step hot path
 * (RKO4.cpp:50-241, rhs_standard.cpp:7-566, solver_poisson_jacobi_nlin.cpp:50-265,
 * solver_poisson_multigrid.cpp:246-418, field_interpolation.cpp:56-315), with the
 * reference's compile-time term switches (rhs_standard.hpp:22-30) turned into a
 * runtime bitmask and with the terms the reference's driver does not enable
 * (Laplacian diffusion, masking penalization, spectral-viscosity cutoff, a
 * residual-based Poisson stop and an FAS V-cycle) added.  Only tests/, bench.py's
 * CPU-baseline leg and __graft_entry__.smoke() call it, to compare the CUDA path with.
 */
#ifndef KF_ORACLE_H_
#define KF_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

/* term bits, named after the reference's switches (rhs_standard.hpp:22-30) */
#define KFO_POISSON (1 << 0)      /* _RHS_POISSON: nonlinear Poisson solve      */
#define KFO_DISSIPATION (1 << 1)  /* _RHS_DISSIPATION: friction tau * u         */
#define KFO_SVISCOSITY (1 << 2)   /* _RHS_SVISCOSITY: spectral viscosity        */
#define KFO_E_INT (1 << 3)        /* _RHS_E_INT: grad(phi), filtered            */
#define KFO_PRESSURE (1 << 4)     /* _RHS_DIFFUSION (sic): grad(s)/theta        */
#define KFO_E_EXT (1 << 5)        /* _RHS_E_EXT: mean-flow M d/dx               */
#define KFO_CONTINUITY (1 << 6)   /* _RHS_CONTINUITY: div u + u.grad s          */
#define KFO_ADVECTION (1 << 7)    /* _RHS_ADVECTION: (u.grad) u                 */
#define KFO_PENALIZATION (1 << 8) /* masking penalization (effect_penalization) */
#define KFO_DIFFUSION (1 << 9)    /* Laplacian diffusion D lap(u), D lap(s)     */
#define KFO_SHIPPED 0xFF          /* the set rhs_standard.hpp:22-30 enables     */

/* Poisson solver modes */
#define KFO_PS_JACOBI_REF 0   /* NLJ, relative-update stop (solver_poisson_jacobi_nlin.cpp:258) */
#define KFO_PS_JACOBI_RES 1   /* NLJ, stop on max-norm residual <= res_tol                  */
#define KFO_PS_CASCADIC 2     /* kielflow.cpp:207-217 cascadic MG plan                       */
#define KFO_PS_FAS 3          /* FAS V-cycle, red-black point-Newton smoother                */

typedef struct {
    int n;           /* cubic grid n^3                                           */
    double L;        /* box side; axis_CoEqSt(-L/2, L, n)                        */
    double M;        /* Mach number (parameters::M)                              */
    double tau;      /* ion-neutral friction (parameters::tau)                   */
    double theta;    /* Te/Ti (parameters::theta)                                */
    double diff_D;   /* Laplacian diffusion coefficient (KFO_DIFFUSION)          */
    double sv_eps;   /* spectral viscosity amplitude (rhs_standard.cpp:57: 0.5)  */
    double sv_cut;   /* SV applied only where |k~| > sv_cut (0 = everywhere)     */
    double pen_eta;  /* penalization damping eta_d (<= 0)                        */
    int terms;       /* KFO_* bitmask                                            */
    int poisson_mode;
    int nlj_max_it;      /* sweeps cap (negative -> 1000, as the reference)      */
    double nlj_limit;    /* relative-update limit (KFO_PS_JACOBI_REF)            */
    double res_tol;      /* residual stop (KFO_PS_JACOBI_RES, KFO_PS_FAS)        */
    int mg_levels;       /* FAS levels (finest n, coarsest n >> (levels-1))      */
    int mg_pre, mg_post; /* FAS smoothing sweeps                                 */
    double coarse_tol;   /* FAS coarsest-level residual target                   */
    int max_cycles;      /* FAS V-cycle cap per solve                            */
    int phi_extrap;      /* linear extrapolation of phi in time for the start    */
    double stretch_m;    /* 0: axis_CoEqSt; > 0: axis_CoSiSt(-L/2, L, n, m) on   */
                         /* all three axes (sine-stretched, axis_SiSt.cpp)       */
    double mg_omega;     /* FAS: over-relaxation of the point Newton step (0: 1) */
} kfo_config;

typedef struct kfo_ctx kfo_ctx;

typedef struct {
    int last_iterations;  /* sweeps (Jacobi) or V-cycles (FAS) of the last solve */
    int total_iterations;
    int solves;
    double last_residual; /* max-norm residual after the last solve              */
    int not_converged;    /* solves that hit their cap                           */
} kfo_poisson_stats;

kfo_ctx *kfo_create(const kfo_config *cfg);
void kfo_destroy(kfo_ctx *c);
void kfo_set_state(kfo_ctx *c, const double *ux, const double *uy, const double *uz,
                   const double *s);
void kfo_get_state(kfo_ctx *c, double *ux, double *uy, double *uz, double *s);
void kfo_set_sources(kfo_ctx *c, const double *nd, const double *mask);
void kfo_set_phi(kfo_ctx *c, const double *phi);
void kfo_get_phi(kfo_ctx *c, double *phi);
int kfo_rhs(kfo_ctx *c, double t);
/* positions val_at(i), i = -1..n (n + 2 values), of the context's axis */
void kfo_positions(kfo_ctx *c, double *out);
/* the derivative's metric factor 1/dS of direction 0 after the 2/3 filter
 * (OP_partial_derivative.cpp:60-80), along that axis: n values */
void kfo_metric(kfo_ctx *c, double *out);
/* OP_partial_derivative on the context's grid: out = d/dx_dir of in (half spectra) */
void kfo_deriv(kfo_ctx *c, int dir, const double *in, double *out);
/* the right-hand side's masking penalization of one field (the restatement of
 * effect_penalization::execute, effect_penalization.cpp:21-44): out <- r2c((1 - H)
 * c2r(out) + H pen_eta (c2r(in) - fix)), H = the mask of kfo_set_sources */
void kfo_penalize(kfo_ctx *c, double fix, const double *in, double *out);
int kfo_rk4(kfo_ctx *c, double dt, int nsteps);
double kfo_time(kfo_ctx *c);
int kfo_poisson(kfo_ctx *c, double *phi_io, const double *rho);
void kfo_poisson_stats_get(kfo_ctx *c, kfo_poisson_stats *out);
double kfo_residual(kfo_ctx *c, const double *phi, const double *rho);
/* tables used by the RHS (for tests): dealias mask, SV, phi filter (each Nc) */
void kfo_tables(kfo_ctx *c, double *dealias, double *sv, double *phifilt);
/* standalone transforms with the reference's normalisation (c2r scaled 1/N) */
void kfo_r2c(int n, const double *in, double *out);
void kfo_c2r(int n, const double *in, double *out);
/* inter-grid transfer: kind 0 = trilinear n -> 2n, 1 = injection n -> n/2,
 * 2 = full-weighting n -> n/2 */
void kfo_transfer(int kind, int n, double L, const double *in, double *out);

#ifdef __cplusplus
}
#endif

#endif
