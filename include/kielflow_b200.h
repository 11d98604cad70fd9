/*
 * kielflow_b200.h -- C ABI of the B200 (sm_100a) time-step hot path of kielflow.
 *
 * One context = one cubic periodic grid resident on one GPU: the spectral
 * state (u'_x, u'_y, u'_z, s = ln n as half spectra), the potential phi, the
 * dust charge n_d and the penalization mask, plus all work buffers.  Host
 * arrays use the reference's layouts:
 *   real field      field_real::val, double[n*n*n], index k + n*(j + n*i)
 *                   (field_base.hpp:23-24)
 *   spectral field  field_imag::val, fftw_complex[n*n*(n/2+1)] = interleaved
 *                   (re, im) doubles (field_imag.cpp:16,23), FFTW r2c layout,
 *                   forward unnormalised, inverse scaled by 1/N
 *                   (OP_FFT.cpp:49-63, OP_iFFT.cpp:49-64).
 * Every call returns KF_OK (0) or a negative KF_ERR_* code; kf_last_error()
 * gives the message.  A context is not thread-safe; distinct contexts are
 * independent.  No call copies device data to the host unless it says so.
 */
#ifndef KIELFLOW_B200_H_
#define KIELFLOW_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KF_OK 0
#define KF_ERR_ARG (-1)           /* invalid argument or unsupported grid        */
#define KF_ERR_CUDA (-2)          /* CUDA runtime error (message has the name)   */
#define KF_ERR_NAN (-3)           /* NaN/Inf detected in phi (cf. reference      */
                                  /* solver_poisson_jacobi_nlin.cpp:78-82,95-99) */
#define KF_ERR_NOT_CONVERGED (-4) /* Poisson solve hit its iteration cap         */
#define KF_ERR_NO_DEVICE (-5)     /* no CUDA device / wrong architecture         */

/* right-hand-side terms (runtime form of rhs_standard.hpp:22-30) */
#define KF_T_POISSON (1 << 0)      /* nonlinear Poisson solve for phi            */
#define KF_T_DISSIPATION (1 << 1)  /* ion-neutral friction tau u                 */
#define KF_T_SVISCOSITY (1 << 2)   /* spectral viscosity field_SV                */
#define KF_T_E_INT (1 << 3)        /* -grad phi (filtered)                       */
#define KF_T_PRESSURE (1 << 4)     /* -grad s / theta  (the reference's          */
                                   /*  _RHS_DIFFUSION switch)                    */
#define KF_T_E_EXT (1 << 5)        /* mean flow  -M d/dx                          */
#define KF_T_CONTINUITY (1 << 6)   /* -div u - u.grad s                          */
#define KF_T_ADVECTION (1 << 7)    /* -(u.grad) u                                */
#define KF_T_PENALIZATION (1 << 8) /* masking penalization of the dust grain     */
#define KF_T_DIFFUSION (1 << 9)    /* Laplacian diffusion D lap(u), D lap(s)     */
#define KF_T_SHIPPED 0xFF          /* the set the reference's build enables       */

/* Poisson solver */
#define KF_PS_JACOBI_REF 0 /* nonlinear Jacobi, relative-update stop (reference)  */
#define KF_PS_JACOBI_RES 1 /* nonlinear Jacobi, max-norm residual stop            */
#define KF_PS_CASCADIC 2   /* the reference's cascadic multigrid plan             */
#define KF_PS_FAS 3        /* FAS V-cycles, red-black point-Newton smoother       */

/* bulk precision */
#define KF_FP64 0
#define KF_FP32_BULK 1 /* FFTs, products, RK4 in FP32; Poisson in FP64 */

/* Context configuration.  Fields are only ever appended; a caller that
 * zero-initializes the struct (kf_config c = {}) gets the documented default
 * (0) of every field it does not set. */
typedef struct {
    int n;             /* cubic grid n^3: 16, 32, 64, 96, 128 or 256                 */
    double L;          /* box side; axes axis_CoEqSt(-L/2, L, n), or axis_CoSiSt      */
                       /* with stretch_m                                             */
    double M;          /* Mach number (parameters::M)                                */
    double tau;        /* friction (parameters::tau)                                 */
    double theta;      /* Te/Ti (parameters::theta)                                  */
    double diff_D;     /* Laplacian diffusion coefficient                            */
    double sv_eps;     /* spectral-viscosity amplitude (0.5 in rhs_standard.cpp:57)  */
    double sv_cut;     /* SV only where |k~| > sv_cut (0: everywhere)                */
    double pen_eta;    /* penalization damping eta_d (<= 0)                          */
    int terms;         /* KF_T_* bitmask                                             */
    int poisson_mode;  /* KF_PS_*                                                    */
    int nlj_max_it;    /* Jacobi sweep cap (negative: 1000, as the reference)        */
    double nlj_limit;  /* relative-update limit (KF_PS_JACOBI_REF)                   */
    double res_tol;    /* max-norm residual target (KF_PS_JACOBI_RES, KF_PS_FAS);     */
                       /* KF_PS_FAS with res_tol <= 0: exactly max_cycles V-cycles  */
                       /* per solve (a smooth map of the inputs, for derivative     */
                       /* checks by finite differences)                             */
    int mg_levels;     /* FAS levels, finest n ... coarsest n >> (levels-1)          */
    int mg_pre;        /* FAS pre-smoothing sweeps                                   */
    int mg_post;       /* FAS post-smoothing sweeps                                  */
    double coarse_tol; /* FAS coarsest-level residual target                         */
    int max_cycles;    /* FAS V-cycle cap per solve                                  */
    int phi_extrap;    /* 1: start each Poisson solve at a new time from the linear  */
                       /*    extrapolation of the last two solutions in time         */
    int precision;     /* KF_FP64 or KF_FP32_BULK                                    */
    double stretch_m;  /* 0: axis_CoEqSt(-L/2, L, n) axes.  > 0: axis_CoSiSt(-L/2, L,  */
                       /* n, stretch_m) on all three axes (x = S(l0 + L i/n),        */
                       /* S(x) = x - m sin(2 pi x/L), axis_SiSt.cpp; the frontend's  */
                       /* grid uses m = L (1 - 0.3)/(2 pi), frontend.cpp:285-287);   */
                       /* 2 pi m / L < 1.  Derivatives then take the chain-rule path */
                       /* of OP_partial_derivative.cpp:104-136 and the Poisson       */
                       /* stencils the stretched spacings (H_create).  Not with      */
                       /* kf_adjoint_run.                                           */
    double mg_omega;   /* KF_PS_FAS: over-relaxation of the smoother's point Newton  */
                       /* step, phi <- phi - omega f/f' (0: 1, the plain step).     */
                       /* Red-black over-relaxation near 1.2 cuts the V-cycles per  */
                       /* solve by about a quarter on these problems                */
} kf_config;

typedef struct kf_ctx kf_ctx;

typedef struct {
    int solves;             /* Poisson solves since creation                    */
    int last_iterations;    /* sweeps (Jacobi) or V-cycles (FAS) of the last one */
    long long total_iterations;
    double last_residual;   /* max-norm residual at exit of the last solve      */
    int not_converged;      /* solves that hit their cap                        */
    double charge;          /* sum(e^s - e^phi + n_d) h^3 (FP64)                */
    double kinetic;         /* sum 0.5 e^s |u|^2 h^3, u = u' + M e_x (FP64)     */
    long long stage_cycles[4]; /* FAS V-cycles spent in RK stages 1..4          */
} kf_diag_out;

/* Context lifetime.  Replaces constructing the reference's rhs_standard
 * (rhs_standard.cpp:7-85), solver_poisson_jacobi_nlin / solver_poisson_multigrid
 * (kielflow.cpp:197-217) and Runge_kutta_O4 (RKO4.cpp:41-47). */
int kf_ctx_create(const kf_config *cfg, kf_ctx **out);
int kf_ctx_destroy(kf_ctx *ctx);
const char *kf_last_error(const kf_ctx *ctx);
/* Make the context issue its work on an existing cudaStream_t (NULL: own stream). */
int kf_set_stream(kf_ctx *ctx, void *cuda_stream);
int kf_synchronize(kf_ctx *ctx);

/* State transfer (host, reference layout).  set = H2D, get = D2H. */
int kf_set_state(kf_ctx *ctx, const double *FUx, const double *FUy, const double *FUz,
                 const double *Fni);
int kf_get_state(kf_ctx *ctx, double *FUx, double *FUy, double *FUz, double *Fni);
/* dust charge n_d and penalization mask H, real fields (NULL: leave as is) */
int kf_set_sources(kf_ctx *ctx, const double *nd, const double *mask);
int kf_set_phi(kf_ctx *ctx, const double *phi);
int kf_get_phi(kf_ctx *ctx, double *phi);

/* interface_rhs::solve (interface_rhs.hpp:11-12; rhs_standard.cpp:89-566):
 * replaces the context's state by its time derivative, in place.  t is
 * accepted for interface parity; the right-hand side is autonomous. */
int kf_rhs_eval(kf_ctx *ctx, double t);

/* interface_ode_solver::solve (interface_ODE_solver.hpp:11-12; RKO4.cpp:50-241):
 * nsteps classic RK4 steps of size dt on the device-resident state.  With
 * KF_PS_FAS (or no Poisson solve) and the profile off, each step is one
 * replay of a captured CUDA graph whose stage times, warm starts and V-cycle
 * loops are decided on the device, and the call returns after the steps have
 * finished; a solve that missed its tolerance is then reported for the call
 * (KF_ERR_NOT_CONVERGED / KF_ERR_NAN) rather than at its stage.  Otherwise
 * the host drives every stage (the Jacobi and cascadic solvers) and the call
 * may return before the GPU has finished. */
int kf_rk4_steps(kf_ctx *ctx, int nsteps, double dt);

/* ------------------------------------------------------------ the time loop
 * kielflow.cpp:172-182: the input files hold the ion density on a linear
 * scale; the state evolves s = ln n.  kf_set_state_linear sets the state
 * from u' spectra and the spectrum Fn of n, forming s^ = r2c(log(c2r(Fn)))
 * on the device. */
int kf_set_state_linear(kf_ctx *ctx, const double *FUx, const double *FUy, const double *FUz,
                        const double *Fn);

/* The fields the reference's save_slice / save_all receive
 * (kielflow.cpp:290-324): the u' spectra, Fn = r2c(exp(c2r(s^))) (linear
 * density) and FPh = r2c(phi) with phi of the last stage solve.  Host arrays,
 * Nc interleaved complex each; NULL entries skip. */
int kf_get_output(kf_ctx *ctx, double *FUx, double *FUy, double *FUz, double *Fn, double *FPh);

#define KF_OUT_SLICE 1  /* save_slice step  */
#define KF_OUT_BACKUP 2 /* save_all backup  */
typedef struct {
    int step;       /* loop index: the state has advanced step + 1 RK4 steps  */
    double t;       /* the reference's t_total at the output: t0 + step * dt  */
                    /* (accumulated; it lags the state by one dt, as there)   */
    int kind;       /* KF_OUT_SLICE | KF_OUT_BACKUP                           */
    const double *FUx, *FUy, *FUz, *Fn, *FPh; /* as kf_get_output; valid     */
                                              /* during the callback only     */
} kf_output;
typedef void (*kf_output_fn)(const kf_output *out, void *user);

/* The time loop of kielflow.cpp:277-331: `iterations` RK4 steps of size dt;
 * after step `step` a slice is due when the reference's counter i_output
 * (counter.hpp: starts at 0, incremented after every step, reset at an output)
 * has reached slice_every, a backup likewise with backup_every (0: never) --
 * with 10 and 50, slices follow loop steps 10, 20, ... and backups 50, 100, ....
 * The output fields are formed on the device and copied to pinned host memory
 * on a side stream while the next steps run; fn is called from this thread,
 * in step order, once an output's copy has finished (at most two are in
 * flight).  With out_dir, the files of the reference's loop are written there
 * as well: slice_NNNN.kfh (step, 4 digits at least) and backup_at_STEP.kfh,
 * in the format of kf_save.  Returns after the last step and the last
 * callback. */
int kf_run(kf_ctx *ctx, int iterations, double dt, double t0, int slice_every, int backup_every,
           const char *out_dir, kf_output_fn fn, void *user);

/* Files.  The reference writes HDF5 (IO.cpp:60-505, 1295-1340): root datasets
 * version, date, path, time; group domain with type_/m_/l0_/N_/L_ + axis
 * letter; group parameters ("mach number M", "damping ratio tau",
 * "temperature ratio theta", "velocity diffusion mu", "magnetization beta");
 * group data with Ux, Uy, Uz, ni (linear density), Ph in real space -- the
 * whole grid in a backup (save_all), the plane z = 0 in a slice (save_slice,
 * index N*(0 - l0)/L).  HDF5 is not available to this library, so the same
 * hierarchy is written as a .kfh container: "KFH1", u32 entry count, then per
 * entry u16 name length, name (the HDF5 path, "data/Ux"), u8 type (1 f64,
 * 2 i32, 3 string, 4 i64), u8 rank, u64 dims[rank], little-endian payload.
 * "velocity diffusion mu" holds diff_D, "magnetization beta" 0. */
#define KF_FILE_SLICE 1
#define KF_FILE_BACKUP 2
typedef struct {
    int n;            /* N_x (= N_y = N_z required)                     */
    int kind;         /* KF_FILE_SLICE (2-D data) or KF_FILE_BACKUP     */
    double L, l0, time, M, tau, theta, mu, beta;
    int type;         /* domain/type_x: 1 axis_CoEqSt, 3 axis_CoSiSt    */
    double m;         /* domain/m_x (the stretching parameter)          */
} kf_file_info;
int kf_file_info_read(const char *path, kf_file_info *info);
/* write the context's current state (and phi) as a slice or backup file */
int kf_save(kf_ctx *ctx, const char *path, int kind, double t);
/* load a backup file into the state and phi (load_field_imag + the ln
 * transform of kielflow.cpp:156-182); the grid must match the context's */
int kf_load(kf_ctx *ctx, const char *path, double *t_out);

/* The frontend's initial state (frontend.cpp:255-330, create_input_from_
 * MGsolver and the filtering after it) on the context's grid:
 * phi solves lap phi = e^phi - (n_background + n_d) from phi = 0 with the
 * context's Poisson solver and its n_d (kf_set_sources), n = exp(-theta phi),
 * both filtered by exp(-2000 k~^15) in k-space, u' = 0; the state takes
 * s^ = r2c(log n) (the load of kielflow.cpp:172-182) and phi the filtered
 * potential.  The reference solves with n_background = 0; on a periodic box
 * that equation has a solution only if the dust charge is positive (the box
 * integral gives sum e^phi = sum n_d), so for a negative grain pass 1, the
 * uniform ion density the right-hand side's rho = e^s + n_d has at s = 0.
 * (The reference's frontend builds stretched axis_CoSiSt grids, which this
 * library does not support.) */
int kf_frontend_state(kf_ctx *ctx, double n_background);

/* interface_ode_solver::solve on host arrays, in place (the reference's call:
 * RKO4.cpp:50-241 on field_imag data): set the state from the four arrays,
 * advance nsteps steps, write the result back; returns when the result is
 * in the arrays.  With the captured step, u' is uploaded on a second stream
 * while stage 1 solves its Poisson problem (which needs s only), so most of
 * the upload is hidden; page-locked host arrays are needed for the overlap
 * (pageable ones work, without it). */
int kf_step_host(kf_ctx *ctx, int nsteps, double dt, double *FUx, double *FUy, double *FUz, double *Fni);

/* Batched form of kf_rk4_steps for independent contexts (a parameter sweep;
 * grids may differ): dts[i] is context i's step.  One host thread queues every
 * context's captured step on the context's own stream, step by step, so the
 * instances' kernels overlap on the GPU; returns after all have finished.  Each
 * context must qualify for the captured step (KF_PS_FAS or no Poisson solve,
 * profile off).  The first failing context's code is returned; its message is
 * in kf_last_error(that context) and kf_last_error(NULL). */
int kf_batch_rk4_steps(kf_ctx *const *ctxs, int nctx, int nsteps, const double *dts);

/* Kernel variants of a context (no reference counterpart: the reference's
 * FFTW plans are chosen by FFTW_MEASURE inside fftw_plan_dft_*, OP_FFT.cpp).
 * fft_plan: radix plan of every transform kernel, 0 or 1 (two factorisations
 * of each supported n into radix stages, with different threads per line);
 * rbgs_rows: the red-black smoother, 4, 8 (the default) or 16 for half-sweep
 * kernels with that many rows per block, or 0 for the streaming sweep (one
 * TMA-staged pass per sweep, the residual fused into the last pre-smoothing
 * sweep) on multigrid levels with n a multiple of 64 and the 8-row half-sweep
 * kernel below them.  Results do not depend on rbgs_rows (same arithmetic
 * per point, bit for bit) and agree between the fft plans to rounding. */
typedef struct kf_tune_out {
    int fft_plan;          /* chosen radix plan */
    int rbgs_rows;         /* chosen smoother: rows per k_rbgs block (4, 8, 16), or 0 */
                           /* for the streaming TMA-staged sweep (levels n >= 64)   */
    int fft_radices[2][4]; /* radix stages of plans 0 and 1 (0 = unused) */
    int fft_threads[2];    /* threads per transformed line of plans 0 and 1 */
    double fft_ms[2];      /* one right-hand side without its Poisson solve, per plan */
    double rbgs_ms[4];     /* one finest-level smoothing sweep with 4, 8, 16 rows and */
                           /* with the streaming sweep (-1: not available)          */
} kf_tune_out;

/* Time the variants on the context's own buffers (reps timed calls each,
 * reps <= 0: 5), keep the fastest of each kind and drop the context's captured
 * graphs so they are rebuilt with the choices.  The state, the potential and
 * the time are unchanged (the right-hand side runs with the potential held,
 * the smoother sweeps a copy of it).  out may be NULL. */
int kf_autotune(kf_ctx *ctx, int reps, kf_tune_out *out);

/* Set the variants directly (the values kf_autotune reports; e.g. one tuning
 * applied to every instance of a sweep).  KF_ERR_ARG for other values. */
int kf_set_tuning(kf_ctx *ctx, int fft_plan, int rbgs_rows);

/* Levels of at most 16^3 points below the finest, in FAS V-cycles that reach
 * a level below them (the 16^3 and 8^3 levels of the 6-level 256^3 cycle):
 * on = 1 (the default) runs them, with the correction they return, as one
 * block with the levels in shared memory (one launch instead of 16 kernels
 * that each last about their launch latency); on = 0 level by level.  The
 * potentials are the same bit for bit.  KF_ERR_ARG for other values. */
int kf_set_coarse_block(kf_ctx *ctx, int on);

/* In the captured step (kf_rk4_steps, kf_step_host, kf_batch_rk4_steps), the
 * transforms of u' and s that feed the products do not depend on phi: on = 1
 * (the default) runs them on a second stream of the context beside each
 * stage's Poisson solve, on = 0 after it.  Same kernels and inputs, so the
 * same results bit for bit.  KF_ERR_ARG for other values. */
int kf_set_overlap(kf_ctx *ctx, int on);

/* interface_poisson_solver::solve (interface_poisson_solver.hpp:18): phi_io is
 * the initial guess and the result, rho is read only; host arrays, n^3 doubles. */
int kf_poisson_solve(kf_ctx *ctx, double *phi_io, const double *rho);

/* diagnostics: Poisson statistics and FP64 conserved-quantity reductions */
int kf_diag(kf_ctx *ctx, kf_diag_out *out);

/* The standalone spectral operators on host arrays (OP_FFT.cpp:49-63,
 * OP_iFFT.cpp:49-64): r2c unnormalised, c2r scaled by 1/N. */
int kf_fft_r2c(kf_ctx *ctx, const double *in_real, double *out_complex);
int kf_fft_c2r(kf_ctx *ctx, const double *in_complex, double *out_real);

/* Device pointers of the resident state (4 half spectra, interleaved complex
 * in the context's bulk precision) for zero-copy consumers; NULL entries skip. */
int kf_state_device_ptrs(kf_ctx *ctx, void **FUx, void **FUy, void **FUz, void **Fni);

/* Kernel launches issued by this context since creation (measurement aid). */
long long kf_launch_count(const kf_ctx *ctx);

/* Kernel profile: when enabled, every launch is bracketed by CUDA events on the
 * context's stream and its algorithmic bytes (distinct inputs + outputs) are
 * recorded per kernel class; enabling or disabling resets the totals.
 * Classes 0..18; kf_profile_class_name gives the kernel name of each. */
int kf_profile_enable(kf_ctx *ctx, int on);
int kf_profile_read(kf_ctx *ctx, int cls, double *ms, long long *launches, double *bytes);
const char *kf_profile_class_name(int cls);

/* ------------------------------------------------------------------ adjoint
 * kf_adjoint_run -- no counterpart in the reference (the reference has no
 * differentiation).  Gradients of the wake-potential functional
 *     J = h^3 sum_x w(x) phi_T(x),   phi_T = Poisson solution of the state
 *                                            after nsteps RK4 steps of size dt
 * by the discrete adjoint of the FP64 time step: the transpose of every
 * transform, product and linear term of the right-hand side, the adjoint of the
 * converged Poisson solve  (-lap_h + diag e^phi) rho_bar = phi_bar  by linear
 * multigrid, and the reverse RK4 recursion, with the forward states recomputed
 * from checkpoints stored every ckpt_every steps.  Starts from the context's
 * state, phi (the first solve's initial guess) and time; dt is held fixed.
 * Requires a KF_FP64 context in KF_PS_FAS mode with KF_T_POISSON and
 * KF_T_E_INT.  w: n^3 host doubles.  dJ_dn0 (n^3, may be NULL) receives the
 * gradient with respect to the initial density n0 where the state's s^ =
 * r2c(ln n0); lam0 (8*Nc doubles = the 4 half spectra, may be NULL) receives
 * the gradient with respect to the initial spectral state.  On return the
 * context holds the final state, phi_T and time t + nsteps*dt. */
#define KF_ADJ_STORE_PHI 1 /* keep phi of every stage from the forward pass: the */
                           /* recomputation then solves no Poisson problem       */
                           /* (4 n^3 doubles per step of extra device memory)    */
#define KF_ADJ_J_ONLY 2    /* forward pass and J only (finite-difference checks) */
typedef struct {
    double J;
    double dJ_dM;        /* Mach number (parameters::M)                          */
    double dJ_dtau;      /* friction (parameters::tau)                           */
    double dJ_dnd;       /* d/de J(n_d -> (1+e) n_d) at e = 0: Q dJ/dQ for a     */
                         /* dust charge n_d proportional to Q                    */
    double fwd_ms;       /* device time of the checkpointed forward pass + J     */
    double bwd_ms;       /* device time of recomputation + adjoint sweep         */
    long long adj_cycles;/* V-cycles of the linear adjoint Poisson solves        */
    int adj_solves;
    int checkpoints;
} kf_grad_out;
int kf_adjoint_run(kf_ctx *ctx, int nsteps, double dt, int ckpt_every, int flags, const double *w,
                   kf_grad_out *out, double *dJ_dn0, double *lam0);

/* kf_fft_r2c_noalloc -- no counterpart in the reference.  The forward 3-D
 * transform of kf_fft_r2c for callers that cannot let a library allocate
 * device memory (a host that owns a fixed device pool and only lends its
 * plugins buffers, or a time-critical loop that cannot afford cudaMalloc's
 * latency and device-wide synchronisation).  It needs no context and
 * allocates nothing: in_real (n^3 doubles) and out_complex (n*n*(n/2+1)
 * interleaved complex doubles) are device-accessible buffers the caller
 * owns; the one intermediate array lives in a static device array of
 * 2,166,784 bytes that every GPU loading this library holds until exit, so
 * n is limited to 16, 32 or 64 (other n: KF_ERR_ARG).  Work is queued on
 * cuda_stream (NULL: the legacy default stream) and the call returns
 * without waiting.  All calls on one device share that array: calls that
 * overlap on the GPU race and must be serialised by the caller.  The first
 * call on each device is a warm-up: it looks up the array's device address
 * and, under lazy module loading (the CUDA default), loads the module, which
 * places the array in device memory and synchronises; make it before the
 * allocation-free part of the program and before any stream capture (a
 * captured first call returns KF_ERR_ARG).  Later uncaptured calls look the
 * address up again, so it stays right after a cudaDeviceReset.  An error
 * already pending from earlier work is reported (KF_ERR_CUDA) and left
 * pending.  Errors are reported by kf_last_error(NULL). */
int kf_fft_r2c_noalloc(int n, const double *in_real, double *out_complex, void *cuda_stream);

#ifdef __cplusplus
}
#endif

#endif
