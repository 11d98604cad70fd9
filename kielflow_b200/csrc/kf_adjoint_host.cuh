// kf_adjoint_host.cuh -- host driver of the discrete adjoint (kf_adjoint_run).
//
// Included by kf_capi.cu after the forward driver: it uses kf_ctx, Impl's
// transform passes (through c->adj_fn), the Launch bookkeeping and the FAS
// level buffers.  FP64 only.
//
// Objective  J = h^3 sum w phi_T,  phi_T the Poisson solution of the final
// state.  Reverse sweep, per RK4 step (RKO4.cpp:105-238) taken backwards:
//   Kbar4 = dt/6 lam                    Xbar4 = f'(X4)^T Kbar4
//   Kbar3 = dt/3 lam + dt   Xbar4       Xbar3 = f'(X3)^T Kbar3
//   Kbar2 = dt/3 lam + dt/2 Xbar3       Xbar2 = f'(X2)^T Kbar2
//   Kbar1 = dt/6 lam + dt/2 Xbar2       Xbar1 = f'(X1)^T Kbar1
//   lam  <- lam + Xbar1 + Xbar2 + Xbar3 + Xbar4
// where f'(X)^T (vjp below) is the transpose of rhs_standard::solve at the
// stage input X with the stage's converged phi, including the implicit
// dependence of phi on s through the Poisson problem.  Stage inputs and
// potentials of one checkpoint segment are recomputed forward (bit-identical
// to the first pass: same kernels, same warm starts) and kept on the device.

#include <algorithm>

namespace {

constexpr double kAdjRtol = 1e-10;  // adjoint Poisson: max residual <= kAdjRtol * max |phi_bar|
constexpr int kAdjMaxCycles = 60;
constexpr double kAdjCoarseRtol = 1e-4;  // coarsest level: residual reduction per visit

struct Snap {
    void *Y[4] = {};
    double *phi = nullptr, *phi_a = nullptr;
    double tau_a = 0., tau_b = 0., t = 0.;
    int nhist = 0;
};

struct AdjState {
    void *lam[4] = {}, *lacc[4] = {}, *Kb[4] = {}, *Xb[4] = {};
    // physical cotangents: 0-2 U_c, 3+3c+d d_d U_c, 12-14 d_d s, 15 s_d, 16-19 rl_q
    double *RB[20] = {};
    void *Ta[20] = {}, *Tb[20] = {};  // their r2c (Ta) and the intermediate pass (Tb)
    void *phib = nullptr;             // cotangent of phihat
    double *phibar = nullptr, *rhob = nullptr, *c0 = nullptr, *w = nullptr, *out = nullptr;
    double *bprev = nullptr;  // source of the previous adjoint Poisson solve (warm start)
    double *sums = nullptr;   // <b, bprev>, <bprev, bprev>
    std::vector<double *> cl;  // e^phi on every level (cl[0] = c0)
    double *part = nullptr, *acc = nullptr, *h_acc = nullptr;
    std::vector<Snap> ck;
    Snap fin;
    std::vector<void *> segX;      // stage inputs of one segment: 16 per step
    std::vector<double *> segPhi;  // stage potentials of one segment: 4 per step
    std::vector<double *> allPhi;  // KF_ADJ_STORE_PHI: 4 per step of the whole run
    cudaGraphExec_t graph = nullptr;
    long long graph_kernels = 0;
    long long cycles = 0;
    int solves = 0;
};

void dfree(kf_ctx *c, void *p) {
    auto it = std::find(c->allocs.begin(), c->allocs.end(), p);
    if (it != c->allocs.end()) {
        c->allocs.erase(it);
        cudaFree(p);
    }
}

Geo<double> geo64(kf_ctx *c) {
    return Geo<double>{c->n, c->nzc, (const double *)c->kv, c->q2, dealias_threshold(), c->pb};
}

Snap snap_alloc(kf_ctx *c) {
    Snap s;
    for (int q = 0; q < 4; ++q) s.Y[q] = dalloc<void>(c, 16 * c->Nc);
    s.phi = dalloc<double>(c, 8 * c->N);
    if (c->cfg.phi_extrap) s.phi_a = dalloc<double>(c, 8 * c->N);
    return s;
}

void snap_save(kf_ctx *c, Snap &s) {
    copy_state(c, s.Y, c->Y);
    CK(cudaMemcpyAsync(s.phi, c->phi, 8 * c->N, cudaMemcpyDeviceToDevice, c->st));
    if (s.phi_a) CK(cudaMemcpyAsync(s.phi_a, c->phi_a, 8 * c->N, cudaMemcpyDeviceToDevice, c->st));
    s.tau_a = c->tau_a;
    s.tau_b = c->tau_b;
    s.t = c->t;
    s.nhist = c->nhist;
}

void snap_load(kf_ctx *c, const Snap &s) {
    copy_state(c, c->Y, s.Y);
    copy_state(c, c->Ys, s.Y);
    CK(cudaMemcpyAsync(c->phi, s.phi, 8 * c->N, cudaMemcpyDeviceToDevice, c->st));
    if (s.phi_a) CK(cudaMemcpyAsync(c->phi_a, s.phi_a, 8 * c->N, cudaMemcpyDeviceToDevice, c->st));
    c->tau_a = s.tau_a;
    c->tau_b = s.tau_b;
    c->t = s.t;
    c->nhist = s.nhist;
}

// Job lists of the adjoint's transform passes (Impl::adj_pass), appended to
// the context's lists, which are uploaded again.
void build_adj_jobs(kf_ctx *c) {
    AdjState &a = *c->adj;
    std::vector<AxisJob> &J = c->hj;
    std::vector<ZJob> &Z = c->hz;
    const bool pen = c->cfg.terms & T_PENALIZATION;
    auto aj = [&](const void *in, void *out, int mul) { J.push_back(AxisJob{in, out, mul, 0}); };
    auto zj = [&](const void *ia, int ma, const void *ib, int mb, void *oa, void *ob) {
        Z.push_back(ZJob{ia, ib, oa, ob, ma, mb});
    };
    void **CX = c->CX, **CY = c->CY, **R = c->R;
    // 1: f_bar_q = c2r_unscaled(P Kbar_q / w)   (P only with penalization: K = P r2c(f))
    c->jV_x = (int)J.size();
    for (int q = 0; q < 4; ++q) aj(a.Kb[q], CX[q], pen ? MUL_P : MUL_NONE);
    c->jV_y = (int)J.size();
    for (int q = 0; q < 4; ++q) aj(CX[q], CY[q], MUL_NONE);
    c->zV = (int)Z.size();
    zj(CY[0], MUL_HALF, CY[1], MUL_HALF, R[20], R[21]);
    zj(CY[2], MUL_HALF, CY[3], MUL_HALF, R[22], R[23]);
    // 2: r2c of the physical cotangents (s_d's comes later, after the Poisson adjoint)
    std::vector<int> f;
    for (int i = 0; i < 15; ++i) f.push_back(i);
    if (pen)
        for (int i = 16; i < 20; ++i) f.push_back(i);
    c->zW = (int)Z.size();
    for (size_t i = 0; i < f.size(); i += 2) {
        const int A = f[i], B = i + 1 < f.size() ? f[i + 1] : -1;
        zj(a.RB[A], 0, B >= 0 ? a.RB[B] : nullptr, 0, a.Ta[A], B >= 0 ? a.Ta[B] : nullptr);
    }
    c->nWz = (int)Z.size() - c->zW;
    c->nWf = (int)f.size();
    c->jW_y = (int)J.size();
    for (int i : f) aj(a.Ta[i], a.Tb[i], MUL_NONE);
    c->jW_x = (int)J.size();
    for (int i : f) aj(a.Tb[i], a.Ta[i], MUL_NONE);
    // 4: r2c of s_d_bar
    c->zS = (int)Z.size();
    zj(a.RB[15], 0, nullptr, 0, a.Ta[15], nullptr);
    c->jS_y = (int)J.size();
    aj(a.Ta[15], a.Tb[15], MUL_NONE);
    c->jS_x = (int)J.size();
    aj(a.Tb[15], a.Ta[15], MUL_NONE);
    // 3: phi_bar = c2r_unscaled(phihat_bar / w)
    c->jP_x = (int)J.size();
    aj(a.phib, CX[0], MUL_NONE);
    c->jP_y = (int)J.size();
    aj(CX[0], CY[0], MUL_NONE);
    c->zP = (int)Z.size();
    zj(CY[0], MUL_HALF, nullptr, 0, a.phibar, nullptr);
    // 5: dJ/ds0 = c2r_unscaled(lam_s / w) -> RB[0];  s0 = c2r(s^) -> RB[1]
    c->jQ_x = (int)J.size();
    aj(a.lam[3], CX[0], MUL_NONE);
    aj(c->Y[3], CX[1], MUL_NONE);
    c->jQ_y = (int)J.size();
    aj(CX[0], CY[0], MUL_NONE);
    aj(CX[1], CY[1], MUL_NONE);
    c->zQ = (int)Z.size();
    zj(CY[0], MUL_HALF, nullptr, 0, a.RB[0], nullptr);
    zj(CY[1], MUL_NONE, nullptr, 0, a.RB[1], nullptr);
    AxisJob *dj = dalloc<AxisJob>(c, sizeof(AxisJob) * J.size());
    ZJob *dz = dalloc<ZJob>(c, sizeof(ZJob) * Z.size());
    CK(cudaMemcpy(dj, J.data(), sizeof(AxisJob) * J.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dz, Z.data(), sizeof(ZJob) * Z.size(), cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(c->st));
    dfree(c, c->dj);
    dfree(c, c->dz);
    c->dj = dj;
    c->dz = dz;
}

void adj_init(kf_ctx *c) {
    if (c->adj) return;
    c->adj = new AdjState;
    AdjState &a = *c->adj;
    const size_t cb = 16 * c->Nc, rb = 8 * c->N;
    for (int q = 0; q < 4; ++q) {
        a.lam[q] = dalloc<void>(c, cb);
        a.lacc[q] = dalloc<void>(c, cb);
        a.Kb[q] = dalloc<void>(c, cb);
        a.Xb[q] = dalloc<void>(c, cb);
    }
    for (int i = 0; i < 20; ++i) {
        a.RB[i] = dalloc<double>(c, rb);
        a.Ta[i] = dalloc<void>(c, cb);
        a.Tb[i] = dalloc<void>(c, cb);
        CK(cudaMemset(a.RB[i], 0, rb));
    }
    a.phib = dalloc<void>(c, cb);
    a.phibar = dalloc<double>(c, rb);
    a.rhob = dalloc<double>(c, rb);
    a.c0 = dalloc<double>(c, rb);
    a.w = dalloc<double>(c, rb);
    a.out = dalloc<double>(c, rb);
    a.bprev = dalloc<double>(c, rb);
    a.sums = dalloc<double>(c, 4 * sizeof(double));
    CK(cudaMemset(a.rhob, 0, rb));
    CK(cudaMemset(a.bprev, 0, rb));
    a.cl.assign(c->lv.size(), nullptr);
    a.cl[0] = a.c0;
    for (size_t l = 1; l < c->lv.size(); ++l) {
        const long n = c->lv[l].n;
        a.cl[l] = dalloc<double>(c, 8 * n * n * n);
    }
    a.part = dalloc<double>(c, sizeof(double) * 4 * 1184);
    a.acc = dalloc<double>(c, sizeof(double) * 4);
    CK(cudaMallocHost(&a.h_acc, sizeof(double) * 4));
    a.fin = snap_alloc(c);
    CK(cudaFuncSetAttribute(k_coarse_solve_lin, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    build_adj_jobs(c);
}

void adj_release(kf_ctx *c) {
    if (!c->adj) return;
    if (c->adj->graph) cudaGraphExecDestroy(c->adj->graph);
    if (c->adj->h_acc) cudaFreeHost(c->adj->h_acc);
    delete c->adj;  // device buffers are in c->allocs
    c->adj = nullptr;
}

void acc4(kf_ctx *c, int nb) {
    Launch L_(c, KC_ADJ_PW, 32. * nb);
    k_accumulate4<<<1, 32, 0, c->st>>>(c->adj->part, nb, c->adj->acc);
}

// ------------------------------------------------------------------ adjoint Poisson
// (-lap_h + diag c) psi = b with c = e^phi: linear FAS V-cycles on the forward
// solver's levels (same stencil, restriction and prolongation); level 0 works
// on psi = rhob, b = phibar.
struct ALev {
    double *psi, *b, *r, *phi0, *cc;
};

ALev alev(kf_ctx *c, int l) {
    AdjState &a = *c->adj;
    LevelBuf &L = c->lv[l];
    if (l == 0) return ALev{a.rhob, a.phibar, L.r, nullptr, a.c0};
    return ALev{L.phi, L.rho, L.r, L.phi0, a.cl[l]};
}

void avcycle(kf_ctx *c, int l) {
    LevelBuf &L = c->lv[l];
    const ALev A = alev(c, l);
    const kf_config &cf = c->cfg;
    const int n = L.n;
    const long N = (long)n * n * n;
    if (l == (int)c->lv.size() - 1) {
        Launch L_(c, KC_ADJ_MG, 32. * N);
        const int bs = N >= 1024 ? 1024 : (int)((N + 31) / 32 * 32);
        k_coarse_solve_lin<<<1, bs, (size_t)(24 * N + 24 * n), c->st>>>(A.psi, A.b, A.cc, L.lev(), kAdjCoarseRtol,
                                                                        400);
        return;
    }
    smooth(c, L, A.psi, A.b, A.cc, cf.mg_pre, KC_ADJ_MG);
    {
        Launch L_(c, KC_ADJ_MG, 32. * N);
        if (col_level(n))
            k_residual_col<8, COL_PI, false, true><<<dim3(n / 64, n / 8, n / COL_PI), mg_block(), 0, c->st>>>(
                A.psi, A.b, L.lev(), A.r, nullptr, A.cc);
        else
            k_residual_lin<<<mg_grid(n, n), mg_block(), 0, c->st>>>(A.psi, A.b, A.cc, L.lev(), A.r);
    }
    LevelBuf &Lc = c->lv[l + 1];
    const ALev C = alev(c, l + 1);
    const long Nc3 = (long)Lc.n * Lc.n * Lc.n;
    {
        Launch L_(c, KC_ADJ_MG, 8. * N + 32. * Nc3);
        k_restrict<<<mg_grid(Lc.n, Lc.n), mg_block(), 0, c->st>>>(A.r, A.psi, n, C.r, C.psi, C.phi0);
    }
    {
        Launch L_(c, KC_ADJ_MG, 32. * Nc3);
        k_fas_rhs_lin<<<mg_grid(Lc.n, Lc.n), mg_block(), 0, c->st>>>(C.psi, C.r, C.cc, Lc.lev(), C.b);
    }
    avcycle(c, l + 1);
    {
        Launch L_(c, KC_ADJ_MG, 24. * Nc3);
        k_correction<<<mg_grid(Lc.n, Lc.n), mg_block(), 0, c->st>>>(C.psi, C.phi0, Lc.n);
    }
    {
        Launch L_(c, KC_ADJ_MG, 16. * N + 8. * Nc3);
        k_prolong_add<<<mg_grid(Lc.n, Lc.n), mg_block(), 0, c->st>>>(A.psi, C.phi0, nullptr, L.gam, n);
    }
    smooth(c, L, A.psi, A.b, A.cc, cf.mg_post, KC_ADJ_MG);
    CK(cudaGetLastError());
}

void run_avcycle(kf_ctx *c) {
    AdjState &a = *c->adj;
    if (c->prof) {
        avcycle(c, 0);
        return;
    }
    if (!a.graph) {
        const long long l0 = c->launches;
        CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        avcycle(c, 0);
        cudaGraph_t g = nullptr;
        CK(cudaStreamEndCapture(c->st, &g));
        cudaError_t e = cudaGraphInstantiate(&a.graph, g, 0);
        cudaGraphDestroy(g);
        CK(e);
        a.graph_kernels = c->launches - l0;
        c->launches = l0;
    }
    CK(cudaGraphLaunch(a.graph, c->st));
    c->launches += a.graph_kernels;
}

double read_max64(kf_ctx *c) {
    CK(cudaMemcpyAsync(c->h_max, c->d_max, 64 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    unsigned long long m = 0;
    for (int s = 0; s < 64; ++s) m = c->h_max[s] > m ? c->h_max[s] : m;
    double r;
    std::memcpy(&r, &m, sizeof(double));
    return r;
}

double adj_resmax(kf_ctx *c) {
    AdjState &a = *c->adj;
    LevelBuf &L = c->lv[0];
    CK(cudaMemsetAsync(c->d_max, 0, 64 * sizeof(unsigned long long), c->st));
    {
        Launch L_(c, KC_ADJ_MG, 24. * c->N);
        dim3 g = mg_grid(L.n, L.n);
        g.z = L.n < 16 ? L.n : 16;
        if (col_level(L.n))
            k_residual_col<8, COL_PI, true, true, false><<<dim3(L.n / 64, L.n / 8, L.n / COL_PI), mg_block(), 0, c->st>>>(
                a.rhob, a.phibar, L.lev(), nullptr, c->d_max, a.c0);
        else
            k_resmax_lin<<<g, mg_block(), 0, c->st>>>(a.rhob, a.phibar, a.c0, L.lev(), c->d_max);
    }
    CK(cudaGetLastError());
    return read_max64(c);
}

// rhob <- (-lap_h + diag e^phi)^-1 phibar, phi = c->phi; warm start: rhob as it stands
void adj_poisson(kf_ctx *c) {
    AdjState &a = *c->adj;
    const long N = c->N;
    {
        Launch L_(c, KC_ADJ_MG, 16. * N);
        k_exp<<<nblk(N, 256), 256, 0, c->st>>>(c->phi, a.c0, N);
    }
    for (size_t l = 1; l < c->lv.size(); ++l) {
        const LevelBuf &L = c->lv[l];
        Launch L_(c, KC_ADJ_MG, 16. * L.n * L.n * L.n);
        k_inject<<<mg_grid(L.n, L.n), mg_block(), 0, c->st>>>(a.c0, c->n, c->n / L.n, a.cl[l]);
    }
    CK(cudaMemsetAsync(c->d_max, 0, 64 * sizeof(unsigned long long), c->st));
    {
        Launch L_(c, KC_ADJ_MG, 8. * N);
        k_absmax<<<red_blocks(N), 256, 0, c->st>>>(a.phibar, N, c->d_max);
    }
    const double bmax = read_max64(c);
    if (bmax != bmax) throw KfError{KF_ERR_NAN, "NaN in the adjoint Poisson source"};
    a.solves++;
    if (bmax == 0.) {
        CK(cudaMemsetAsync(a.rhob, 0, 8 * N, c->st));
        return;
    }
    // warm start: the previous solution times the least-squares factor of
    // this source on the previous one (consecutive stage sources are close
    // to proportional)
    {
        const int nb = red_blocks(N);
        {
            Launch L_(c, KC_ADJ_MG, 16. * N);
            k_dot2<RBS><<<nb, RBS, 0, c->st>>>(a.phibar, a.bprev, N, a.part);
        }
        CK(cudaMemsetAsync(a.sums, 0, 4 * sizeof(double), c->st));
        {
            Launch L_(c, KC_ADJ_MG, 32. * nb);
            k_accumulate4<<<1, 32, 0, c->st>>>(a.part, nb, a.sums);
        }
        Launch L_(c, KC_ADJ_MG, 32. * N);
        k_warm_scale<<<nblk(N, 256), 256, 0, c->st>>>(a.rhob, a.bprev, a.phibar, a.sums, N);
    }
    const double tol = kAdjRtol * bmax;
    double r = adj_resmax(c);
    int cyc = 0;
    while (r > tol && cyc < kAdjMaxCycles) {
        run_avcycle(c);
        ++cyc;
        r = adj_resmax(c);
    }
    a.cycles += cyc;
    if (r != r) throw KfError{KF_ERR_NAN, "NaN in the adjoint Poisson solve"};
    if (r > tol) throw KfError{KF_ERR_NOT_CONVERGED, "adjoint Poisson solve did not reach its tolerance"};
}

// ------------------------------------------------------------------ one stage VJP
VjpAsmArgs asm_args(kf_ctx *c, int stage_two) {
    AdjState &a = *c->adj;
    VjpAsmArgs va;
    for (int i = 0; i < 20; ++i) va.CA[i] = (const double2 *)a.Ta[i];
    for (int q = 0; q < 4; ++q) {
        va.Kbar[q] = (const double2 *)a.Kb[q];
        va.Y[q] = (const double2 *)c->Ys[q];
        va.Ybar[q] = (double2 *)a.Xb[q];
    }
    va.SV = (const double *)c->SV;
    va.PF = (const double *)c->PF;
    va.phib = (double2 *)a.phib;
    va.tau = c->cfg.tau;
    va.theta = c->cfg.theta;
    va.M = c->cfg.M;
    va.D = c->cfg.diff_D;
    va.invN = 1. / (double)c->N;
    va.terms = c->cfg.terms;
    va.stage_two = stage_two;
    va.part = a.part;
    return va;
}

// s-part of the Poisson path: s_d_bar (RB[15]) += rhob e^{s_d}, dJ/dn_d, then
// Xb_s += P (w/N) r2c(s_d_bar).  Needs R[0] = s_d and phibar of the stage.
void vjp_poisson_tail(kf_ctx *c) {
    AdjState &a = *c->adj;
    const long N = c->N;
    adj_poisson(c);
    const int nb = red_blocks(N);
    {
        Launch L_(c, KC_ADJ_PW, 32. * N);
        k_poisson_vjp_tail<RBS><<<nb, RBS, 0, c->st>>>(a.rhob, (const double *)c->R[0], c->nd, a.RB[15], N, a.part);
    }
    acc4(c, nb);
    c->adj_fn(c, 4);
    {
        Launch L_(c, KC_ADJ_PW, 48. * c->Nc);
        k_vjp_assemble<RBS><<<red_blocks(c->Nc), RBS, 0, c->st>>>(asm_args(c, 1), geo64(c));
    }
    CK(cudaGetLastError());
}

// Xb = f'(X)^T Kb at the stage input X (4 fields) with the stage potential PHi;
// parameter gradients accumulate into a.acc.
void vjp(kf_ctx *c, void *const *X, const double *PHi) {
    AdjState &a = *c->adj;
    const kf_config &cf = c->cfg;
    const long N = c->N;
    copy_state(c, c->Ys, X);
    CK(cudaMemcpyAsync(c->phi, PHi, 8 * N, cudaMemcpyDeviceToDevice, c->st));
    c->adj_fn(c, 0);  // s_d, U, dU, ds
    c->adj_fn(c, 1);  // f_bar -> R[20..23]
    ProdVjpArgs pa;
    for (int q = 0; q < 4; ++q) {
        pa.fb[q] = (const double *)c->R[20 + q];
        pa.rlb[q] = a.RB[16 + q];
    }
    for (int d = 0; d < 3; ++d) {
        pa.U[d] = (const double *)c->R[1 + d];
        pa.ds[d] = (const double *)c->R[13 + d];
        pa.Ub[d] = a.RB[d];
        pa.dsb[d] = a.RB[12 + d];
        for (int e = 0; e < 3; ++e) {
            pa.dU[d][e] = (const double *)c->R[4 + 3 * d + e];
            pa.dUb[d][e] = a.RB[3 + 3 * d + e];
        }
    }
    pa.H = (const double *)c->H;
    pa.sdb = a.RB[15];
    pa.eta = cf.pen_eta;
    pa.terms = cf.terms;
    pa.N = N;
    pa.part = a.part;
    const int nb = red_blocks(N);
    {
        Launch L_(c, KC_ADJ_PW, 8. * N * 40);
        k_prod_vjp<RBS><<<nb, RBS, 0, c->st>>>(pa);
    }
    acc4(c, nb);
    c->adj_fn(c, 2);  // r2c of the physical cotangents -> Ta
    const int nbc = red_blocks(c->Nc);
    {
        Launch L_(c, KC_ADJ_PW, 16. * c->Nc * 30);
        k_vjp_assemble<RBS><<<nbc, RBS, 0, c->st>>>(asm_args(c, 0), geo64(c));
    }
    acc4(c, nbc);
    c->adj_fn(c, 3);  // phi_bar
    vjp_poisson_tail(c);
}

void adj_stage(kf_ctx *c, int mode, double ca, double cb) {
    AdjState &a = *c->adj;
    AdjStageArgs s;
    for (int q = 0; q < 4; ++q) {
        s.lam[q] = (double *)a.lam[q];
        s.lacc[q] = (double *)a.lacc[q];
        s.Kb[q] = (double *)a.Kb[q];
        s.Xb[q] = (const double *)a.Xb[q];
    }
    const long M = 2 * c->Nc;
    Launch L_(c, KC_ADJ_PW, 4. * M * 8 * (mode == 1 ? 5 : 3));
    k_adj_stage<<<dim3(nblk(M, 256), 4), 256, 0, c->st>>>(s, ca, cb, mode, M);
}

// phi_T of the state in Y (time c->t), as a stage solve would find it
void final_solve(kf_ctx *c) {
    c->t_stage = c->t;
    c->adj_fn(c, 6);
    {
        Launch L_(c, KC_RHO, 24. * c->N);
        k_rho<double><<<nblk(c->N, 256), 256, 0, c->st>>>((const double *)c->R[0], c->nd, c->rho, c->N);
    }
    const bool newtime = phi_guess(c);
    if (poisson(c)) throw KfError{KF_ERR_NOT_CONVERGED, "Poisson solve did not reach its tolerance"};
    if (c->cfg.phi_extrap && newtime) {
        c->nhist = c->nhist < 2 ? c->nhist + 1 : 2;
        c->tau_b = c->t_stage;
    }
}

void adj_run(kf_ctx *c, int nsteps, double dt, int E, int flags, const double *w, kf_grad_out *out,
             double *dJ_dn0, double *lam0) {
    const kf_config &cf = c->cfg;
    if (!out || !w) throw KfError{KF_ERR_ARG, "null argument"};
    if (nsteps < 0 || E < 1) throw KfError{KF_ERR_ARG, "nsteps >= 0 and ckpt_every >= 1 required"};
    if (c->fp32) throw KfError{KF_ERR_ARG, "the adjoint needs a KF_FP64 context"};
    if (cf.poisson_mode != KF_PS_FAS) throw KfError{KF_ERR_ARG, "the adjoint needs poisson_mode KF_PS_FAS"};
    if (!(cf.terms & T_POISSON) || !(cf.terms & T_E_INT))
        throw KfError{KF_ERR_ARG, "the adjoint needs KF_T_POISSON and KF_T_E_INT"};
    adj_init(c);
    AdjState &a = *c->adj;
    const bool jonly = flags & KF_ADJ_J_ONLY;
    const bool sphi = (flags & KF_ADJ_STORE_PHI) && !jonly;
    const long N = c->N;
    const int nck = nsteps > 0 ? (nsteps + E - 1) / E : 0;
    const int seg = nsteps < E ? nsteps : E;
    if (!jonly) {
        while ((int)a.ck.size() < nck) a.ck.push_back(snap_alloc(c));
        while ((int)a.segX.size() < 16 * seg) a.segX.push_back(dalloc<void>(c, 16 * c->Nc));
        if (!sphi)
            while ((int)a.segPhi.size() < 4 * seg) a.segPhi.push_back(dalloc<double>(c, 8 * N));
        if (sphi)
            while ((int)a.allPhi.size() < 4 * nsteps) a.allPhi.push_back(dalloc<double>(c, 8 * N));
    }
    CK(cudaMemcpyAsync(a.w, w, 8 * N, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemsetAsync(a.acc, 0, 4 * sizeof(double), c->st));
    a.cycles = 0;
    a.solves = 0;
    cudaEvent_t ev[3];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    struct EvGuard {
        cudaEvent_t *e;
        ~EvGuard() {
            for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]);
        }
    } eg{ev};
    CK(cudaEventRecord(ev[0], c->st));
    // forward pass with checkpoints
    for (int s = 0; s < nsteps; ++s) {
        if (!jonly && s % E == 0) snap_save(c, a.ck[s / E]);
        rk4_step(c, dt, nullptr, sphi ? &a.allPhi[4 * (size_t)s] : nullptr, nullptr);
    }
    final_solve(c);
    const int nb = red_blocks(N);
    {
        Launch L_(c, KC_ADJ_PW, 16. * N);
        k_dot_w<RBS><<<nb, RBS, 0, c->st>>>(a.w, c->phi, N, a.part);
    }
    acc4(c, nb);
    CK(cudaEventRecord(ev[1], c->st));
    if (!jonly) {
        const double h = cf.L / c->n, h3 = h * h * h;
        snap_save(c, a.fin);
        // lam_T: the Poisson path of phi_T only
        for (int q = 0; q < 4; ++q) CK(cudaMemsetAsync(a.Xb[q], 0, 16 * c->Nc, c->st));
        {
            Launch L_(c, KC_ADJ_PW, 16. * N);
            k_scale<<<nblk(N, 256), 256, 0, c->st>>>(a.w, a.phibar, h3, N);
        }
        CK(cudaMemsetAsync(a.RB[15], 0, 8 * N, c->st));
        vjp_poisson_tail(c);
        for (int q = 0; q < 4; ++q)
            CK(cudaMemcpyAsync(a.lam[q], a.Xb[q], 16 * c->Nc, cudaMemcpyDeviceToDevice, c->st));
        for (int g = nck - 1; g >= 0; --g) {
            const int s0 = g * E, s1 = std::min(nsteps, s0 + E);
            snap_load(c, a.ck[g]);
            for (int s = s0; s < s1; ++s) {
                void *const *X = &a.segX[16 * (size_t)(s - s0)];
                if (sphi)
                    rk4_step(c, dt, X, nullptr, &a.allPhi[4 * (size_t)s]);
                else
                    rk4_step(c, dt, X, &a.segPhi[4 * (size_t)(s - s0)], nullptr);
            }
            for (int s = s1 - 1; s >= s0; --s) {
                void *const *X = &a.segX[16 * (size_t)(s - s0)];
                double *const *PH = sphi ? &a.allPhi[4 * (size_t)s] : &a.segPhi[4 * (size_t)(s - s0)];
                adj_stage(c, 0, dt / 6., 0.);
                vjp(c, X + 12, PH[3]);
                adj_stage(c, 1, dt / 3., dt);
                vjp(c, X + 8, PH[2]);
                adj_stage(c, 1, dt / 3., 0.5 * dt);
                vjp(c, X + 4, PH[1]);
                adj_stage(c, 1, dt / 6., 0.5 * dt);
                vjp(c, X + 0, PH[0]);
                adj_stage(c, 2, 0., 0.);
            }
        }
        // gradient with respect to the initial state
        if (nck > 0) snap_load(c, a.ck[0]);
        if (dJ_dn0) {
            c->adj_fn(c, 5);
            {
                Launch L_(c, KC_ADJ_PW, 24. * N);
                k_dn0<<<nblk(N, 256), 256, 0, c->st>>>(a.RB[0], a.RB[1], a.out, N);
            }
            CK(cudaMemcpyAsync(dJ_dn0, a.out, 8 * N, cudaMemcpyDeviceToHost, c->st));
        }
        if (lam0)
            for (int q = 0; q < 4; ++q)
                CK(cudaMemcpyAsync(lam0 + 2 * c->Nc * q, a.lam[q], 16 * c->Nc, cudaMemcpyDeviceToHost, c->st));
        snap_load(c, a.fin);
    }
    CK(cudaEventRecord(ev[2], c->st));
    CK(cudaMemcpyAsync(a.h_acc, a.acc, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaGetLastError());
    float f_ms = 0.f, b_ms = 0.f;
    CK(cudaEventElapsedTime(&f_ms, ev[0], ev[1]));
    CK(cudaEventElapsedTime(&b_ms, ev[1], ev[2]));
    const double h = cf.L / c->n;
    out->J = a.h_acc[3] * h * h * h;
    out->dJ_dM = jonly ? 0. : a.h_acc[0];
    out->dJ_dtau = jonly ? 0. : a.h_acc[1];
    out->dJ_dnd = jonly ? 0. : a.h_acc[2];
    out->fwd_ms = f_ms;
    out->bwd_ms = jonly ? 0. : b_ms;
    out->adj_cycles = a.cycles;
    out->adj_solves = a.solves;
    out->checkpoints = jonly ? 0 : nck;
}

}  // namespace

extern "C" int kf_adjoint_run(kf_ctx *c, int nsteps, double dt, int ckpt_every, int flags, const double *w,
                              kf_grad_out *out, double *dJ_dn0, double *lam0) {
    return guarded(c, [&] {
        if (c->stretched) throw KfError{KF_ERR_ARG, "the discrete adjoint needs equidistant axes (stretch_m = 0)"};
        adj_run(c, nsteps, dt, ckpt_every, flags, w, out, dJ_dn0, lam0);
    });
}
