// kf_capi.cu -- host driver and C ABI (include/kielflow_b200.h).
//
// The right-hand side of rhs_standard::solve (rhs_standard.cpp:89-566) is run as
// six rounds of kernels on device-resident buffers:
//   A  inverse x/y passes of s^ (P s^, i k_x P s^, i k_y P s^) and the z pass of
//      P s^  ->  s_d;  rho = exp(s_d) + n_d;  Poisson solve -> phi
//   B  phi^ = r2c(phi)                                    (E-force, :218-226)
//   C  (penalization) rl_q = -lin_q in k-space
//   D  inverse passes generating U_c, d_d U_c, d_d s (and c2r(rl_q))
//   E  physical-space products (advection, u.grad s) [+ penalization]
//   F  forward z/y passes, then the forward x pass fused with the assembly
//      K_q = -(lin_q + F_q)   (or P F_q with penalization)
// RK4 (RKO4.cpp:50-241) combines four such evaluations with k_rk.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <memory>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/kielflow_b200.h"
#include "kf_adjoint.cuh"
#include "kf_graph.cuh"
#include "kf_march.cuh"
#include "kf_passes.cuh"
#include "kf_pointwise.cuh"
#include "kf_poisson.cuh"
#include "kf_stretch.cuh"

using namespace kf;

namespace {

struct KfError {
    int code;
    std::string msg;
};

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) throw KfError{KF_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

struct LevelBuf {
    int n = 0;
    double *dd = nullptr, *dp = nullptr, *dm = nullptr, *ip = nullptr, *im = nullptr, *gam = nullptr;
    double *phi = nullptr, *rho = nullptr, *r = nullptr, *phi0 = nullptr;
    double *t = nullptr;  // second potential of the streaming smoother (k_rbgs_march), n >= MT_TK
    std::shared_ptr<AxTab> tab;  // host copy of dd, ip, im for k_rbgs_t (n <= KF_TAB_N)
    Lev lev() const { return Lev{n, dd, dp, dm, ip, im}; }
};

constexpr int RBS = 256;  // reduction block size

// Colour-split copy of the finest rho for the half sweeps (0: they read rho).
#ifndef KF_RHO_CS
#define KF_RHO_CS 1
#endif

// Half sweeps with the i and j axis tables passed as a kernel parameter
// (k_rbgs_t; 0: k_rbgs reads them from global memory).
#ifndef KF_RBGS_TAB
#define KF_RBGS_TAB 1
#endif


struct AdjState;  // discrete-adjoint buffers (allocated by the first kf_adjoint_run)
struct OutState;  // output buffers of kf_run / kf_get_output (allocated on first use)

}  // namespace

struct kf_ctx {
    kf_config cfg;
    int n = 0, nzc = 0;
    long N = 0, Nc = 0;
    bool fp32 = false;
    size_t es = 8, cs = 16;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    std::string err;
    long long launches = 0;
    std::vector<void *> allocs;

    void *Y[4] = {}, *Ys[4] = {}, *ACC[4] = {}, *K[4] = {};
    void *CX[12] = {}, *CY[16] = {}, *R[24] = {}, *phihat = nullptr, *LIN[4] = {};
    double *phi = nullptr, *rho = nullptr, *nd = nullptr;
    double *rho_cs = nullptr;  // colour-split copy of rho for the finest half sweeps (rho_split)
    void *H = nullptr, *phiT = nullptr;
    void *kv = nullptr, *SV = nullptr, *PF = nullptr, *tw = nullptr;
    double *q2 = nullptr;
    int *pb = nullptr;  // x-pass 2/3-rule bounds per (j, kz) column (dealias_bounds)
    double *stage64 = nullptr;
    std::vector<LevelBuf> lv;
    double *partial = nullptr;
    int npartial = 0;
    double *red = nullptr;
    double *h_red = nullptr;
    int *d_sweeps = nullptr;
    unsigned long long *d_max = nullptr, *h_max = nullptr;
    int *d_err = nullptr, *h_err = nullptr;  // kernel error word (bit 0: a bounded copy wait gave up)
    // RK4 time (Runge_kutta_O4::t_) and the phi history for extrapolated starts
    double t = 0., t_stage = 0.;
    double *phi_a = nullptr;
    double tau_a = 0., tau_b = 0.;
    int nhist = 0;
    AxisJob *dj = nullptr;
    ZJob *dz = nullptr;
    // job-list offsets (into dj / dz) and counts
    int jA_x = 0, jA_y = 0, zA = 0, zB = 0, jB_y = 0, jB_x = 0, jD_x = 0, nD_x = 0, jD_y = 0, nD_y = 0;
    int zD = 0, nzD = 0, zF = 0, jF_y = 0, jF_x = 0, jT_x = 0, jT_y = 0, zT = 0, jTf_y = 0, jTf_x = 0;
    int jG_x = 0, jG_y = 0, zG = 0;
    // sine-stretched axes: the chain-rule right-hand side's buffers, metric
    // tables and job lists (allocated only when cfg.stretch_m != 0)
    bool stretched = false;
    void *SX[15] = {};
    void *met = nullptr;    // filtered 1/dS per index (bulk precision)
    double *vol = nullptr;  // dS per index (cell widths / h) for the diagnostics
    int jS_Dx = 0, jS_Dy = 0, zS_D = 0, zS_F = 0, jS_Fy = 0, jS_Fx = 0, jS_Gx = 0, jS_Gy = 0, zS_G = 0;
    int zS_I = 0, jS_Iy = 0, jS_Ix = 0, jS_Kx = 0, jS_Ky = 0, zS_K = 0, zS_Kf = 0, jS_Kfy = 0, jS_Kfx = 0;
    // Jacobi state carried between sweeps and solves (solver_poisson_jacobi_nlin.hpp:66-95)
    double norm_max = 0., norm_sum = 0., norm_max_old = -1., norm_sum_old = -1.;
    double sup = 0., inf = 0., omega = 1.;
    kf_diag_out diag{};
    // kernel profiling (CUDA events around each launch, when enabled)
    bool prof = false;
    struct ProfRec { int cls; cudaEvent_t a, b; double bytes; };
    std::vector<ProfRec> recs;
    std::vector<cudaEvent_t> evfree;
    double prof_ms[32] = {}, prof_bytes[32] = {};
    long long prof_n[32] = {};
    std::vector<AxisJob> hj;
    std::vector<ZJob> hz;
    // the FAS V-cycle captured once as a CUDA graph (replayed every cycle)
    cudaGraphExec_t vgraph = nullptr;
    long long vgraph_kernels = 0;
    // the part of a V-cycle after the finest level's residual (adaptive solves)
    cudaGraphExec_t vgraph_tail = nullptr;
    long long vgraph_tail_kernels = 0;
    // per-(precision, n) entry points
    void (*rhs_fn)(kf_ctx *) = nullptr;
    void (*r2c_fn)(kf_ctx *) = nullptr;
    void (*c2r_fn)(kf_ctx *) = nullptr;
    void (*inv_state_fn)(kf_ctx *) = nullptr;
    void (*adj_fn)(kf_ctx *, int) = nullptr;
    // discrete adjoint: buffers, job-list offsets, and the "phi given" switch
    // under which a right-hand side uses c->phi as it stands (no solve)
    AdjState *adj = nullptr;
    OutState *out = nullptr;
    bool phi_given = false;
    int fftv = 0;     // radix-plan variant of the transform kernels (kf_autotune)
    int rbgs_by = 8;  // smoother variant (kf_autotune): k_rbgs rows per block, or 0 for k_rbgs_march
    bool march_maps = false;  // the driver's tensor-map encoder is available
    bool coarse_block = true;  // levels <= 16^3 of a V-cycle in one k_coarse_cycle block (kf_set_coarse_block)
    int cc_level = -1;         // entry level of k_coarse_cycle, or -1 (cc_setup)
    CoarseCycle ccyc{};
    size_t cc_smem = 0;
    int stage_idx = 0;  // RK stage of the right-hand side being evaluated (0..3)
    // one RK4 step captured as a CUDA graph (FAS or no Poisson, profile off):
    // time / warm-start history and solve statistics live on the device
    bool capturing = false;
    cudaStream_t st_body = nullptr;  // stream on which conditional bodies are captured
    // round D's transforms of u' and s, which do not depend on phi, run in a
    // captured step on st_side beside the Poisson solve (kf_set_overlap)
    bool overlap_d = true;
    cudaStream_t st_side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    DevTime *dtime = nullptr;
    DevPois *dpois = nullptr;
    DevPois hpois{};  // last values read back
    cudaGraphExec_t step_graph = nullptr;
    // the same step whose stage 1 waits for ev_u (the u' upload of kf_step_host)
    // after its Poisson solve, before the first use of u'
    cudaGraphExec_t step_graph_wait = nullptr;
    bool capture_wait_u = false;
    cudaStream_t st_copy = nullptr;
    cudaEvent_t ev_u = nullptr;
    double *stage64b = nullptr;  // FP32-bulk staging of the copy stream
    double step_dt = 0.;
    long long step_kernels = 0, cycle_kernels = 0, head_kernels = 0;
    int jV_x = 0, jV_y = 0, zV = 0, zW = 0, nWz = 0, nWf = 0, jW_y = 0, jW_x = 0, zS = 0, jS_y = 0, jS_x = 0;
    int jP_x = 0, jP_y = 0, zP = 0, jQ_x = 0, jQ_y = 0, zQ = 0;
};

namespace {

// Host-side NVTX range (profiler timelines and ncu --nvtx filters): each RK4
// stage, each Poisson solve, each replay of a captured step.  Header-only NVTX:
// without a profiler attached the calls return at once.
struct NvtxRange {
    explicit NvtxRange(const char *s) { nvtxRangePushA(s); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

template <typename P> P *dalloc(kf_ctx *c, size_t bytes) {
    void *p = nullptr;
    CK(cudaMalloc(&p, bytes ? bytes : 16));
    c->allocs.push_back(p);
    return static_cast<P *>(p);
}

inline int nblk(long work, int bs) { return (int)((work + bs - 1) / bs); }

// Kernel classes for the profile (kf_profile_read); names in kf_profile_class_name.
enum KCls { KC_AXIS_INV, KC_AXIS_FWD, KC_Z_C2R, KC_Z_R2C, KC_XASM, KC_PROD, KC_LIN, KC_RHO, KC_RK,
            KC_JACOBI, KC_RBGS, KC_RESID, KC_TRANSFER, KC_COARSE, KC_REDUCE, KC_MISC, KC_ADJ_PW, KC_ADJ_MG,
            KC_MG_COARSE, KC_MARCH, KC_MARCH_RES,
            KC_N };
const char *const kKClsName[KC_N] = {"k_axis_pass(inverse)", "k_axis_pass(forward)", "k_z_c2r", "k_z_r2c",
                                     "k_xfwd_assemble", "k_products", "k_lin", "k_rho", "k_rk", "k_jacobi",
                                     "k_rbgs", "k_residual", "k_restrict/k_fas_rhs/k_prolong/k_inject",
                                     "k_coarse_solve/k_coarse_cycle", "k_reduce_final", "conversion/diagnostics",
                                     "adjoint pointwise (k_prod_vjp/k_vjp_assemble/k_adj_stage/...)",
                                     "adjoint Poisson (linear multigrid)",
                                     "FAS levels below the finest (k_rbgs/k_residual/transfers)",
                                     "k_rbgs_march(sweep)", "k_rbgs_march(sweep+residual)"};

void prof_flush(kf_ctx *c) {
    if (c->recs.empty()) return;
    CK(cudaStreamSynchronize(c->st));
    for (auto &r : c->recs) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, r.a, r.b));
        c->prof_ms[r.cls] += ms;
        c->prof_n[r.cls] += 1;
        c->prof_bytes[r.cls] += r.bytes;
        c->evfree.push_back(r.a);
        c->evfree.push_back(r.b);
    }
    c->recs.clear();
}

cudaEvent_t prof_event(kf_ctx *c) {
    if (c->evfree.empty()) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        return e;
    }
    cudaEvent_t e = c->evfree.back();
    c->evfree.pop_back();
    return e;
}

// One kernel launch: counts it and, when profiling, brackets it with events
// on the context's stream and records its algorithmic bytes.
struct Launch {
    kf_ctx *c;
    int cls;
    double bytes;
    cudaEvent_t a = nullptr;
    Launch(kf_ctx *c_, int cls_, double bytes_) : c(c_), cls(cls_), bytes(bytes_) {
        c->launches++;
        if (c->prof) {
            if (c->recs.size() > 16384) prof_flush(c);
            a = prof_event(c);
            CK(cudaEventRecord(a, c->st));
        }
    }
    ~Launch() noexcept(false) {
        if (c->prof) {
            cudaEvent_t b = prof_event(c);
            CK(cudaEventRecord(b, c->st));
            c->recs.push_back(kf_ctx::ProfRec{cls, a, b, bytes});
        }
    }
};

// ------------------------------------------------------------------ host tables
double k_val_at(int i, int n, double L) {  // axis_EqSt.cpp:57-61
    double pi = acos(-1.);
    return ((i <= n / 2) ? (2. * pi * i / L) : (2. * pi * (i - n) / L));
}
// Position of index i (-1 <= i <= n) on the box axis [-L/2, L/2):
// axis_CoEqSt for m == 0 (axis_EqSt.cpp:52-55), else axis_CoSiSt with the
// periodic extension of its val_at (axis_SiSt.cpp:93-116) and
// S(x) = x - m sin(2 pi x / L) (:153-157).
double val_at(int i, int n, double L, double m = 0.) {
    if (m == 0.) return -0.5 * L + i * (L / n);
    int shift = 0;
    if (i < 0) {
        do {
            shift += 1;
        } while (i + shift * n < 0);
    }
    if (i >= n) {
        do {
            shift -= 1;
        } while (i + shift * n >= n - 1);
    }
    const double pi = acos(-1.);
    const double x = -0.5 * L + L * double(i + shift * n) / (n);
    return (x - m * sin(2. * pi * x / L)) - shift * L;
}
// dS/dx of the stretched axis at index i (axis_SiSt.cpp:158-164)
double dS_at(int i, int n, double L, double m) {
    const double pi = acos(-1.);
    const double x = -0.5 * L + (L / n) * i;
    return 1. - (2. * pi * m / L) * cos(2. * pi * x / L);
}
// 1/dS of each index after the 2/3 filter: OP_partial_derivative.cpp:60-80
// forms it on the whole grid (FFT, OP_dealiasing, inverse FFT); the field
// depends on one index only, so that is one 1-D DFT pair along the axis with
// the filter of the (k, 0, 0) line, done here in long double.
std::vector<double> metric_table(int n, double L, double m, double thr) {
    std::vector<double> f(n), q2(n), out(n);
    const double kmax = k_val_at(n / 2, n, L);
    for (int i = 0; i < n; ++i) {
        f[i] = 1. / dS_at(i, n, L, m);
        q2[i] = pow(k_val_at(i, n, L) / kmax, 2.);
    }
    const long double twopi = 6.283185307179586476925286766559005768L;
    std::vector<long double> acc(n, 0.L);
    for (int kk = 0; kk < n; ++kk) {
        if (!(q2[kk] + q2[0] + q2[0] < thr)) continue;
        long double Fr = 0.L, Fi = 0.L;
        for (int i = 0; i < n; ++i) {
            const long double a = twopi * (long double)((long)kk * i % n) / n;
            Fr += f[i] * cosl(a);
            Fi -= f[i] * sinl(a);
        }
        for (int i = 0; i < n; ++i) {
            const long double a = twopi * (long double)((long)kk * i % n) / n;
            acc[i] += Fr * cosl(a) - Fi * sinl(a);
        }
    }
    for (int i = 0; i < n; ++i) out[i] = (double)(acc[i] / n);
    return out;
}

// The 2/3 rule of OP_dealiasing.hpp:24-30 on one (j, kz) column of the x
// pass, (q2[i] + q2[j]) + q2[kz] < thr, as a bound b: keep(i) == (min(i, n - i)
// <= b).  The bound is the largest such m in [0, n/2] (-1: none), and the
// equivalence is checked on every i of the column with the same additions as
// the device; a column where it fails gets -2 (the kernels then test each
// element).
std::vector<int> dealias_bounds(const std::vector<double> &q2, int n, double thr) {
    const int nzc = n / 2 + 1;
    std::vector<int> pb((size_t)n * nzc);
    for (int j = 0; j < n; ++j)
        for (int k = 0; k < nzc; ++k) {
            int b = -1;
            for (int m = 0; m <= n / 2; ++m)
                if ((q2[m] + q2[j]) + q2[k] < thr) b = m;
            bool ok = true;
            for (int i = 0; i < n && ok; ++i) {
                const bool keep = (q2[i] + q2[j]) + q2[k] < thr;
                ok = keep == ((i <= n / 2 ? i : n - i) <= b);
            }
            pb[(size_t)j * nzc + k] = ok ? b : -2;
        }
    return pb;
}

// ------------------------------------------------------------------ Poisson driver
void reduce_read(kf_ctx *c, int nb) {
    {
        Launch L_(c, KC_REDUCE, 0.);
        k_reduce_final<RBS><<<1, RBS, 0, c->st>>>(c->partial, nb, c->red);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_red, c->red, sizeof(double) * KF_RED, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
}

int red_blocks(long N) {
    long nb = (N + RBS - 1) / RBS;
    return (int)(nb < 1184 ? nb : 1184);
}

// Levels on which the column form of the residual runs (whole warps along k,
// columns of COL_PI planes).  At 256^3 (one B200): 99.6 us against 155.9 us for
// k_residual<1, 1>; the column form of the half sweep measured slower (201-225
// us per sweep against 150 us: its per-thread chain of Newton steps is
// latency-bound), so the half sweep stays one point per thread.
constexpr int COL_PI = 16;
bool col_level(int n) { return n >= 64 && n % 64 == 0 && n % COL_PI == 0; }

// The kernel error word: queued for reading before a synchronisation
// (kerr_fetch) and checked after it (kerr_check, which clears it)
void kerr_fetch(kf_ctx *c) {
    CK(cudaMemcpyAsync(c->h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
}
void kerr_check(kf_ctx *c) {
    if (*c->h_err) {
        *c->h_err = 0;
        CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
        throw KfError{KF_ERR_CUDA, "a shared-memory copy of the multigrid smoother did not land within its wait limit"};
    }
}

double max_residual(kf_ctx *c, const LevelBuf &L, const double *phi, const double *rho, bool fast) {
    const long N = (long)L.n * L.n * L.n;
    CK(cudaMemsetAsync(c->d_max, 0, 64 * sizeof(unsigned long long), c->st));
    {
        Launch L_(c, KC_RESID, 16. * N);
        dim3 g = mg_grid(L.n, L.n);
        g.z = L.n < 16 ? L.n : 16;  // each block strides over the i-planes
        if (fast && col_level(L.n))
            k_residual_col<8, COL_PI, true, false, false>
                <<<dim3(L.n / 64, L.n / 8, L.n / COL_PI), mg_block(), 0, c->st>>>(phi, rho, L.lev(), nullptr, c->d_max);
        else if (fast)
            k_resmax<true><<<g, mg_block(), 0, c->st>>>(phi, rho, L.lev(), c->d_max);
        else
            k_resmax<false><<<g, mg_block(), 0, c->st>>>(phi, rho, L.lev(), c->d_max);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_max, c->d_max, 64 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->st));
    kerr_fetch(c);
    CK(cudaStreamSynchronize(c->st));
    kerr_check(c);
    unsigned long long m = 0;
    for (int s = 0; s < 64; ++s) m = c->h_max[s] > m ? c->h_max[s] : m;
    double r;
    std::memcpy(&r, &m, sizeof(double));
    return r;
}

// solver_poisson_jacobi_nlin::solve (:50-108) on one level; phi, tmp: level-sized.
int jacobi_solve(kf_ctx *c, const LevelBuf &L, double *phi, double *tmp, const double *rho, int max_it,
                 double limit_max, bool resstop, double tol) {
    const long N = (long)L.n * L.n * L.n;
    const int nb = red_blocks(N);
    c->sup = 0.;
    c->inf = 0.;
    int iteration = 0;
    c->omega = 1.;
    bool converged = false;
    c->norm_sum_old = -1.;
    if (max_it < 0) max_it = 1000;
    double *cur = phi, *oth = tmp;
    double rlast = 0.;
    while (!converged && iteration < max_it) {
        iteration++;
        c->norm_sum_old = c->norm_sum;
        c->norm_max_old = c->norm_max;
        {
            Launch L_(c, KC_JACOBI, 24. * N);
            k_jacobi<RBS><<<nb, RBS, 0, c->st>>>(cur, oth, rho, L.lev(), c->omega, c->partial);
        }
        reduce_read(c, nb);
        std::swap(cur, oth);
        c->norm_max = c->h_red[0];
        c->norm_sum = c->h_red[1];
        c->sup = c->h_red[2];
        c->inf = c->h_red[3];
        rlast = c->h_red[4];
        if (rlast != rlast || c->norm_max != c->norm_max) throw KfError{KF_ERR_NAN, "NaN in the Jacobi sweep"};
        // Carre's over-relaxation factor (:237-252)
        c->norm_sum = c->norm_sum / ((double)N);
        if ((c->norm_max < c->norm_max_old) && (iteration > 1)) {
            double lambda = c->norm_sum / c->norm_sum_old;
            c->omega = 2. / (1. + sqrt(1. - pow(lambda + c->omega - 1., 2.) / (lambda * pow(c->omega, 2.))));
        } else {
            c->omega = .5;
        }
        if (c->omega != c->omega) c->omega = .5;
        bool conv_rel = c->norm_max < limit_max * (c->sup - c->inf);
        converged = resstop ? (rlast <= tol) : conv_rel;
    }
    if (cur != phi) CK(cudaMemcpyAsync(phi, cur, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->st));
    c->diag.last_iterations = iteration;
    c->diag.total_iterations += iteration;
    c->diag.last_residual = rlast;
    if (!converged) c->diag.not_converged++;
    return converged ? 0 : 1;
}

// over-relaxation factor of the FAS smoother's Newton step (0 selects 1)
double mg_omega(const kf_config &cf) { return cf.mg_omega > 0. ? cf.mg_omega : 1.; }

// ------------------------------------------------------- streaming smoother
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (EncodeTiledFn)p;
    }();
    return fn;
}

// Tensor map of an n^3 FP64 level whose copies are single rows of MT_PITCH
// doubles (x = k fastest, then j, then i)
bool row_map(CUtensorMap *m, const double *base, int n) {
    const EncodeTiledFn f = encode_tiled();
    if (!f) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)n};
    const cuuint64_t strides[2] = {(cuuint64_t)n * 8, (cuuint64_t)n * n * 8};
    const cuuint32_t box[3] = {MT_PITCH, 1, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// planes per CTA of the streaming smoother: at least three waves of CTAs at
// 256^3 (128 tiles x 8 chunks), the ghost planes (2 H per chunk) small
int march_ci(int n) { return n >= 256 ? 32 : (n >= 128 ? 16 : 8); }
constexpr int MT_TJ = 8;

bool march_level(const LevelBuf &L) { return L.n >= MT_TK && L.n % MT_TK == 0 && L.n % MT_TJ == 0; }

bool march_ok(const kf_ctx *c, const LevelBuf &L) { return c->rbgs_by == 0 && c->march_maps && L.t && march_level(L); }

void march_attrs() {
    CK(cudaFuncSetAttribute(k_rbgs_march<MM_RES, MT_TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)march_smem<MM_RES, MT_TJ>(32)));
    CK(cudaFuncSetAttribute(k_rbgs_march<MM_SWEEP, MT_TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)march_smem<MM_SWEEP, MT_TJ>(32)));
    CK(cudaFuncSetAttribute(k_rbgs_march<MM_SWEEP_RES, MT_TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)march_smem<MM_SWEEP_RES, MT_TJ>(32)));
}

// One streaming pass on level L: src -> dst (a whole red-black sweep) and/or
// the residual r of the result, max |r| into `slots` when given.
template <int MODE>
void march(kf_ctx *c, const LevelBuf &L, const double *src, const double *rho, double *dst, double *r,
           unsigned long long *slots, int cls) {
    const int n = L.n, ci = march_ci(n);
    CUtensorMap mp, mr;
    if (!row_map(&mp, src, n) || !row_map(&mr, rho, n))
        throw KfError{KF_ERR_CUDA, "cuTensorMapEncodeTiled refused a multigrid level"};
    MarchArgs a{dst, r, src, rho, L.dd, L.ip, L.im, slots, c->d_err, n, ci, n / MT_TK, mg_omega(c->cfg)};
    const dim3 g((n / MT_TK) * (n / MT_TJ), n / ci);
    const long N = (long)n * n * n;
    Launch L_(c, cls, (MODE == MM_SWEEP_RES ? 32. : 24.) * N);
    k_rbgs_march<MODE, MT_TJ><<<g, MT_THREADS, march_smem<MODE, MT_TJ>(ci), c->st>>>(mp, mr, a);
}

// `sweeps` red-black Gauss-Seidel sweeps on level L (phi in place), two
// half-sweep launches each.  cc: the adjoint's e^phi (linear point solve) or
// nullptr (Newton step).
void smooth_plain(kf_ctx *c, LevelBuf &L, double *phi, const double *rho, const double *cc, int sweeps, int cls);

void smooth(kf_ctx *c, LevelBuf &L, double *phi, const double *rho, const double *cc, int sweeps, int cls) {
    if (!cc && march_ok(c, L) && phi != L.t) {
        // streaming passes phi -> t -> phi; an odd sweep first in place
        if (sweeps & 1) smooth_plain(c, L, phi, rho, nullptr, 1, cls);
        const int mc = cls == KC_RBGS ? KC_MARCH : cls;
        for (int s = 0; s + 1 < sweeps; s += 2) {
            march<MM_SWEEP>(c, L, phi, rho, L.t, nullptr, nullptr, mc);
            march<MM_SWEEP>(c, L, L.t, rho, phi, nullptr, nullptr, mc);
        }
        return;
    }
    smooth_plain(c, L, phi, rho, cc, sweeps, cls);
}

// `sweeps` red-black sweeps as two half-sweep launches each (k_rbgs, or
// k_rbgs_lin with the adjoint's e^phi).  (Sweeping a level larger than L2 in
// chunks of i-planes, black one plane behind red so that the black half finds
// its data in L2, gives the same potentials bit for bit but measured slower at
// 256^3: 156 / 169 / 181 / 214 us per sweep for 1 / 2 / 4 / 8 chunks.  So did
// threads that update one (j, k) on 2 or 4 planes two apart, sharing the axis
// tables and the planes between their points: 20.4 / 20.2 ms against 18.9 ms
// for 240 half sweeps; L1 use fell from 89 to 62 %, but occupancy halved and
// the DRAM throughput, 4.5 TB/s on 1.33x the algorithmic bytes, stayed.)

void smooth_plain(kf_ctx *c, LevelBuf &L, double *phi, const double *rho, const double *cc, int sweeps, int cls) {
    const int n = L.n;
    const long N = (long)n * n * n;
    const int by = c->rbgs_by ? c->rbgs_by : 8;
    const double om = mg_omega(c->cfg);
    const dim3 g((n / 2 + 31) / 32, (n + by - 1) / by, n), b(32, by);
    for (int s = 0; s < sweeps; ++s)
        for (int color = 0; color < 2; ++color) {
            Launch L_(c, cls, 16. * N);
            if (cc && L.tab) {
                if (by == 4)
                    k_rbgs_lin_t<4><<<g, b, 0, c->st>>>(phi, rho, cc, L.lev(), color, om, *L.tab);
                else if (by == 16)
                    k_rbgs_lin_t<16><<<g, b, 0, c->st>>>(phi, rho, cc, L.lev(), color, om, *L.tab);
                else
                    k_rbgs_lin_t<8><<<g, b, 0, c->st>>>(phi, rho, cc, L.lev(), color, om, *L.tab);
            } else if (cc) {
                if (by == 4)
                    k_rbgs_lin<4><<<g, b, 0, c->st>>>(phi, rho, cc, L.lev(), color, om);
                else if (by == 16)
                    k_rbgs_lin<16><<<g, b, 0, c->st>>>(phi, rho, cc, L.lev(), color, om);
                else
                    k_rbgs_lin<8><<<g, b, 0, c->st>>>(phi, rho, cc, L.lev(), color, om);
            } else if (L.tab && rho == c->rho && c->rho_cs) {
                // the finest level reads the colour-split copy (rho_split at the solve's start)
                if (by == 4)
                    k_rbgs_t<4, true><<<g, b, 0, c->st>>>(phi, c->rho_cs, L.lev(), color, om, *L.tab);
                else if (by == 16)
                    k_rbgs_t<16, true><<<g, b, 0, c->st>>>(phi, c->rho_cs, L.lev(), color, om, *L.tab);
                else
                    k_rbgs_t<8, true><<<g, b, 0, c->st>>>(phi, c->rho_cs, L.lev(), color, om, *L.tab);
            } else if (L.tab) {
                if (by == 4)
                    k_rbgs_t<4><<<g, b, 0, c->st>>>(phi, rho, L.lev(), color, om, *L.tab);
                else if (by == 16)
                    k_rbgs_t<16><<<g, b, 0, c->st>>>(phi, rho, L.lev(), color, om, *L.tab);
                else
                    k_rbgs_t<8><<<g, b, 0, c->st>>>(phi, rho, L.lev(), color, om, *L.tab);
            } else {
                if (by == 4)
                    k_rbgs<4><<<g, b, 0, c->st>>>(phi, rho, L.lev(), color, om);
                else if (by == 16)
                    k_rbgs<16><<<g, b, 0, c->st>>>(phi, rho, L.lev(), color, om);
                else
                    k_rbgs<8><<<g, b, 0, c->st>>>(phi, rho, L.lev(), color, om);
            }
        }
}

void vcycle(kf_ctx *c, int l);

// First part of a V-cycle on level l (not the coarsest): pre-smoothing and the
// residual L.r; with_max also leaves max |L.r| in the d_max slots.
void vcycle_head(kf_ctx *c, int l, bool with_max) {
    LevelBuf &L = c->lv[l];
    const kf_config &cf = c->cfg;
    const int n = L.n;
    const long N = (long)n * n * n;
    if (march_ok(c, L) && cf.mg_pre >= 1) {
        // the last pre-smoothing sweep fused with the residual (and its max):
        // the sweeps before it leave the potential in L.t
        int s = cf.mg_pre - 1;
        const int cls = l == 0 ? KC_MARCH : KC_MG_COARSE;
        if (s > 0 && s % 2 == 0) {
            smooth_plain(c, L, L.phi, L.rho, nullptr, 1, l == 0 ? KC_RBGS : KC_MG_COARSE);
            --s;
        }
        if (s == 0) {
            CK(cudaMemcpyAsync(L.t, L.phi, 8 * (size_t)N, cudaMemcpyDeviceToDevice, c->st));
        } else {
            march<MM_SWEEP>(c, L, L.phi, L.rho, L.t, nullptr, nullptr, cls);
            for (; s > 1; s -= 2) {
                march<MM_SWEEP>(c, L, L.t, L.rho, L.phi, nullptr, nullptr, cls);
                march<MM_SWEEP>(c, L, L.phi, L.rho, L.t, nullptr, nullptr, cls);
            }
        }
        if (with_max) CK(cudaMemsetAsync(c->d_max, 0, 64 * sizeof(unsigned long long), c->st));
        march<MM_SWEEP_RES>(c, L, L.t, L.rho, L.phi, L.r, with_max ? c->d_max : nullptr,
                            l == 0 ? KC_MARCH_RES : KC_MG_COARSE);
        return;
    }
    smooth(c, L, L.phi, L.rho, nullptr, cf.mg_pre, l == 0 ? KC_RBGS : KC_MG_COARSE);
    if (with_max) CK(cudaMemsetAsync(c->d_max, 0, 64 * sizeof(unsigned long long), c->st));
    Launch L_(c, l == 0 ? KC_RESID : KC_MG_COARSE, 24. * N);
    if (col_level(n)) {
        const dim3 gc(n / 64, n / 8, n / COL_PI);
        if (with_max)
            k_residual_col<8, COL_PI, true><<<gc, mg_block(), 0, c->st>>>(L.phi, L.rho, L.lev(), L.r, c->d_max);
        else
            k_residual_col<8, COL_PI, false><<<gc, mg_block(), 0, c->st>>>(L.phi, L.rho, L.lev(), L.r, nullptr);
    } else if (with_max) {
        dim3 g = mg_grid(n, n);
        g.z = n < 16 ? n : 16;  // each block strides over n/16 i-planes (ncu, 256^3: 158 us; 64 groups 169 us)
        k_residual<true, true><<<g, mg_block(), 0, c->st>>>(L.phi, L.rho, L.lev(), L.r, c->d_max);
    } else {
        k_residual<true><<<mg_grid(n, n), mg_block(), 0, c->st>>>(L.phi, L.rho, L.lev(), L.r);
    }
}

// The rest of the V-cycle on level l: restriction, the coarse cycle, the
// correction and post-smoothing.
void vcycle_tail(kf_ctx *c, int l) {
    LevelBuf &L = c->lv[l];
    const kf_config &cf = c->cfg;
    const int n = L.n;
    const long N = (long)n * n * n;
    LevelBuf &Lc = c->lv[l + 1];
    const long Nc3 = (long)Lc.n * Lc.n * Lc.n;
    {
        Launch L_(c, l == 0 ? KC_TRANSFER : KC_MG_COARSE, 8. * N + 32. * Nc3);
        k_restrict<<<mg_grid(Lc.n, Lc.n), mg_block(), 0, c->st>>>(L.r, L.phi, n, Lc.r, Lc.phi, Lc.phi0);
    }
    if (l + 1 == c->cc_level) {
        // the levels from l + 1 down in one block: FAS right-hand side, cycle, correction
        Launch L_(c, KC_COARSE, 40. * Nc3);
        k_coarse_cycle<<<1, 1024, c->cc_smem, c->st>>>(Lc.phi, Lc.phi0, Lc.r, c->ccyc, cf.mg_pre, cf.mg_post,
                                                       cf.coarse_tol, 1000, mg_omega(cf), c->d_sweeps);
    } else {
        {
            Launch L_(c, l == 0 ? KC_TRANSFER : KC_MG_COARSE, 24. * Nc3);
            k_fas_rhs<<<mg_grid(Lc.n, Lc.n), mg_block(), 0, c->st>>>(Lc.phi, Lc.r, Lc.lev(), Lc.rho);
        }
        vcycle(c, l + 1);
        {
            Launch L_(c, l == 0 ? KC_TRANSFER : KC_MG_COARSE, 24. * Nc3);
            k_correction<<<mg_grid(Lc.n, Lc.n), mg_block(), 0, c->st>>>(Lc.phi, Lc.phi0, Lc.n);
        }
    }
    {
        Launch L_(c, l == 0 ? KC_TRANSFER : KC_MG_COARSE, 16. * N + 8. * Nc3);
        k_prolong_add<<<mg_grid(Lc.n, Lc.n), mg_block(), 0, c->st>>>(L.phi, Lc.phi0, nullptr, L.gam, n);
    }
    smooth(c, L, L.phi, L.rho, nullptr, cf.mg_post, l == 0 ? KC_RBGS : KC_MG_COARSE);
    CK(cudaGetLastError());
}

void vcycle(kf_ctx *c, int l) {
    LevelBuf &L = c->lv[l];
    const kf_config &cf = c->cfg;
    const int n = L.n;
    const long N = (long)n * n * n;
    if (l == (int)c->lv.size() - 1) {
        Launch L_(c, KC_COARSE, 16. * N);
        const int bs = N >= 1024 ? 1024 : (int)((N + 31) / 32 * 32);
        k_coarse_solve<<<1, bs, (size_t)(16 * N + 24 * n), c->st>>>(L.phi, L.rho, L.lev(), cf.coarse_tol, 1000,
                                                                   c->d_sweeps, mg_omega(cf));
        return;
    }
    vcycle_head(c, l, false);
    vcycle_tail(c, l);
}

// One FAS V-cycle on the finest level: replayed from a CUDA graph captured on
// first use (one launch instead of ~70), or launched kernel by kernel while
// the per-launch profile is on.
void run_vcycle(kf_ctx *c) {
    if (c->prof) {
        vcycle(c, 0);
        return;
    }
    if (!c->vgraph) {
        const long long l0 = c->launches;
        CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        vcycle(c, 0);
        cudaGraph_t g = nullptr;
        CK(cudaStreamEndCapture(c->st, &g));
        cudaError_t e = cudaGraphInstantiate(&c->vgraph, g, 0);
        cudaGraphDestroy(g);
        CK(e);
        c->vgraph_kernels = c->launches - l0;
        c->launches = l0;
    }
    CK(cudaGraphLaunch(c->vgraph, c->st));
    c->launches += c->vgraph_kernels;
}

// vcycle_tail(c, 0), replayed from its own graph as run_vcycle does
void run_vcycle_tail(kf_ctx *c) {
    if (c->prof) {
        vcycle_tail(c, 0);
        return;
    }
    if (!c->vgraph_tail) {
        const long long l0 = c->launches;
        CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        vcycle_tail(c, 0);
        cudaGraph_t g = nullptr;
        CK(cudaStreamEndCapture(c->st, &g));
        cudaError_t e = cudaGraphInstantiate(&c->vgraph_tail, g, 0);
        cudaGraphDestroy(g);
        CK(e);
        c->vgraph_tail_kernels = c->launches - l0;
        c->launches = l0;
    }
    CK(cudaGraphLaunch(c->vgraph_tail, c->st));
    c->launches += c->vgraph_tail_kernels;
}

// max over the 64 d_max slots (IEEE bit patterns of non-negative doubles)
double read_max_slots(kf_ctx *c) {
    CK(cudaMemcpyAsync(c->h_max, c->d_max, 64 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->st));
    kerr_fetch(c);
    CK(cudaStreamSynchronize(c->st));
    kerr_check(c);
    unsigned long long m = 0;
    for (int s = 0; s < 64; ++s) m = c->h_max[s] > m ? c->h_max[s] : m;
    double r;
    std::memcpy(&r, &m, sizeof(double));
    return r;
}

// The colour-split copy of c->rho that the finest half sweeps read: made at
// the start of every FAS solve, so it follows whatever wrote c->rho.
void rho_split(kf_ctx *c) {
    if (!c->rho_cs) return;
    const int n = c->n;
    Launch L_(c, KC_RHO, 16. * c->N);
    k_rho_split<<<mg_grid(n / 2, n), mg_block(), 0, c->st>>>(c->rho, c->rho_cs, n);
    CK(cudaGetLastError());
}

// Poisson solve on c->phi with source c->rho.  Returns KF_OK or KF_ERR_NOT_CONVERGED.
int poisson(kf_ctx *c) {
    NvtxRange nv("kf Poisson solve");
    const kf_config &cf = c->cfg;
    c->diag.solves++;
    LevelBuf &L0 = c->lv[0];
    int rc = 0;
    if (cf.poisson_mode == KF_PS_JACOBI_REF || cf.poisson_mode == KF_PS_JACOBI_RES) {
        rc = jacobi_solve(c, L0, c->phi, L0.r, c->rho, cf.nlj_max_it, cf.nlj_limit,
                          cf.poisson_mode == KF_PS_JACOBI_RES, cf.res_tol);
        if (cf.poisson_mode == KF_PS_JACOBI_REF) {
            c->diag.last_residual = max_residual(c, L0, c->phi, c->rho, false);
            rc = 0;  // the reference's plan has no failure on a sweep cap
        }
    } else if (cf.poisson_mode == KF_PS_CASCADIC) {
        // kielflow.cpp:207-217 through solver_poisson_multigrid.cpp:246-418
        const int steps[4] = {0, -1, -1, -1};
        const double tol[4] = {0.01, 0.0005, 0.0001, 0.0001};
        const int n = c->n;
        LevelBuf &L3 = c->lv[3];
        {
            Launch L_(c, KC_TRANSFER, 16. * L3.n * L3.n * L3.n);
            k_inject<<<mg_grid(L3.n, L3.n), mg_block(), 0, c->st>>>(c->phi, n, 8, L3.phi);
        }
        for (int cas = 0; cas < 4; ++cas) {
            const int l = 3 - cas;
            LevelBuf &L = c->lv[l];
            const long Nl = (long)L.n * L.n * L.n;
            if (cas > 0) {
                double *dst = l == 0 ? c->phi : L.phi;
                Launch L_(c, KC_TRANSFER, 9. * Nl);
                k_prolong_set<<<mg_grid(L.n, L.n), mg_block(), 0, c->st>>>(dst, c->lv[l + 1].phi, L.gam, L.n);
            }
            const double *rho_l = c->rho;
            if (l > 0) {
                {
                    Launch L_(c, KC_TRANSFER, 16. * Nl);
                    k_inject<<<mg_grid(L.n, L.n), mg_block(), 0, c->st>>>(c->rho, n, n / L.n, L.rho);
                }
                rho_l = L.rho;
            }
            double *phi_l = l == 0 ? c->phi : L.phi;
            jacobi_solve(c, L, phi_l, L.r, rho_l, steps[cas], tol[cas], false, 0.);
        }
        c->diag.last_residual = max_residual(c, L0, c->phi, c->rho, false);
        rc = 0;
    } else if (!(cf.res_tol > 0.)) {
        // fixed number of V-cycles: the result is a smooth function of rho
        // and of the initial guess (no data-dependent stopping)
        rho_split(c);
        for (int cyc = 0; cyc < cf.max_cycles; ++cyc) run_vcycle(c);
        const double r = max_residual(c, L0, c->phi, c->rho, true);
        c->diag.last_iterations = cf.max_cycles;
        c->diag.total_iterations += cf.max_cycles;
        c->diag.stage_cycles[c->stage_idx & 3] += cf.max_cycles;
        c->diag.last_residual = r;
        if (r != r) throw KfError{KF_ERR_NAN, "NaN in the multigrid solve"};
    } else if (c->lv.size() > 1) {
        // test after each cycle's pre-smoothing on the residual the cycle
        // computes anyway; the rest of the cycle only when it fails
        rho_split(c);
        double r = 0.;
        int cyc = 0;
        for (;;) {
            vcycle_head(c, 0, true);
            CK(cudaGetLastError());
            r = read_max_slots(c);
            if (!(r > cf.res_tol) || cyc >= cf.max_cycles) break;
            run_vcycle_tail(c);
            ++cyc;
        }
        c->diag.last_iterations = cyc;
        c->diag.stage_cycles[c->stage_idx & 3] += cyc;
        c->diag.total_iterations += cyc;
        c->diag.last_residual = r;
        if (r != r) throw KfError{KF_ERR_NAN, "NaN in the multigrid solve"};
        if (r > cf.res_tol) {
            c->diag.not_converged++;
            rc = 1;
        }
    } else {
        rho_split(c);
        double r = max_residual(c, L0, c->phi, c->rho, true);
        int cyc = 0;
        while (r > cf.res_tol && cyc < cf.max_cycles) {
            run_vcycle(c);
            ++cyc;
            r = max_residual(c, L0, c->phi, c->rho, true);
        }
        c->diag.last_iterations = cyc;
        c->diag.stage_cycles[c->stage_idx & 3] += cyc;
        c->diag.total_iterations += cyc;
        c->diag.last_residual = r;
        if (r != r) throw KfError{KF_ERR_NAN, "NaN in the multigrid solve"};
        if (r > cf.res_tol) {
            c->diag.not_converged++;
            rc = 1;
        }
    }
    if (c->diag.last_residual != c->diag.last_residual) throw KfError{KF_ERR_NAN, "NaN in phi"};
    return rc;
}

// Start of a solve at time t_stage: linear extrapolation of the last two
// solutions at distinct times (returns whether t_stage is a new time).
bool phi_guess(kf_ctx *c) {
    const double t = c->t_stage;
    const bool newtime = c->nhist == 0 || t != c->tau_b;
    if (!c->cfg.phi_extrap || !newtime || c->nhist == 0) return newtime;
    if (c->nhist >= 2) {
        const double w = (t - c->tau_b) / (c->tau_b - c->tau_a);
        Launch L_(c, KC_MISC, 24. * c->N);
        k_extrap<<<nblk(c->N, 256), 256, 0, c->st>>>(c->phi, c->phi_a, w, c->N);
    } else {
        CK(cudaMemcpyAsync(c->phi_a, c->phi, 8 * c->N, cudaMemcpyDeviceToDevice, c->st));
    }
    c->tau_a = c->tau_b;
    return newtime;
}

// The stage's Poisson solve inside the capture of a step graph: device-side
// warm start, then the FAS loop as a conditional WHILE node whose body (one
// V-cycle + the max-residual test) is captured on st_body.
void poisson_captured(kf_ctx *c) {
    const kf_config &cf = c->cfg;
    const bool extrap = cf.phi_extrap != 0;
    if (extrap) {
        Launch L_(c, KC_MISC, 24. * c->N);
        k_guess<<<nblk(c->N, 256), 256, 0, c->st>>>(c->phi, c->phi_a, c->dtime, c->N);
    }
    if (extrap) {
        Launch L_(c, KC_MISC, 0.);
        k_guess_post<<<1, 32, 0, c->st>>>(c->dtime);
    }
    LevelBuf &L0 = c->lv[0];
    const bool fixed = !(cf.res_tol > 0.);
    rho_split(c);
    c->head_kernels = 0;
    if (!fixed && c->lv.size() > 1) {
        // WHILE { head of the cycle (pre-smoothing, residual with its max);
        //         k_fas_check_mid;  IF { rest of the cycle } }
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, nullptr, nullptr));
        cudaGraphConditionalHandle hw, hi;
        CK(cudaGraphConditionalHandleCreate(&hw, g, 0, 0));
        CK(cudaGraphConditionalHandleCreate(&hi, g, 0, 0));
        {
            Launch L_(c, KC_MISC, 0.);
            k_fas_begin<<<1, 32, 0, c->st>>>(c->dpois, hw);
        }
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &ndeps));
        cudaGraphNodeParams wp = {cudaGraphNodeTypeConditional};
        wp.conditional.handle = hw;
        wp.conditional.type = cudaGraphCondTypeWhile;
        wp.conditional.size = 1;
        cudaGraphNode_t wnode;
        CK(cudaGraphAddNode(&wnode, g, deps, ndeps, &wp));
        CK(cudaStreamUpdateCaptureDependencies(c->st, &wnode, 1, cudaStreamSetCaptureDependencies));
        cudaGraph_t body = wp.conditional.phGraph_out[0];
        const long long l0 = c->launches;
        cudaStream_t outer = c->st;
        c->st = c->st_body;
        cudaError_t e = cudaStreamBeginCaptureToGraph(c->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            try {
                vcycle_head(c, 0, true);
                {
                    Launch L_(c, KC_MISC, 0.);
                    k_fas_check_mid<<<1, 32, 0, c->st>>>(c->d_max, c->dpois, cf.res_tol, cf.max_cycles, c->stage_idx,
                                                         hw, hi);
                }
                c->head_kernels = c->launches - l0;
                cudaGraph_t gb = nullptr;
                CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &gb, &deps, &ndeps));
                cudaGraphNodeParams ip = {cudaGraphNodeTypeConditional};
                ip.conditional.handle = hi;
                ip.conditional.type = cudaGraphCondTypeIf;
                ip.conditional.size = 1;
                cudaGraphNode_t inode;
                CK(cudaGraphAddNode(&inode, gb, deps, ndeps, &ip));
                CK(cudaStreamUpdateCaptureDependencies(c->st, &inode, 1, cudaStreamSetCaptureDependencies));
                cudaGraph_t body_out = nullptr;
                CK(cudaStreamEndCapture(c->st, &body_out));
                CK(cudaStreamBeginCaptureToGraph(c->st, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeThreadLocal));
                vcycle_tail(c, 0);
                e = cudaStreamEndCapture(c->st, &body_out);
            } catch (...) {
                cudaGraph_t junk = nullptr;
                cudaStreamEndCapture(c->st, &junk);
                c->st = outer;
                throw;
            }
        }
        c->st = outer;
        CK(e);
        c->cycle_kernels = c->launches - l0;
        if (extrap) {
            Launch L_(c, KC_MISC, 0.);
            k_hist_post<<<1, 32, 0, c->st>>>(c->dtime);
        }
        CK(cudaGetLastError());
        return;
    }
    auto resmax = [&](cudaStream_t st) {
        CK(cudaMemsetAsync(c->d_max, 0, 64 * sizeof(unsigned long long), st));
        Launch L_(c, KC_RESID, 16. * c->N);
        dim3 g = mg_grid(L0.n, L0.n);
        g.z = L0.n < 16 ? L0.n : 16;
        if (col_level(L0.n))
            k_residual_col<8, COL_PI, true, false, false>
                <<<dim3(L0.n / 64, L0.n / 8, L0.n / COL_PI), mg_block(), 0, st>>>(c->phi, c->rho, L0.lev(), nullptr,
                                                                                  c->d_max);
        else
            k_resmax<true><<<g, mg_block(), 0, st>>>(c->phi, c->rho, L0.lev(), c->d_max);
    };
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, nullptr, nullptr));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    resmax(c->st);
    {
        Launch L_(c, KC_MISC, 0.);
        k_fas_check<<<1, 32, 0, c->st>>>(c->d_max, c->dpois, cf.res_tol, cf.max_cycles, 1, fixed, c->stage_idx, h);
    }
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &ndeps));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
    CK(cudaStreamUpdateCaptureDependencies(c->st, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const long long l0 = c->launches;
    cudaStream_t outer = c->st;
    c->st = c->st_body;
    CK(cudaStreamBeginCaptureToGraph(c->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    vcycle(c, 0);
    resmax(c->st);
    {
        Launch L_(c, KC_MISC, 0.);
        k_fas_check<<<1, 32, 0, c->st>>>(c->d_max, c->dpois, cf.res_tol, cf.max_cycles, 0, fixed, c->stage_idx, h);
    }
    cudaGraph_t body_out = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->st, &body_out);
    c->st = outer;
    CK(e);
    c->cycle_kernels = c->launches - l0;
    if (extrap) {
        Launch L_(c, KC_MISC, 0.);
        k_hist_post<<<1, 32, 0, c->st>>>(c->dtime);
    }
    CK(cudaGetLastError());
}

// ------------------------------------------------------------------ per-(T, N) implementation
template <typename T, int N> struct Impl {
    typedef typename C2<T>::type T2;
    static constexpr int TC = Tile<T>::TC, LZ = ZTile<T>::LZ, NZC = N / 2 + 1;
    template <int V> static constexpr int PV = PlanV<N, V>::P;

    static Geo<T> geo(kf_ctx *c) {
        return Geo<T>{c->n, c->nzc, (const T *)c->kv, c->q2, dealias_threshold(), c->pb};
    }

    static void set_attrs() {
        static bool done = false;
        if (done) return;
        const int big = 200 * 1024;
        CK(cudaFuncSetAttribute(k_axis_pass<T, N, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        CK(cudaFuncSetAttribute(k_axis_pass<T, N, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        set_attrs_v<0>(big);
        set_attrs_v<1>(big);
        done = true;
    }

    template <int V> static void set_attrs_v(int big) {
        CK(cudaFuncSetAttribute(k_axis_pipe<T, N, -1, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        CK(cudaFuncSetAttribute(k_axis_pipe<T, N, +1, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        CK(cudaFuncSetAttribute(k_z_c2r<T, N, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        CK(cudaFuncSetAttribute(k_z_r2c<T, N, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        CK(cudaFuncSetAttribute(k_xfwd_assemble<T, N, V, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        CK(cudaFuncSetAttribute(k_xfwd_assemble<T, N, V, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    }

    static double job_bytes(kf_ctx *c, int off, int njobs) {
        std::vector<const void *> u;
        for (int j = 0; j < njobs; ++j) {
            const void *p = c->hj[off + j].in;
            bool seen = false;
            for (auto q : u) seen |= q == p;
            if (!seen) u.push_back(p);
        }
        return (double)(u.size() + njobs) * c->Nc * sizeof(T2);
    }
    // resident blocks per SM x SMs of the pipelined pass (its grid)
    template <int V> static int pipe_grid(int sign) {
        static int g[2] = {0, 0};
        int &v = g[sign > 0];
        if (!v) {
            int dev = 0, sms = 0, per = 0;
            CK(cudaGetDevice(&dev));
            CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            const size_t smem = axis_pipe_smem<T, N>(32);
            if (sign < 0)
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_axis_pipe<T, N, -1, V>, TC * PV<V>, smem));
            else
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_axis_pipe<T, N, +1, V>, TC * PV<V>, smem));
            v = (per > 0 ? per : 1) * sms;
        }
        return v;
    }
    template <int V> static void axis_v(kf_ctx *c, int off, int njobs, int ax, int sign) {
        const int ntiles = ax == 0 ? (N * NZC + TC - 1) / TC : N * ((NZC + TC - 1) / TC);
        const int total = njobs * ntiles, grid = std::min(total, pipe_grid<V>(sign));
        const size_t smem = axis_pipe_smem<T, N>(njobs);
        if (sign < 0)
            k_axis_pipe<T, N, -1, V><<<grid, TC * PV<V>, smem, c->st>>>(c->dj + off, njobs, ax, geo(c),
                                                                      (const T2 *)c->tw, total);
        else
            k_axis_pipe<T, N, +1, V><<<grid, TC * PV<V>, smem, c->st>>>(c->dj + off, njobs, ax, geo(c),
                                                                      (const T2 *)c->tw, total);
    }
    static void axis(kf_ctx *c, int off, int njobs, int ax, int sign) {
        Launch L_(c, sign > 0 ? KC_AXIS_INV : KC_AXIS_FWD, job_bytes(c, off, njobs));
        if (c->fftv)
            axis_v<1>(c, off, njobs, ax, sign);
        else
            axis_v<0>(c, off, njobs, ax, sign);
    }
    static double z_bytes(kf_ctx *c, int off, int njobs, bool c2r) {
        std::vector<const void *> u;
        int outs = 0;
        for (int j = 0; j < njobs; ++j) {
            const ZJob &z = c->hz[off + j];
            for (const void *p : {z.inA, z.inB}) {
                if (!p) continue;
                bool seen = false;
                for (auto q : u) seen |= q == p;
                if (!seen) u.push_back(p);
            }
            outs += (z.outA ? 1 : 0) + (z.outB ? 1 : 0);
        }
        const double cb = (double)c->Nc * sizeof(T2), rb = (double)c->N * sizeof(T);
        return c2r ? u.size() * cb + outs * rb : u.size() * rb + outs * cb;
    }
    // scale < 0: the 1/N of c2r; otherwise the given factor (1 for transposes)
    static void zc2r(kf_ctx *c, int off, int njobs, double scale = -1.) {
        const int nrows = N * N;
        const int ntiles = (nrows + LZ - 1) / LZ;
        const size_t smem = ZSmem<T, N, true>::bytes;
        Launch L_(c, KC_Z_C2R, z_bytes(c, off, njobs, true));
        const T sc = (T)(scale < 0. ? 1. / ((double)N * N * N) : scale);
        if (c->fftv)
            k_z_c2r<T, N, 1><<<njobs * ntiles, LZ * PV<1>, smem, c->st>>>(c->dz + off, njobs, nrows, geo(c),
                                                                        (const T2 *)c->tw, sc);
        else
            k_z_c2r<T, N, 0><<<njobs * ntiles, LZ * PV<0>, smem, c->st>>>(c->dz + off, njobs, nrows, geo(c),
                                                                        (const T2 *)c->tw, sc);
    }
    static void zr2c(kf_ctx *c, int off, int njobs) {
        const int nrows = N * N;
        const int ntiles = (nrows + LZ - 1) / LZ;
        const size_t smem = ZSmem<T, N, false>::bytes;
        Launch L_(c, KC_Z_R2C, z_bytes(c, off, njobs, false));
        if (c->fftv)
            k_z_r2c<T, N, 1><<<njobs * ntiles, LZ * PV<1>, smem, c->st>>>(c->dz + off, njobs, nrows, (const T2 *)c->tw);
        else
            k_z_r2c<T, N, 0><<<njobs * ntiles, LZ * PV<0>, smem, c->st>>>(c->dz + off, njobs, nrows, (const T2 *)c->tw);
    }
    static RhsArgs<T> rargs(kf_ctx *c) {
        RhsArgs<T> a;
        for (int q = 0; q < 4; ++q) a.Y[q] = (const T2 *)c->Ys[q];
        a.phihat = (const T2 *)c->phihat;
        a.SV = (const T *)c->SV;
        a.PF = (const T *)c->PF;
        a.tau = (T)c->cfg.tau;
        a.theta = (T)c->cfg.theta;
        a.M = (T)c->cfg.M;
        a.D = (T)c->cfg.diff_D;
        a.terms = c->cfg.terms;
        return a;
    }

    // rounds A (P s, d_x s, d_y s and s_d = c2r(P s)), the Poisson solve and
    // B (phi^ = r2c(phi)), shared by both right-hand sides
    // Round D's jobs on u' and s (the first 6 x, 9 y and 8 z jobs of its
    // lists): every input is the stage state or round A's output.
    static void round_D_us(kf_ctx *c) {
        axis(c, c->jD_x, 6, 0, +1);
        axis(c, c->jD_y, 9, 1, +1);
        zc2r(c, c->zD, 8);
    }

    // In a captured step, fork round_D_us onto st_side after round A; rhs
    // joins it before the products.  The branch writes CX[2..7], CY[3..11]
    // and R[1..15], which nothing between the fork and the join touches (the
    // Poisson solve, round B in CX[8] / CY[12], k_lin, round D's LIN part).
    // (Measured at 256^3 FP32 bulk: +1 to +2.4 % per step; the Poisson chain
    // at a higher stream priority than the branch was slower than equal
    // priorities, and the branch's transform passes on half the persistent
    // grid were no faster.)
    static bool fork_D(kf_ctx *c) {
        if (!(c->capturing && c->overlap_d)) return false;
        CK(cudaEventRecord(c->ev_fork, c->st));
        CK(cudaStreamWaitEvent(c->st_side, c->ev_fork, 0));
        if (c->capture_wait_u && c->stage_idx == 0)
            CK(cudaStreamWaitEvent(c->st_side, c->ev_u, cudaEventWaitExternal));
        cudaStream_t main = c->st;
        c->st = c->st_side;
        try {
            round_D_us(c);
        } catch (...) {
            c->st = main;
            throw;
        }
        c->st = main;
        CK(cudaEventRecord(c->ev_join, c->st_side));
        return true;
    }

    static bool rounds_AB(kf_ctx *c, bool fork = false) {
        const int Tm = c->cfg.terms;
        const bool pen = Tm & T_PENALIZATION;
        const bool pois = (Tm & T_POISSON) && (Tm & T_E_INT);
        // A
        axis(c, c->jA_x, 2, 0, +1);
        axis(c, c->jA_y, 3, 1, +1);
        if (pois || pen) zc2r(c, c->zA, 1);
        const bool forked = fork && fork_D(c);
        if (pois && !c->phi_given) {
            {
                Launch L_(c, KC_RHO, (double)c->N * (sizeof(T) + 16));
                k_rho<T><<<nblk(c->N, 256), 256, 0, c->st>>>((const T *)c->R[0], c->nd, c->rho, c->N);
            }
            CK(cudaGetLastError());
            if (c->capturing) {
                poisson_captured(c);
            } else {
                const bool newtime = phi_guess(c);
                int rc = poisson(c);
                if (rc) throw KfError{KF_ERR_NOT_CONVERGED, "Poisson solve did not reach its tolerance"};
                if (c->cfg.phi_extrap && newtime) {
                    c->nhist = c->nhist < 2 ? c->nhist + 1 : 2;
                    c->tau_b = c->t_stage;
                }
            }
        }
        // B
        if (c->capturing && c->capture_wait_u && c->stage_idx == 0)
            CK(cudaStreamWaitEvent(c->st, c->ev_u, cudaEventWaitExternal));
        if (Tm & T_E_INT) {
            if (c->fp32) {
                Launch L_(c, KC_MISC, (double)c->N * (8 + sizeof(T)));
                k_from_f64<T><<<nblk(c->N, 256), 256, 0, c->st>>>((T *)c->phiT, c->phi, c->N);
            }
            zr2c(c, c->zB, 1);
            axis(c, c->jB_y, 1, 1, -1);
            axis(c, c->jB_x, 1, 0, -1);
        }
        return forked;
    }

    // one right-hand-side evaluation: Ys -> K
    static void rhs(kf_ctx *c) {
        const int Tm = c->cfg.terms;
        const bool pen = Tm & T_PENALIZATION;
        const bool forked = rounds_AB(c, true);
        // C
        if (pen) {
            Launch L_(c, KC_LIN, (double)c->Nc * (9 * sizeof(T2) + 2 * sizeof(T)));
            k_lin<T><<<mg_grid(NZC, N), mg_block(), 0, c->st>>>(rargs(c), geo(c), (T2 *)c->LIN[0], (T2 *)c->LIN[1],
                                                               (T2 *)c->LIN[2], (T2 *)c->LIN[3]);
        }
        // D: the u', s part (unless forked) and the linear terms' part
        if (!forked) {
            axis(c, c->jD_x, pen ? 10 : 6, 0, +1);
            axis(c, c->jD_y, pen ? 13 : 9, 1, +1);
            zc2r(c, c->zD, pen ? 10 : 8);
        } else {
            if (pen) {
                axis(c, c->jD_x + 6, 4, 0, +1);
                axis(c, c->jD_y + 9, 4, 1, +1);
                zc2r(c, c->zD + 8, 2);
            }
            CK(cudaStreamWaitEvent(c->st, c->ev_join, 0));
        }
        // E
        ProdArgs<T> pa;
        for (int q = 0; q < 3; ++q) {
            pa.U[q] = (const T *)c->R[1 + q];
            pa.ds[q] = (const T *)c->R[13 + q];
            for (int d = 0; d < 3; ++d) pa.dU[q][d] = (const T *)c->R[4 + 3 * q + d];
        }
        for (int q = 0; q < 4; ++q) {
            pa.rl[q] = (const T *)c->R[16 + q];
            pa.out[q] = (T *)c->R[20 + q];
        }
        pa.sd = (const T *)c->R[0];
        pa.H = (const T *)c->H;
        pa.M = (T)c->cfg.M;
        pa.eta = (T)c->cfg.pen_eta;
        pa.terms = Tm;
        pa.N = c->N;
        {
            Launch L_(c, KC_PROD, (double)c->N * sizeof(T) * (19 + (pen ? 6 : 0)));
            k_products<T><<<nblk(c->N, 256), 256, 0, c->st>>>(pa);
        }
        // F
        zr2c(c, c->zF, 2);
        axis(c, c->jF_y, 4, 1, -1);
        const int ntiles = (N * NZC + TC - 1) / TC;
        {
            const double cb = (double)c->Nc * sizeof(T2), rb = (double)c->Nc * sizeof(T);
            Launch L_(c, KC_XASM, pen ? 8 * cb : 8 * cb + 4 * cb + ((Tm & T_E_INT) ? cb : 0.) + 2 * rb);
            const size_t sm = (size_t)N * TC * sizeof(T2);
            const AxisJob *j = c->dj + c->jF_x;
            if (c->fftv && pen)
                k_xfwd_assemble<T, N, 1, true><<<ntiles, TC * PV<1>, sm, c->st>>>(j, geo(c), rargs(c), (const T2 *)c->tw);
            else if (c->fftv)
                k_xfwd_assemble<T, N, 1, false><<<ntiles, TC * PV<1>, sm, c->st>>>(j, geo(c), rargs(c), (const T2 *)c->tw);
            else if (pen)
                k_xfwd_assemble<T, N, 0, true><<<ntiles, TC * PV<0>, sm, c->st>>>(j, geo(c), rargs(c), (const T2 *)c->tw);
            else
                k_xfwd_assemble<T, N, 0, false><<<ntiles, TC * PV<0>, sm, c->st>>>(j, geo(c), rargs(c), (const T2 *)c->tw);
        }
        CK(cudaGetLastError());
    }

    // The right-hand side on sine-stretched axes: every derivative takes the
    // chain-rule path D_d F = r2c(m_d c2r(P i k_d F)) of
    // OP_partial_derivative.cpp:104-136, so the derivative terms that
    // rhs() folds into k-space become transform pairs:
    //   C' linear parts, F1                 D' raw derivatives (15 c2r)
    //   E' times the metric                 F' their r2c (15)
    //   G' c2r(P D_d u'_c), c2r(P D_d s)    H' products (rhs_standard.cpp:323-436)
    //   I' r2c of the products              J' assembly
    //   K' penalization of the finished right-hand side, then the 2/3 filter
    static void rhs_stretched(kf_ctx *c) {
        const int Tm = c->cfg.terms;
        const bool pen = Tm & T_PENALIZATION;
        const long Nc = c->Nc, Nr = c->N;
        const double cb = (double)Nc * sizeof(T2), rb = (double)Nr * sizeof(T);
        rounds_AB(c);
        {  // C'
            Launch L_(c, KC_LIN, 4 * cb + 6 * cb + 2 * rb);
            k_sl_lin<T><<<nblk(Nc, 256), 256, 0, c->st>>>(rargs(c), geo(c), (T2 *)c->LIN[0], (T2 *)c->LIN[1],
                                                            (T2 *)c->LIN[2], (T2 *)c->LIN[3], (T2 *)c->CX[10]);
        }
        // D'
        axis(c, c->jS_Dx, 8, 0, +1);
        axis(c, c->jS_Dy, 12, 1, +1);
        zc2r(c, c->zS_D, 10);
        {  // E'
            ScaleArgs<T> sa;
            for (int j = 0; j < 15; ++j) sa.f[j] = (T *)c->R[4 + j];
            sa.met = (const T *)c->met;
            sa.n = c->n;
            sa.N = Nr;
            Launch L_(c, KC_PROD, 30. * rb);
            k_sl_scale<T><<<nblk(Nr, 256), 256, 0, c->st>>>(sa);
        }
        // F'
        zr2c(c, c->zS_F, 8);
        axis(c, c->jS_Fy, 15, 1, -1);
        axis(c, c->jS_Fx, 15, 0, -1);
        const bool prod = Tm & (T_ADVECTION | T_CONTINUITY);
        if (prod) {
            // G'
            axis(c, c->jS_Gx, 12, 0, +1);
            axis(c, c->jS_Gy, 12, 1, +1);
            zc2r(c, c->zS_G, 6);
            {  // H'
                ProdArgs<T> pa{};
                for (int q = 0; q < 3; ++q) {
                    pa.U[q] = (const T *)c->R[1 + q];
                    pa.ds[q] = (const T *)c->R[13 + q];
                    for (int d = 0; d < 3; ++d) pa.dU[q][d] = (const T *)c->R[4 + 3 * q + d];
                }
                for (int q = 0; q < 4; ++q) pa.out[q] = (T *)c->R[20 + q];
                pa.M = (T)c->cfg.M;
                pa.terms = Tm & (T_ADVECTION | T_CONTINUITY);
                pa.N = Nr;
                Launch L_(c, KC_PROD, 19. * rb);
                k_products<T><<<nblk(Nr, 256), 256, 0, c->st>>>(pa);
            }
            // I'
            zr2c(c, c->zS_I, 2);
            axis(c, c->jS_Iy, 4, 1, -1);
            axis(c, c->jS_Ix, 4, 0, -1);
        }
        {  // J'
            AsmArgs<T> aa;
            for (int q = 0; q < 4; ++q) {
                aa.lin[q] = (const T2 *)c->LIN[q];
                aa.pr[q] = prod ? (const T2 *)c->SX[8 + q] : nullptr;
                aa.K[q] = (T2 *)c->K[q];
            }
            for (int j = 0; j < 15; ++j) aa.dn[j] = (const T2 *)c->CY[j];
            aa.M = (T)c->cfg.M;
            aa.terms = Tm;
            aa.Nc = Nc;
            Launch L_(c, KC_XASM, 27 * cb);
            k_sl_assemble<T><<<nblk(Nc, 256), 256, 0, c->st>>>(aa);
        }
        if (pen) {  // K'
            axis(c, c->jS_Kx, 4, 0, +1);
            axis(c, c->jS_Ky, 4, 1, +1);
            zc2r(c, c->zS_K, 2);
            {
                ProdArgs<T> pa{};
                for (int q = 0; q < 3; ++q) pa.U[q] = (const T *)c->R[1 + q];
                for (int q = 0; q < 4; ++q) {
                    pa.rl[q] = (const T *)c->R[20 + q];
                    pa.out[q] = (T *)c->R[20 + q];
                }
                pa.sd = (const T *)c->R[0];
                pa.H = (const T *)c->H;
                pa.M = (T)c->cfg.M;
                pa.eta = (T)c->cfg.pen_eta;
                pa.terms = T_PENALIZATION;
                pa.N = Nr;
                Launch L_(c, KC_PROD, 13. * rb);
                k_products<T><<<nblk(Nr, 256), 256, 0, c->st>>>(pa);
            }
            zr2c(c, c->zS_Kf, 2);
            axis(c, c->jS_Kfy, 4, 1, -1);
            axis(c, c->jS_Kfx, 4, 0, -1);
            Launch L_(c, KC_MISC, 8 * cb);
            k_sl_dealias4<T><<<nblk(Nc, 256), 256, 0, c->st>>>(geo(c), (T2 *)c->K[0], (T2 *)c->K[1],
                                                                 (T2 *)c->K[2], (T2 *)c->K[3]);
        }
        CK(cudaGetLastError());
    }

    // standalone transforms on R[0] <-> CX[0] (through CY[0])
    static void r2c(kf_ctx *c) {
        zr2c(c, c->zT, 1);
        axis(c, c->jTf_y, 1, 1, -1);
        axis(c, c->jTf_x, 1, 0, -1);
        CK(cudaGetLastError());
    }
    static void c2r(kf_ctx *c) {
        axis(c, c->jT_x, 1, 0, +1);
        axis(c, c->jT_y, 1, 1, +1);
        zc2r(c, c->zT + 1, 1);
        CK(cudaGetLastError());
    }
    // transform passes of the discrete adjoint (job lists of build_adj_jobs)
    static void adj_pass(kf_ctx *c, int which) {
        switch (which) {
            case 0:  // forward intermediates s_d, U_c, d_d U_c, d_d s of the stage input in Ys
                axis(c, c->jA_x, 2, 0, +1);
                axis(c, c->jA_y, 3, 1, +1);
                zc2r(c, c->zA, 1);
                axis(c, c->jD_x, 6, 0, +1);
                axis(c, c->jD_y, 9, 1, +1);
                zc2r(c, c->zD, 8);
                break;
            case 1:  // f_bar = r2c^T(P Kbar) = c2r_unscaled(P Kbar / w)
                axis(c, c->jV_x, 4, 0, +1);
                axis(c, c->jV_y, 4, 1, +1);
                zc2r(c, c->zV, 2, 1.);
                break;
            case 2:  // r2c of the physical cotangents
                zr2c(c, c->zW, c->nWz);
                axis(c, c->jW_y, c->nWf, 1, -1);
                axis(c, c->jW_x, c->nWf, 0, -1);
                break;
            case 3:  // phi_bar = r2c^T(phihat_bar)
                axis(c, c->jP_x, 1, 0, +1);
                axis(c, c->jP_y, 1, 1, +1);
                zc2r(c, c->zP, 1, 1.);
                break;
            case 4:  // r2c of s_d_bar
                zr2c(c, c->zS, 1);
                axis(c, c->jS_y, 1, 1, -1);
                axis(c, c->jS_x, 1, 0, -1);
                break;
            case 5:  // r2c^T of the s cotangent, and c2r of the state's s
                axis(c, c->jQ_x, 2, 0, +1);
                axis(c, c->jQ_y, 2, 1, +1);
                zc2r(c, c->zQ, 1, 1.);
                zc2r(c, c->zQ + 1, 1);
                break;
            case 6:  // s_d only (the Poisson source of the state in Ys)
                axis(c, c->jA_x, 2, 0, +1);
                axis(c, c->jA_y, 3, 1, +1);
                zc2r(c, c->zA, 1);
                break;
        }
        CK(cudaGetLastError());
    }
    // inverse transforms of the (undealiased) state into R[20..23] for diagnostics
    static void inv_state(kf_ctx *c) {
        axis(c, c->jG_x, 4, 0, +1);
        axis(c, c->jG_y, 4, 1, +1);
        zc2r(c, c->zG, 2);
        CK(cudaGetLastError());
    }
};

template <typename T> struct Dispatch {
    static bool pick(kf_ctx *c) {
        switch (c->n) {
#define KF_CASE(NN)                                    \
    case NN:                                           \
        Impl<T, NN>::set_attrs();                      \
        c->rhs_fn = c->stretched ? &Impl<T, NN>::rhs_stretched : &Impl<T, NN>::rhs; \
        c->r2c_fn = &Impl<T, NN>::r2c;                 \
        c->c2r_fn = &Impl<T, NN>::c2r;                 \
        c->inv_state_fn = &Impl<T, NN>::inv_state;     \
        c->adj_fn = &Impl<T, NN>::adj_pass;            \
        return true;
            KF_CASE(16)
            KF_CASE(32)
            KF_CASE(64)
            KF_CASE(96)
            KF_CASE(128)
            KF_CASE(256)
#undef KF_CASE
            default:
                return false;
        }
    }
};

// radix stages and threads per line of the two transform plans of length n
template <int NN> void plan_info_n(int rad[2][4], int thr[2]) {
    for (int i = 0; i < 4; ++i) {
        rad[0][i] = PlanV<NN, 0>::radix[i];
        rad[1][i] = PlanV<NN, 1>::radix[i];
    }
    thr[0] = PlanV<NN, 0>::P;
    thr[1] = PlanV<NN, 1>::P;
}
void plan_info(int n, int rad[2][4], int thr[2]) {
    switch (n) {
        case 16: plan_info_n<16>(rad, thr); break;
        case 32: plan_info_n<32>(rad, thr); break;
        case 64: plan_info_n<64>(rad, thr); break;
        case 96: plan_info_n<96>(rad, thr); break;
        case 128: plan_info_n<128>(rad, thr); break;
        case 256: plan_info_n<256>(rad, thr); break;
        default: break;
    }
}

// FP64 sums of the charge density e^s - e^phi + n_d and the kinetic energy
// density 0.5 e^s |M e_x + u'|^2 (block partials in slots 0 and 1).
template <typename T>
__global__ void __launch_bounds__(RBS) k_diag_sums(const T *__restrict__ s, const T *__restrict__ ux,
                                                   const T *__restrict__ uy, const T *__restrict__ uz,
                                                   const double *__restrict__ phi, const double *__restrict__ nd,
                                                   double M, long N, double *__restrict__ partial,
                                                   const double *__restrict__ vol, int n) {
    __shared__ double sh[2 * RBS];
    double ch = 0., kin = 0.;
    for (long i = (long)blockIdx.x * RBS + threadIdx.x; i < N; i += (long)gridDim.x * RBS) {
        // cell volume / h^3: 1, or dS(x) dS(y) dS(z) on stretched axes
        double w = 1.;
        if (vol) w = vol[i / ((long)n * n)] * vol[(i / n) % n] * vol[i % n];
        const double n_i = exp((double)s[i]);
        ch += w * (n_i - exp(phi[i]) + nd[i]);
        const double vx = M + (double)ux[i], vy = (double)uy[i], vz = (double)uz[i];
        kin += w * (0.5 * n_i * (vx * vx + vy * vy + vz * vz));
    }
    sh[threadIdx.x] = kin;
    sh[RBS + threadIdx.x] = ch;
    __syncthreads();
    for (int w = RBS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sh[threadIdx.x] += sh[threadIdx.x + w];
            sh[RBS + threadIdx.x] += sh[RBS + threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[(long)blockIdx.x * KF_RED + 0] = sh[0];
        partial[(long)blockIdx.x * KF_RED + 1] = sh[RBS];
    }
}

__global__ void k_diag_final(const double *__restrict__ partial, int nb, double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double a = 0., b = 0.;
        for (int i = 0; i < nb; ++i) {
            a += partial[(long)i * KF_RED + 0];
            b += partial[(long)i * KF_RED + 1];
        }
        out[0] = a;
        out[1] = b;
    }
}

void build_tables(kf_ctx *c) {
    const int n = c->n, nzc = c->nzc;
    const double L = c->cfg.L;
    std::vector<double> kv(n), q2(n);
    const double kmax = k_val_at(n / 2, n, L);
    const double kzq = k_val_at(nzc / 2, n, L);  // operations.hpp:25 quirk: field_imag::Nz = n/2+1
    for (int i = 0; i < n; ++i) {
        kv[i] = k_val_at(i, n, L);
        q2[i] = pow(kv[i] / kmax, 2.);
    }
    std::vector<double> SV(c->Nc), PF(c->Nc);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < nzc; ++k) {
                const size_t ijk = (size_t)k + nzc * ((size_t)j + (size_t)i * n);
                const double kx = kv[i], ky = kv[j], kz = kv[k];
                // rhs_standard.cpp:64-71 (field_SV), optional cut at sv_cut
                const double knorm = sqrt(pow(kx / kmax, 2.) + pow(ky / kmax, 2.) + pow(kz / kmax, 2.));
                const double filter = 1. - exp(-8. * pow(sqrt(knorm), 8.));
                double svv = c->cfg.sv_eps * filter;
                if (c->cfg.sv_cut > 0. && !(knorm > c->cfg.sv_cut)) svv = 0.;
                SV[ijk] = svv;
                // operations.hpp:35-40 with the filter of rhs_standard.cpp:220
                const double kq = sqrt(pow(kx / kmax, 2.) + pow(ky / kmax, 2.) + pow(kz / kzq, 2.));
                PF[ijk] = exp(-2000. * pow(kq, 15.));
            }
    // twiddles W_N^m = exp(-2 pi i m / N), long double
    std::vector<double> tw(2 * n);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < n; ++m) {
        long double a = twopi * (long double)m / (long double)n;
        tw[2 * m] = (double)cosl(a);
        tw[2 * m + 1] = (double)(-sinl(a));
    }
    c->q2 = dalloc<double>(c, sizeof(double) * n);
    CK(cudaMemcpy(c->q2, q2.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    {
        const std::vector<int> pb = dealias_bounds(q2, n, dealias_threshold());
        c->pb = dalloc<int>(c, sizeof(int) * pb.size());
        CK(cudaMemcpy(c->pb, pb.data(), sizeof(int) * pb.size(), cudaMemcpyHostToDevice));
    }
    if (c->fp32) {
        std::vector<float> kvf(n), SVf(c->Nc), PFf(c->Nc), twf(2 * n);
        for (int i = 0; i < n; ++i) kvf[i] = (float)kv[i];
        for (long i = 0; i < c->Nc; ++i) { SVf[i] = (float)SV[i]; PFf[i] = (float)PF[i]; }
        for (int i = 0; i < 2 * n; ++i) twf[i] = (float)tw[i];
        c->kv = dalloc<void>(c, 4 * n);
        c->SV = dalloc<void>(c, 4 * c->Nc);
        c->PF = dalloc<void>(c, 4 * c->Nc);
        c->tw = dalloc<void>(c, 8 * n);
        CK(cudaMemcpy(c->kv, kvf.data(), 4 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c->SV, SVf.data(), 4 * c->Nc, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c->PF, PFf.data(), 4 * c->Nc, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c->tw, twf.data(), 8 * n, cudaMemcpyHostToDevice));
    } else {
        c->kv = dalloc<void>(c, 8 * n);
        c->SV = dalloc<void>(c, 8 * c->Nc);
        c->PF = dalloc<void>(c, 8 * c->Nc);
        c->tw = dalloc<void>(c, 16 * n);
        CK(cudaMemcpy(c->kv, kv.data(), 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c->SV, SV.data(), 8 * c->Nc, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c->PF, PF.data(), 8 * c->Nc, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c->tw, tw.data(), 16 * n, cudaMemcpyHostToDevice));
    }
    if (c->stretched) {
        const std::vector<double> met = metric_table(n, L, c->cfg.stretch_m, dealias_threshold());
        std::vector<double> vol(n);
        for (int i = 0; i < n; ++i) vol[i] = dS_at(i, n, L, c->cfg.stretch_m);
        c->met = dalloc<void>(c, c->es * n);
        c->vol = dalloc<double>(c, 8 * n);
        if (c->fp32) {
            std::vector<float> mf(met.begin(), met.end());
            CK(cudaMemcpy(c->met, mf.data(), 4 * n, cudaMemcpyHostToDevice));
        } else {
            CK(cudaMemcpy(c->met, met.data(), 8 * n, cudaMemcpyHostToDevice));
        }
        CK(cudaMemcpy(c->vol, vol.data(), 8 * n, cudaMemcpyHostToDevice));
    }
}

void cc_setup(kf_ctx *c);


void build_levels(kf_ctx *c) {
    const kf_config &cf = c->cfg;
    int nl = 1;
    if (cf.poisson_mode == KF_PS_FAS) nl = cf.mg_levels > 1 ? cf.mg_levels : 1;
    if (cf.poisson_mode == KF_PS_CASCADIC) nl = 4;
    for (int l = 1; l < nl; ++l)
        if ((c->n >> l) < 2 || ((c->n >> (l - 1)) % 2))
            throw KfError{KF_ERR_ARG, "too many multigrid levels for this grid"};
    if (cf.poisson_mode == KF_PS_CASCADIC && c->n % 8) throw KfError{KF_ERR_ARG, "cascadic plan needs n % 8 == 0"};
    if (cf.poisson_mode == KF_PS_FAS && ((long)(c->n >> (nl - 1)) * (c->n >> (nl - 1)) * (c->n >> (nl - 1)) > 8192))
        throw KfError{KF_ERR_ARG, "coarsest FAS level above 8192 points (shared-memory solve); add levels"};
    CK(cudaFuncSetAttribute(k_coarse_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    march_attrs();
    c->march_maps = encode_tiled() != nullptr;  // before the levels: L.t depends on it
    c->lv.resize(nl);
    for (int l = 0; l < nl; ++l) {
        LevelBuf &L = c->lv[l];
        const int n = c->n >> l;
        L.n = n;
        const double Lb = cf.L;
        std::vector<double> H(n + 1), dd(n), dp(n), dm(n), ip(n), im(n), gam(n, 0.);
        const double sm = cf.stretch_m;
        for (int i = 0; i < n + 1; ++i) H[i] = val_at(i, n, Lb, sm) - val_at(i - 1, n, Lb, sm);  // H_create (:112-126)
        for (int i = 0; i < n; ++i) {
            dd[i] = 2. / (H[i + 1] * H[i]);
            dp[i] = H[i + 1] * (H[i + 1] + H[i]);
            dm[i] = H[i] * (H[i + 1] + H[i]);
            ip[i] = 2. / dp[i];
            im[i] = 2. / dm[i];
        }
        for (int m = 1; m < n; m += 2) {  // OP_hto2h gamma on this (fine) axis
            const double x1 = val_at(m - 1, n, Lb, sm), x2 = val_at(m + 1, n, Lb, sm), x = val_at(m, n, Lb, sm);
            gam[m] = (x - x1) / (x2 - x1);
        }
        L.dd = dalloc<double>(c, 8 * n);
        L.dp = dalloc<double>(c, 8 * n);
        L.dm = dalloc<double>(c, 8 * n);
        L.gam = dalloc<double>(c, 8 * n);
        L.ip = dalloc<double>(c, 8 * n);
        L.im = dalloc<double>(c, 8 * n);
        CK(cudaMemcpy(L.ip, ip.data(), 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(L.im, im.data(), 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(L.dd, dd.data(), 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(L.dp, dp.data(), 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(L.dm, dm.data(), 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(L.gam, gam.data(), 8 * n, cudaMemcpyHostToDevice));
        if (KF_RBGS_TAB && n <= KF_TAB_N) {
            L.tab = std::make_shared<AxTab>();
            for (int m = 0; m < n; ++m) {
                L.tab->dd[m] = dd[m];
                L.tab->ip[m] = ip[m];
                L.tab->im[m] = im[m];
            }
        }
        const size_t bytes = sizeof(double) * (size_t)n * n * n;
        L.r = dalloc<double>(c, bytes);
        if (cf.poisson_mode == KF_PS_FAS && march_level(L) && c->march_maps) {
            L.t = dalloc<double>(c, bytes);
            CUtensorMap probe;  // the encoder must accept this level's row copies
            if (!row_map(&probe, L.t, n)) L.t = nullptr;
        }
        if (l == 0) {
            L.phi = c->phi;
            L.rho = c->rho;
        } else {
            L.phi = dalloc<double>(c, bytes);
            L.rho = dalloc<double>(c, bytes);
            L.phi0 = dalloc<double>(c, bytes);
        }
    }
    CK(cudaFuncSetAttribute(k_coarse_cycle, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    cc_setup(c);
}

// The entry level of k_coarse_cycle: the first level below the finest with
// n <= 16 that has at least one level below it, when the levels from it down
// fit the kernel (KF_CC_LEVELS, 200 KB of shared memory); -1 otherwise or
// with the block switched off.
void cc_setup(kf_ctx *c) {
    c->cc_level = -1;
    const int nl = (int)c->lv.size();
    if (!c->coarse_block || c->cfg.poisson_mode != KF_PS_FAS) return;
    int lb = 1;
    while (lb < nl && c->lv[lb].n > 16) ++lb;
    if (lb >= nl - 1 || nl - lb > KF_CC_LEVELS) return;
    CoarseCycle C{};
    C.nl = nl - lb;
    for (int m = 0; m < C.nl; ++m) {
        const LevelBuf &L = c->lv[lb + m];
        C.n[m] = L.n;
        C.dd[m] = L.dd;
        C.ip[m] = L.ip;
        C.im[m] = L.im;
        C.gam[m] = L.gam;
    }
    const size_t b = coarse_cycle_smem(C);
    if (b > 200 * 1024) return;
    c->ccyc = C;
    c->cc_smem = b;
    c->cc_level = lb;
}

void build_jobs(kf_ctx *c) {
    std::vector<AxisJob> J;
    std::vector<ZJob> Z;
    auto aj = [&](const void *in, void *out, int mul) { J.push_back(AxisJob{in, out, mul, 0}); };
    auto zj = [&](const void *ia, int ma, const void *ib, int mb, void *oa, void *ob) {
        Z.push_back(ZJob{ia, ib, oa, ob, ma, mb});
    };
    void **CX = c->CX, **CY = c->CY, **R = c->R;
    // A
    c->jA_x = (int)J.size();
    aj(c->Ys[3], CX[0], MUL_P);
    aj(c->Ys[3], CX[1], MUL_P_IK);
    c->jA_y = (int)J.size();
    aj(CX[0], CY[0], MUL_NONE);
    aj(CX[0], CY[1], MUL_IK);
    aj(CX[1], CY[2], MUL_NONE);
    c->zA = (int)Z.size();
    zj(CY[0], MUL_NONE, nullptr, 0, R[0], nullptr);
    // B
    c->zB = (int)Z.size();
    zj(c->phiT, 0, nullptr, 0, CX[8], nullptr);  // CX[8], CY[12]: not written by round D's u', s part
    c->jB_y = (int)J.size();
    aj(CX[8], CY[12], MUL_NONE);
    c->jB_x = (int)J.size();
    aj(CY[12], c->phihat, MUL_NONE);
    // D
    c->jD_x = (int)J.size();
    for (int q = 0; q < 3; ++q) {
        aj(c->Ys[q], CX[2 + 2 * q], MUL_P);
        aj(c->Ys[q], CX[3 + 2 * q], MUL_P_IK);
    }
    for (int q = 0; q < 4; ++q) aj(c->LIN[q], CX[8 + q], MUL_NONE);
    c->jD_y = (int)J.size();
    for (int q = 0; q < 3; ++q) {
        aj(CX[2 + 2 * q], CY[3 + 3 * q], MUL_NONE);
        aj(CX[2 + 2 * q], CY[4 + 3 * q], MUL_IK);
        aj(CX[3 + 2 * q], CY[5 + 3 * q], MUL_NONE);
    }
    for (int q = 0; q < 4; ++q) aj(CX[8 + q], CY[12 + q], MUL_NONE);
    c->zD = (int)Z.size();
    for (int q = 0; q < 3; ++q) {
        zj(CY[3 + 3 * q], MUL_NONE, CY[3 + 3 * q], MUL_IK, R[1 + q], R[4 + 3 * q + 2]);  // U_c, d_z U_c
        zj(CY[4 + 3 * q], MUL_NONE, CY[5 + 3 * q], MUL_NONE, R[4 + 3 * q + 1], R[4 + 3 * q + 0]);  // d_y, d_x
    }
    zj(CY[1], MUL_NONE, CY[2], MUL_NONE, R[14], R[13]);  // d_y s, d_x s
    zj(CY[0], MUL_IK, nullptr, 0, R[15], nullptr);       // d_z s
    zj(CY[12], MUL_NONE, CY[13], MUL_NONE, R[16], R[17]);
    zj(CY[14], MUL_NONE, CY[15], MUL_NONE, R[18], R[19]);
    // F
    c->zF = (int)Z.size();
    zj(R[20], 0, R[21], 0, CX[0], CX[1]);
    zj(R[22], 0, R[23], 0, CX[2], CX[3]);
    c->jF_y = (int)J.size();
    for (int q = 0; q < 4; ++q) aj(CX[q], CY[q], MUL_NONE);
    c->jF_x = (int)J.size();
    for (int q = 0; q < 4; ++q) aj(CY[q], c->K[q], MUL_NONE);
    // standalone transforms: r2c R[0] -> CX[0] ; c2r CX[0] -> R[0]
    c->zT = (int)Z.size();
    zj(R[0], 0, nullptr, 0, CX[1], nullptr);
    zj(CY[0], MUL_NONE, nullptr, 0, R[0], nullptr);
    c->jTf_y = (int)J.size();
    aj(CX[1], CY[1], MUL_NONE);
    c->jTf_x = (int)J.size();
    aj(CY[1], CX[0], MUL_NONE);
    c->jT_x = (int)J.size();
    aj(CX[0], CX[1], MUL_NONE);
    c->jT_y = (int)J.size();
    aj(CX[1], CY[0], MUL_NONE);
    // diagnostics: c2r of the state (Y) -> R[20..23]
    c->jG_x = (int)J.size();
    for (int q = 0; q < 4; ++q) aj(c->Y[q], CX[q], MUL_NONE);
    c->jG_y = (int)J.size();
    for (int q = 0; q < 4; ++q) aj(CX[q], CY[q], MUL_NONE);
    c->zG = (int)Z.size();
    zj(CY[0], MUL_NONE, CY[1], MUL_NONE, R[20], R[21]);
    zj(CY[2], MUL_NONE, CY[3], MUL_NONE, R[22], R[23]);
    if (c->stretched) {
        void **SX = c->SX;
        // D': raw derivatives c2r(P i k_d F) of u'_c (R[4+3c+d], with U_c in
        // R[1+c]), of s (R[13+d]; its x and y passes are round A's) and of F1
        // (in CX[10]; R[16+d])
        c->jS_Dx = (int)J.size();
        for (int q = 0; q < 3; ++q) {
            aj(c->Ys[q], CX[2 + 2 * q], MUL_P);
            aj(c->Ys[q], CX[3 + 2 * q], MUL_P_IK);
        }
        aj(CX[10], CX[8], MUL_P);
        aj(CX[10], CX[9], MUL_P_IK);
        c->jS_Dy = (int)J.size();
        for (int q = 0; q < 3; ++q) {
            aj(CX[2 + 2 * q], CY[3 + 3 * q], MUL_NONE);
            aj(CX[2 + 2 * q], CY[4 + 3 * q], MUL_IK);
            aj(CX[3 + 2 * q], CY[5 + 3 * q], MUL_NONE);
        }
        aj(CX[8], CY[12], MUL_NONE);
        aj(CX[8], CY[13], MUL_IK);
        aj(CX[9], CY[14], MUL_NONE);
        c->zS_D = (int)Z.size();
        for (int q = 0; q < 3; ++q) {
            zj(CY[3 + 3 * q], MUL_NONE, CY[3 + 3 * q], MUL_IK, R[1 + q], R[4 + 3 * q + 2]);
            zj(CY[4 + 3 * q], MUL_NONE, CY[5 + 3 * q], MUL_NONE, R[4 + 3 * q + 1], R[4 + 3 * q + 0]);
        }
        zj(CY[1], MUL_NONE, CY[2], MUL_NONE, R[14], R[13]);
        zj(CY[0], MUL_IK, nullptr, 0, R[15], nullptr);
        zj(CY[14], MUL_NONE, CY[13], MUL_NONE, R[16], R[17]);
        zj(CY[12], MUL_IK, nullptr, 0, R[18], nullptr);
        // F': r2c of the 15 scaled derivatives R[4..18] -> CY[0..14]
        c->zS_F = (int)Z.size();
        for (int j = 0; j < 14; j += 2) zj(R[4 + j], 0, R[5 + j], 0, CY[j], CY[j + 1]);
        zj(R[18], 0, nullptr, 0, CY[14], nullptr);
        c->jS_Fy = (int)J.size();
        for (int j = 0; j < 15; ++j) aj(CY[j], SX[j], MUL_NONE);
        c->jS_Fx = (int)J.size();
        for (int j = 0; j < 15; ++j) aj(SX[j], CY[j], MUL_NONE);
        // G': c2r(P D_d u'_c), c2r(P D_d s) -> R[4..15] (the products' operands)
        c->jS_Gx = (int)J.size();
        for (int j = 0; j < 12; ++j) aj(CY[j], SX[j], MUL_P);
        c->jS_Gy = (int)J.size();
        for (int j = 0; j < 12; ++j) aj(SX[j], CX[j], MUL_NONE);
        c->zS_G = (int)Z.size();
        for (int j = 0; j < 12; j += 2) zj(CX[j], MUL_NONE, CX[j + 1], MUL_NONE, R[4 + j], R[5 + j]);
        // I': r2c of the products R[20..23] -> SX[8..11]
        c->zS_I = (int)Z.size();
        zj(R[20], 0, R[21], 0, SX[0], SX[1]);
        zj(R[22], 0, R[23], 0, SX[2], SX[3]);
        c->jS_Iy = (int)J.size();
        for (int q = 0; q < 4; ++q) aj(SX[q], SX[4 + q], MUL_NONE);
        c->jS_Ix = (int)J.size();
        for (int q = 0; q < 4; ++q) aj(SX[4 + q], SX[8 + q], MUL_NONE);
        // K': penalization, K -> R[20..23] -> K
        c->jS_Kx = (int)J.size();
        for (int q = 0; q < 4; ++q) aj(c->K[q], SX[q], MUL_NONE);
        c->jS_Ky = (int)J.size();
        for (int q = 0; q < 4; ++q) aj(SX[q], SX[4 + q], MUL_NONE);
        c->zS_K = (int)Z.size();
        zj(SX[4], MUL_NONE, SX[5], MUL_NONE, R[20], R[21]);
        zj(SX[6], MUL_NONE, SX[7], MUL_NONE, R[22], R[23]);
        c->zS_Kf = (int)Z.size();
        zj(R[20], 0, R[21], 0, SX[0], SX[1]);
        zj(R[22], 0, R[23], 0, SX[2], SX[3]);
        c->jS_Kfy = (int)J.size();
        for (int q = 0; q < 4; ++q) aj(SX[q], SX[4 + q], MUL_NONE);
        c->jS_Kfx = (int)J.size();
        for (int q = 0; q < 4; ++q) aj(SX[4 + q], c->K[q], MUL_NONE);
    }
    c->hj = J;
    c->hz = Z;
    c->dj = dalloc<AxisJob>(c, sizeof(AxisJob) * J.size());
    c->dz = dalloc<ZJob>(c, sizeof(ZJob) * Z.size());
    CK(cudaMemcpy(c->dj, J.data(), sizeof(AxisJob) * J.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->dz, Z.data(), sizeof(ZJob) * Z.size(), cudaMemcpyHostToDevice));
}

void create(kf_ctx *c) {
    const kf_config &cf = c->cfg;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) throw KfError{KF_ERR_NO_DEVICE, "no CUDA device"};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) throw KfError{KF_ERR_NO_DEVICE, "this library targets sm_100a (B200)"};
    if (cf.precision != KF_FP64 && cf.precision != KF_FP32_BULK) throw KfError{KF_ERR_ARG, "precision"};
    if (cf.pen_eta > 0.) throw KfError{KF_ERR_ARG, "penalization damping must be <= 0 (effect_penalization.cpp:7-12)"};
    if (!(cf.L > 0.) || !(cf.theta != 0.)) throw KfError{KF_ERR_ARG, "L > 0 and theta != 0 required"};
    if (!(cf.stretch_m >= 0.) || !(2. * acos(-1.) * cf.stretch_m < cf.L))
        throw KfError{KF_ERR_ARG, "stretch_m must satisfy 0 <= 2 pi m < L (a monotone axis_CoSiSt map)"};
    if (!(cf.mg_omega >= 0.) || !(cf.mg_omega < 2.))
        throw KfError{KF_ERR_ARG, "mg_omega must lie in [0, 2) (0: the plain Newton step)"};
    c->stretched = cf.stretch_m != 0.;
    c->fp32 = cf.precision == KF_FP32_BULK;
    c->es = c->fp32 ? 4 : 8;
    c->cs = 2 * c->es;
    c->n = cf.n;
    c->nzc = cf.n / 2 + 1;
    c->N = (long)cf.n * cf.n * cf.n;
    c->Nc = (long)cf.n * cf.n * c->nzc;
    bool ok = c->fp32 ? Dispatch<float>::pick(c) : Dispatch<double>::pick(c);
    if (!ok) throw KfError{KF_ERR_ARG, "grid size must be one of 16, 32, 64, 96, 128, 256"};
    CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    c->own_stream = true;
    CK(cudaStreamCreateWithFlags(&c->st_body, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->st_side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    const size_t cb = c->cs * c->Nc, rb = c->es * c->N;
    for (int q = 0; q < 4; ++q) {
        c->Y[q] = dalloc<void>(c, cb);
        c->Ys[q] = dalloc<void>(c, cb);
        c->ACC[q] = dalloc<void>(c, cb);
        c->K[q] = dalloc<void>(c, cb);
        c->LIN[q] = dalloc<void>(c, cb);
    }
    for (int i = 0; i < 12; ++i) c->CX[i] = dalloc<void>(c, cb);
    for (int i = 0; i < 16; ++i) c->CY[i] = dalloc<void>(c, cb);
    for (int i = 0; i < 24; ++i) c->R[i] = dalloc<void>(c, rb);
    if (c->stretched)
        for (int i = 0; i < 15; ++i) c->SX[i] = dalloc<void>(c, cb);
    c->phihat = dalloc<void>(c, cb);
    c->phi = dalloc<double>(c, 8 * c->N);
    c->rho = dalloc<double>(c, 8 * c->N);
    if (KF_RHO_CS && c->cfg.poisson_mode == KF_PS_FAS && c->n >= 64 && c->n <= KF_TAB_N)
        c->rho_cs = dalloc<double>(c, 8 * c->N);
    c->nd = dalloc<double>(c, 8 * c->N);
    c->H = dalloc<void>(c, rb);
    c->phiT = c->fp32 ? dalloc<void>(c, rb) : (void *)c->phi;
    c->stage64 = dalloc<double>(c, (size_t)16 * (c->Nc > c->N ? c->Nc : c->N));
    CK(cudaMemset(c->phi, 0, 8 * c->N));
    CK(cudaMemset(c->nd, 0, 8 * c->N));
    CK(cudaMemset(c->H, 0, rb));
    for (int q = 0; q < 4; ++q) {
        CK(cudaMemset(c->Y[q], 0, cb));
        CK(cudaMemset(c->Ys[q], 0, cb));
    }
    c->npartial = 1184;
    c->partial = dalloc<double>(c, sizeof(double) * KF_RED * c->npartial);
    c->red = dalloc<double>(c, sizeof(double) * 8);
    c->d_sweeps = dalloc<int>(c, sizeof(int) * 4);
    c->d_err = dalloc<int>(c, sizeof(int));
    CK(cudaMemset(c->d_err, 0, sizeof(int)));
    CK(cudaMallocHost(&c->h_err, sizeof(int)));
    c->d_max = dalloc<unsigned long long>(c, 64 * sizeof(unsigned long long));
    CK(cudaMallocHost(&c->h_max, 64 * sizeof(unsigned long long)));
    if (cf.phi_extrap) c->phi_a = dalloc<double>(c, 8 * c->N);
    CK(cudaMallocHost(&c->h_red, sizeof(double) * 8));
    c->dtime = dalloc<DevTime>(c, sizeof(DevTime));
    c->dpois = dalloc<DevPois>(c, sizeof(DevPois));
    CK(cudaMemset(c->dtime, 0, sizeof(DevTime)));
    CK(cudaMemset(c->dpois, 0, sizeof(DevPois)));
    build_tables(c);
    build_levels(c);
    build_jobs(c);
    CK(cudaDeviceSynchronize());
}

// H2D of a host FP64 array of `count` doubles into a bulk-precision device array
void put_bulk(kf_ctx *c, void *dst, const double *src, long count) {
    if (!c->fp32) {
        CK(cudaMemcpyAsync(dst, src, 8 * count, cudaMemcpyHostToDevice, c->st));
    } else {
        CK(cudaMemcpyAsync(c->stage64, src, 8 * count, cudaMemcpyHostToDevice, c->st));
        Launch L_(c, KC_MISC, 12. * count);
        k_from_f64<float><<<nblk(count, 256), 256, 0, c->st>>>((float *)dst, c->stage64, count);
    }
}

void get_bulk(kf_ctx *c, double *dst, const void *src, long count) {
    if (!c->fp32) {
        CK(cudaMemcpyAsync(dst, src, 8 * count, cudaMemcpyDeviceToHost, c->st));
    } else {
        {
            Launch L_(c, KC_MISC, 12. * count);
            k_to_f64<float><<<nblk(count, 256), 256, 0, c->st>>>(c->stage64, (const float *)src, count);
        }
        CK(cudaMemcpyAsync(dst, c->stage64, 8 * count, cudaMemcpyDeviceToHost, c->st));
    }
}

void copy_state(kf_ctx *c, void *const *dst, void *const *src) {
    for (int q = 0; q < 4; ++q)
        CK(cudaMemcpyAsync(dst[q], src[q], c->cs * c->Nc, cudaMemcpyDeviceToDevice, c->st));
}

void rk_launch(kf_ctx *c, double cdt, int mode) {
    const long M = c->Nc;
    for (int q = 0; q < 4; ++q) {
        Launch L_(c, KC_RK, (double)M * c->cs * (mode == 1 ? 5 : 4));
        if (c->fp32)
            k_rk<float><<<nblk(M, 256), 256, 0, c->st>>>((float2 *)c->Y[q], (float2 *)c->ACC[q], (float2 *)c->Ys[q],
                                                        (const float2 *)c->K[q], (float)cdt, mode, M);
        else
            k_rk<double><<<nblk(M, 256), 256, 0, c->st>>>((double2 *)c->Y[q], (double2 *)c->ACC[q], (double2 *)c->Ys[q],
                                                         (const double2 *)c->K[q], cdt, mode, M);
    }
    CK(cudaGetLastError());
}

// One RK4 step (RKO4.cpp:105-238) on Y (== Ys on entry).  Optional hooks of
// the adjoint: X (16 buffers) receives the four stage inputs, PH (4) the four
// stage potentials; with PHin the stage potentials are taken from there and
// no Poisson problem is solved.
void rk4_step(kf_ctx *c, double dt, void *const *X, double *const *PH, double *const *PHin) {
    const double t0 = c->t;
    const double ts[4] = {t0, t0 + 0.5 * dt, t0 + 0.5 * dt, t0 + 1.0 * dt};
    const double cdt[4] = {0.5 * dt, 0.5 * dt, 1.0 * dt, dt / 6.};
    const int mode[4] = {0, 1, 1, 2};
    static const char *const kStage[4] = {"kf RK4 stage 1", "kf RK4 stage 2", "kf RK4 stage 3", "kf RK4 stage 4"};
    for (int i = 0; i < 4; ++i) {
        NvtxRange nv(kStage[i]);
        c->t_stage = ts[i];
        c->stage_idx = i;
        if (X) copy_state(c, X + 4 * i, c->Ys);
        if (PHin) {
            CK(cudaMemcpyAsync(c->phi, PHin[i], 8 * c->N, cudaMemcpyDeviceToDevice, c->st));
            c->phi_given = true;
        }
        c->rhs_fn(c);
        c->phi_given = false;
        if (PH) CK(cudaMemcpyAsync(PH[i], c->phi, 8 * c->N, cudaMemcpyDeviceToDevice, c->st));
        rk_launch(c, cdt[i], mode[i]);
    }
    copy_state(c, c->Ys, c->Y);
    c->t = t0 + dt;
}

// Whether kf_rk4_steps replays a captured step graph: every decision of the
// step can be taken on the device (FAS or no Poisson solve; the Jacobi and
// cascadic solvers steer their sweeps from the host) and the per-launch
// profile is off.  KIELFLOW_B200_NO_GRAPH=1 forces the host-driven path.
bool graph_path(kf_ctx *c) {
    const kf_config &cf = c->cfg;
    static const bool off = [] {
        const char *e = std::getenv("KIELFLOW_B200_NO_GRAPH");
        return e && e[0] == '1';
    }();
    if (c->prof || off) return false;
    const bool pois = (cf.terms & T_POISSON) && (cf.terms & T_E_INT);
    return !pois || cf.poisson_mode == KF_PS_FAS;
}

// Capture one RK4 step (the sequence of rk4_step) with device-side stage
// times, warm starts and convergence loops; with wait_u, stage 1 waits for
// ev_u after its Poisson solve.
void capture_step(kf_ctx *c, double dt, bool wait_u, cudaGraphExec_t *out);

void build_step_graph(kf_ctx *c, double dt, bool with_wait = false) {
    if (c->step_graph && c->step_dt != dt) {
        cudaGraphExecDestroy(c->step_graph);
        c->step_graph = nullptr;
        if (c->step_graph_wait) cudaGraphExecDestroy(c->step_graph_wait);
        c->step_graph_wait = nullptr;
    }
    if (!c->step_graph) capture_step(c, dt, false, &c->step_graph);
    if (with_wait && !c->step_graph_wait) capture_step(c, dt, true, &c->step_graph_wait);
    c->step_dt = dt;
}

void capture_step(kf_ctx *c, double dt, bool wait_u, cudaGraphExec_t *out) {
    const double xs[4] = {0., 0.5 * dt, 0.5 * dt, 1.0 * dt};
    const double cdt[4] = {0.5 * dt, 0.5 * dt, 1.0 * dt, dt / 6.};
    const int mode[4] = {0, 1, 1, 2};
    const kf_config &cf = c->cfg;
    const bool pois = (cf.terms & T_POISSON) && (cf.terms & T_E_INT);
    const long long l0 = c->launches;
    c->cycle_kernels = 0;
    c->capturing = true;
    c->capture_wait_u = wait_u;
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    try {
        for (int i = 0; i < 4; ++i) {
            {
                Launch L_(c, KC_MISC, 0.);
                k_time<<<1, 32, 0, c->st>>>(c->dtime, xs[i], 0);
            }
            c->stage_idx = i;
            c->rhs_fn(c);
            rk_launch(c, cdt[i], mode[i]);
        }
        copy_state(c, c->Ys, c->Y);
        {
            Launch L_(c, KC_MISC, 0.);
            k_time<<<1, 32, 0, c->st>>>(c->dtime, dt, 1);
        }
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(c->st, &g);
        if (g) cudaGraphDestroy(g);
        c->capturing = false;
        c->capture_wait_u = false;
        c->launches = l0;
        throw;
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->st, &g);
    c->capturing = false;
    c->capture_wait_u = false;
    CK(e);
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    c->step_kernels = c->launches - l0 - (pois ? 4 * c->cycle_kernels : 0);
    c->launches = l0;
}

// nsteps replays of the step graph; the host's time and warm-start record is
// handed to the device before and read back after, with the solve statistics.
void graph_begin(kf_ctx *c, double dt) {
    build_step_graph(c, dt);
    DevTime ht{c->t, c->t_stage, c->tau_a, c->tau_b, c->nhist, 0, 0, 0};
    CK(cudaMemcpyAsync(c->dtime, &ht, sizeof(DevTime), cudaMemcpyHostToDevice, c->st));
}

void graph_step(kf_ctx *c) {
    NvtxRange nv("kf RK4 step (captured graph)");
    CK(cudaGraphLaunch(c->step_graph, c->st));
    c->launches += c->step_kernels;
}

void graph_end(kf_ctx *c) {
    DevTime ht;
    DevPois hp;
    CK(cudaMemcpyAsync(&ht, c->dtime, sizeof(DevTime), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&hp, c->dpois, sizeof(DevPois), cudaMemcpyDeviceToHost, c->st));
    kerr_fetch(c);
    CK(cudaStreamSynchronize(c->st));
    kerr_check(c);
    c->t = ht.t;
    c->t_stage = ht.t_stage;
    c->tau_a = ht.tau_a;
    c->tau_b = ht.tau_b;
    c->nhist = ht.nhist;
    const DevPois &o = c->hpois;
    c->launches += (hp.total_cycles - o.total_cycles) * c->cycle_kernels + (hp.solves - o.solves) * c->head_kernels;
    c->diag.solves += hp.solves - o.solves;
    c->diag.total_iterations += hp.total_cycles - o.total_cycles;
    if (hp.solves != o.solves) {
        c->diag.last_iterations = hp.last_cycles;
        c->diag.last_residual = hp.last_residual;
    }
    c->diag.not_converged += hp.not_converged - o.not_converged;
    for (int s = 0; s < 4; ++s) c->diag.stage_cycles[s] += hp.stage_cycles[s] - o.stage_cycles[s];
    const bool nan = hp.nans != o.nans, nc = hp.not_converged != o.not_converged;
    c->hpois = hp;
    if (nan) throw KfError{KF_ERR_NAN, "NaN in the multigrid solve"};
    if (nc) throw KfError{KF_ERR_NOT_CONVERGED, "Poisson solve did not reach its tolerance"};
}

void rk4_steps_graph(kf_ctx *c, int nsteps, double dt) {
    graph_begin(c, dt);
    for (int s = 0; s < nsteps; ++s) graph_step(c);
    graph_end(c);
}

// interface_ode_solver::solve with the state in host arrays, in place: the
// upload of s goes first on the compute stream; u' is uploaded on a copy
// stream while stage 1's Poisson solve runs (the captured step of the first
// step waits for it just before it needs u'); the result is copied back.
void step_host(kf_ctx *c, int nsteps, double dt, double *const *host) {
    if (!c->st_copy) {
        CK(cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->ev_u, cudaEventDisableTiming));
        if (c->fp32) c->stage64b = dalloc<double>(c, 16 * (size_t)c->Nc);
    }
    build_step_graph(c, dt, true);
    put_bulk(c, c->Y[3], host[3], 2 * c->Nc);
    CK(cudaMemcpyAsync(c->Ys[3], c->Y[3], c->cs * c->Nc, cudaMemcpyDeviceToDevice, c->st));
    for (int q = 0; q < 3; ++q) {
        if (!c->fp32) {
            CK(cudaMemcpyAsync(c->Y[q], host[q], 16 * c->Nc, cudaMemcpyHostToDevice, c->st_copy));
        } else {
            CK(cudaMemcpyAsync(c->stage64b, host[q], 16 * c->Nc, cudaMemcpyHostToDevice, c->st_copy));
            const long M = 2 * c->Nc;
            Launch L_(c, KC_MISC, 12. * M);
            k_from_f64<float><<<nblk(M, 256), 256, 0, c->st_copy>>>((float *)c->Y[q], c->stage64b, M);
        }
        CK(cudaMemcpyAsync(c->Ys[q], c->Y[q], c->cs * c->Nc, cudaMemcpyDeviceToDevice, c->st_copy));
    }
    CK(cudaEventRecord(c->ev_u, c->st_copy));
    c->nhist = 0;  // as kf_set_state
    DevTime ht{c->t, c->t_stage, c->tau_a, c->tau_b, c->nhist, 0, 0, 0};
    CK(cudaMemcpyAsync(c->dtime, &ht, sizeof(DevTime), cudaMemcpyHostToDevice, c->st));
    CK(cudaGraphLaunch(c->step_graph_wait, c->st));
    c->launches += c->step_kernels;
    for (int s = 1; s < nsteps; ++s) graph_step(c);
    graph_end(c);
    for (int q = 0; q < 4; ++q) get_bulk(c, host[q], c->Y[q], 2 * c->Nc);
    CK(cudaStreamSynchronize(c->st));
}

template <typename F> int guarded(kf_ctx *c, F f) {
    if (!c) return KF_ERR_ARG;
    try {
        f();
        return KF_OK;
    } catch (const KfError &e) {
        c->err = e.msg;
        return e.code;
    } catch (const std::exception &e) {
        c->err = e.what();
        return KF_ERR_ARG;
    }
}

}  // namespace

#include "kf_adjoint_host.cuh"
#include "kf_driver.cuh"

namespace {

// Captured graphs hold the kernel variants they were captured with; dropped
// when the variants change and rebuilt by their next use.
void drop_graphs(kf_ctx *c) {
    CK(cudaStreamSynchronize(c->st));
    if (c->vgraph) cudaGraphExecDestroy(c->vgraph);
    c->vgraph = nullptr;
    if (c->vgraph_tail) cudaGraphExecDestroy(c->vgraph_tail);
    c->vgraph_tail = nullptr;
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
    if (c->step_graph_wait) cudaGraphExecDestroy(c->step_graph_wait);
    c->step_graph_wait = nullptr;
    if (c->adj && c->adj->graph) {
        cudaGraphExecDestroy(c->adj->graph);
        c->adj->graph = nullptr;
    }
}

// milliseconds per call of f: two untimed calls, then reps calls between
// CUDA events on the context's stream
template <typename F> double time_candidate(kf_ctx *c, int reps, F f) {
    cudaEvent_t a = nullptr, b = nullptr;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    float ms = 0.f;
    cudaError_t e = cudaSuccess;
    try {
        f();
        f();
        CK(cudaEventRecord(a, c->st));
        for (int r = 0; r < reps; ++r) f();
        CK(cudaEventRecord(b, c->st));
        CK(cudaEventSynchronize(b));
        e = cudaEventElapsedTime(&ms, a, b);
    } catch (...) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        throw;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CK(e);
    return (double)ms / reps;
}

void autotune(kf_ctx *c, int reps, kf_tune_out *o) {
    if (c->capturing) throw KfError{KF_ERR_ARG, "kf_autotune during a capture"};
    kf_tune_out r{};
    plan_info(c->n, r.fft_radices, r.fft_threads);
    // transform plans: the right-hand side with the potential held writes
    // only scratch arrays and K (the stage derivative, consumed within a step)
    const bool pg = c->phi_given;
    const int si = c->stage_idx, fv = c->fftv, by = c->rbgs_by;
    c->phi_given = true;
    c->stage_idx = 0;
    try {
        for (int v = 0; v < 2; ++v) {
            c->fftv = v;
            copy_state(c, c->Ys, c->Y);
            r.fft_ms[v] = time_candidate(c, reps, [&] { c->rhs_fn(c); });
        }
    } catch (...) {
        c->phi_given = pg;
        c->stage_idx = si;
        c->fftv = fv;
        throw;
    }
    c->phi_given = pg;
    c->stage_idx = si;
    r.fft_plan = r.fft_ms[1] < r.fft_ms[0] ? 1 : 0;
    // smoother shapes: sweeps of a copy of the finest-level potential
    // (rows 0: the streaming k_rbgs_march where the level allows it)
    const int rows[4] = {4, 8, 16, 0};
    r.rbgs_rows = by;
    if (c->rho && !c->lv.empty()) {
        LevelBuf &L0 = c->lv[0];
        double *tmp = nullptr;
        CK(cudaMalloc(&tmp, 8 * (size_t)c->N));
        try {
            CK(cudaMemcpyAsync(tmp, c->phi, 8 * (size_t)c->N, cudaMemcpyDeviceToDevice, c->st));
            rho_split(c);  // the finest half sweeps read the colour-split copy
            int best = -1;
            for (int k = 0; k < 4; ++k) {
                c->rbgs_by = rows[k];
                if (rows[k] == 0 && !march_ok(c, L0)) {
                    r.rbgs_ms[k] = -1.;
                    continue;
                }
                r.rbgs_ms[k] =
                    0.5 * time_candidate(c, reps, [&] { smooth(c, L0, tmp, c->rho, nullptr, 2, KC_RBGS); });
                if (best < 0 || r.rbgs_ms[k] < r.rbgs_ms[best]) best = k;
            }
            r.rbgs_rows = rows[best];
        } catch (...) {
            c->rbgs_by = by;
            c->fftv = fv;
            cudaStreamSynchronize(c->st);
            cudaFree(tmp);
            throw;
        }
        CK(cudaStreamSynchronize(c->st));
        CK(cudaFree(tmp));
    }
    c->fftv = r.fft_plan;
    c->rbgs_by = r.rbgs_rows;
    drop_graphs(c);
    if (o) *o = r;
}

}  // namespace

// Message of the last failure that has no context (kf_ctx_create and the
// context-free entry points); kf_last_error(NULL) returns it.
std::string &kf_global_error() {
    static thread_local std::string s;
    return s;
}

extern "C" {

int kf_ctx_create(const kf_config *cfg, kf_ctx **out) {
    if (!cfg || !out) return KF_ERR_ARG;
    kf_ctx *c = new kf_ctx;
    c->cfg = *cfg;
    int rc = guarded(c, [&] { create(c); });
    if (rc) {
        kf_global_error() = c->err;
        kf_ctx_destroy(c);
        *out = nullptr;
        return rc;
    }
    *out = c;
    return KF_OK;
}

int kf_ctx_destroy(kf_ctx *c) {
    if (!c) return KF_ERR_ARG;
    if (c->st) cudaStreamSynchronize(c->st);
    for (auto &r : c->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : c->evfree) cudaEventDestroy(e);
    if (c->vgraph) cudaGraphExecDestroy(c->vgraph);
    if (c->vgraph_tail) cudaGraphExecDestroy(c->vgraph_tail);
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    if (c->step_graph_wait) cudaGraphExecDestroy(c->step_graph_wait);
    if (c->ev_u) cudaEventDestroy(c->ev_u);
    if (c->st_copy) cudaStreamDestroy(c->st_copy);
    if (c->st_body) cudaStreamDestroy(c->st_body);
    if (c->st_side) cudaStreamDestroy(c->st_side);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    adj_release(c);
    out_release(c);
    for (void *p : c->allocs) cudaFree(p);
    if (c->h_red) cudaFreeHost(c->h_red);
    if (c->h_max) cudaFreeHost(c->h_max);
    if (c->h_err) cudaFreeHost(c->h_err);
    if (c->st && c->own_stream) cudaStreamDestroy(c->st);
    delete c;
    return KF_OK;
}

const char *kf_last_error(const kf_ctx *c) { return c ? c->err.c_str() : kf_global_error().c_str(); }

int kf_set_stream(kf_ctx *c, void *stream) {
    return guarded(c, [&] {
        CK(cudaStreamSynchronize(c->st));
        if (c->own_stream) CK(cudaStreamDestroy(c->st));
        if (stream) {
            c->st = (cudaStream_t)stream;
            c->own_stream = false;
        } else {
            CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
            c->own_stream = true;
        }
    });
}

int kf_synchronize(kf_ctx *c) {
    return guarded(c, [&] { CK(cudaStreamSynchronize(c->st)); CK(cudaGetLastError()); });
}

int kf_set_state(kf_ctx *c, const double *ux, const double *uy, const double *uz, const double *s) {
    return guarded(c, [&] {
        if (!ux || !uy || !uz || !s) throw KfError{KF_ERR_ARG, "null state array"};
        const double *src[4] = {ux, uy, uz, s};
        for (int q = 0; q < 4; ++q) put_bulk(c, c->Y[q], src[q], 2 * c->Nc);
        copy_state(c, c->Ys, c->Y);
        c->nhist = 0;
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_get_state(kf_ctx *c, double *ux, double *uy, double *uz, double *s) {
    return guarded(c, [&] {
        double *dst[4] = {ux, uy, uz, s};
        for (int q = 0; q < 4; ++q)
            if (dst[q]) get_bulk(c, dst[q], c->Y[q], 2 * c->Nc);
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_set_sources(kf_ctx *c, const double *nd, const double *mask) {
    return guarded(c, [&] {
        if (nd) CK(cudaMemcpyAsync(c->nd, nd, 8 * c->N, cudaMemcpyHostToDevice, c->st));
        if (mask) put_bulk(c, c->H, mask, c->N);
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_set_phi(kf_ctx *c, const double *phi) {
    return guarded(c, [&] {
        CK(cudaMemcpyAsync(c->phi, phi, 8 * c->N, cudaMemcpyHostToDevice, c->st));
        c->nhist = 0;
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_get_phi(kf_ctx *c, double *phi) {
    return guarded(c, [&] {
        CK(cudaMemcpyAsync(phi, c->phi, 8 * c->N, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_rhs_eval(kf_ctx *c, double t) {
    return guarded(c, [&] {
        c->t_stage = t;  // selects the start of the Poisson solve only
        c->stage_idx = 0;
        copy_state(c, c->Ys, c->Y);
        c->rhs_fn(c);
        copy_state(c, c->Y, c->K);
        copy_state(c, c->Ys, c->K);
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_step_host(kf_ctx *c, int nsteps, double dt, double *ux, double *uy, double *uz, double *s) {
    return guarded(c, [&] {
        if (!ux || !uy || !uz || !s) throw KfError{KF_ERR_ARG, "null state array"};
        if (nsteps < 0) throw KfError{KF_ERR_ARG, "nsteps < 0"};
        double *host[4] = {ux, uy, uz, s};
        if (nsteps > 0 && graph_path(c)) {
            step_host(c, nsteps, dt, host);
            return;
        }
        for (int q = 0; q < 4; ++q) put_bulk(c, c->Y[q], host[q], 2 * c->Nc);
        copy_state(c, c->Ys, c->Y);
        c->nhist = 0;
        for (int k = 0; k < nsteps; ++k) rk4_step(c, dt, nullptr, nullptr, nullptr);
        for (int q = 0; q < 4; ++q) get_bulk(c, host[q], c->Y[q], 2 * c->Nc);
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_rk4_steps(kf_ctx *c, int nsteps, double dt) {
    return guarded(c, [&] {
        if (nsteps < 0) throw KfError{KF_ERR_ARG, "nsteps < 0"};
        // Ys == Y on entry; stage times t, t + dt/2, t + dt/2, t + dt (RKO4.cpp:105-212)
        if (nsteps > 0 && graph_path(c)) {
            rk4_steps_graph(c, nsteps, dt);
            return;
        }
        for (int s = 0; s < nsteps; ++s) rk4_step(c, dt, nullptr, nullptr, nullptr);
        CK(cudaGetLastError());
    });
}

int kf_autotune(kf_ctx *c, int reps, kf_tune_out *out) {
    return guarded(c, [&] { autotune(c, reps > 0 ? reps : 5, out); });
}

int kf_set_tuning(kf_ctx *c, int fft_plan, int rbgs_rows) {
    return guarded(c, [&] {
        if ((fft_plan != 0 && fft_plan != 1) ||
            (rbgs_rows != 0 && rbgs_rows != 4 && rbgs_rows != 8 && rbgs_rows != 16))
            throw KfError{KF_ERR_ARG, "kf_set_tuning: fft_plan 0 or 1, rbgs_rows 0, 4, 8 or 16"};
        if (c->capturing) throw KfError{KF_ERR_ARG, "kf_set_tuning during a capture"};
        const bool changed = fft_plan != c->fftv || rbgs_rows != c->rbgs_by;
        c->fftv = fft_plan;
        c->rbgs_by = rbgs_rows;
        if (changed) drop_graphs(c);
    });
}

int kf_set_coarse_block(kf_ctx *c, int on) {
    return guarded(c, [&] {
        if (on != 0 && on != 1) throw KfError{KF_ERR_ARG, "kf_set_coarse_block: on is 0 or 1"};
        if (c->capturing) throw KfError{KF_ERR_ARG, "kf_set_coarse_block during a capture"};
        if (c->coarse_block == (on == 1)) return;
        c->coarse_block = on == 1;
        cc_setup(c);
        drop_graphs(c);
    });
}

int kf_set_overlap(kf_ctx *c, int on) {
    return guarded(c, [&] {
        if (on != 0 && on != 1) throw KfError{KF_ERR_ARG, "kf_set_overlap: on is 0 or 1"};
        if (c->capturing) throw KfError{KF_ERR_ARG, "kf_set_overlap during a capture"};
        if (c->overlap_d == (on == 1)) return;
        c->overlap_d = on == 1;
        drop_graphs(c);
    });
}

int kf_batch_rk4_steps(kf_ctx *const *ctxs, int nctx, int nsteps, const double *dts) {
    if (!ctxs || !dts || nctx < 0 || nsteps < 0) {
        kf_global_error() = "kf_batch_rk4_steps: invalid argument";
        return KF_ERR_ARG;
    }
    for (int i = 0; i < nctx; ++i) {
        if (!ctxs[i]) {
            kf_global_error() = "kf_batch_rk4_steps: null context";
            return KF_ERR_ARG;
        }
        if (!graph_path(ctxs[i])) {
            ctxs[i]->err = "kf_batch_rk4_steps needs a context whose step can be captured "
                           "(KF_PS_FAS or no Poisson solve, profile off)";
            kf_global_error() = ctxs[i]->err;
            return KF_ERR_ARG;
        }
    }
    int rc = KF_OK;
    std::vector<char> begun(nctx, 0);
    for (int i = 0; i < nctx && rc == KF_OK; ++i) {
        rc = guarded(ctxs[i], [&] { graph_begin(ctxs[i], dts[i]); });
        begun[i] = rc == KF_OK;
        if (rc != KF_OK) kf_global_error() = ctxs[i]->err;
    }
    // step-major: every instance's step s is queued before any step s + 1
    for (int s = 0; s < nsteps && rc == KF_OK; ++s)
        for (int i = 0; i < nctx && rc == KF_OK; ++i) {
            rc = guarded(ctxs[i], [&] { graph_step(ctxs[i]); });
            if (rc != KF_OK) kf_global_error() = ctxs[i]->err;
        }
    for (int i = 0; i < nctx; ++i) {
        if (!begun[i]) continue;
        const int r = guarded(ctxs[i], [&] { graph_end(ctxs[i]); });
        if (r != KF_OK && rc == KF_OK) {
            rc = r;
            kf_global_error() = ctxs[i]->err;
        }
    }
    return rc;
}

int kf_poisson_solve(kf_ctx *c, double *phi_io, const double *rho) {
    int rc = guarded(c, [&] {
        if (!phi_io || !rho) throw KfError{KF_ERR_ARG, "null array"};
        CK(cudaMemcpyAsync(c->phi, phi_io, 8 * c->N, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(c->rho, rho, 8 * c->N, cudaMemcpyHostToDevice, c->st));
        int r = poisson(c);
        CK(cudaMemcpyAsync(phi_io, c->phi, 8 * c->N, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        if (r) throw KfError{KF_ERR_NOT_CONVERGED, "Poisson solve did not reach its tolerance"};
    });
    return rc;
}

int kf_diag(kf_ctx *c, kf_diag_out *out) {
    return guarded(c, [&] {
        if (!out) throw KfError{KF_ERR_ARG, "null output"};
        c->inv_state_fn(c);
        const int nb = red_blocks(c->N);
        Launch L_(c, KC_MISC, (double)c->N * (4 * c->es + 16));
        if (c->fp32)
            k_diag_sums<float><<<nb, RBS, 0, c->st>>>((const float *)c->R[23], (const float *)c->R[20],
                                                     (const float *)c->R[21], (const float *)c->R[22], c->phi, c->nd,
                                                     c->cfg.M, c->N, c->partial, c->vol, c->n);
        else
            k_diag_sums<double><<<nb, RBS, 0, c->st>>>((const double *)c->R[23], (const double *)c->R[20],
                                                      (const double *)c->R[21], (const double *)c->R[22], c->phi,
                                                      c->nd, c->cfg.M, c->N, c->partial, c->vol, c->n);
        k_diag_final<<<1, 32, 0, c->st>>>(c->partial, nb, c->red);
        c->launches++;
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(c->h_red, c->red, sizeof(double) * 2, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        const double h = c->cfg.L / c->n, h3 = h * h * h;
        *out = c->diag;
        out->kinetic = c->h_red[0] * h3;
        out->charge = c->h_red[1] * h3;
    });
}

int kf_fft_r2c(kf_ctx *c, const double *in, double *out) {
    return guarded(c, [&] {
        put_bulk(c, c->R[0], in, c->N);
        c->r2c_fn(c);
        get_bulk(c, out, c->CX[0], 2 * c->Nc);
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_fft_c2r(kf_ctx *c, const double *in, double *out) {
    return guarded(c, [&] {
        put_bulk(c, c->CX[0], in, 2 * c->Nc);
        c->c2r_fn(c);
        get_bulk(c, out, c->R[0], c->N);
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_state_device_ptrs(kf_ctx *c, void **ux, void **uy, void **uz, void **s) {
    return guarded(c, [&] {
        void **o[4] = {ux, uy, uz, s};
        for (int q = 0; q < 4; ++q)
            if (o[q]) *o[q] = c->Y[q];
    });
}

long long kf_launch_count(const kf_ctx *c) { return c ? c->launches : -1; }

int kf_profile_enable(kf_ctx *c, int on) {
    return guarded(c, [&] {
        prof_flush(c);
        for (int k = 0; k < KC_N; ++k) {
            c->prof_ms[k] = 0.;
            c->prof_bytes[k] = 0.;
            c->prof_n[k] = 0;
        }
        c->prof = on != 0;
    });
}

int kf_profile_read(kf_ctx *c, int cls, double *ms, long long *launches, double *bytes) {
    return guarded(c, [&] {
        if (cls < 0 || cls >= KC_N) throw KfError{KF_ERR_ARG, "kernel class out of range"};
        prof_flush(c);
        if (ms) *ms = c->prof_ms[cls];
        if (launches) *launches = c->prof_n[cls];
        if (bytes) *bytes = c->prof_bytes[cls];
    });
}

const char *kf_profile_class_name(int cls) { return (cls >= 0 && cls < KC_N) ? kKClsName[cls] : ""; }

}  // extern "C"
