/*
 * kf_oracle.cpp -- CPU restatement of the reference's RK4 time-step hot path.
 *
 * TEST INFRASTRUCTURE.  This is the restatement the CUDA path is compared with; it
 * is never linked into kielflow_b200/.  Every function cites the reference code
 * it restates (paths relative to the reference project).  The arithmetic is kept
 * in the reference's operation order so that, with the same FFT (fftw_shim.c)
 * and -ffp-contract=off, the shipped configuration reproduces the reference
 * compiled here (oracle/_ref) bit for bit; the tests pin that.
 *
 * Additions the reference's driver does not enable (each switchable at run time):
 *  - KFO_DIFFUSION: Laplacian diffusion  d/dt q += -D |k|^2 q^  (the formula of
 *    effect_diffusion.cpp:16-44, without its re/im slip at :39-40);
 *  - KFO_PENALIZATION: masking penalization of the finished right-hand side,
 *    f <- (1-H) f + H eta_d (q - q_fix)   (effect_penalization.cpp:35), applied
 *    in physical space and followed by the 2/3 filter as rhs_standard.cpp:491-532
 *    does for its own penalization block;
 *  - sv_cut: spectral viscosity only where |k~| > sv_cut;
 *  - KFO_PS_JACOBI_RES: the Jacobi sweeps of solver_poisson_jacobi_nlin with a
 *    max-norm residual stop;
 *  - KFO_PS_FAS: an FAS V-cycle (red-black point-Newton smoother built from
 *    iteration_loop's point update, optionally over-relaxed by mg_omega,
 *    injection for phi, full weighting for the
 *    residual, the trilinear OP_hto2h for the correction).
 */
#include "kf_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

extern "C" {
#include "fftw3.h"
}

namespace {

typedef std::vector<double> vec;

/* f(i) for i in [0, n) on the host's cores (kfs_parallel): every use below
 * gives each i work whose result does not depend on any other i (pointwise
 * passes, independent transform lines, the points of one red-black colour,
 * per-plane partial maxima), so the threads change no result; the sums whose
 * order matters (the Jacobi sweep's statistics) stay sequential. */
template <class F> void par_for(long n, long min_items, const F &f) {
    kfs_parallel(
        n, min_items,
        [](long b, long e, void *ctx) {
            const F &g = *static_cast<const F *>(ctx);
            for (long i = b; i < e; ++i) g(i);
        },
        (void *)&f);
}

/* axis_CoEqSt (axis_EqSt.cpp:52-61) and, with m > 0, axis_CoSiSt: the
 * periodic sine-stretched axis x = S(l0 + L i/N), S(x) = x - m sin(2 pi x/L)
 * (axis_SiSt.cpp:93-116 val_at, :153-164 S and dS; k_val_at :120-124 is the
 * equidistant one). */
struct axis_eq {
    double l0, L;
    int N;
    double m = 0.;
    double S(double x) const {
        const double pi = acos(-1.);
        return x - m * sin(2. * pi * x / L);
    }
    double val_at(int index) const {
        if (m == 0.) return l0 + index * (L / N);
        int shift = 0;
        if (index < 0) {
            do {
                shift += 1;
            } while (index + shift * N < 0);
        }
        if (index >= N) {
            do {
                shift -= 1;
            } while (index + shift * N >= N - 1);
        }
        double x = l0 + L * double(index + shift * N) / (N);
        return S(x) - shift * L;
    }
    double dS(int index) const {
        const double pi = acos(-1.);
        double x = l0 + (L / N) * index;
        return 1. - (2. * pi * m / L) * cos(2. * pi * x / L);
    }
    double k_val_at(int i) const {
        double pi = acos(-1.);
        return ((i <= N / 2) ? (2. * pi * i / L) : (2. * pi * (i - N) / L));
    }
};

/* Point Newton solve of A - D x - exp(x) = 0 (newton_method.hpp:16-63 with the
 * lambdas of solver_poisson_jacobi_nlin.cpp:197-199). */
inline double newton_point(double x, double A, double D) {
    const double eps = 0.05;
    const int Nmax = 20;
    double omega = 1.;
    double g = 0.8;
    double dx = 0.;
    double dx_alt = (A - D * x - exp(x)) / (-D - exp(x));
    int i = 0;
    do {
        x -= omega * dx;
        dx = (A - D * x - exp(x)) / (-D - exp(x));
        omega = fabs(dx) > fabs(dx_alt) ? g * omega : (1. - g) * omega + g * 1.;
        dx_alt = dx;
        ++i;
    } while (fabs(dx) > eps && i < Nmax);
    return x - dx;
}

/* Per-level stencil coefficients from the axis spacings
 * (solver_poisson_jacobi_nlin.cpp:112-126 H_create, :177-189). */
struct level {
    int n;
    axis_eq ax;
    vec H;                  /* H[i] = val_at(i) - val_at(i-1), i = 0..n */
    vec dd, den_p, den_m;   /* 2/(H[i+1]H[i]), H[i+1](H[i+1]+H[i]), H[i](H[i+1]+H[i]) */
    vec inv_p, inv_m;       /* 2/den_p, 2/den_m: stencil weights of the FAS cycle      */
    void init(int n_, double L, double m) {
        n = n_;
        ax.l0 = -0.5 * L;
        ax.L = L;
        ax.N = n_;
        ax.m = m;
        H.resize(n + 1);
        for (int i = 0; i < n + 1; ++i) H[i] = ax.val_at(i) - ax.val_at(i - 1);
        dd.resize(n);
        den_p.resize(n);
        den_m.resize(n);
        inv_p.resize(n);
        inv_m.resize(n);
        for (int i = 0; i < n; ++i) {
            dd[i] = 2. / (H[i + 1] * H[i]);
            den_p[i] = H[i + 1] * (H[i + 1] + H[i]);
            den_m[i] = H[i] * (H[i + 1] + H[i]);
            inv_p[i] = 2. / den_p[i];
            inv_m[i] = 2. / den_m[i];
        }
    }
    inline size_t idx(int i, int j, int k) const { return (size_t)k + n * ((size_t)j + (size_t)i * n); }
    inline int wrap(int i) const { return i < 0 ? i + n : (i >= n ? i - n : i); }
    /* D and A of iteration_loop (:177-189) at (i,j,k) for field p and source rho */
    inline void coeffs(const double *p, const double *rho, int i, int j, int k, double &A,
                       double &D) const {
        D = 2. / (H[i + 1] * H[i]);
        D += 2. / (H[j + 1] * H[j]);
        D += 2. / (H[k + 1] * H[k]);
        A = p[idx(wrap(i + 1), j, k)] / den_p[i];
        A += p[idx(wrap(i - 1), j, k)] / den_m[i];
        A += p[idx(i, wrap(j + 1), k)] / den_p[j];
        A += p[idx(i, wrap(j - 1), k)] / den_m[j];
        A += p[idx(i, j, wrap(k + 1))] / den_p[k];
        A += p[idx(i, j, wrap(k - 1))] / den_m[k];
        A = 2. * A;
        A += rho[idx(i, j, k)];
    }
    /* pointwise residual f(phi) = A - D phi - exp(phi) = lap_h phi + rho - e^phi */
    inline double resid(const double *p, const double *rho, int i, int j, int k) const {
        double A, D;
        coeffs(p, rho, i, j, k, A, D);
        double x = p[idx(i, j, k)];
        return A - D * x - exp(x);
    }
    /* the same stencil with the weights 2/den precomputed (FAS cycle): the
     * factor 2 of :187 is folded into the weights, the divisions become products */
    inline void coeffs_fast(const double *p, const double *rho, int i, int j, int k, double &A,
                            double &D) const {
        D = dd[i] + dd[j] + dd[k];
        A = p[idx(wrap(i + 1), j, k)] * inv_p[i];
        A += p[idx(wrap(i - 1), j, k)] * inv_m[i];
        A += p[idx(i, wrap(j + 1), k)] * inv_p[j];
        A += p[idx(i, wrap(j - 1), k)] * inv_m[j];
        A += p[idx(i, j, wrap(k + 1))] * inv_p[k];
        A += p[idx(i, j, wrap(k - 1))] * inv_m[k];
        if (rho) A += rho[idx(i, j, k)];
    }
    inline double resid_fast(const double *p, const double *rho, int i, int j, int k) const {
        double A, D;
        coeffs_fast(p, rho, i, j, k, A, D);
        double x = p[idx(i, j, k)];
        return A - D * x - exp(x);
    }
};

}  // namespace

struct kfo_ctx {
    kfo_config cfg;
    int n, nzc;
    size_t N, Nc;
    axis_eq ax;
    vec kv;                    /* k_val_at(i) */
    vec P, SV, PF, K2;         /* dealias mask, SV table, phi filter, |k|^2  (Nc) */
    vec FU[3], Fs;             /* state (interleaved complex) */
    bool stretched = false;    /* axis_CoSiSt: derivatives take the chain-rule path */
    vec dsv[3];                /* filtered 1/dS per direction (N), OP_partial_derivative.cpp:60-80 */
    vec Phi, nd, mask;         /* real fields */
    /* Jacobi solver state that persists across calls (solver_poisson_jacobi_nlin.hpp:66-95) */
    double norm_max = 0., norm_sum = 0., norm_max_old = -1., norm_sum_old = -1.;
    double supremum = 0., infinum = 0., omega_SOR = 1.;
    kfo_poisson_stats stats{};
    std::vector<level> lv;     /* lv[0] finest */
    /* time of the RK4 driver (Runge_kutta_O4::t_, RKO4.cpp:42,240) and the phi
     * history used to extrapolate the start of each solve at a new time */
    double t = 0.;
    vec phi_a;
    double tau_a = 0., tau_b = 0.;
    int nhist = 0;
};

namespace {

void r2c(const kfo_ctx *c, const vec &in, vec &out) {
    out.resize(2 * c->Nc);
    kfs_r2c_3d(c->n, c->n, c->n, in.data(), out.data());
}

/* OP_iFFT::operator() (OP_iFFT.cpp:49-64): c2r then scale by Norm = 1/N */
void c2r(const kfo_ctx *c, const vec &in, vec &out) {
    out.resize(c->N);
    kfs_c2r_3d(c->n, c->n, c->n, in.data(), out.data());
    double Norm = 1. / ((double)c->N);
    par_for((long)(c->N), 16384, [&](long i) { out[i] = out[i] * Norm; });
}

/* OP_dealiasing::operator() (OP_dealiasing.cpp:5-13) */
void dealias(const kfo_ctx *c, vec &F) {
    par_for((long)c->Nc, 16384, [&](long i) {
        F[2 * i] *= c->P[i];
        F[2 * i + 1] *= c->P[i];
    });
}

/* effect_penalization::execute (effect_penalization.cpp:21-44), masking form,
 * on one finished right-hand-side field: out <- r2c((1 - H) c2r(out)
 * + H eta_d (q - q_fix)), with q the field's state in physical space
 * (the reference forms it as iFFT of its `in`); b: scratch */
void penalize(const kfo_ctx *c, const vec &q, double fix, vec &out, vec &b) {
    c2r(c, out, b);
    par_for((long)c->N, 16384,
            [&](long i) { b[i] = (1. - c->mask[i]) * b[i] + c->mask[i] * c->cfg.pen_eta * (q[i] - fix); });
    r2c(c, b, out);
}

/* OP_partial_derivative::operator() (OP_partial_derivative.cpp:104-136): i k
 * times the input; on a stretched axis, then dealiased, taken to physical
 * space, multiplied by the filtered 1/dS of the direction and transformed back. */
void deriv(const kfo_ctx *c, int dir, const vec &in, vec &out) {
    out.resize(2 * c->Nc);
    const int n = c->n, nzc = c->nzc;
    par_for(n, 1, [&](long i) {
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < nzc; ++k) {
                size_t ijk = (size_t)k + nzc * ((size_t)j + (size_t)i * n);
                int q = dir == 0 ? (int)i : (dir == 1 ? j : k);
                double kk = c->kv[q];
                double tmp = in[2 * ijk];
                out[2 * ijk] = -kk * in[2 * ijk + 1];
                out[2 * ijk + 1] = kk * tmp;
            }
    });
    if (!c->stretched) return;
    dealias(c, out);
    vec t;
    c2r(c, out, t);
    const vec &d = c->dsv[dir];
    par_for((long)(c->N), 16384, [&](long i) { t[i] = t[i] * d[i]; });
    r2c(c, t, out);
}

void add(vec &a, const vec &b) {
    par_for((long)(a.size()), 16384, [&](long i) { a[i] += b[i]; });
}

/* ------------------------------------------------------------ Poisson solvers */

/* One Jacobi sweep: iteration_loop (solver_poisson_jacobi_nlin.cpp:140-265)
 * without the unused boundary branch.  Returns max |f(P_old)| (the residual of
 * the input iterate) for the residual stop. */
double jacobi_sweep(kfo_ctx *c, const level &L, const vec &in, vec &out, const vec &rho,
                    int iteration, bool &converged, double limit_max) {
    c->norm_sum_old = c->norm_sum;
    c->norm_max_old = c->norm_max;
    c->norm_max = 0.;
    c->norm_sum = 0.;
    c->supremum = in[0];
    c->infinum = in[0];
    double rmax = 0.;
    const int n = L.n;
    const size_t N = (size_t)n * n * n;
    /* the point updates on the host's cores; the statistics in the
     * reference's point order (its sums are order dependent) */
    vec pnew(N), f0a(N);
    const double om = c->omega_SOR;
    par_for(n, 1, [&](long i) {
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                double A, D;
                L.coeffs(in.data(), rho.data(), (int)i, j, k, A, D);
                const size_t q = L.idx((int)i, j, k);
                double P_old = in[q];
                f0a[q] = A - D * P_old - exp(P_old);
                double P_new = newton_point(P_old, A, D);
                pnew[q] = P_new;
                out[q] = (1. - om) * P_old + om * P_new;
            }
    });
    for (size_t q = 0; q < N; ++q) {
        const double f0 = f0a[q], P_new = pnew[q];
        if (fabs(f0) > rmax) rmax = fabs(f0);
        double delta = fabs(P_new - in[q]);
        c->supremum = (P_new < c->supremum) ? c->supremum : P_new; /* max<double> (o_math.hpp) */
        c->infinum = !(P_new < c->infinum) ? c->infinum : P_new;   /* min<double> (o_math.hpp) */
        c->norm_max = (delta < c->norm_max) ? c->norm_max : delta;
        c->norm_sum += delta;
    }
    /* Carre's SOR factor (:237-252) */
    c->norm_sum = c->norm_sum / ((double)L.n * L.n * L.n);
    if ((c->norm_max < c->norm_max_old) && (iteration > 1)) {
        double lambda = c->norm_sum / c->norm_sum_old;
        double omega_new =
            2. / (1. + sqrt(1. - pow(lambda + c->omega_SOR - 1., 2.) /
                                     (lambda * pow(c->omega_SOR, 2.))));
        c->omega_SOR = omega_new;
    } else {
        c->omega_SOR = .5;
    }
    if (c->omega_SOR != c->omega_SOR) c->omega_SOR = .5;
    if (c->norm_max < limit_max * (c->supremum - c->infinum)) converged = true;
    return rmax;
}

/* solver_poisson_jacobi_nlin::solve (:50-108).  residual_stop selects the
 * max-norm residual test instead of the relative-update test of :258. */
int jacobi_solve(kfo_ctx *c, const level &L, vec &phi, const vec &rho, int &max_iterations,
                 double limit_max, bool residual_stop, double res_tol) {
    c->supremum = 0.;
    c->infinum = 0.;
    int iteration = 0;
    c->omega_SOR = 1.;
    bool converged = false;
    c->norm_sum_old = -1.;
    vec Phi_n(phi.size());
    if (max_iterations < 0) max_iterations = 1000;
    while (!converged && (iteration < max_iterations)) {
        iteration++;
        bool conv_rel = false;
        double r = jacobi_sweep(c, L, phi, Phi_n, rho, iteration, conv_rel, limit_max);
        phi = Phi_n;
        if (residual_stop) {
            c->stats.last_residual = r;
            converged = r <= res_tol;
        } else {
            converged = conv_rel;
        }
    }
    c->stats.last_iterations = iteration;
    c->stats.total_iterations += iteration;
    if (!converged) c->stats.not_converged++;
    return iteration;
}

/* OP_2htoh_lvl0 / OP_4htoh / OP_8htoh: injection (field_interpolation.cpp:233-315) */
void inject(int nf, int step, const vec &in, vec &out) {
    int nc = nf / step;
    out.assign((size_t)nc * nc * nc, 0.);
    par_for(nc, 1, [&](long i) {
        for (int j = 0; j < nc; ++j)
            for (int k = 0; k < nc; ++k)
                out[(size_t)k + nc * ((size_t)j + (size_t)i * nc)] =
                    in[(size_t)(step * k) + nf * ((size_t)(step * j) + (size_t)(step * i) * nf)];
    });
}

/* OP_hto2h: trilinear prolongation in z, then y, then x passes
 * (field_interpolation.cpp:56-147), on the axis of the fine level. */
void prolong(int nc, double L, double m, const vec &in, vec &out) {
    int nf = 2 * nc;
    axis_eq ax{-0.5 * L, L, nf, m};
    out.assign((size_t)nf * nf * nf, 0.);
    auto id = [nf](int i, int j, int k) { return (size_t)k + nf * ((size_t)j + (size_t)i * nf); };
    auto w = [nf](int i) { return i < 0 ? i + nf : (i > nf - 1 ? i - nf : i); };
    /* each pass reads only points the earlier passes wrote */
    par_for(nc, 1, [&](long i) {
        for (int j = 0; j < nc; j++)
            for (int k = 0; k < nc; k++)
                out[id(2 * (int)i, 2 * j, 2 * k)] = in[(size_t)k + nc * ((size_t)j + (size_t)i * nc)];
    });
    par_for(nf / 2, 1, [&](long ii) {
        const int i = 2 * (int)ii;
        for (int j = 0; j < nf; j += 2)
            for (int k = 1; k < nf; k += 2) {
                double z1 = ax.val_at(k - 1), z2 = ax.val_at(k + 1), z = ax.val_at(k);
                double g = (z - z1) / (z2 - z1);
                out[id(i, j, k)] = (1. - g) * out[id(i, j, w(k - 1))] + g * out[id(i, j, w(k + 1))];
            }
    });
    par_for(nf / 2, 1, [&](long ii) {
        const int i = 2 * (int)ii;
        for (int j = 1; j < nf; j += 2) {
            double y1 = ax.val_at(j - 1), y2 = ax.val_at(j + 1), y = ax.val_at(j);
            double g = (y - y1) / (y2 - y1);
            for (int k = 0; k < nf; k += 1)
                out[id(i, j, k)] = (1. - g) * out[id(i, w(j - 1), k)] + g * out[id(i, w(j + 1), k)];
        }
    });
    par_for(nf / 2, 1, [&](long ii) {
        const int i = 2 * (int)ii + 1;
        double x1 = ax.val_at(i - 1), x2 = ax.val_at(i + 1), x = ax.val_at(i);
        double g = (x - x1) / (x2 - x1);
        for (int j = 0; j < nf; j += 1)
            for (int k = 0; k < nf; k += 1)
                out[id(i, j, k)] = (1. - g) * out[id(w(i - 1), j, k)] + g * out[id(w(i + 1), j, k)];
    });
}

/* Full-weighting restriction n -> n/2 (new for the FAS cycle): tensor product of
 * (1/4, 1/2, 1/4) around the injected point, periodic, summed x-outer, z-inner. */
void restrict_fw(int nf, const vec &in, vec &out) {
    int nc = nf / 2;
    out.assign((size_t)nc * nc * nc, 0.);
    const double w[3] = {0.25, 0.5, 0.25};
    par_for(nc, 1, [&](long il) {
        const int i = (int)il;
        for (int j = 0; j < nc; ++j)
            for (int k = 0; k < nc; ++k) {
                double s = 0.;
                for (int a = -1; a <= 1; ++a) {
                    int I = (2 * i + a + nf) % nf;
                    double sy = 0.;
                    for (int b = -1; b <= 1; ++b) {
                        int J = (2 * j + b + nf) % nf;
                        double sz = 0.;
                        for (int cc = -1; cc <= 1; ++cc) {
                            int K = (2 * k + cc + nf) % nf;
                            sz += w[cc + 1] * in[(size_t)K + nf * ((size_t)J + (size_t)I * nf)];
                        }
                        sy += w[b + 1] * sz;
                    }
                    s += w[a + 1] * sy;
                }
                out[(size_t)k + nc * ((size_t)j + (size_t)i * nc)] = s;
            }
    });
}

double max_resid(const level &L, const vec &phi, const vec &rho) {
    /* per-plane maxima, then their maximum: f > r never takes a NaN, and the
     * maximum of the other values does not depend on the order */
    vec rp(L.n, 0.);
    par_for(L.n, 1, [&](long i) {
        double r = 0.;
        for (int j = 0; j < L.n; ++j)
            for (int k = 0; k < L.n; ++k) {
                double f = fabs(L.resid(phi.data(), rho.data(), (int)i, j, k));
                if (f > r) r = f;
            }
        rp[i] = r;
    });
    double r = 0.;
    for (double v : rp)
        if (v > r) r = v;
    return r;
}

double max_resid_fast(const level &L, const vec &phi, const vec &rho) {
    /* per-plane maxima, then their maximum: f > r never takes a NaN, and the
     * maximum of the other values does not depend on the order */
    vec rp(L.n, 0.);
    par_for(L.n, 1, [&](long i) {
        double r = 0.;
        for (int j = 0; j < L.n; ++j)
            for (int k = 0; k < L.n; ++k) {
                double f = fabs(L.resid_fast(phi.data(), rho.data(), (int)i, j, k));
                if (f > r) r = f;
            }
        rp[i] = r;
    });
    double r = 0.;
    for (double v : rp)
        if (v > r) r = v;
    return r;
}

/* Red-black Gauss-Seidel-Newton sweep: at each point one Newton step on the
 * point equation A - D x - e^x = 0 of iteration_loop (:177-199), in place,
 * colour (i+j+k)%2 == 0 first. */
void rbgs_sweep(const level &L, vec &phi, const vec &rho, double om) {
    /* the points of one colour read only points of the other */
    for (int color = 0; color < 2; ++color)
        par_for(L.n, 1, [&](long il) {
            const int i = (int)il;
            for (int j = 0; j < L.n; ++j)
                for (int k = (i + j + color) & 1; k < L.n; k += 2) {
                    double A, D;
                    L.coeffs_fast(phi.data(), rho.data(), i, j, k, A, D);
                    const size_t q = L.idx(i, j, k);
                    const double x = phi[q], ex = exp(x);
                    phi[q] = x - om * ((A - D * x - ex) / (-D - ex));
                }
        });
}

/* N(phi) = -lap_h phi + e^phi = -f(phi; rho = 0) at every point */
void apply_N(const level &L, const vec &phi, vec &out) {
    out.resize(phi.size());
    par_for(L.n, 1, [&](long i) {
        for (int j = 0; j < L.n; ++j)
            for (int k = 0; k < L.n; ++k) {
                size_t q = L.idx((int)i, j, k);
                out[q] = 0. - L.resid_fast(phi.data(), nullptr, (int)i, j, k);
            }
    });
}

void fas_head(kfo_ctx *c, int l, vec &phi, const vec &rho, vec &r);
void fas_tail(kfo_ctx *c, int l, vec &phi, const vec &rho, const vec &r);

void fas_vcycle(kfo_ctx *c, int l, vec &phi, const vec &rho) {
    const level &L = c->lv[l];
    const kfo_config &cf = c->cfg;
    const double om = cf.mg_omega > 0. ? cf.mg_omega : 1.; /* over-relaxed point Newton step */
    if (l == (int)c->lv.size() - 1) {
        /* coarsest level: relaxed until its max residual is at most
           max(coarse_tol, 1e-4 x its value at entry), at most 1000 sweeps */
        double r0 = 0.;
        for (int s = 0; s < 1000; ++s) {
            const double r = max_resid_fast(L, phi, rho);
            if (s == 0) r0 = r;
            if (r <= std::max(cf.coarse_tol, 1e-4 * r0)) break;
            rbgs_sweep(L, phi, rho, om);
        }
        return;
    }
    vec r;
    fas_head(c, l, phi, rho, r);
    fas_tail(c, l, phi, rho, r);
}

/* first part of a V-cycle on level l (not the coarsest): pre-smoothing and the
 * residual r of the pre-smoothed iterate */
void fas_head(kfo_ctx *c, int l, vec &phi, const vec &rho, vec &r) {
    const level &L = c->lv[l];
    const kfo_config &cf = c->cfg;
    const double om = cf.mg_omega > 0. ? cf.mg_omega : 1.;
    for (int s = 0; s < cf.mg_pre; ++s) rbgs_sweep(L, phi, rho, om);
    r.assign(phi.size(), 0.);
    par_for(L.n, 1, [&](long i) {
        for (int j = 0; j < L.n; ++j)
            for (int k = 0; k < L.n; ++k)
                r[L.idx((int)i, j, k)] = L.resid_fast(phi.data(), rho.data(), (int)i, j, k);
    });
}

/* the rest: restriction, the coarse cycle, the correction, post-smoothing */
void fas_tail(kfo_ctx *c, int l, vec &phi, const vec &rho, const vec &r) {
    const level &L = c->lv[l];
    const kfo_config &cf = c->cfg;
    const double om = cf.mg_omega > 0. ? cf.mg_omega : 1.;
    vec phic, rc, Nc, rhoc;
    inject(L.n, 2, phi, phic);
    restrict_fw(L.n, r, rc);
    const level &Lc = c->lv[l + 1];
    apply_N(Lc, phic, Nc); /* -lap_c phic + e^phic */
    rhoc.resize(phic.size());
    par_for((long)(phic.size()), 16384, [&](long q) { rhoc[q] = Nc[q] + rc[q]; });
    vec phic0 = phic;
    fas_vcycle(c, l + 1, phic, rhoc);
    par_for((long)(phic.size()), 16384, [&](long q) { phic[q] = phic[q] - phic0[q]; });
    vec e;
    prolong(Lc.n, cf.L, cf.stretch_m, phic, e);
    par_for((long)(phi.size()), 16384, [&](long q) { phi[q] += e[q]; });
    for (int s = 0; s < cf.mg_post; ++s) rbgs_sweep(L, phi, rho, om);
}

/* solver_poisson_multigrid::solve with the plan of kielflow.cpp:207-217
 * (solver_poisson_multigrid.cpp:246-418): {down3, up, up, up}, steps {0,-1,-1,-1},
 * tolerances {1e-2, 5e-4, 1e-4, 1e-4}, each level relaxed by the Jacobi solver. */
void cascadic_solve(kfo_ctx *c, vec &phi, const vec &rho) {
    const int n = c->n;
    const int steps[4] = {0, -1, -1, -1};
    const double tol[4] = {0.01, 0.0005, 0.0001, 0.0001};
    vec cur = phi, nxt;
    int ncur = n;
    for (int cas = 0; cas < 4; ++cas) {
        if (cas == 0) {
            inject(ncur, 8, cur, nxt);
            ncur /= 8;
        } else {
            prolong(ncur, c->cfg.L, c->cfg.stretch_m, cur, nxt);
            ncur *= 2;
        }
        vec rho_n;
        inject(n, n / ncur, rho, rho_n); /* repeated injection == one strided injection */
        level L;
        L.init(ncur, c->cfg.L, c->cfg.stretch_m);
        int max_it = steps[cas];
        jacobi_solve(c, L, nxt, rho_n, max_it, tol[cas], false, 0.);
        cur.swap(nxt);
    }
    phi.swap(cur);
}

int poisson(kfo_ctx *c, vec &phi, const vec &rho) {
    const kfo_config &cf = c->cfg;
    c->stats.solves++;
    if (cf.poisson_mode == KFO_PS_JACOBI_REF || cf.poisson_mode == KFO_PS_JACOBI_RES) {
        int max_it = cf.nlj_max_it;
        jacobi_solve(c, c->lv[0], phi, rho, max_it, cf.nlj_limit,
                     cf.poisson_mode == KFO_PS_JACOBI_RES, cf.res_tol);
        if (cf.poisson_mode == KFO_PS_JACOBI_REF) c->stats.last_residual = max_resid(c->lv[0], phi, rho);
    } else if (cf.poisson_mode == KFO_PS_CASCADIC) {
        cascadic_solve(c, phi, rho);
        c->stats.last_residual = max_resid(c->lv[0], phi, rho);
    } else if (cf.res_tol > 0. && c->lv.size() > 1) {
        /* the stop test runs on the residual of each cycle's pre-smoothed
         * iterate (the one the cycle restricts); the rest of the cycle only
         * when it fails, so the returned phi has the tested residual */
        int cyc = 0;
        double r = 0.;
        vec rv;
        for (;;) {
            fas_head(c, 0, phi, rho, rv);
            r = 0.;
            for (double v : rv) {
                const double a = std::fabs(v);
                if (a != a) {
                    r = a;
                    break;
                }
                r = std::max(r, a);
            }
            if (!(r > cf.res_tol) || cyc >= cf.max_cycles) break;
            fas_tail(c, 0, phi, rho, rv);
            ++cyc;
        }
        c->stats.last_iterations = cyc;
        c->stats.total_iterations += cyc;
        c->stats.last_residual = r;
        if (r > cf.res_tol) c->stats.not_converged++;
    } else {
        double r = max_resid_fast(c->lv[0], phi, rho);
        int cyc = 0;
        while (r > cf.res_tol && cyc < cf.max_cycles) {
            fas_vcycle(c, 0, phi, rho);
            ++cyc;
            r = max_resid_fast(c->lv[0], phi, rho);
        }
        c->stats.last_iterations = cyc;
        c->stats.total_iterations += cyc;
        c->stats.last_residual = r;
        if (r > cf.res_tol) c->stats.not_converged++;
    }
    for (double v : phi)
        if (v != v) return -3;
    return 0;
}

/* ------------------------------------------------------------------ the RHS */

/* Start of the Poisson solve at time t: with two earlier solutions at distinct
 * times, phi <- phi_b + (t - tau_b)/(tau_b - tau_a) (phi_b - phi_a). */
void phi_guess(kfo_ctx *c, double t, bool &newtime) {
    newtime = c->nhist == 0 || t != c->tau_b;
    if (!c->cfg.phi_extrap || !newtime || c->nhist == 0) return;
    if (c->nhist >= 2) {
        const double w = (t - c->tau_b) / (c->tau_b - c->tau_a);
        par_for((long)c->N, 16384, [&](long i) {
            const double b = c->Phi[i], a = c->phi_a[i];
            c->Phi[i] = b + w * (b - a);
            c->phi_a[i] = b;
        });
    } else {
        c->phi_a = c->Phi;
    }
    c->tau_a = c->tau_b;
}

void phi_record(kfo_ctx *c, double t, bool newtime) {
    if (!c->cfg.phi_extrap || !newtime) return;
    c->nhist = c->nhist < 2 ? c->nhist + 1 : 2;
    c->tau_b = t;
}

/* rhs_standard::solve (rhs_standard.cpp:89-566) with runtime term switches. */
int rhs(kfo_ctx *c, vec *FU, vec &Fni, double t) {
    const int T = c->cfg.terms;
    const kfo_config &cf = c->cfg;
    const size_t Nc = c->Nc, N = c->N;
    vec F1(2 * Nc), F2(2 * Nc), b1(N), b2(N), FBu[3], FBn(2 * Nc);
    for (int q = 0; q < 3; ++q) FBu[q].assign(2 * Nc, 0.);
    int rc = 0;
    /* [Poisson] :100-113 */
    if ((T & KFO_POISSON) && (T & KFO_E_INT)) {
        F1 = Fni;
        dealias(c, F1);
        c2r(c, F1, b1);
        par_for((long)(N), 16384, [&](long i) { b1[i] = exp(b1[i]) + c->nd[i]; });
        bool newtime;
        phi_guess(c, t, newtime);
        rc = poisson(c, c->Phi, b1);
        if (rc) return rc;
        phi_record(c, t, newtime);
    }
    /* [dissipation & spectral viscosity] :119-209 */
    const bool diss = T & KFO_DISSIPATION, sv = T & KFO_SVISCOSITY;
    par_for((long)Nc, 16384, [&](long i) {
        for (int q = 0; q < 3; ++q)
            for (int ri = 0; ri < 2; ++ri) {
                double u = FU[q][2 * i + ri];
                FBu[q][2 * i + ri] = diss && sv ? (cf.tau + c->SV[i]) * u
                                   : diss       ? cf.tau * u
                                   : sv         ? c->SV[i] * u
                                                : 0.;
            }
        for (int ri = 0; ri < 2; ++ri) FBn[2 * i + ri] = sv ? c->SV[i] * Fni[2 * i + ri] : 0.;
    });
    /* [Laplacian diffusion] (new term; -D |k|^2 q^ in d/dt, +D |k|^2 q^ in FB) */
    if (T & KFO_DIFFUSION) {
        par_for((long)Nc, 16384, [&](long i) {
            for (int ri = 0; ri < 2; ++ri) {
                for (int q = 0; q < 3; ++q) FBu[q][2 * i + ri] += cf.diff_D * c->K2[i] * FU[q][2 * i + ri];
                FBn[2 * i + ri] += cf.diff_D * c->K2[i] * Fni[2 * i + ri];
            }
        });
    }
    /* [E-force + pressure] :218-248 */
    const bool pres = T & KFO_PRESSURE, eint = T & KFO_E_INT;
    if (pres || eint) {
        if (eint) {
            r2c(c, c->Phi, F1);
            if (pres)
                par_for((long)Nc, 16384, [&](long i) {
                    F1[2 * i] *= c->PF[i];
                    F1[2 * i + 1] *= c->PF[i];
                });
        }
        if (pres && eint) {
            par_for((long)Nc, 16384, [&](long i) {
                F1[2 * i] += Fni[2 * i] / cf.theta;
                F1[2 * i + 1] += Fni[2 * i + 1] / cf.theta;
            });
        } else if (pres) {
            par_for((long)Nc, 16384, [&](long i) {
                F1[2 * i] = Fni[2 * i] / cf.theta;
                F1[2 * i + 1] = Fni[2 * i + 1] / cf.theta;
            });
        }
        for (int d = 0; d < 3; ++d) {
            deriv(c, d, F1, F2);
            add(FBu[d], F2);
        }
    }
    /* [prep] :253-273 */
    for (int q = 0; q < 3; ++q) dealias(c, FU[q]);
    dealias(c, Fni);
    vec U[3];
    for (int q = 0; q < 3; ++q) c2r(c, FU[q], U[q]);
    vec dFU[3][3]; /* dFU[c][d] = d_d FU_c */
    for (int q = 0; q < 3; ++q)
        for (int d = 0; d < 3; ++d) deriv(c, d, FU[q], dFU[q][d]);
    /* [mean flow] :279-311 */
    if (T & KFO_E_EXT) {
        for (int q = 0; q < 3; ++q)
            par_for((long)(2 * Nc), 16384, [&](long i) { FBu[q][i] += cf.M * dFU[q][0][i]; });
        deriv(c, 0, Fni, F1);
        par_for((long)(2 * Nc), 16384, [&](long i) { FBn[i] += cf.M * F1[i]; });
    }
    /* [continuity] :315-345 */
    if (T & KFO_CONTINUITY) {
        add(FBn, dFU[0][0]);
        add(FBn, dFU[1][1]);
        add(FBn, dFU[2][2]);
        if (!(T & KFO_E_EXT)) deriv(c, 0, Fni, F1); /* :322 relies on :305 */
        dealias(c, F1);
        c2r(c, F1, b1);
        par_for((long)(N), 16384, [&](long i) { b2[i] = b1[i] * U[0][i]; });
        deriv(c, 1, Fni, F1);
        dealias(c, F1);
        c2r(c, F1, b1);
        par_for((long)(N), 16384, [&](long i) { b2[i] += b1[i] * U[1][i]; });
        deriv(c, 2, Fni, F1);
        dealias(c, F1);
        c2r(c, F1, b1);
        par_for((long)(N), 16384, [&](long i) { b2[i] += b1[i] * U[2][i]; });
        r2c(c, b2, F1);
        add(FBn, F1);
    }
    /* [advection] :388-439 */
    if (T & KFO_ADVECTION) {
        for (int q = 0; q < 3; ++q)
            for (int d = 0; d < 3; ++d) dealias(c, dFU[q][d]);
        for (int q = 0; q < 3; ++q) {
            c2r(c, dFU[q][0], b1);
            par_for((long)(N), 16384, [&](long i) { b2[i] = U[0][i] * b1[i]; });
            c2r(c, dFU[q][1], b1);
            par_for((long)(N), 16384, [&](long i) { b2[i] += U[1][i] * b1[i]; });
            c2r(c, dFU[q][2], b1);
            par_for((long)(N), 16384, [&](long i) { b2[i] += U[2][i] * b1[i]; });
            r2c(c, b2, F1);
            add(FBu[q], F1);
        }
    }
    /* [out] :538-560 */
    vec sd;
    if (T & KFO_PENALIZATION) c2r(c, Fni, sd); /* dealiased s in physical space */
    for (int q = 0; q < 3; ++q)
        par_for((long)(2 * Nc), 16384, [&](long i) { FU[q][i] = -FBu[q][i]; });
    par_for((long)(2 * Nc), 16384, [&](long i) { Fni[i] = -FBn[i]; });
    /* [penalization] masking form of effect_penalization.cpp:35 on the finished
     * right-hand side, then the 2/3 filter (cf. rhs_standard.cpp:491-532) */
    if (T & KFO_PENALIZATION) {
        const double qfix[4] = {-cf.M, 0., 0., -10.};
        for (int q = 0; q < 4; ++q) {
            vec &out = q < 3 ? FU[q] : Fni;
            penalize(c, q < 3 ? U[q] : sd, qfix[q], out, b1);
            dealias(c, out);
        }
    }
    return 0;
}

}  // namespace

extern "C" {

kfo_ctx *kfo_create(const kfo_config *cfg) {
    kfo_ctx *c = new kfo_ctx;
    c->cfg = *cfg;
    const int n = cfg->n;
    c->n = n;
    c->nzc = n / 2 + 1;
    c->N = (size_t)n * n * n;
    c->Nc = (size_t)n * n * c->nzc;
    c->ax = axis_eq{-0.5 * cfg->L, cfg->L, n, cfg->stretch_m};
    c->kv.resize(n);
    for (int i = 0; i < n; ++i) c->kv[i] = c->ax.k_val_at(i);
    const double kmax = c->ax.k_val_at(n / 2);
    const double kzq = c->ax.k_val_at(c->nzc / 2); /* operations.hpp:25 (field_imag::Nz = n/2+1) */
    c->P.resize(c->Nc);
    c->SV.resize(c->Nc);
    c->PF.resize(c->Nc);
    c->K2.resize(c->Nc);
    par_for(n, 1, [&](long i) {
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < c->nzc; ++k) {
                size_t ijk = (size_t)k + c->nzc * ((size_t)j + (size_t)i * n);
                double kx = c->kv[i], ky = c->kv[j], kz = c->kv[k];
                /* OP_dealiasing.hpp:24-30 with the 2/3 rule of rhs_standard.cpp:22 */
                double kabs = sqrt(pow(kx / kmax, 2.) + pow(ky / kmax, 2.) + pow(kz / kmax, 2.));
                c->P[ijk] = kabs < (2. / 3.) ? 1. : 0.;
                /* rhs_standard.cpp:64-71 */
                double knorm = sqrt(pow(kx / kmax, 2.) + pow(ky / kmax, 2.) + pow(kz / kmax, 2.));
                double filter = 1. - exp(-8. * pow(sqrt(knorm), 8.));
                double svv = cfg->sv_eps * filter;
                if (cfg->sv_cut > 0. && !(knorm > cfg->sv_cut)) svv = 0.;
                c->SV[ijk] = svv;
                /* operations.hpp:35-40 with the filter of rhs_standard.cpp:220 */
                double kq = sqrt(pow(kx / kmax, 2.) + pow(ky / kmax, 2.) + pow(kz / kzq, 2.));
                c->PF[ijk] = exp(-2000. * pow(kq, 15.));
                c->K2[ijk] = kx * kx + ky * ky + kz * kz;
            }
    });
    for (int q = 0; q < 3; ++q) c->FU[q].assign(2 * c->Nc, 0.);
    c->Fs.assign(2 * c->Nc, 0.);
    c->Phi.assign(c->N, 0.);
    c->nd.assign(c->N, 0.);
    c->mask.assign(c->N, 0.);
    int levels = cfg->poisson_mode == KFO_PS_FAS ? (cfg->mg_levels > 0 ? cfg->mg_levels : 1) : 1;
    c->lv.resize(levels);
    for (int l = 0; l < levels; ++l) c->lv[l].init(n >> l, cfg->L, cfg->stretch_m);
    /* OP_partial_derivative.cpp:60-80: dS_val = 1/dS of the direction's index,
     * dealiased through FFT, the 2/3 filter and the inverse FFT */
    c->stretched = cfg->stretch_m != 0.;
    if (c->stretched)
        for (int d = 0; d < 3; ++d) {
            vec f(c->N), F;
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j)
                    for (int k = 0; k < n; ++k) {
                        const int q = d == 0 ? i : (d == 1 ? j : k);
                        f[(size_t)k + n * ((size_t)j + (size_t)i * n)] = 1. / c->ax.dS(q);
                    }
            r2c(c, f, F);
            dealias(c, F);
            c2r(c, F, c->dsv[d]);
        }
    return c;
}

void kfo_destroy(kfo_ctx *c) { delete c; }

void kfo_positions(kfo_ctx *c, double *out) {
    for (int i = -1; i <= c->n; ++i) out[i + 1] = c->ax.val_at(i);
}

void kfo_deriv(kfo_ctx *c, int dir, const double *in, double *out) {
    vec a(in, in + 2 * c->Nc), b;
    deriv(c, dir, a, b);
    std::memcpy(out, b.data(), sizeof(double) * 2 * c->Nc);
}

void kfo_penalize(kfo_ctx *c, double fix, const double *in, double *out) {
    vec a(in, in + 2 * c->Nc), o(out, out + 2 * c->Nc), q, b;
    c2r(c, a, q);
    penalize(c, q, fix, o, b);
    std::memcpy(out, o.data(), sizeof(double) * 2 * c->Nc);
}

void kfo_metric(kfo_ctx *c, double *out) {
    const int n = c->n;
    for (int i = 0; i < n; ++i) out[i] = c->stretched ? c->dsv[0][(size_t)i * n * n] : 1.;
}

void kfo_set_state(kfo_ctx *c, const double *ux, const double *uy, const double *uz,
                   const double *s) {
    const double *src[3] = {ux, uy, uz};
    for (int q = 0; q < 3; ++q) std::memcpy(c->FU[q].data(), src[q], sizeof(double) * 2 * c->Nc);
    std::memcpy(c->Fs.data(), s, sizeof(double) * 2 * c->Nc);
    c->nhist = 0;
}

void kfo_get_state(kfo_ctx *c, double *ux, double *uy, double *uz, double *s) {
    double *dst[3] = {ux, uy, uz};
    for (int q = 0; q < 3; ++q) std::memcpy(dst[q], c->FU[q].data(), sizeof(double) * 2 * c->Nc);
    std::memcpy(s, c->Fs.data(), sizeof(double) * 2 * c->Nc);
}

void kfo_set_sources(kfo_ctx *c, const double *nd, const double *mask) {
    if (nd) std::memcpy(c->nd.data(), nd, sizeof(double) * c->N);
    if (mask) std::memcpy(c->mask.data(), mask, sizeof(double) * c->N);
}

void kfo_set_phi(kfo_ctx *c, const double *phi) {
    std::memcpy(c->Phi.data(), phi, sizeof(double) * c->N);
    c->nhist = 0;
}
void kfo_get_phi(kfo_ctx *c, double *phi) { std::memcpy(phi, c->Phi.data(), sizeof(double) * c->N); }

int kfo_rhs(kfo_ctx *c, double t) {
    /* the right-hand side is autonomous (rhs_standard.cpp never reads t); t
     * only selects the start of the Poisson solve */
    return rhs(c, c->FU, c->Fs, t);
}

/* Runge_kutta_O4::solve (RKO4.cpp:50-241) */
int kfo_rk4(kfo_ctx *c, double dt, int nsteps) {
    const size_t M = 2 * c->Nc;
    for (int s = 0; s < nsteps; ++s) {
        vec R0[4], R1[4], R2[4], R3[4], R4[4];
        vec *Y[4] = {&c->FU[0], &c->FU[1], &c->FU[2], &c->Fs};
        for (int q = 0; q < 4; ++q) { R0[q] = *Y[q]; R1[q] = *Y[q]; }
        const double t0 = c->t;
        int rc = rhs(c, R1, R1[3], t0);
        if (rc) return rc;
        for (int q = 0; q < 4; ++q) {
            R2[q].resize(M);
            par_for((long)(M), 16384, [&](long i) { R2[q][i] = R0[q][i] + 0.5 * dt * R1[q][i]; });
        }
        if ((rc = rhs(c, R2, R2[3], t0 + 0.5 * dt))) return rc;
        for (int q = 0; q < 4; ++q) {
            R3[q].resize(M);
            par_for((long)(M), 16384, [&](long i) { R3[q][i] = R0[q][i] + 0.5 * dt * R2[q][i]; });
        }
        if ((rc = rhs(c, R3, R3[3], t0 + 0.5 * dt))) return rc;
        for (int q = 0; q < 4; ++q) {
            R4[q].resize(M);
            par_for((long)(M), 16384, [&](long i) { R4[q][i] = R0[q][i] + 1.0 * dt * R3[q][i]; });
        }
        if ((rc = rhs(c, R4, R4[3], t0 + 1.0 * dt))) return rc;
        for (int q = 0; q < 4; ++q)
            par_for((long)M, 16384, [&](long i) {
                (*Y[q])[i] = R0[q][i] + (dt / 6.) * (1. * R1[q][i] + 2. * R2[q][i] + 2. * R3[q][i] +
                                                      1. * R4[q][i]);
            });
        c->t = t0 + dt;
    }
    return 0;
}

double kfo_time(kfo_ctx *c) { return c->t; }

int kfo_poisson(kfo_ctx *c, double *phi_io, const double *rho) {
    vec phi(phi_io, phi_io + c->N), r(rho, rho + c->N);
    int rc = poisson(c, phi, r);
    std::memcpy(phi_io, phi.data(), sizeof(double) * c->N);
    return rc;
}

void kfo_poisson_stats_get(kfo_ctx *c, kfo_poisson_stats *out) { *out = c->stats; }

double kfo_residual(kfo_ctx *c, const double *phi, const double *rho) {
    vec p(phi, phi + c->N), r(rho, rho + c->N);
    return max_resid(c->lv[0], p, r);
}

void kfo_tables(kfo_ctx *c, double *dealias_out, double *sv, double *phifilt) {
    if (dealias_out) std::memcpy(dealias_out, c->P.data(), sizeof(double) * c->Nc);
    if (sv) std::memcpy(sv, c->SV.data(), sizeof(double) * c->Nc);
    if (phifilt) std::memcpy(phifilt, c->PF.data(), sizeof(double) * c->Nc);
}

void kfo_r2c(int n, const double *in, double *out) { kfs_r2c_3d(n, n, n, in, out); }

void kfo_c2r(int n, const double *in, double *out) {
    size_t N = (size_t)n * n * n;
    kfs_c2r_3d(n, n, n, in, out);
    double Norm = 1. / ((double)N);
    par_for((long)(N), 16384, [&](long i) { out[i] = out[i] * Norm; });
}

void kfo_transfer(int kind, int n, double L, const double *in, double *out) {
    size_t N = (size_t)n * n * n;
    vec a(in, in + N), b;
    if (kind == 0) prolong(n, L, 0., a, b);
    else if (kind == 1) inject(n, 2, a, b);
    else restrict_fw(n, a, b);
    std::memcpy(out, b.data(), sizeof(double) * b.size());
}

}  // extern "C"
