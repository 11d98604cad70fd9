// kf_adjoint.cuh -- kernels of the discrete adjoint of the FP64 time step.
//
// The state is the 2*Nc real numbers (Re, Im) of the four half spectra, and the
// adjoint is the transpose with respect to those coordinates.  With w(kz) = 1
// for kz = 0, n/2 and 2 otherwise, the transposes of the reference's transforms
// (OP_FFT / OP_iFFT: r2c unnormalised, c2r scaled by 1/N, the imaginary parts of
// the kz = 0, n/2 bins ignored) are
//   c2r^T(x) = (w/N) r2c(x),      r2c^T(X) = N c2r(X / w) = c2r_unscaled(X / w),
// and multiplication by i k transposes to multiplication by -i k.
#pragma once

#include "kf_passes.cuh"
#include "kf_poisson.cuh"

namespace kf {

// Block sums of up to 4 partial quantities into part[blockIdx.x * 4 + q].
template <int BS>
__device__ __forceinline__ void block_sum4(double v[4], double *sh, double *part) {
    for (int q = 0; q < 4; ++q) sh[q * BS + threadIdx.x] = v[q];
    __syncthreads();
    for (int w = BS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < 4; ++q) sh[q * BS + threadIdx.x] = __dadd_rn(sh[q * BS + threadIdx.x], sh[q * BS + threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) part[blockIdx.x * 4 + q] = sh[q * BS];
}

// acc[q] += sum over blocks of part[b*4 + q], fixed order (one thread).
__global__ void k_accumulate4(const double *__restrict__ part, int nb, double *__restrict__ acc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int q = 0; q < 4; ++q) {
        double s = 0.;
        for (int b = 0; b < nb; ++b) s = __dadd_rn(s, part[b * 4 + q]);
        acc[q] = __dadd_rn(acc[q], s);
    }
}

// Transpose of the physical-space part of the right-hand side (k_products).
//   pen: f_q = (1-H)(rl_q - pr_q) + H eta (qd_q - qfix_q), qd = (U, s_d), qfix_x = -M
//   no pen: the products enter K through -r2c, fb_q carries c2r_u(Kbar_q / w)
// Outputs the cotangents of U_c, dU[c][d], ds[d], s_d (penalization part), rl_q
// and the block sums of dJ/dM (slot 0).
struct ProdVjpArgs {
    const double *fb[4];
    const double *U[3], *dU[3][3], *ds[3], *H;
    double *Ub[3], *dUb[3][3], *dsb[3], *sdb, *rlb[4];
    double eta;
    int terms;
    long N;
    double *part;
};

template <int BS>
__global__ void __launch_bounds__(BS, 3) k_prod_vjp(ProdVjpArgs a) {
    __shared__ double sh[4 * BS];
    double acc[4] = {0., 0., 0., 0.};
    const bool pen = a.terms & T_PENALIZATION, adv = a.terms & T_ADVECTION, cont = a.terms & T_CONTINUITY;
    for (long i = (long)blockIdx.x * BS + threadIdx.x; i < a.N; i += (long)gridDim.x * BS) {
        double prb[4], qdb[4] = {0., 0., 0., 0.};
        const double h = pen ? a.H[i] : 0.;
        for (int q = 0; q < 4; ++q) {
            const double f = a.fb[q][i];
            if (pen) {
                const double g1 = __dmul_rn(1. - h, f);
                a.rlb[q][i] = g1;
                prb[q] = -g1;
                qdb[q] = __dmul_rn(__dmul_rn(h, a.eta), f);
            } else {
                prb[q] = -f;
            }
        }
        if (pen) acc[0] = __dadd_rn(acc[0], qdb[0]);  // d f_x / d M = H eta
        const double u[3] = {a.U[0][i], a.U[1][i], a.U[2][i]};
        for (int d = 0; d < 3; ++d) {
            double ub = qdb[d];
            if (adv)
                for (int c = 0; c < 3; ++c) ub += prb[c] * a.dU[c][d][i];
            if (cont) ub += prb[3] * a.ds[d][i];
            a.Ub[d][i] = ub;
            for (int c = 0; c < 3; ++c) a.dUb[c][d][i] = adv ? prb[c] * u[d] : 0.;
            a.dsb[d][i] = cont ? prb[3] * u[d] : 0.;
        }
        a.sdb[i] = qdb[3];
    }
    block_sum4<BS>(acc, sh, a.part);
}

// Spectral assembly of the transpose of the right-hand side at one stage.
// CA[0..2]   = r2c(Ubar_c), CA[3+3c+d] = r2c(dUbar[c][d]), CA[12+d] = r2c(dsbar_d),
// CA[15] = r2c(sdbar) (second call only), CA[16+q] = r2c(rlbar_q) (penalization).
// part 1 (stage_two = 0): Ybar_q (=, not +=) from everything but sdbar, phihat-bar,
//   block sums of dJ/dtau (slot 1) and dJ/dM (slot 0).
// part 2 (stage_two = 1): Ybar_s += P (w/N) CA[15].
struct VjpAsmArgs {
    const double2 *CA[20];
    const double2 *Kbar[4];  // no-penalization path: lin-bar = -Kbar
    const double2 *Y[4];     // the stage input
    const double *SV, *PF;
    double2 *Ybar[4];
    double2 *phib;
    double tau, theta, M, D, invN;
    int terms, stage_two;
    double *part;
};

template <int BS>
__global__ void __launch_bounds__(BS, 3) k_vjp_assemble(VjpAsmArgs a, Geo<double> g) {
    __shared__ double sh[4 * BS];
    double acc[4] = {0., 0., 0., 0.};
    const long Nc = (long)g.n * g.n * g.nzc;
    const int Tm = a.terms;
    const bool pen = Tm & T_PENALIZATION;
    for (long idx = (long)blockIdx.x * BS + threadIdx.x; idx < Nc; idx += (long)gridDim.x * BS) {
        const int k = (int)(idx % g.nzc);
        const long r = idx / g.nzc;
        const int j = (int)(r % g.n), i = (int)(r / g.n);
        const double kx = g.kv[i], ky = g.kv[j], kz = g.kv[k];
        const double kk[3] = {kx, ky, kz};
        const bool P = dealias_keep(g.q2, g.thr, i, j, k);
        const double wN = (k == 0 || 2 * k == g.n ? 1. : 2.) * a.invN;
        if (a.stage_two) {
            if (P) {
                const double2 f = a.CA[15][idx];
                double2 y = a.Ybar[3][idx];
                y.x += wN * f.x;
                y.y += wN * f.y;
                a.Ybar[3][idx] = y;
            }
            continue;
        }
        // lin-bar_q
        double2 lb[4];
        for (int q = 0; q < 4; ++q) {
            if (pen) {
                const double2 f = a.CA[16 + q][idx];
                lb[q] = make_double2(-wN * f.x, -wN * f.y);
            } else {
                const double2 f = a.Kbar[q][idx];
                lb[q] = make_double2(-f.x, -f.y);
            }
        }
        const double sv = a.SV[idx];
        const double k2 = kx * kx + ky * ky + kz * kz;
        const bool diss = Tm & T_DISSIPATION, svo = Tm & T_SVISCOSITY;
        const double cf = diss && svo ? (a.tau + sv) : diss ? a.tau : svo ? sv : 0.;
        const double dk = (Tm & T_DIFFUSION) ? a.D * k2 : 0.;
        double2 yb[4];
        // physical-space cotangents mapped back: P (w/N) [F(Ub_c) - i k_d F(dUb[c][d])]
        for (int c = 0; c < 3; ++c) {
            double2 t = make_double2(0., 0.);
            if (P) {
                const double2 fu = a.CA[c][idx];
                t.x = fu.x;
                t.y = fu.y;
                for (int d = 0; d < 3; ++d) {
                    const double2 f = a.CA[3 + 3 * c + d][idx];
                    t.x += kk[d] * f.y;   // -i k (x + i y) = k y - i k x
                    t.y -= kk[d] * f.x;
                }
                t.x *= wN;
                t.y *= wN;
            }
            // linear terms of u_c: (cf + D k^2) u, M i k_x P u, continuity i k_c P u_c in s
            const double2 l = lb[c];
            t.x += (cf + dk) * l.x;
            t.y += (cf + dk) * l.y;
            if ((Tm & T_E_EXT) && P) {
                t.x += a.M * kx * l.y;
                t.y -= a.M * kx * l.x;
            }
            if ((Tm & T_CONTINUITY) && P) {
                t.x += kk[c] * lb[3].y;
                t.y -= kk[c] * lb[3].x;
            }
            yb[c] = t;
            if (diss) {  // d lin / d tau = u
                const double2 u = a.Y[c][idx];
                acc[1] += l.x * u.x + l.y * u.y;
            }
            if (Tm & T_E_EXT && P) {  // d lin / d M = i k_x P u
                const double2 u = a.Y[c][idx];
                acc[0] += l.x * (-kx * u.y) + l.y * (kx * u.x);
            }
        }
        // s: physical part, (SV + D k^2) s, M i k_x P s, pressure i k_c s / theta
        {
            double2 t = make_double2(0., 0.);
            if (P) {
                for (int d = 0; d < 3; ++d) {
                    const double2 f = a.CA[12 + d][idx];
                    t.x += kk[d] * f.y;
                    t.y -= kk[d] * f.x;
                }
                t.x *= wN;
                t.y *= wN;
            }
            const double2 l = lb[3];
            const double cs = ((Tm & T_SVISCOSITY) ? sv : 0.) + dk;
            t.x += cs * l.x;
            t.y += cs * l.y;
            if ((Tm & T_E_EXT) && P) {
                t.x += a.M * kx * l.y;
                t.y -= a.M * kx * l.x;
                const double2 s = a.Y[3][idx];
                acc[0] += l.x * (-kx * s.y) + l.y * (kx * s.x);
            }
            if (Tm & T_PRESSURE)
                for (int c = 0; c < 3; ++c) {
                    t.x += kk[c] * lb[c].y / a.theta;
                    t.y -= kk[c] * lb[c].x / a.theta;
                }
            yb[3] = t;
        }
        for (int q = 0; q < 4; ++q) a.Ybar[q][idx] = yb[q];
        // phihat-bar = sum_c PF (-i k_c) lin-bar_c  (E-force)
        double2 pb = make_double2(0., 0.);
        if (Tm & T_E_INT) {
            const double pf = (Tm & T_PRESSURE) ? a.PF[idx] : 1.;
            for (int c = 0; c < 3; ++c) {
                pb.x += pf * kk[c] * lb[c].y;
                pb.y -= pf * kk[c] * lb[c].x;
            }
        }
        a.phib[idx] = pb;
    }
    block_sum4<BS>(acc, sh, a.part);
}

// sdbar += rhobar * exp(s_d) (rho = exp(s_d) + n_d); block sums of
// sum rhobar * n_d (slot 2): the derivative along n_d -> (1+e) n_d
template <int BS>
__global__ void __launch_bounds__(BS) k_poisson_vjp_tail(const double *__restrict__ rhob, const double *__restrict__ sd,
                                                         const double *__restrict__ nd,
                                                         double *__restrict__ sdb, long N, double *__restrict__ part) {
    __shared__ double sh[4 * BS];
    double acc[4] = {0., 0., 0., 0.};
    for (long i = (long)blockIdx.x * BS + threadIdx.x; i < N; i += (long)gridDim.x * BS) {
        const double rb = rhob[i];
        sdb[i] = __dadd_rn(sdb[i], __dmul_rn(rb, exp(sd[i])));
        acc[2] = __dadd_rn(acc[2], __dmul_rn(rb, nd[i]));
    }
    block_sum4<BS>(acc, sh, part);
}

// y = a x + b y over interleaved complex (real coordinates), four fields via a grid dimension
__global__ void k_axpby(double *__restrict__ y, const double *__restrict__ x, double a, double b, long M) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) y[i] = __dadd_rn(__dmul_rn(a, x[i]), __dmul_rn(b, y[i]));
}

// c = exp(phi)
__global__ void k_exp(const double *__restrict__ phi, double *__restrict__ c, long N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) c[i] = exp(phi[i]);
}

// out = s * in (real)
__global__ void k_scale(const double *__restrict__ in, double *__restrict__ out, double s, long N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = s * in[i];
}

// J partial: block sums of sum w * phi (slot 3)
template <int BS>
__global__ void __launch_bounds__(BS) k_dot_w(const double *__restrict__ w, const double *__restrict__ phi, long N,
                                              double *__restrict__ part) {
    __shared__ double sh[4 * BS];
    double acc[4] = {0., 0., 0., 0.};
    for (long i = (long)blockIdx.x * BS + threadIdx.x; i < N; i += (long)gridDim.x * BS)
        acc[3] = __dadd_rn(acc[3], __dmul_rn(w[i], phi[i]));
    block_sum4<BS>(acc, sh, part);
}

// ---------------------------------------------------------------- linear (adjoint) Poisson
// Solve (-L_h + c) psi = b, c = exp(phi) > 0, with the FAS framework of the
// forward solver: the point equation A - D psi - c psi = 0 (A = 2 sum w psi_nb + b)
// is linear, so the "Newton step" is the exact point solve psi = A / (D + c),
// over-relaxed by om as the forward smoother (om = 1: the point solve itself).

template <int BY = 8>
__global__ void __launch_bounds__(32 * BY) k_rbgs_lin(double *__restrict__ phi, const double *__restrict__ rho,
                                                      const double *__restrict__ cl, Lev L, int color, double om) {
    const int n = L.n;
    const int k2 = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * BY + threadIdx.y, i = blockIdx.z;
    if (2 * k2 >= n || j >= n) return;
    const int k = 2 * k2 + ((i + j + color) & 1);
    double A, D;
    point_coeffs_fast(phi, rho, L, i, j, k, A, D);
    const long q = lidx(i, j, k, n);
    const double y = A / __dadd_rn(D, cl[q]);
    phi[q] = om == 1. ? y : __dadd_rn(phi[q], __dmul_rn(om, __dsub_rn(y, phi[q])));
}

// The same linear half sweep indexed as k_rbgs_t: one 32-bit index with
// wrapped neighbour offsets, the i and j axis tables from the constant bank;
// the loads, the sum and its order are point_coeffs_fast's.
template <int BY = 8>
__global__ void __launch_bounds__(32 * BY) k_rbgs_lin_t(double *__restrict__ phi, const double *__restrict__ rho,
                                                        const double *__restrict__ cl, Lev L, int color, double om,
                                                        const __grid_constant__ AxTab T) {
    const int n = L.n;
    const int k2 = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * BY + threadIdx.y, i = blockIdx.z;
    if (2 * k2 >= n || j >= n) return;
    const int k = 2 * k2 + ((i + j + color) & 1);
    const int nn = n * n;
    const int q = (i * n + j) * n + k;
    const int oip = i == n - 1 ? -(n - 1) * nn : nn, oim = i == 0 ? (n - 1) * nn : -nn;
    const int ojp = j == n - 1 ? -(n - 1) * n : n, ojm = j == 0 ? (n - 1) * n : -n;
    const int okp = k == n - 1 ? -(n - 1) : 1, okm = k == 0 ? n - 1 : -1;
    const double D = __dadd_rn(__dadd_rn(T.dd[i], T.dd[j]), L.dd[k]);
    double A = __dmul_rn(phi[q + oip], T.ip[i]);
    A = __dadd_rn(A, __dmul_rn(phi[q + oim], T.im[i]));
    A = __dadd_rn(A, __dmul_rn(phi[q + ojp], T.ip[j]));
    A = __dadd_rn(A, __dmul_rn(phi[q + ojm], T.im[j]));
    A = __dadd_rn(A, __dmul_rn(phi[q + okp], L.ip[k]));
    A = __dadd_rn(A, __dmul_rn(phi[q + okm], L.im[k]));
    if (rho) A = __dadd_rn(A, rho[q]);
    const double y = A / __dadd_rn(D, cl[q]);
    phi[q] = om == 1. ? y : __dadd_rn(phi[q], __dmul_rn(om, __dsub_rn(y, phi[q])));
}

__global__ void __launch_bounds__(256) k_residual_lin(const double *__restrict__ phi, const double *__restrict__ rho,
                                                      const double *__restrict__ cl, Lev L, double *__restrict__ r) {
    const int n = L.n;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, i = blockIdx.z;
    if (k >= n || j >= n) return;
    double A, D;
    point_coeffs_fast(phi, rho, L, i, j, k, A, D);
    const long id = lidx(i, j, k, n);
    r[id] = __dsub_rn(A, __dmul_rn(__dadd_rn(D, cl[id]), phi[id]));
}

__global__ void __launch_bounds__(256) k_resmax_lin(const double *__restrict__ phi, const double *__restrict__ rho,
                                                    const double *__restrict__ cl, Lev L,
                                                    unsigned long long *__restrict__ out) {
    __shared__ double sh[8];
    const int n = L.n;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
    double af = 0.;
    if (k < n && j < n)
        for (int i = blockIdx.z; i < n; i += gridDim.z) {
            double A, D;
            point_coeffs_fast(phi, rho, L, i, j, k, A, D);
            const long id = lidx(i, j, k, n);
            af = nmax(af, fabs(__dsub_rn(A, __dmul_rn(__dadd_rn(D, cl[id]), phi[id]))));
        }
    for (int o = 16; o > 0; o >>= 1) af = nmax(af, __shfl_xor_sync(0xffffffffu, af, o));
    if (threadIdx.x == 0) sh[threadIdx.y] = af;
    __syncthreads();
    if (threadIdx.y == 0 && threadIdx.x == 0) {
        double m = sh[0];
        for (int w = 1; w < 8; ++w) m = nmax(m, sh[w]);
        atomicMax(out + ((blockIdx.x + blockIdx.y * gridDim.x + blockIdx.z) & 63),
                  (unsigned long long)__double_as_longlong(m));
    }
}

// rho_c = N_c(psi_c) + r_c with N(psi) = -L psi + c psi
__global__ void __launch_bounds__(256) k_fas_rhs_lin(const double *__restrict__ phic, const double *__restrict__ rc,
                                                     const double *__restrict__ cl, Lev L, double *__restrict__ rhoc) {
    const int n = L.n;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, i = blockIdx.z;
    if (k >= n || j >= n) return;
    const long id = lidx(i, j, k, n);
    double A, D;
    point_coeffs_fast(phic, nullptr, L, i, j, k, A, D);
    const double Nc = __dsub_rn(__dmul_rn(__dadd_rn(D, cl[id]), phic[id]), A);
    rhoc[id] = __dadd_rn(Nc, rc[id]);
}

// Coarsest level of the linear solve in one block, staged in shared memory
// (psi, b, c and the axis tables: 24 n^3 + 24 n bytes): red-black sweeps
// until the max residual has dropped by rtol from its value at entry
// (checked every 4 sweeps), or max_sweeps.
__global__ void __launch_bounds__(1024) k_coarse_solve_lin(double *__restrict__ phi, const double *__restrict__ rho,
                                                           const double *__restrict__ cl, Lev L, double rtol,
                                                           int max_sweeps) {
    extern __shared__ __align__(16) double cl_sm[];
    __shared__ double sh[32];
    const int n = L.n, N = n * n * n;
    double *sp = cl_sm, *sb = cl_sm + N, *sc = cl_sm + 2 * N, *sd = cl_sm + 3 * N, *si = sd + n, *sm_ = si + n;
    for (int id = threadIdx.x; id < N; id += blockDim.x) {
        sp[id] = phi[id];
        sb[id] = rho[id];
        sc[id] = cl[id];
    }
    for (int id = threadIdx.x; id < n; id += blockDim.x) {
        sd[id] = L.dd[id];
        si[id] = L.ip[id];
        sm_[id] = L.im[id];
    }
    __syncthreads();
    const Lev Ls{n, sd, nullptr, nullptr, si, sm_};
    double r0 = 0.;
    for (int s = 0;; s += 4) {
        double m = 0.;
        for (int id = threadIdx.x; id < N; id += blockDim.x) {
            const int k = id % n, r = id / n, j = r % n, i = r / n;
            double A, D;
            point_coeffs_fast(sp, sb, Ls, i, j, k, A, D);
            m = nmax(m, fabs(__dsub_rn(A, __dmul_rn(__dadd_rn(D, sc[id]), sp[id]))));
        }
        for (int o = 16; o > 0; o >>= 1) m = nmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32) {
            double t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.;
            for (int o = 16; o > 0; o >>= 1) t = nmax(t, __shfl_xor_sync(0xffffffffu, t, o));
            if (threadIdx.x == 0) sh[0] = t;
        }
        __syncthreads();
        const double res = sh[0];
        __syncthreads();
        if (s == 0) r0 = res;
        if (!(res > rtol * r0) || s >= max_sweeps) break;  // reached, zero, NaN or capped
        for (int sw = 0; sw < 4; ++sw)
            for (int color = 0; color < 2; ++color) {
                const int nh = n / 2;
                for (int id = threadIdx.x; id < N / 2; id += blockDim.x) {
                    const int k2 = id % nh, r = id / nh, j = r % n, i = r / n;
                    const int k = 2 * k2 + ((i + j + color) & 1);
                    double A, D;
                    point_coeffs_fast(sp, sb, Ls, i, j, k, A, D);
                    const int q = (int)lidx(i, j, k, n);
                    sp[q] = A / __dadd_rn(D, sc[q]);
                }
                __syncthreads();
            }
    }
    for (int id = threadIdx.x; id < N; id += blockDim.x) phi[id] = sp[id];
}

// Block sums of <b, bp> (slot 0) and <bp, bp> (slot 1): the least-squares
// factor alpha = <b, bp> / <bp, bp> of the warm start alpha * psi_prev.
template <int BS>
__global__ void __launch_bounds__(BS) k_dot2(const double *__restrict__ b, const double *__restrict__ bp, long N,
                                             double *__restrict__ part) {
    __shared__ double sh[4 * BS];
    double acc[4] = {0., 0., 0., 0.};
    for (long i = (long)blockIdx.x * BS + threadIdx.x; i < N; i += (long)gridDim.x * BS) {
        const double x = b[i], y = bp[i];
        acc[0] += x * y;
        acc[1] += y * y;
    }
    block_sum4<BS>(acc, sh, part);
}

// psi = alpha psi (alpha = sums[0] / sums[1], 0 when sums[1] == 0); bp = b
__global__ void k_warm_scale(double *__restrict__ psi, double *__restrict__ bp, const double *__restrict__ b,
                             const double *__restrict__ sums, long N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double den = sums[1];
    const double alpha = den > 0. ? sums[0] / den : 0.;
    psi[i] *= alpha;
    bp[i] = b[i];
}

// max |x| over N values: block maxima, atomic max on the bit pattern (x >= 0)
// into one of 64 slots
__global__ void __launch_bounds__(256) k_absmax(const double *__restrict__ x, long N,
                                                unsigned long long *__restrict__ out) {
    __shared__ double sh[8];
    double m = 0.;
    for (long i = (long)blockIdx.x * 256 + threadIdx.x; i < N; i += (long)gridDim.x * 256) m = nmax(m, fabs(x[i]));
    for (int o = 16; o > 0; o >>= 1) m = nmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = sh[0];
        for (int w = 1; w < 8; ++w) t = nmax(t, sh[w]);
        atomicMax(out + (blockIdx.x & 63), (unsigned long long)__double_as_longlong(t));
    }
}

// ---------------------------------------------------------------- reverse RK4
// Stage cotangents of one RK4 step (RKO4.cpp:105-238) taken in reverse,
// y' = y + dt/6 (K1 + 2 K2 + 2 K3 + K4), X2 = y + dt/2 K1, X3 = y + dt/2 K2,
// X4 = y + dt K3, over the real coordinates of the four half spectra:
//   mode 0 (before stage 4): Kb = ca lam,           lacc = lam
//   mode 1 (before 3, 2, 1): Kb = ca lam + cb Xb,   lacc += Xb
//   mode 2 (after stage 1):  lam = lacc + Xb
// with Xb the cotangent of the last stage input.  blockIdx.y = field.
struct AdjStageArgs {
    double *lam[4], *lacc[4], *Kb[4];
    const double *Xb[4];
};
__global__ void k_adj_stage(AdjStageArgs a, double ca, double cb, int mode, long M) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int q = blockIdx.y;
    if (i >= M) return;
    const double l = a.lam[q][i];
    if (mode == 0) {
        a.lacc[q][i] = l;
        a.Kb[q][i] = ca * l;
    } else if (mode == 1) {
        const double xb = a.Xb[q][i];
        a.lacc[q][i] += xb;
        a.Kb[q][i] = ca * l + cb * xb;
    } else {
        a.lam[q][i] = a.lacc[q][i] + a.Xb[q][i];
    }
}

// dJ/dn0 = dJ/ds0 * exp(-s0)  (s0 = ln n0)
__global__ void k_dn0(const double *__restrict__ ds0, const double *__restrict__ s0, double *__restrict__ out, long N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = ds0[i] * exp(-s0[i]);
}

}  // namespace kf
