// kf_poisson.cuh -- FP64 kernels of the nonlinear Boltzmann-electron Poisson solve
//   lap_h phi = exp(phi) - rho,   rho = exp(s) + n_d
// (rhs_standard.cpp:100-113; solver_poisson_jacobi_nlin.cpp:140-265).
//
// The point update is the reference's: with the 7-point coefficients of the
// axis spacings H[i] = x_i - x_{i-1},
//   D = sum_axes 2/(H[i+1] H[i]),  A = 2 sum_nb phi_nb / (H(H[i+1]+H[i])) + rho,
// phi_new solves A - D x - e^x = 0 by the damped Newton of newton_method.hpp:16-63.
// Products and sums are spelled with __d*_rn intrinsics where the reference's
// order must not be contracted into FMAs, so that the GPU reproduces the CPU
// arithmetic up to the last-bit differences of exp().
#pragma once

#include <cuda_runtime.h>

namespace kf {

struct Lev {
    int n;
    const double *dd;  // 2/(H[i+1] H[i])
    const double *dp;  // H[i+1] (H[i+1] + H[i])
    const double *dm;  // H[i]   (H[i+1] + H[i])
    const double *ip;  // 2/dp  (FAS cycle weights)
    const double *im;  // 2/dm
};

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }
__device__ __forceinline__ long lidx(int i, int j, int k, int n) { return (long)k + n * ((long)j + (long)i * n); }

__device__ __forceinline__ void point_coeffs(const double *__restrict__ p, const double *__restrict__ rho,
                                             const Lev &L, int i, int j, int k, double &A, double &D) {
    const int n = L.n;
    D = __dadd_rn(__dadd_rn(L.dd[i], L.dd[j]), L.dd[k]);
    A = p[lidx(wrapi(i + 1, n), j, k, n)] / L.dp[i];
    A = __dadd_rn(A, p[lidx(wrapi(i - 1, n), j, k, n)] / L.dm[i]);
    A = __dadd_rn(A, p[lidx(i, wrapi(j + 1, n), k, n)] / L.dp[j]);
    A = __dadd_rn(A, p[lidx(i, wrapi(j - 1, n), k, n)] / L.dm[j]);
    A = __dadd_rn(A, p[lidx(i, j, wrapi(k + 1, n), n)] / L.dp[k]);
    A = __dadd_rn(A, p[lidx(i, j, wrapi(k - 1, n), n)] / L.dm[k]);
    A = __dmul_rn(2., A);
    if (rho) A = __dadd_rn(A, rho[lidx(i, j, k, n)]);
}

// The FAS cycle's stencil: the same operator with the weights 2/den
// precomputed, products instead of divisions.
__device__ __forceinline__ void point_coeffs_fast(const double *__restrict__ p, const double *__restrict__ rho,
                                                  const Lev &L, int i, int j, int k, double &A, double &D) {
    const int n = L.n;
    D = __dadd_rn(__dadd_rn(L.dd[i], L.dd[j]), L.dd[k]);
    A = __dmul_rn(p[lidx(wrapi(i + 1, n), j, k, n)], L.ip[i]);
    A = __dadd_rn(A, __dmul_rn(p[lidx(wrapi(i - 1, n), j, k, n)], L.im[i]));
    A = __dadd_rn(A, __dmul_rn(p[lidx(i, wrapi(j + 1, n), k, n)], L.ip[j]));
    A = __dadd_rn(A, __dmul_rn(p[lidx(i, wrapi(j - 1, n), k, n)], L.im[j]));
    A = __dadd_rn(A, __dmul_rn(p[lidx(i, j, wrapi(k + 1, n), n)], L.ip[k]));
    A = __dadd_rn(A, __dmul_rn(p[lidx(i, j, wrapi(k - 1, n), n)], L.im[k]));
    if (rho) A = __dadd_rn(A, rho[lidx(i, j, k, n)]);
}

template <bool FAST>
__device__ __forceinline__ void coeffs_t(const double *__restrict__ p, const double *__restrict__ rho,
                                         const Lev &L, int i, int j, int k, double &A, double &D) {
    if (FAST) point_coeffs_fast(p, rho, L, i, j, k, A, D);
    else point_coeffs(p, rho, L, i, j, k, A, D);
}

// one Newton step on A - D x - e^x = 0, over-relaxed by om (the FAS
// smoother's point update; om = 1: the plain Newton step)
__device__ __forceinline__ double newton_step(double x, double A, double D, double om) {
    const double ex = exp(x);
    return __dsub_rn(x, __dmul_rn(om, __dsub_rn(__dsub_rn(A, __dmul_rn(D, x)), ex) / __dsub_rn(-D, ex)));
}

__device__ __forceinline__ double f_point(double A, double D, double x) {
    return __dsub_rn(__dsub_rn(A, __dmul_rn(D, x)), exp(x));
}

// newton_method::solve (newton_method.hpp:16-63), eps 0.05, Nmax 20, g 0.8
__device__ __forceinline__ double newton_point(double x, double A, double D) {
    const double g = 0.8;
    double omega = 1.;
    double dx = 0.;
    double ex = exp(x);
    double dx_alt = __dsub_rn(__dsub_rn(A, __dmul_rn(D, x)), ex) / __dsub_rn(-D, ex);
    int i = 0;
    do {
        x = __dsub_rn(x, __dmul_rn(omega, dx));
        ex = exp(x);
        dx = __dsub_rn(__dsub_rn(A, __dmul_rn(D, x)), ex) / __dsub_rn(-D, ex);
        omega = fabs(dx) > fabs(dx_alt) ? __dmul_rn(g, omega) : __dadd_rn(__dmul_rn(1. - g, omega), g * 1.);
        dx_alt = dx;
        ++i;
    } while (fabs(dx) > 0.05 && i < 20);
    return __dsub_rn(x, dx);
}

// ------------------------------------------------------------ reductions
// Block partials of the Jacobi sweep statistics; slot layout per block:
// [0] max|dP|, [1] sum|dP|, [2] max P_new, [3] min P_new, [4] max|f(P_old)|
constexpr int KF_RED = 5;

// NaN-propagating max / min (fmax alone would drop a NaN)
__device__ __forceinline__ double nmax(double a, double b) { return (a != a || b != b) ? a + b : fmax(a, b); }
__device__ __forceinline__ double nmin(double a, double b) { return (a != a || b != b) ? a + b : fmin(a, b); }

template <int BS>
__device__ __forceinline__ void block_reduce5(double v[KF_RED], double *sh, double *out) {
    // sh: [KF_RED][BS]
    for (int s = 0; s < KF_RED; ++s) sh[s * BS + threadIdx.x] = v[s];
    __syncthreads();
    for (int w = BS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            double *a = sh + threadIdx.x, *b = sh + threadIdx.x + w;
            a[0] = nmax(a[0], b[0]);
            a[BS] = __dadd_rn(a[BS], b[BS]);
            a[2 * BS] = nmax(a[2 * BS], b[2 * BS]);
            a[3 * BS] = nmin(a[3 * BS], b[3 * BS]);
            a[4 * BS] = nmax(a[4 * BS], b[4 * BS]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int s = 0; s < KF_RED; ++s) out[s] = sh[s * BS];
}

// Jacobi sweep (iteration_loop, solver_poisson_jacobi_nlin.cpp:140-235)
template <int BS>
__global__ void __launch_bounds__(BS) k_jacobi(const double *__restrict__ in, double *__restrict__ out,
                                               const double *__restrict__ rho, Lev L, double omega,
                                               double *__restrict__ partial) {
    __shared__ double sh[KF_RED * BS];
    const int n = L.n;
    const long N = (long)n * n * n;
    double v[KF_RED] = {0., 0., -INFINITY, INFINITY, 0.};
    if (blockIdx.x == 0 && threadIdx.x == 0) v[2] = v[3] = in[0];  // supremum = infinum = in.val[0] (:158-159)
    for (long id = (long)blockIdx.x * BS + threadIdx.x; id < N; id += (long)gridDim.x * BS) {
        const int k = (int)(id % n);
        const long r = id / n;
        const int j = (int)(r % n), i = (int)(r / n);
        double A, D;
        point_coeffs(in, rho, L, i, j, k, A, D);
        const double P_old = in[id];
        const double f0 = f_point(A, D, P_old);
        const double P_new = newton_point(P_old, A, D);
        const double delta = fabs(__dsub_rn(P_new, P_old));
        out[id] = __dadd_rn(__dmul_rn(1. - omega, P_old), __dmul_rn(omega, P_new));
        v[0] = nmax(v[0], delta);
        v[1] = __dadd_rn(v[1], delta);
        v[2] = nmax(v[2], P_new);
        v[3] = nmin(v[3], P_new);
        v[4] = nmax(v[4], fabs(f0));
    }
    block_reduce5<BS>(v, sh, partial + (long)blockIdx.x * KF_RED);
}

// Final fixed-order reduction of nb block partials into out[0..4].
template <int BS>
__global__ void __launch_bounds__(BS) k_reduce_final(const double *__restrict__ partial, int nb,
                                                     double *__restrict__ out) {
    __shared__ double sh[KF_RED * BS];
    double v[KF_RED] = {0., 0., -INFINITY, INFINITY, 0.};
    for (int b = threadIdx.x; b < nb; b += BS) {
        const double *p = partial + (long)b * KF_RED;
        v[0] = nmax(v[0], p[0]);
        v[1] = __dadd_rn(v[1], p[1]);
        v[2] = nmax(v[2], p[2]);
        v[3] = nmin(v[3], p[3]);
        v[4] = nmax(v[4], p[4]);
    }
    block_reduce5<BS>(v, sh, out);
}

// Launch geometry of the multigrid kernels: block (32, 8), grid
// (ceil(nx/32), ceil(n/8), n) over (k or k/2, j, i) -- no index division.
inline dim3 mg_grid(int nx, int n) { return dim3((nx + 31) / 32, (n + 7) / 8, n); }
inline dim3 mg_block() { return dim3(32, 8, 1); }

// Pointwise residual r = f(phi) = lap_h phi + rho - e^phi on the whole level;
// with MAX also max |r|, so that the convergence test of a cycle needs no pass
// of its own: each block then covers the i-planes blockIdx.z, blockIdx.z +
// gridDim.z, ... (launched with gridDim.z <= 16), takes the block
// maximum and makes one atomic max on the IEEE bit pattern into one of 64 slots.
template <bool FAST, bool MAX = false>
__global__ void __launch_bounds__(256) k_residual(const double *__restrict__ phi, const double *__restrict__ rho,
                                                  Lev L, double *__restrict__ r,
                                                  unsigned long long *__restrict__ slots = nullptr) {
    const int n = L.n;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
    double af = 0.;
    if (k < n && j < n) {
        for (int i = blockIdx.z; i < n; i += (MAX ? gridDim.z : n)) {
            double A, D;
            coeffs_t<FAST>(phi, rho, L, i, j, k, A, D);
            const long id = lidx(i, j, k, n);
            const double f = f_point(A, D, phi[id]);
            r[id] = f;
            af = nmax(af, fabs(f));
        }
    }
    if constexpr (MAX) {
        __shared__ double sh[8];
        for (int o = 16; o > 0; o >>= 1) af = nmax(af, __shfl_xor_sync(0xffffffffu, af, o));
        if (threadIdx.x == 0) sh[threadIdx.y] = af;
        __syncthreads();
        if (threadIdx.y == 0 && threadIdx.x == 0) {
            double m = sh[0];
            for (int w = 1; w < 8; ++w) m = nmax(m, sh[w]);
            atomicMax(slots + ((blockIdx.x + blockIdx.y * gridDim.x + blockIdx.z) & 63),
                      (unsigned long long)__double_as_longlong(m));
        }
    }
}

// max |f(phi)| over the level: each block covers a (32 x 8) tile of (k, j) for
// the i-planes blockIdx.z, blockIdx.z + gridDim.z, ...; block maximum, then an
// atomic max on the IEEE bit pattern (order-free; NaN sorts above +inf) into
// one of 64 slots.
template <bool FAST>
__global__ void __launch_bounds__(256) k_resmax(const double *__restrict__ phi, const double *__restrict__ rho,
                                                Lev L, unsigned long long *__restrict__ out) {
    __shared__ double sh[8];
    const int n = L.n;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
    double af = 0.;
    if (k < n && j < n) {
        for (int i = blockIdx.z; i < n; i += gridDim.z) {
            double A, D;
            coeffs_t<FAST>(phi, rho, L, i, j, k, A, D);
            af = nmax(af, fabs(f_point(A, D, phi[lidx(i, j, k, n)])));
        }
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

// phi <- phi + w (phi - phi_a), phi_a <- old phi  (start of a solve at a new time)
__global__ void k_extrap(double *__restrict__ phi, double *__restrict__ phi_a, double w, long N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double b = phi[i], a = phi_a[i];
    phi[i] = __dadd_rn(b, __dmul_rn(w, __dsub_rn(b, a)));
    phi_a[i] = b;
}

// Red-black Gauss-Seidel-Newton half sweep (colour (i+j+k)%2): one Newton
// step per point; grid over (k/2, j, i), blocks of 32 x BY (the tile shape
// kf_autotune chooses; the arithmetic does not depend on it).
// The axis tables of a level of at most 256 points per axis, passed by value
// as a kernel parameter: entries read with a warp-uniform index (the i and j
// of a half-sweep warp) come from the constant bank instead of L1.
constexpr int KF_TAB_N = 256;
struct AxTab {
    double dd[KF_TAB_N], ip[KF_TAB_N], im[KF_TAB_N];
};

// The point's index and its six periodic neighbours' are one 32-bit base and
// wrapped offsets (n^3 < 2^31 for every supported n <= 256): the loads, the
// sum and its order are point_coeffs_fast's, with fewer integer instructions.
template <int BY = 8>
__global__ void __launch_bounds__(32 * BY) k_rbgs(double *__restrict__ phi, const double *__restrict__ rho, Lev L,
                                                  int color, double om) {
    const int n = L.n;
    const int k2 = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * BY + threadIdx.y, i = blockIdx.z;
    if (2 * k2 >= n || j >= n) return;
    const int k = 2 * k2 + ((i + j + color) & 1);
    const int nn = n * n;
    const int q = (i * n + j) * n + k;
    const int oip = i == n - 1 ? -(n - 1) * nn : nn, oim = i == 0 ? (n - 1) * nn : -nn;
    const int ojp = j == n - 1 ? -(n - 1) * n : n, ojm = j == 0 ? (n - 1) * n : -n;
    const int okp = k == n - 1 ? -(n - 1) : 1, okm = k == 0 ? n - 1 : -1;
    const double D = __dadd_rn(__dadd_rn(L.dd[i], L.dd[j]), L.dd[k]);
    double A = __dmul_rn(phi[q + oip], L.ip[i]);
    A = __dadd_rn(A, __dmul_rn(phi[q + oim], L.im[i]));
    A = __dadd_rn(A, __dmul_rn(phi[q + ojp], L.ip[j]));
    A = __dadd_rn(A, __dmul_rn(phi[q + ojm], L.im[j]));
    A = __dadd_rn(A, __dmul_rn(phi[q + okp], L.ip[k]));
    A = __dadd_rn(A, __dmul_rn(phi[q + okm], L.im[k]));
    A = __dadd_rn(A, rho[q]);
    phi[q] = newton_step(phi[q], A, D, om);
}

// rho split by colour (the finest level's copy for the half sweeps): the
// point of colour c at k = 2 k2 + ((i + j + c) & 1) is element
// c n^3/2 + (i n + j) n/2 + k2, so a half sweep reads only its own colour's
// rho, contiguously (the natural layout makes it read every sector of rho).
__global__ void __launch_bounds__(256) k_rho_split(const double *__restrict__ rho, double *__restrict__ rcs, int n) {
    const int k2 = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, i = blockIdx.z;
    if (2 * k2 >= n || j >= n) return;
    const int row = (i * n + j) * (n / 2) + k2, half = n * n * (n / 2);
    const double2 v = *reinterpret_cast<const double2 *>(rho + 2 * row);
    const int c0 = (i + j) & 1;  // colour of k = 2 k2
    rcs[c0 * half + row] = v.x;
    rcs[(c0 ^ 1) * half + row] = v.y;
}

// The same half sweep with the i and j tables from the constant bank (AxTab);
// CS: rho is the colour-split copy (k_rho_split), the sum and its order unchanged.
template <int BY = 8, bool CS = false>
__global__ void __launch_bounds__(32 * BY) k_rbgs_t(double *__restrict__ phi, const double *__restrict__ rho, Lev L,
                                                    int color, double om, const __grid_constant__ AxTab T) {
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
    if constexpr (CS)
        A = __dadd_rn(A, rho[color * (nn * (n / 2)) + (i * n + j) * (n / 2) + k2]);
    else
        A = __dadd_rn(A, rho[q]);
    phi[q] = newton_step(phi[q], A, D, om);
}

// ------------------------------------------------------------ column form
// k_residual is bound by L1 throughput (about 17 loads per point: 7
// potentials, rho, 9 axis-table entries, most strided).  In the column form a
// thread owns the k-pair (2 k2, 2 k2 + 1) of row j and marches the planes
// i0 ... i0 + PI - 1 of a column: each plane's pair is one 16-byte load, kept
// in registers as the i-neighbour of the next and previous plane; the
// k-neighbours outside the pair come from the neighbouring lanes by warp
// shuffle (the warp's two edge lanes load theirs); the k tables are read once
// per column.  The arithmetic and its order are those of point_coeffs_fast,
// so the results are bit-identical.  Requires n/2 a multiple of 32 (whole
// warps along k), BY | n and PI | n.
// Resident blocks per SM asked of the register allocator for k_residual_col
// (measured at 256^3, 36 launches: 1 -> 120 registers, 4.09 ms; 3 -> 80
// registers, 3.62 ms; 4 -> 64 registers with a 40-byte spill, 3.40 ms).
#ifndef KF_RESCOL_MINB
#define KF_RESCOL_MINB 4
#endif

// The residual r = f(phi) of both points of the pair at every plane of the
// column (16-byte loads of the pairs of rows j, j -+ 1 and of rho, one 16-byte
// store): the pointwise f of k_residual<true>; with MAX also max |r| as
// k_residual<true, true>; without STORE only the maximum (k_resmax<true>).
// LIN: the adjoint's linear residual A - (D + cl) psi (k_residual_lin,
// k_resmax_lin).
template <int BY, int PI, bool MAX, bool LIN = false, bool STORE = true>
__global__ void __launch_bounds__(32 * BY, KF_RESCOL_MINB) k_residual_col(const double *__restrict__ phi, const double *__restrict__ rho,
                                                          Lev L, double *__restrict__ r,
                                                          unsigned long long *__restrict__ slots,
                                                          const double *__restrict__ cl = nullptr) {
    const int n = L.n;
    const int lane = threadIdx.x;
    const int k2 = blockIdx.x * 32 + lane, j = blockIdx.y * BY + threadIdx.y, i0 = blockIdx.z * PI;
    const int jp = j + 1 == n ? 0 : j + 1, jm = j == 0 ? n - 1 : j - 1;
    const int ka = 2 * k2, kb = ka + 1;
    const int kl = ka == 0 ? n - 1 : ka - 1, kr = kb + 1 == n ? 0 : kb + 1;
    const double dda = L.dd[ka], ipa = L.ip[ka], ima = L.im[ka];
    const double ddb = L.dd[kb], ipb = L.ip[kb], imb = L.im[kb];
    const double ddj = L.dd[j], ipj = L.ip[j], imj = L.im[j];
    // 32-bit element indices (n^3 < 2^31 for every supported n): q = the
    // pair at (i, j, ka); the j, k and next-plane neighbours as offsets
    const int nn = n * n, ojp = (jp - j) * n, ojm = (jm - j) * n, okl = kl - ka, okr = kr - ka;
    int q = (i0 * n + j) * n + ka;
    double2 pm = *reinterpret_cast<const double2 *>(phi + ((wrapi(i0 - 1, n) * n + j) * n + ka));
    double2 pc = *reinterpret_cast<const double2 *>(phi + q);
    double af = 0.;
#pragma unroll 2
    for (int ii = 0; ii < PI; ++ii) {
        const int i = i0 + ii;
        const int qn = i + 1 == n ? q - (n - 1) * nn : q + nn;
        const double2 pn = *reinterpret_cast<const double2 *>(phi + qn);
        const double2 pjp = *reinterpret_cast<const double2 *>(phi + q + ojp);
        const double2 pjm = *reinterpret_cast<const double2 *>(phi + q + ojm);
        const double2 rr = *reinterpret_cast<const double2 *>(rho + q);
        double fromR = __shfl_down_sync(0xffffffffu, pc.x, 1);
        double fromL = __shfl_up_sync(0xffffffffu, pc.y, 1);
        if (lane == 31) fromR = phi[q + okr];
        if (lane == 0) fromL = phi[q + okl];
        const double ipi = L.ip[i], imi = L.im[i], ddi = L.dd[i];
        double Aa = __dmul_rn(pn.x, ipi);
        Aa = __dadd_rn(Aa, __dmul_rn(pm.x, imi));
        Aa = __dadd_rn(Aa, __dmul_rn(pjp.x, ipj));
        Aa = __dadd_rn(Aa, __dmul_rn(pjm.x, imj));
        Aa = __dadd_rn(Aa, __dmul_rn(pc.y, ipa));
        Aa = __dadd_rn(Aa, __dmul_rn(fromL, ima));
        Aa = __dadd_rn(Aa, rr.x);
        double Ab = __dmul_rn(pn.y, ipi);
        Ab = __dadd_rn(Ab, __dmul_rn(pm.y, imi));
        Ab = __dadd_rn(Ab, __dmul_rn(pjp.y, ipj));
        Ab = __dadd_rn(Ab, __dmul_rn(pjm.y, imj));
        Ab = __dadd_rn(Ab, __dmul_rn(fromR, ipb));
        Ab = __dadd_rn(Ab, __dmul_rn(pc.x, imb));
        Ab = __dadd_rn(Ab, rr.y);
        const double Da = __dadd_rn(__dadd_rn(ddi, ddj), dda), Db = __dadd_rn(__dadd_rn(ddi, ddj), ddb);
        double fa, fb;
        if constexpr (LIN) {
            const double2 cp = *reinterpret_cast<const double2 *>(cl + q);
            fa = __dsub_rn(Aa, __dmul_rn(__dadd_rn(Da, cp.x), pc.x));
            fb = __dsub_rn(Ab, __dmul_rn(__dadd_rn(Db, cp.y), pc.y));
        } else {
            fa = f_point(Aa, Da, pc.x);
            fb = f_point(Ab, Db, pc.y);
        }
        if (STORE) *reinterpret_cast<double2 *>(r + q) = make_double2(fa, fb);
        if (MAX) af = nmax(af, nmax(fabs(fa), fabs(fb)));
        pm = pc;
        pc = pn;
        q = qn;
    }
    if constexpr (MAX) {
        __shared__ double sh[BY];
        for (int o = 16; o > 0; o >>= 1) af = nmax(af, __shfl_xor_sync(0xffffffffu, af, o));
        if (lane == 0) sh[threadIdx.y] = af;
        __syncthreads();
        if (threadIdx.y == 0 && lane == 0) {
            double m = sh[0];
            for (int w = 1; w < BY; ++w) m = nmax(m, sh[w]);
            atomicMax(slots + ((blockIdx.x + blockIdx.y * gridDim.x + blockIdx.z * gridDim.x * gridDim.y) & 63),
                      (unsigned long long)__double_as_longlong(m));
        }
    }
}

// Block-wide max of m (NaN-propagating) over up to 1024 threads; sh: 32 doubles.
__device__ __forceinline__ double block_nmax(double m, double *sh) {
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
    return res;
}

// One red-black half sweep (k_rbgs's point update) of a level the block holds.
__device__ __forceinline__ void block_half_sweep(double *sp, const double *sr, const Lev &Ls, int color,
                                                 double om) {
    const int n = Ls.n;
    const int M = n * n * n / 2, nh = n / 2;
    for (int id = threadIdx.x; id < M; id += blockDim.x) {
        const int k2 = id % nh;
        const int r = id / nh;
        const int j = r % n, i = r / n;
        const int k = 2 * k2 + ((i + j + color) & 1);
        double A, D;
        point_coeffs_fast(sp, sr, Ls, i, j, k, A, D);
        const int q = (int)lidx(i, j, k, n);
        sp[q] = newton_step(sp[q], A, D, om);
    }
    __syncthreads();
}

// Coarsest-level relaxation of a level the block holds: red-black sweeps until
// max |f| <= max(tol, 1e-4 max |f| at entry), checked before every sweep (as
// the host loop of the oracle); returns the number of sweeps.
__device__ __forceinline__ int block_coarse_relax(double *sp, const double *sr, const Lev &Ls, double tol,
                                                  int max_sweeps, double om, double *sh) {
    const int n = Ls.n;
    const int N = n * n * n;
    int s = 0;
    double r0 = 0.;
    for (;; ++s) {
        double m = 0.;
        for (int id = threadIdx.x; id < N; id += blockDim.x) {
            const int k = id % n;
            const int r = id / n;
            const int j = r % n, i = r / n;
            double A, D;
            point_coeffs_fast(sp, sr, Ls, i, j, k, A, D);
            m = nmax(m, fabs(f_point(A, D, sp[id])));
        }
        const double res = block_nmax(m, sh);
        if (s == 0) r0 = res;
        if (!(res > fmax(tol, 1e-4 * r0)) || s >= max_sweeps) break;  // converged, NaN or capped
        block_half_sweep(sp, sr, Ls, 0, om);
        block_half_sweep(sp, sr, Ls, 1, om);
    }
    return s;
}

// Coarsest-level solve in one block: the level (phi, rho and the axis tables)
// is staged in shared memory, block_coarse_relax runs, then phi is written
// back.  Dynamic shared memory: 16 n^3 + 24 n bytes.
__global__ void __launch_bounds__(1024) k_coarse_solve(double *__restrict__ phi, const double *__restrict__ rho,
                                                       Lev L, double tol, int max_sweeps,
                                                       int *__restrict__ sweeps_out, double om) {
    extern __shared__ __align__(16) double cs_sm[];
    __shared__ double sh[32];
    const int n = L.n;
    const int N = n * n * n;
    double *sp = cs_sm, *sr = cs_sm + N, *sd = cs_sm + 2 * N, *si = sd + n, *sm_ = si + n;
    for (int id = threadIdx.x; id < N; id += blockDim.x) {
        sp[id] = phi[id];
        sr[id] = rho[id];
    }
    for (int id = threadIdx.x; id < n; id += blockDim.x) {
        sd[id] = L.dd[id];
        si[id] = L.ip[id];
        sm_[id] = L.im[id];
    }
    __syncthreads();
    const Lev Ls{n, sd, nullptr, nullptr, si, sm_};
    const int s = block_coarse_relax(sp, sr, Ls, tol, max_sweeps, om, sh);
    for (int id = threadIdx.x; id < N; id += blockDim.x) phi[id] = sp[id];
    if (threadIdx.x == 0) *sweeps_out = s;
}

// e = phic - phic0 on the coarse level (the correction the prolongation carries)
__global__ void __launch_bounds__(256) k_correction(const double *__restrict__ phic, double *__restrict__ phic0,
                                                    int nc) {
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, i = blockIdx.z;
    if (k >= nc || j >= nc) return;
    const long q = lidx(i, j, k, nc);
    phic0[q] = __dsub_rn(phic[q], phic0[q]);
}

// Full-weighting restriction of r (fine nf) at the coarse point (i, j, k)
__device__ __forceinline__ double fw_point(const double *__restrict__ r, int nf, int i, int j, int k) {
    const double w[3] = {0.25, 0.5, 0.25};
    double s = 0.;
    for (int a = -1; a <= 1; ++a) {
        const int I = (2 * i + a + nf) % nf;
        double sy = 0.;
        for (int b = -1; b <= 1; ++b) {
            const int J = (2 * j + b + nf) % nf;
            double sz = 0.;
            for (int c = -1; c <= 1; ++c) {
                const int K = (2 * k + c + nf) % nf;
                sz = __dadd_rn(sz, __dmul_rn(w[c + 1], r[lidx(I, J, K, nf)]));
            }
            sy = __dadd_rn(sy, __dmul_rn(w[b + 1], sz));
        }
        s = __dadd_rn(s, __dmul_rn(w[a + 1], sy));
    }
    return s;
}

// Full-weighting restriction of r (fine n) and injection of phi:
// rc = FW(r), phic = phic0 = phi[2i,2j,2k]  (field_interpolation.cpp:233-259 for phi)
__global__ void __launch_bounds__(256) k_restrict(const double *__restrict__ r, const double *__restrict__ phi, int nf,
                                                  double *__restrict__ rc, double *__restrict__ phic,
                                                  double *__restrict__ phic0) {
    const int nc = nf / 2;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, i = blockIdx.z;
    if (k >= nc || j >= nc) return;
    const long id = lidx(i, j, k, nc);
    rc[id] = fw_point(r, nf, i, j, k);
    const double p = phi[lidx(2 * i, 2 * j, 2 * k, nf)];
    phic[id] = p;
    phic0[id] = p;
}

// rho_c = N_c(phi_c) + r_c with N(phi) = -lap_h phi + e^phi, at one point
__device__ __forceinline__ double fas_rho_point(const double *__restrict__ phic, double rc, const Lev &L, int i, int j,
                                                int k) {
    double A, D;
    point_coeffs_fast(phic, nullptr, L, i, j, k, A, D);
    const double Nc = __dsub_rn(0., f_point(A, D, phic[lidx(i, j, k, L.n)]));
    return __dadd_rn(Nc, rc);
}

__global__ void __launch_bounds__(256) k_fas_rhs(const double *__restrict__ phic, const double *__restrict__ rc, Lev L,
                                                 double *__restrict__ rhoc) {
    const int n = L.n;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, i = blockIdx.z;
    if (k >= n || j >= n) return;
    const long id = lidx(i, j, k, n);
    rhoc[id] = fas_rho_point(phic, rc[id], L, i, j, k);
}

// Trilinear prolongation of e = phic - phic0 in the z, y, x pass order of
// OP_hto2h (field_interpolation.cpp:56-147), added to phi:  phi += P e.
// gam[m] = (x_m - x_{m-1}) / (x_{m+1} - x_{m-1}) on the fine axis (odd m).
__device__ __forceinline__ double e_c(const double *pc, const double *pc0, int nc, int I, int J, int K) {
    const long q = lidx(I, J, K, nc);
    return pc0 ? __dsub_rn(pc[q], pc0[q]) : pc[q];
}
__device__ __forceinline__ double pz(const double *pc, const double *pc0, const double *gam, int nf, int i, int j, int k) {
    const int nc = nf / 2;
    if ((k & 1) == 0) return e_c(pc, pc0, nc, i / 2, j / 2, k / 2);
    const double g = gam[k];
    const int k1 = (k - 1) / 2, k2 = ((k + 1) % nf) / 2;
    return __dadd_rn(__dmul_rn(1. - g, e_c(pc, pc0, nc, i / 2, j / 2, k1)), __dmul_rn(g, e_c(pc, pc0, nc, i / 2, j / 2, k2)));
}
__device__ __forceinline__ double py(const double *pc, const double *pc0, const double *gam, int nf, int i, int j, int k) {
    if ((j & 1) == 0) return pz(pc, pc0, gam, nf, i, j, k);
    const double g = gam[j];
    return __dadd_rn(__dmul_rn(1. - g, pz(pc, pc0, gam, nf, i, j - 1, k)),
                     __dmul_rn(g, pz(pc, pc0, gam, nf, i, (j + 1) % nf, k)));
}
// The coarse cell (I, J, K): the 8 fine points (2I+a, 2J+b, 2K+c) from the 8
// corner values, with OP_hto2h's z, y, x passes and gammas (the same
// operations per fine point as interpolating the whole field pass by pass).
__device__ __forceinline__ void prolong_cell(double *__restrict__ phi, const double *__restrict__ e,
                                             const double *__restrict__ gam, int nf, int I, int J, int K) {
    const int nc = nf / 2;
    const int I1 = I + 1 == nc ? 0 : I + 1, J1 = J + 1 == nc ? 0 : J + 1, K1 = K + 1 == nc ? 0 : K + 1;
    // corner values e[I+di][J+dj][K+dk]
    double c[2][2][2];
    c[0][0][0] = e[lidx(I, J, K, nc)];
    c[0][0][1] = e[lidx(I, J, K1, nc)];
    c[0][1][0] = e[lidx(I, J1, K, nc)];
    c[0][1][1] = e[lidx(I, J1, K1, nc)];
    c[1][0][0] = e[lidx(I1, J, K, nc)];
    c[1][0][1] = e[lidx(I1, J, K1, nc)];
    c[1][1][0] = e[lidx(I1, J1, K, nc)];
    c[1][1][1] = e[lidx(I1, J1, K1, nc)];
    const double gz = gam[2 * K + 1], gy = gam[2 * J + 1], gx = gam[2 * I + 1];
    // z pass on the even (i, j) columns: zc[di][dj][c] for fine k = 2K + c
    double zc[2][2][2];
#pragma unroll
    for (int di = 0; di < 2; ++di)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj) {
            zc[di][dj][0] = c[di][dj][0];
            zc[di][dj][1] = __dadd_rn(__dmul_rn(1. - gz, c[di][dj][0]), __dmul_rn(gz, c[di][dj][1]));
        }
    // y pass on the even i planes: yc[di][b][c] for fine j = 2J + b
    double yc[2][2][2];
#pragma unroll
    for (int di = 0; di < 2; ++di)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            yc[di][0][cc] = zc[di][0][cc];
            yc[di][1][cc] = __dadd_rn(__dmul_rn(1. - gy, zc[di][0][cc]), __dmul_rn(gy, zc[di][1][cc]));
        }
    // x pass and the update of the 8 fine points
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const double v = a == 0 ? yc[0][b][cc]
                                        : __dadd_rn(__dmul_rn(1. - gx, yc[0][b][cc]), __dmul_rn(gx, yc[1][b][cc]));
                const long q = lidx(2 * I + a, 2 * J + b, 2 * K + cc, nf);
                phi[q] = __dadd_rn(phi[q], v);
            }
}

// phi += P e, one thread per coarse cell
__global__ void __launch_bounds__(256) k_prolong_add(double *__restrict__ phi, const double *__restrict__ e,
                                                     const double *__restrict__ unused,
                                                     const double *__restrict__ gam, int nf) {
    (void)unused;
    const int nc = nf / 2;
    const int K = blockIdx.x * 32 + threadIdx.x, J = blockIdx.y * 8 + threadIdx.y, I = blockIdx.z;
    if (K >= nc || J >= nc) return;
    prolong_cell(phi, e, gam, nf, I, J, K);
}

// ------------------------------------------------------------ coarse levels in one block
// Levels of at most 16^3 points hold at most 4096 points: the kernels of one
// V-cycle there (half-sweeps, residual, restriction, FAS right-hand side,
// coarsest solve, correction, prolongation: 14 launches from the 16^3 level
// down to 8^3) each run for about the time of their launch.  k_coarse_cycle
// runs all of it in one block with every level in shared memory, from the
// entry level's injected potential and restricted residual (k_restrict) to
// its correction e = phi - phi0 (left in phi0 for k_prolong_add), with the
// per-point arithmetic of the level-by-level kernels, so the potentials are
// the same bit for bit.
constexpr int KF_CC_LEVELS = 4;

struct CoarseCycle {
    int nl;  // levels held: 0 = the entry level, nl - 1 = the coarsest (2 <= nl <= KF_CC_LEVELS)
    int n[KF_CC_LEVELS];
    const double *dd[KF_CC_LEVELS], *ip[KF_CC_LEVELS], *im[KF_CC_LEVELS];
    const double *gam[KF_CC_LEVELS];  // fine-axis gammas of level m (prolongation from m + 1)
};

// Shared memory of k_coarse_cycle: per level phi, rho, r, phi0 (n^3 each) and
// four axis tables (n each).
inline size_t coarse_cycle_smem(const CoarseCycle &C) {
    size_t b = 0;
    for (int m = 0; m < C.nl; ++m) b += 8 * (4 * (size_t)C.n[m] * C.n[m] * C.n[m] + 4 * (size_t)C.n[m]);
    return b;
}

// Level m of the shared-memory layout of k_coarse_cycle.
struct CcLevel {
    double *P, *R, *F, *P0;  // phi, rho, r, phi0
    Lev L;                   // n and the tables dd, ip, im (in shared memory)
    double *G;               // gammas (in shared memory)
};
__device__ __forceinline__ CcLevel cc_level(const CoarseCycle &C, double *sm, int m) {
    for (int l = 0; l < m; ++l) sm += 4 * (C.n[l] * C.n[l] * C.n[l] + C.n[l]);
    const int n = C.n[m], N = n * n * n;
    double *t = sm + 4 * N;
    return CcLevel{sm, sm + N, sm + 2 * N, sm + 3 * N, Lev{n, t, nullptr, nullptr, t + n, t + 2 * n}, t + 3 * n};
}

__global__ void __launch_bounds__(1024) k_coarse_cycle(double *__restrict__ phi, double *__restrict__ phi0,
                                                       const double *__restrict__ r, CoarseCycle C, int pre,
                                                       int post, double tol, int max_sweeps, double om,
                                                       int *__restrict__ sweeps_out) {
    extern __shared__ __align__(16) double cc_sm[];
    __shared__ double sh[32];
    for (int m = 0; m < C.nl; ++m) {
        const CcLevel V = cc_level(C, cc_sm, m);
        double *dd = const_cast<double *>(V.L.dd), *ip = const_cast<double *>(V.L.ip);
        double *im = const_cast<double *>(V.L.im);
        for (int t = threadIdx.x; t < V.L.n; t += blockDim.x) {
            dd[t] = C.dd[m][t];
            ip[t] = C.ip[m][t];
            im[t] = C.im[m][t];
            V.G[t] = C.gam[m] ? C.gam[m][t] : 0.;
        }
    }
    {
        const CcLevel V = cc_level(C, cc_sm, 0);
        const int N = C.n[0] * C.n[0] * C.n[0];
        for (int id = threadIdx.x; id < N; id += blockDim.x) {
            V.P[id] = phi[id];
            V.R[id] = r[id];
        }
    }
    __syncthreads();
    // the entry level's FAS right-hand side (k_fas_rhs) in place of its r;
    // on the levels below, the restriction leaves r in R the same way
    for (int m = 0; m < C.nl; ++m) {
        const CcLevel V = cc_level(C, cc_sm, m);
        const int n = V.L.n, N = n * n * n;
        for (int id = threadIdx.x; id < N; id += blockDim.x) {
            const int k = id % n, j = (id / n) % n, i = id / (n * n);
            V.R[id] = fas_rho_point(V.P, V.R[id], V.L, i, j, k);
        }
        __syncthreads();
        if (m + 1 == C.nl) break;
        // pre-smoothing, residual (k_residual<true>), restriction and injection (k_restrict)
        for (int s = 0; s < pre; ++s) {
            block_half_sweep(V.P, V.R, V.L, 0, om);
            block_half_sweep(V.P, V.R, V.L, 1, om);
        }
        for (int id = threadIdx.x; id < N; id += blockDim.x) {
            const int k = id % n, j = (id / n) % n, i = id / (n * n);
            double A, D;
            point_coeffs_fast(V.P, V.R, V.L, i, j, k, A, D);
            V.F[id] = f_point(A, D, V.P[id]);
        }
        __syncthreads();
        const CcLevel W = cc_level(C, cc_sm, m + 1);
        const int nc = n / 2, Ncc = nc * nc * nc;
        for (int id = threadIdx.x; id < Ncc; id += blockDim.x) {
            const int k = id % nc, j = (id / nc) % nc, i = id / (nc * nc);
            W.R[id] = fw_point(V.F, n, i, j, k);
            const double p = V.P[lidx(2 * i, 2 * j, 2 * k, n)];
            W.P[id] = p;
            W.P0[id] = p;
        }
        __syncthreads();
    }
    const CcLevel Vc = cc_level(C, cc_sm, C.nl - 1);
    const int s = block_coarse_relax(Vc.P, Vc.R, Vc.L, tol, max_sweeps, om, sh);
    for (int m = C.nl - 2; m >= 0; --m) {
        // correction (k_correction), prolongation (k_prolong_add), post-smoothing
        const CcLevel V = cc_level(C, cc_sm, m), W = cc_level(C, cc_sm, m + 1);
        const int n = V.L.n, nc = n / 2, Ncc = nc * nc * nc;
        for (int id = threadIdx.x; id < Ncc; id += blockDim.x) W.P0[id] = __dsub_rn(W.P[id], W.P0[id]);
        __syncthreads();
        for (int id = threadIdx.x; id < Ncc; id += blockDim.x) {
            const int K = id % nc, J = (id / nc) % nc, I = id / (nc * nc);
            prolong_cell(V.P, W.P0, V.G, n, I, J, K);
        }
        __syncthreads();
        for (int t = 0; t < post; ++t) {
            block_half_sweep(V.P, V.R, V.L, 0, om);
            block_half_sweep(V.P, V.R, V.L, 1, om);
        }
    }
    const CcLevel V0 = cc_level(C, cc_sm, 0);
    const int N = C.n[0] * C.n[0] * C.n[0];
    for (int id = threadIdx.x; id < N; id += blockDim.x) {
        const double p = V0.P[id];
        phi[id] = p;
        phi0[id] = __dsub_rn(p, phi0[id]);
    }
    if (threadIdx.x == 0 && sweeps_out) *sweeps_out = s;
}

// Strided injection (OP_2htoh_lvl0 / OP_4htoh / OP_8htoh)
__global__ void __launch_bounds__(256) k_inject(const double *__restrict__ in, int nf, int step,
                                                double *__restrict__ out) {
    const int nc = nf / step;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, i = blockIdx.z;
    if (k >= nc || j >= nc) return;
    out[lidx(i, j, k, nc)] = in[lidx(step * i, step * j, step * k, nf)];
}

// OP_hto2h (plain, not a correction): out(2n) = trilinear(in(n)); used by the
// cascadic plan.  Same pass order as k_prolong_add with phic0 == 0.
__global__ void __launch_bounds__(256) k_prolong_set(double *__restrict__ out, const double *__restrict__ pc,
                                                     const double *__restrict__ gam, int nf) {
    const double *zero = nullptr;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, i = blockIdx.z;
    if (k >= nf || j >= nf) return;
    const long id = lidx(i, j, k, nf);
    double e;
    if ((i & 1) == 0) {
        e = py(pc, zero, gam, nf, i, j, k);
    } else {
        const double g = gam[i];
        e = __dadd_rn(__dmul_rn(1. - g, py(pc, zero, gam, nf, i - 1, j, k)),
                      __dmul_rn(g, py(pc, zero, gam, nf, (i + 1) % nf, j, k)));
    }
    out[id] = e;
}

}  // namespace kf
