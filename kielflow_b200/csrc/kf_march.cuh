// kf_march.cuh -- the FAS cycle's red-black smoother as one streaming pass per
// sweep (FP64): TMA-staged tiles, temporal blocking of the two colour
// half-sweeps in shared memory, and the residual fused into the last pass.
//
// The arithmetic per point is the one of k_rbgs / k_residual (kf_poisson.cuh):
// the 7-point operator of the axis spacings H[i] (solver_poisson_jacobi_nlin.cpp
// :177-211, weights 2/den precomputed) and one over-relaxed Newton step on
// A - D x - e^x = 0, in the same order of operations, so a launch of this kernel
// gives the potentials of two k_rbgs launches bit for bit.
//
// Layout.  A CTA owns a tile of TK = 64 (k, contiguous) x TJ (j) points and a
// chunk of CI i-planes.  It streams the planes i0 - H ... i0 + CI + H - 1 of phi
// (and of rho) through a ring of shared-memory slots; each staged plane is the
// tile plus a halo (H rows in j, HK columns in k), fetched as one 80-double row
// per TMA copy (cp.async.bulk.tensor.3d, the row's j and i coordinates wrapped
// on the host side of the copy, so the periodic box needs no special case in j
// and i; the k halo of the two edge tiles is patched with plain loads).  At
// plane step t the stages run as a wavefront, stage s on plane t - 1 - s:
//   MM_SWEEP      colour 0 (margin 1), colour 1 (margin 0)  -> phi_out
//   MM_SWEEP_RES  colour 0 (margin 2), colour 1 (margin 1), residual (margin 0)
//                                                             -> phi_out, r, max|r|
//   MM_RES        residual only                              -> r, max|r|
// (margin m: the stage covers the tile grown by m points in j, k and i, what
// the later stages read).  Each colour update in a slot is in place: the
// points of one colour read only points of the other, and the wavefront order
// (stage 0 on plane p before stage 1 on plane p - 1 within a step) gives every
// read the value the two-launch sweep gives it.  The input phi is never
// written (phi_out is another array): neighbouring tiles read their halos
// from it while this tile runs.
//
// Waits on the copies are bounded: a wait that gives up sets *err, waits (also
// bounded) for the copies still in flight, and the CTA returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kf_poisson.cuh"

namespace kf {

constexpr int MT_TK = 64;     // interior points of a tile along k
constexpr int MT_PITCH = 80;  // doubles per staged row = the TMA box width (640 B, 5 x 128 B)
constexpr int MT_THREADS = 256;

enum MarchMode : int { MM_RES = 0, MM_SWEEP = 1, MM_SWEEP_RES = 2 };

template <int MODE, int TJ, int PF_ = 2> struct MarchShape {
    static constexpr int NST = MODE == MM_RES ? 1 : (MODE == MM_SWEEP ? 2 : 3);  // stages per plane
    static constexpr int H = NST;              // phi halo rows (j) and ghost planes (i)
    static constexpr int HK = (NST + 1) & ~1;  // phi halo columns (k): even, so the copy's x is 16-byte aligned
    static constexpr int RH = NST - 1;         // rho halo rows
    static constexpr int RK = 2;               // rho halo columns (>= NST - 1, even)
    static constexpr int PF = PF_;             // planes fetched ahead
    static constexpr int S = NST + PF + 1;     // ring slots
    static constexpr int PROWS = TJ + 2 * H;   // staged phi rows
    static constexpr int RROWS = TJ + 2 * RH;  // staged rho rows
    static constexpr int PSLOT = PROWS * MT_PITCH;  // doubles per phi slot
    static constexpr int RSLOT = RROWS * MT_PITCH;  // doubles per rho slot
    static constexpr int NPATCH = 2 * (HK * PROWS + RK * RROWS);  // k-wrap patch values (both edges)
    static_assert(2 * HK + MT_TK <= MT_PITCH, "phi tile does not fit the staged row");
    static_assert(2 * RK + MT_TK <= MT_PITCH, "rho tile does not fit the staged row");
    static_assert(NPATCH <= MT_THREADS, "one patch value per thread");
    static_assert((TJ * MT_TK / 2) % MT_THREADS == 0, "whole 16-byte phi stores per thread and plane");
};

// dynamic shared memory of a launch with chunks of ci planes
template <int MODE, int TJ, int PF = 2> inline size_t march_smem(int ci) {
    using Sh = MarchShape<MODE, TJ, PF>;
    const int np = ci + 2 * Sh::H;
    return 128 + 8 * (size_t)Sh::S * (Sh::PSLOT + Sh::RSLOT)  // ring (128: base alignment)
           + 8 * (size_t)3 * (MT_PITCH + Sh::PROWS + np)      // axis tables
           + 8 * (size_t)Sh::S                                 // mbarriers
           + 8 * 32;                                           // reduction scratch
}

struct MarchArgs {
    double *phi_out;             // MM_SWEEP, MM_SWEEP_RES
    double *r_out;               // MM_RES, MM_SWEEP_RES
    const double *phi_in;        // the staged potential (for the k-wrap patches)
    const double *rho;
    const double *dd, *ip, *im;  // axis tables of the level (kf_poisson.cuh Lev)
    unsigned long long *slots;   // 64 slots of max |r| (IEEE bit patterns), or nullptr
    int *err;                    // bit 0 set when a copy wait gives up
    int n, ci, ntk;              // grid, planes per chunk, tiles along k
    double om;                   // over-relaxation of the Newton step
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// true once the phase of the given parity has completed; false after about
// `limit` clock cycles (a copy that never lands)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit) {
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) return false;
    }
}

// one row of a 3-D tensor (x fastest) into shared memory, completing on bar
__device__ __forceinline__ void tma_row(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ int wrapn(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// One colour update of the point at staged offset o: the arithmetic of
// point_coeffs_fast + newton_step (kf_poisson.cuh) on the staged planes.
struct MarchPoint {
    int o, ro, rr, cc;
};

// MODE: MM_*; TJ: tile rows; PF: planes fetched ahead; PAIR: each thread
// takes two points at a time (loads of both, then both Newton steps), for
// independent work in flight; MINB: resident CTAs per SM the registers allow.
template <int MODE, int TJ, int PF = 2, bool PAIR = false, int MINB = 2>
__global__ void __launch_bounds__(MT_THREADS, MINB)
    k_rbgs_march(const __grid_constant__ CUtensorMap tm_phi, const __grid_constant__ CUtensorMap tm_rho,
                 MarchArgs a) {
    using Sh = MarchShape<MODE, TJ, PF>;
    constexpr int NST = Sh::NST, H = Sh::H, HK = Sh::HK, RH = Sh::RH, RK = Sh::RK, S = Sh::S;
    constexpr int W = MT_PITCH;
    constexpr bool SWEEP = MODE != MM_RES, RES = MODE != MM_SWEEP;
    constexpr long long WAIT_LIMIT = 4000000000LL;  // about 2 s at the boost clock

    extern __shared__ unsigned char march_raw[];
    double *ring = (double *)(((uintptr_t)march_raw + 127) & ~(uintptr_t)127);
    double *sphi = ring;                   // S slots x PROWS x W
    double *srho = sphi + S * Sh::PSLOT;   // S slots x RROWS x W
    const int n = a.n, ci = a.ci, np = ci + 2 * H;
    double *tk = srho + S * Sh::RSLOT;     // k tables: dd, ip, im  [W each]
    double *tj = tk + 3 * W;               // j tables [PROWS each]
    double *ti = tj + 3 * Sh::PROWS;       // i tables [np each]
    uint64_t *bar = (uint64_t *)(ti + 3 * np);
    double *red = (double *)(bar + S);

    const int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int kt = tile % a.ntk, jt = tile / a.ntk;
    const int k0 = kt * MT_TK, j0 = jt * TJ, i0 = blockIdx.y * ci;
    const bool left = k0 == 0, right = k0 + MT_TK == n;

    // axis tables of the tile, wrapped (n >= MT_TK, so one wrap suffices)
    for (int c = tid; c < W; c += MT_THREADS) {
        const int k = wrapn(k0 - HK + c, n);
        tk[c] = a.dd[k];
        tk[W + c] = a.ip[k];
        tk[2 * W + c] = a.im[k];
    }
    for (int r = tid; r < Sh::PROWS; r += MT_THREADS) {
        const int j = wrapn(j0 - H + r, n);
        tj[r] = a.dd[j];
        tj[Sh::PROWS + r] = a.ip[j];
        tj[2 * Sh::PROWS + r] = a.im[j];
    }
    for (int p = tid; p < np; p += MT_THREADS) {
        const int i = wrapn(i0 - H + p, n);
        ti[p] = a.dd[i];
        ti[np + p] = a.ip[i];
        ti[2 * np + p] = a.im[i];
    }
    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(bar + s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // copies of plane p (phi and rho rows) by warp 0
    auto issue = [&](int p) {
        const int s = p % S;
        const int iw = wrapn(i0 - H + p, n);
        const int lane = tid;  // warp 0 only
        if (lane == 0) mbar_expect_tx(bar + s, (uint32_t)(8 * W * (Sh::PROWS + Sh::RROWS)));
        __syncwarp();
        for (int r = lane; r < Sh::PROWS + Sh::RROWS; r += 32) {
            if (r < Sh::PROWS)
                tma_row(sphi + s * Sh::PSLOT + r * W, &tm_phi, k0 - HK, wrapn(j0 - H + r, n), iw, bar + s);
            else
                tma_row(srho + s * Sh::RSLOT + (r - Sh::PROWS) * W, &tm_rho, k0 - RK,
                        wrapn(j0 - RH + r - Sh::PROWS, n), iw, bar + s);
        }
    };
    // k-wrap patch of plane p: this thread's slot address and source value
    const int npatch = (left ? Sh::NPATCH / 2 : 0) + (right ? Sh::NPATCH / 2 : 0);
    auto patch_src = [&](int p, double *&dst) -> double {
        int q = tid;
        const bool lft = left && q < Sh::NPATCH / 2;
        if (left && !lft) q -= Sh::NPATCH / 2;
        const int iw = wrapn(i0 - H + p, n);
        const int s = p % S;
        const int nphi = HK * Sh::PROWS;
        if (q < nphi) {
            const int r = q / HK, c = q % HK;
            const int col = lft ? c : HK + MT_TK + c;  // staged column
            const int k = lft ? n - HK + c : c;        // wrapped source column
            const int j = wrapn(j0 - H + r, n);
            dst = sphi + s * Sh::PSLOT + r * W + col;
            return a.phi_in[((long)iw * n + j) * n + k];
        }
        q -= nphi;
        const int r = q / RK, c = q % RK;
        const int col = lft ? c : RK + MT_TK + c;
        const int k = lft ? n - RK + c : c;
        const int j = wrapn(j0 - RH + r, n);
        dst = srho + s * Sh::RSLOT + r * W + col;
        return a.rho[((long)iw * n + j) * n + k];
    };

    bool ok = true;
    // prologue: planes 0 .. PF + 1 in flight; planes 0, 1 landed and patched
    int nissued = np < PF + 2 ? np : PF + 2, nlanded = 0;
    if (tid < 32)
        for (int p = 0; p < nissued; ++p) issue(p);
    double pv = 0.;
    double *pdst = nullptr;
    for (int p = 0; p < 2; ++p) {
        ok = ok && mbar_wait(bar + (p % S), (uint32_t)((p / S) & 1), WAIT_LIMIT);
        if (ok) nlanded = p + 1;
        if (ok && tid < npatch) {
            const double v = patch_src(p, pdst);
            *pdst = v;
        }
    }
    if (tid < npatch && 2 < np) pv = patch_src(2, pdst);
    double amax = 0.;

    for (int t = 2; t < np && !__syncthreads_or(!ok); ++t) {
        ok = mbar_wait(bar + (t % S), (uint32_t)((t / S) & 1), WAIT_LIMIT);
        if (__syncthreads_or(!ok)) break;
        nlanded = t + 1;
        if (tid < npatch) *pdst = pv;
        __syncthreads();
#pragma unroll
        for (int s = 0; s < NST; ++s) {
            const int p = t - 1 - s;
            if (p < s + 1 || p >= np - 1 - s) continue;  // outside this stage's planes (uniform)
            const int m = NST - 1 - s;                   // margin of the stage
            const int iu = i0 - H + p;                   // unwrapped plane index (parity)
            const double *pm = sphi + ((p - 1) % S) * Sh::PSLOT;
            double *pc = sphi + (p % S) * Sh::PSLOT;
            const double *pp = sphi + ((p + 1) % S) * Sh::PSLOT;
            const double *rc = srho + (p % S) * Sh::RSLOT;
            const double ddi = ti[p], ipi = ti[np + p], imi = ti[2 * np + p];
            const bool is_res = RES && s == NST - 1;
            if (!is_res) {
                const int color = s;  // colour 0, then colour 1
                const int ppr = MT_TK / 2 + m;  // points of the colour per row
                const int items = (TJ + 2 * m) * ppr;
                auto locate = [&](int it) {
                    const int row = it / ppr, pr = it - row * ppr;
                    const int ju = j0 - m + row;
                    const int ks = k0 - m;
                    const int k = ks + 2 * pr + ((color + iu + ju + ks) & 1);
                    MarchPoint P;
                    P.rr = row + H - m;
                    P.cc = k - k0 + HK;
                    P.o = P.rr * W + P.cc;
                    P.ro = (row + RH - m) * W + (k - k0 + RK);
                    return P;
                };
                auto coeffs = [&](const MarchPoint &P, double &A, double &D) {
                    const double *q = pc + P.o;
                    A = __dmul_rn(pp[P.o], ipi);
                    A = __dadd_rn(A, __dmul_rn(pm[P.o], imi));
                    A = __dadd_rn(A, __dmul_rn(q[W], tj[Sh::PROWS + P.rr]));
                    A = __dadd_rn(A, __dmul_rn(q[-W], tj[2 * Sh::PROWS + P.rr]));
                    A = __dadd_rn(A, __dmul_rn(q[1], tk[W + P.cc]));
                    A = __dadd_rn(A, __dmul_rn(q[-1], tk[2 * W + P.cc]));
                    A = __dadd_rn(A, rc[P.ro]);
                    D = __dadd_rn(__dadd_rn(ddi, tj[P.rr]), tk[P.cc]);
                };
                if constexpr (PAIR) {
                    // the points of one colour read only the other colour:
                    // both loads before both stores give the same values
                    for (int it = tid; it < items; it += 2 * MT_THREADS) {
                        const int it2 = it + MT_THREADS;
                        const bool two = it2 < items;
                        const MarchPoint P0 = locate(it), P1 = locate(two ? it2 : it);
                        double A0, D0, A1, D1;
                        coeffs(P0, A0, D0);
                        coeffs(P1, A1, D1);
                        const double x0 = pc[P0.o], x1 = pc[P1.o];
                        const double y0 = newton_step(x0, A0, D0, a.om);
                        const double y1 = newton_step(x1, A1, D1, a.om);
                        pc[P0.o] = y0;
                        if (two) pc[P1.o] = y1;
                    }
                } else {
                    for (int it = tid; it < items; it += MT_THREADS) {
                        const MarchPoint P = locate(it);
                        double A, D;
                        coeffs(P, A, D);
                        pc[P.o] = newton_step(pc[P.o], A, D, a.om);
                    }
                }
                __syncthreads();
                if (SWEEP && s == 1 && p >= H && p < H + ci) {
                    // the plane's potential is final: 16-byte stores of the interior
#pragma unroll
                    for (int u = 0; u < TJ * MT_TK / 2 / MT_THREADS; ++u) {
                        const int e = tid + u * MT_THREADS;
                        const int row = e / (MT_TK / 2), c2 = e % (MT_TK / 2);
                        const double2 v = *(const double2 *)(pc + (row + H) * W + HK + 2 * c2);
                        *(double2 *)(a.phi_out + ((long)wrapn(iu, n) * n + j0 + row) * n + k0 + 2 * c2) = v;
                    }
                }
            } else {
                // residual on the tile's interior of plane p (all points)
                const int iw = wrapn(iu, n);
                for (int it = tid; it < TJ * MT_TK; it += MT_THREADS) {
                    const int row = it / MT_TK, kk = it % MT_TK;
                    const int rr = row + H, cc = kk + HK;
                    const int o = rr * W + cc;
                    const double *q = pc + o;
                    double A = __dmul_rn(pp[o], ipi);
                    A = __dadd_rn(A, __dmul_rn(pm[o], imi));
                    A = __dadd_rn(A, __dmul_rn(q[W], tj[Sh::PROWS + rr]));
                    A = __dadd_rn(A, __dmul_rn(q[-W], tj[2 * Sh::PROWS + rr]));
                    A = __dadd_rn(A, __dmul_rn(q[1], tk[W + cc]));
                    A = __dadd_rn(A, __dmul_rn(q[-1], tk[2 * W + cc]));
                    A = __dadd_rn(A, rc[(row + RH) * W + kk + RK]);
                    const double D = __dadd_rn(__dadd_rn(ddi, tj[rr]), tk[cc]);
                    const double f = f_point(A, D, q[0]);
                    a.r_out[((long)iw * n + j0 + row) * n + k0 + kk] = f;
                    amax = nmax(amax, fabs(f));
                }
            }
        }
        // the slots of planes t + PF (the oldest planes) are free now
        fence_proxy_async();
        __syncthreads();
        if (t + PF < np) {
            if (tid < 32) issue(t + PF);
            nissued = t + PF + 1;
        }
        if (tid < npatch && t + 1 < np) pv = patch_src(t + 1, pdst);
    }

    if (__syncthreads_or(!ok)) {
        // a copy did not land in time: record it, let the copies still in
        // flight finish (bounded waits) before the CTA's shared memory is
        // released, and return
        if (tid == 0) {
            atomicOr(a.err, 1);
            for (int p = nlanded; p < nissued; ++p) mbar_wait(bar + (p % S), (uint32_t)((p / S) & 1), WAIT_LIMIT / 8);
        }
        return;
    }
    if (RES && a.slots) {
        for (int o = 16; o > 0; o >>= 1) amax = nmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        if ((tid & 31) == 0) red[tid >> 5] = amax;
        __syncthreads();
        if (tid == 0) {
            double mx = red[0];
            for (int w = 1; w < MT_THREADS / 32; ++w) mx = nmax(mx, red[w]);
            atomicMax(a.slots + ((blockIdx.x + blockIdx.y * gridDim.x) & 63),
                      (unsigned long long)__double_as_longlong(mx));
        }
    }
}

}  // namespace kf
