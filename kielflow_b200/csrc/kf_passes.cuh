// kf_passes.cuh -- the transform passes of the spectral right-hand side.
//
// A 3-D real transform of the reference's layout (real n^3, half spectrum
// n x n x (n/2+1), z fastest; field_base.hpp:23-24, field_imag.cpp:16) is done
// in three passes, each one read and one write of HBM:
//   inverse : x pass (complex) -> y pass (complex) -> z pass (c2r, x 1/N)
//   forward : z pass (r2c)     -> y pass (complex) -> x pass (complex)
// The x and y passes load a tile of TC contiguous columns by the whole line
// (coalesced 128-byte row segments), transform it with the Stockham engine and
// store it back in place of the same tile of another buffer.  The z passes
// pack two real rows into one complex line (z = a + i b).  Loads apply the
// spectral multipliers of the right-hand side (2/3 mask, i k) so derivative
// fields are generated on the fly instead of being written out.
#pragma once

#include "kf_fft.cuh"
#include "kf_types.cuh"

namespace kf {

// Columns per x/y-pass tile: one 128-byte row segment per line by default.
#ifndef KF_TC64
#define KF_TC64 8
#endif
#ifndef KF_TC32
#define KF_TC32 16
#endif
template <typename T> struct Tile { static constexpr int TC = sizeof(T) == 8 ? KF_TC64 : KF_TC32; };


template <typename T2>
__device__ __forceinline__ T2 mul_ik(T2 a, decltype(T2::x) k) {  // i k a
    return mk<T2>(-k * a.y, k * a.x);
}

// --------------------------------------------------------------- x / y pass
// axis 0: columns are the flattened (j, kz) plane, line index i, stride n*nzc.
// axis 1: columns are kz within an x-plane, line index j, stride nzc.
// gridDim.x = njobs * ntiles (job fastest so that jobs sharing an input run
// together and hit L2).
template <typename T, int N, int SIGN>
__global__ void __launch_bounds__(Tile<T>::TC * Plan<N>::P)
k_axis_pass(const AxisJob *__restrict__ jobs, int njobs, int axis, Geo<T> g,
            const typename C2<T>::type *__restrict__ tw) {
    typedef typename C2<T>::type T2;
    constexpr int TC = Tile<T>::TC, P = Plan<N>::P, E = N / P;
    extern __shared__ __align__(16) unsigned char kf_smem[];
    T2 *sm = reinterpret_cast<T2 *>(kf_smem);
    const int job = blockIdx.x % njobs, tile = blockIdx.x / njobs;
    const AxisJob J = jobs[job];
    const T2 *__restrict__ in = static_cast<const T2 *>(J.in);
    T2 *__restrict__ out = static_cast<T2 *>(J.out);
    const int c = threadIdx.x % TC, p = threadIdx.x / TC;
    const int n = g.n, nzc = g.nzc;
    long base;
    long rstride;
    int jj = 0, kk = 0;
    bool valid;
    if (axis == 0) {
        const int col = tile * TC + c;
        valid = col < n * nzc;
        base = col;
        rstride = (long)n * nzc;
        jj = col / nzc;
        kk = col - jj * nzc;
    } else {
        const int tpp = (nzc + TC - 1) / TC;
        const int plane = tile / tpp;
        kk = (tile - plane * tpp) * TC + c;
        valid = kk < nzc;
        base = (long)plane * n * nzc + kk;
        rstride = nzc;
    }
    const int pbnd = valid && (J.mul == MUL_P || J.mul == MUL_P_IK) ? dealias_bound(g.pb, jj, kk, g.nzc) : -2;
    T2 v[E];
#pragma unroll
    for (int q = 0; q < E; ++q) {
        const int row = reg_row<N, P, Plan<N>::R1>(p, q);
        T2 x = valid ? in[base + row * rstride] : mk<T2>((T)0, (T)0);
        if (J.mul == MUL_P || J.mul == MUL_P_IK) {
            if (!dealias_keep_b(g.q2, g.thr, pbnd, g.n, row, jj, kk)) x = mk<T2>((T)0, (T)0);
        }
        if (J.mul == MUL_P_IK || J.mul == MUL_IK) x = mul_ik(x, g.kv[row]);
        v[q] = x;
    }
    Plan<N>::template fft<T2, SIGN>(v, sm + c, StrideAddr{TC}, p, tw);
    if (valid) {
#pragma unroll
        for (int q = 0; q < E; ++q) {
            const int row = reg_row<N, P, Plan<N>::RL>(p, q);
            out[base + row * rstride] = v[q];
        }
    }
}

// ------------------------------------------------- pipelined x / y pass
// The x / y pass as a persistent kernel: each block walks tiles t, t + grid,
// ... and while tile t is transformed in registers, the loads of the next
// tile are in flight as cp.async copies into a staging buffer (shared memory
// beside the exchange buffer).  Every thread stages exactly the elements it
// later reads, so the staging buffer needs no barrier; the exchange buffer
// keeps the FFT's own.  Same tiles, multipliers, transforms and stores as
// k_axis_pass, so the same results.
__device__ __forceinline__ void cp_async_copy(void *smem, const float2 *g) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_copy(void *smem, const double2 *g) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <int PENDING> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

template <typename T> struct AxisTile {
    typedef typename C2<T>::type T2;
    const T2 *in;
    T2 *out;
    int base, rstride;  // element indices: n * n * (n/2 + 1) < 2^31 for every supported n
    int jj, kk, mul;
    bool valid;
};

// Tile `tile` of job `job` (global tile index tile * njobs + job), column c.
template <typename T, int N>
__device__ __forceinline__ AxisTile<T> axis_tile(const AxisJob *__restrict__ jobs, int job, int tile, int axis,
                                                 int c) {
    typedef typename C2<T>::type T2;
    constexpr int TC = Tile<T>::TC, n = N, nzc = N / 2 + 1;
    AxisTile<T> G;
    const AxisJob J = jobs[job];
    G.in = static_cast<const T2 *>(J.in);
    G.out = static_cast<T2 *>(J.out);
    G.mul = J.mul;
    G.jj = 0;
    G.kk = 0;
    if (axis == 0) {
        const int col = tile * TC + c;
        G.valid = col < n * nzc;
        G.base = col;
        G.rstride = n * nzc;
        G.jj = col / nzc;
        G.kk = col - G.jj * nzc;
    } else {
        constexpr int tpp = (nzc + TC - 1) / TC;
        const int plane = tile / tpp;
        G.kk = (tile - plane * tpp) * TC + c;
        G.valid = G.kk < nzc;
        G.base = plane * n * nzc + G.kk;
        G.rstride = nzc;
    }
    return G;
}

// Resident blocks per SM that the transform kernels ask the register
// allocator for: as many as their shared memory allows (TILES tiles of
// N x TC elements per block), at most CAP, and no more than leave FLOOR
// registers per thread.  Without this bound the allocator spends 128-224
// registers per thread on the 256-point transforms and two blocks fit; with
// it the same code fits 64-85 registers (FP32) without spilling.
template <typename T, int N, int V, int TILES, int CAP, int FLOOR> struct PipeMinBlocks {
    static constexpr long threads = (long)Tile<T>::TC * PlanV<N, V>::P;
    static constexpr long smem = (long)TILES * N * Tile<T>::TC * sizeof(typename C2<T>::type);
    static constexpr long by_smem = (227L * 1024) / smem;
    static constexpr long by_regs = 65536L / (threads * FLOOR);
    static constexpr long lim = by_smem < by_regs ? by_smem : by_regs;
    static constexpr int value = lim < 1 ? 1 : (lim < CAP ? (int)lim : CAP);
};

// Staging slots per k_axis_pipe block: the tile being transformed was loaded
// into one slot while the next KF_PIPE_DEPTH - 1 tiles load into the others.
// (Two slots, 96 KB per block at 256^3, measured slower: 13.5 against 12.2 ms
// for the 48 inverse launches of a 20-step run; the shared memory they take
// from the L1 cache is what the twiddle and table loads hit.)
#ifndef KF_PIPE_DEPTH
#define KF_PIPE_DEPTH 1
#endif

// Shared memory of a k_axis_pipe launch: the exchange tile and KF_PIPE_DEPTH
// staging tiles.  (Held to fewer registers for three resident blocks, or with
// its twiddles, k values and job descriptors staged in shared memory, the
// one-slot pass measured no faster: 12.5 and 13.8 ms against 12.4 ms for 48
// launches.)
template <typename T, int N> inline size_t axis_pipe_smem(int) {
    return (1 + KF_PIPE_DEPTH) * (size_t)N * Tile<T>::TC * sizeof(typename C2<T>::type);
}

// Resident blocks per SM asked of the register allocator for k_axis_pipe
// (0: no request; 3 fits the FP32 256-point pass in 80 registers without
// spilling: its 48 inverse launches of 20 steps took 12.0-12.1 ms against
// 13.7 ms with 125 registers and 2 blocks), and for the FP32 k_z_c2r (12
// blocks, 40 registers with spills: 8.0 against 7.5 ms; not used).
#ifndef KF_PIPE_MINB
#define KF_PIPE_MINB 3
#endif
#ifndef KF_ZC2R_MINB
#define KF_ZC2R_MINB 0
#endif

template <typename T, int N, int SIGN, int V = 0>
__global__ void __launch_bounds__(Tile<T>::TC * PlanV<N, V>::P,
                                  (KF_PIPE_MINB ? PipeMinBlocks<T, N, V, 1 + KF_PIPE_DEPTH, (KF_PIPE_MINB > 0 ? KF_PIPE_MINB : 1), 64>::value : 1))
k_axis_pipe(const AxisJob *__restrict__ jobs, int njobs, int axis, Geo<T> g,
            const typename C2<T>::type *__restrict__ tw, int total) {
    typedef typename C2<T>::type T2;
    constexpr int TC = Tile<T>::TC, P = PlanV<N, V>::P, E = N / P;
    constexpr int D = KF_PIPE_DEPTH;
    extern __shared__ __align__(16) unsigned char kf_smem[];
    T2 *sm = reinterpret_cast<T2 *>(kf_smem);  // exchange [N][TC]
    T2 *stg0 = sm + N * TC;                     // staging  [D][N][TC]
    const int c = threadIdx.x % TC, p = threadIdx.x / TC;
    int t = blockIdx.x;
    if (t >= total) return;
    // (job, tile) of global tile t = tile * njobs + job, advanced by the grid
    // stride without a division per tile: for the tile being transformed (c*)
    // and for the next one to stage (p*)
    const int GS = gridDim.x, Gq = GS / njobs, Gr = GS - Gq * njobs;
    auto adv = [&](int &j, int &tl) {
        j += Gr;
        tl += Gq;
        if (j >= njobs) {
            j -= njobs;
            ++tl;
        }
    };
    int cj = t % njobs, ct = t / njobs;
    int pj = cj, pt = ct, ptt = t;
    // Each thread stages exactly the elements it reads back, so the slots need
    // no barrier.  One commit group per tile (empty past the end), so that
    // cp.async.wait_group D - 1 always leaves the current tile complete.
    auto prefetch = [&](int slot) {
        if (ptt < total) {
            const AxisTile<T> G = axis_tile<T, N>(jobs, pj, pt, axis, c);
            T2 *st = stg0 + slot * (N * TC);
#pragma unroll
            for (int q = 0; q < E; ++q) {
                const int row = reg_row<N, P, PlanV<N, V>::R1>(p, q);
                T2 *dst = st + row * TC + c;
                if (G.valid)
                    cp_async_copy(dst, G.in + G.base + row * G.rstride);
                else
                    *dst = mk<T2>((T)0, (T)0);
            }
        }
        cp_async_commit();
        ptt += GS;
        adv(pj, pt);
    };
#pragma unroll
    for (int d = 0; d < D; ++d) prefetch(d);
    for (int it = 0; t < total; t += GS, ++it) {
        const int slot = it % D;
        const AxisTile<T> cur = axis_tile<T, N>(jobs, cj, ct, axis, c);
        adv(cj, ct);
        // the 2/3 rule of this column as an index bound (one table read per tile)
        const int pbnd = cur.valid && (cur.mul == MUL_P || cur.mul == MUL_P_IK)
                             ? dealias_bound(g.pb, cur.jj, cur.kk, g.nzc)
                             : -2;
        cp_async_wait<D - 1>();
        const T2 *stg = stg0 + slot * (N * TC);
        T2 v[E];
#pragma unroll
        for (int q = 0; q < E; ++q) {
            const int row = reg_row<N, P, PlanV<N, V>::R1>(p, q);
            T2 x = stg[row * TC + c];
            if (cur.mul == MUL_P || cur.mul == MUL_P_IK) {
                if (!dealias_keep_b(g.q2, g.thr, pbnd, g.n, row, cur.jj, cur.kk)) x = mk<T2>((T)0, (T)0);
            }
            if (cur.mul == MUL_P_IK || cur.mul == MUL_IK) x = mul_ik(x, g.kv[row]);
            v[q] = x;
        }
        prefetch(slot);
        PlanV<N, V>::template fft<T2, SIGN>(v, sm + c, StrideAddr{TC}, p, tw);
        if (cur.valid) {
#pragma unroll
            for (int q = 0; q < E; ++q) {
                const int row = reg_row<N, P, PlanV<N, V>::RL>(p, q);
                cur.out[cur.base + row * cur.rstride] = v[q];
            }
        }
    }
}

// --------------------------------------------------------------- z c2r pass
// LZ line pairs per block; thread = p + P*l.  Half rows are staged in shared
// memory, multiplied, extended by Hermitian symmetry (the imaginary parts of
// the kz = 0 and kz = n/2 bins are dropped, as a c2r transform does), packed
// as A + iB, transformed backwards and written as two real rows scaled by
// `scale` (the 1/N of OP_iFFT.cpp:59-61).
// Line pairs per z-pass block (4 and 16 measured no faster than 8 at 256^3:
// the c2r launches took 7.36 and 8.01 ms against 7.33 ms over 20 steps).
#ifndef KF_ZLZ
#define KF_ZLZ 8
#endif
template <typename T> struct ZTile { static constexpr int LZ = KF_ZLZ; };

// Shared memory of a z pass: its line buffers (the c2r staging of two half
// spectra per line pair, reused by the transform).
template <typename T, int N, bool C2R> struct ZSmem {
    typedef typename C2<T>::type T2;
    static constexpr int LZ = ZTile<T>::LZ, NZC = N / 2 + 1, LS = PadLen<N>::value;
    static constexpr int lines = C2R ? (2 * LZ * NZC > LZ * LS ? 2 * LZ * NZC : LZ * LS) : LZ * LS;
    static constexpr size_t bytes = (size_t)lines * sizeof(T2);
};

template <typename T, int N, int V = 0>
__global__ void __launch_bounds__(ZTile<T>::LZ * PlanV<N, V>::P, (sizeof(T) == 4 && KF_ZC2R_MINB > 0 ? KF_ZC2R_MINB : 1))
k_z_c2r(const ZJob *__restrict__ jobs, int njobs, int nrows, Geo<T> g,
        const typename C2<T>::type *__restrict__ tw, T scale) {
    typedef typename C2<T>::type T2;
    constexpr int LZ = ZTile<T>::LZ, P = PlanV<N, V>::P, E = N / P, NZC = N / 2 + 1;
    constexpr int LS = PadLen<N>::value;  // padded line of the exchange buffer
    extern __shared__ __align__(16) unsigned char kf_smem[];
    T2 *half = reinterpret_cast<T2 *>(kf_smem);  // [2][LZ][NZC], staging of the half spectra
    T2 *xch = half;                              // [LZ][LS], reused by the transform once staged
    const int job = blockIdx.x % njobs, tile = blockIdx.x / njobs;
    const ZJob J = jobs[job];
    const int r0 = tile * LZ;
    const T2 *inA = static_cast<const T2 *>(J.inA);
    const T2 *inB = static_cast<const T2 *>(J.inB);
    // raw half spectra -> shared memory with asynchronous copies (all of a
    // thread's loads in flight at once); the multipliers are applied below.
    // The tile's LZ rows of a half spectrum are one contiguous run of
    // LZ * NZC elements from row r0.
    const int lim = (nrows - r0) * NZC;  // elements of the run inside the field
    const long off = (long)r0 * NZC;
    for (int e = threadIdx.x; e < LZ * NZC; e += blockDim.x) {
        if (e < lim) {
            cp_async_copy(half + e, inA + off + e);
            if (inB)
                cp_async_copy(half + LZ * NZC + e, inB + off + e);
            else
                half[LZ * NZC + e] = mk<T2>((T)0, (T)0);
        } else {
            half[e] = mk<T2>((T)0, (T)0);
            half[LZ * NZC + e] = mk<T2>((T)0, (T)0);
        }
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    const int p = threadIdx.x % P, l = threadIdx.x / P;
    const T2 *hA = half + l * NZC;
    const T2 *hB = half + LZ * NZC + l * NZC;
    // staged element kk (0 <= kk < NZC) times its job's multiplier, with the
    // imaginary parts of the kz = 0 and kz = n/2 bins dropped
    auto staged = [&](const T2 *h, int kk, int mul) {
        T2 x = h[kk];
        if (mul == MUL_IK) x = mul_ik(x, g.kv[kk]);
        if (mul == MUL_HALF && kk > 0 && 2 * kk < N) x = mk<T2>((T)0.5 * x.x, (T)0.5 * x.y);
        if (kk == 0 || 2 * kk == N) x.y = (T)0;
        return x;
    };
    T2 v[E];
#pragma unroll
    for (int q = 0; q < E; ++q) {
        const int k = reg_row<N, P, PlanV<N, V>::R1>(p, q);
        T2 a, b;
        if (k < NZC) {
            a = staged(hA, k, J.mulA);
            b = staged(hB, k, J.mulB);
        } else {
            a = staged(hA, N - k, J.mulA);
            b = staged(hB, N - k, J.mulB);
            a.y = -a.y;
            b.y = -b.y;
        }
        v[q] = mk<T2>(a.x - b.y, a.y + b.x);  // A + iB
    }
    __syncthreads();  // staging consumed: the exchange buffer may overwrite it
    PlanV<N, V>::template fft<T2, +1>(v, xch + l * LS, PadAddr{}, p, tw);
    const int r = r0 + l;
    if (r < nrows) {
        T *oA = static_cast<T *>(J.outA) + (long)r * N;
        T *oB = J.outB ? static_cast<T *>(J.outB) + (long)r * N : nullptr;
#pragma unroll
        for (int q = 0; q < E; ++q) {
            const int z = reg_row<N, P, PlanV<N, V>::RL>(p, q);
            oA[z] = v[q].x * scale;
            if (oB) oB[z] = v[q].y * scale;
        }
    }
}

// --------------------------------------------------------------- z r2c pass
template <typename T, int N, int V = 0>
__global__ void __launch_bounds__(ZTile<T>::LZ * PlanV<N, V>::P)
k_z_r2c(const ZJob *__restrict__ jobs, int njobs, int nrows,
        const typename C2<T>::type *__restrict__ tw) {
    typedef typename C2<T>::type T2;
    constexpr int LZ = ZTile<T>::LZ, P = PlanV<N, V>::P, E = N / P, NZC = N / 2 + 1;
    constexpr int LS = PadLen<N>::value;
    extern __shared__ __align__(16) unsigned char kf_smem[];
    T2 *xch = reinterpret_cast<T2 *>(kf_smem);  // [LZ][LS], padded lines
    const int job = blockIdx.x % njobs, tile = blockIdx.x / njobs;
    const ZJob J = jobs[job];
    const int r0 = tile * LZ;
    const int p = threadIdx.x % P, l = threadIdx.x / P;
    const int r = r0 + l;
    const T *iA = static_cast<const T *>(J.inA);
    const T *iB = static_cast<const T *>(J.inB);
    T2 v[E];
#pragma unroll
    for (int q = 0; q < E; ++q) {
        const int z = reg_row<N, P, PlanV<N, V>::R1>(p, q);
        T a = (T)0, b = (T)0;
        if (r < nrows) {
            a = iA[(long)r * N + z];
            if (iB) b = iB[(long)r * N + z];
        }
        v[q] = mk<T2>(a, b);
    }
    T2 *line = xch + l * LS;
    const PadAddr pa;
    PlanV<N, V>::template fft<T2, -1>(v, line, pa, p, tw);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < E; ++q) line[pa(reg_row<N, P, PlanV<N, V>::RL>(p, q))] = v[q];
    __syncthreads();
    // the tile's LZ output rows of a half spectrum are one contiguous run of
    // LZ * NZC elements from row r0
    const int lim = (nrows - r0) * NZC;
    T2 *oA = static_cast<T2 *>(J.outA) + (long)r0 * NZC;
    T2 *oB = J.outB ? static_cast<T2 *>(J.outB) + (long)r0 * NZC : nullptr;
    for (int idx = threadIdx.x; idx < LZ * NZC && idx < lim; idx += blockDim.x) {
        const int ll = idx / NZC, k = idx - ll * NZC;
        const T2 zk = xch[ll * LS + pa(k)];
        const T2 zm = xch[ll * LS + pa(k == 0 ? 0 : N - k)];
        const T cr = zm.x, ci = -zm.y;  // conj(Z[N-k])
        oA[idx] = mk<T2>((T)0.5 * (zk.x + cr), (T)0.5 * (zk.y + ci));
        if (oB) oB[idx] = mk<T2>((T)0.5 * (zk.y - ci), (T)-0.5 * (zk.x - cr));
    }
}

// --------------------------------------------- spectral linear terms (FB parts)
// lin_q is the part of rhs_standard's FBuffer_q (the negated right-hand side)
// that is computed in k-space, in the reference's order of accumulation:
//   u_c: (tau+SV) u^ [+ D|k|^2 u^] + i k_c (PF phi^ + s^/theta) + M i k_x P u^
//        (rhs_standard.cpp:119-140, 218-248, 279-295)
//   s  : SV s^ [+ D|k|^2 s^] + M i k_x P s^ + i k.P u^
//        (rhs_standard.cpp:135-139, 304-319)
// b: the column's 2/3-rule bound (dealias_bound), or -2 for the exact test.
template <typename T>
__device__ __forceinline__ typename C2<T>::type lin_term(const RhsArgs<T> &a, const Geo<T> &g, int q,
                                                         int i, int j, int k, long idx, int b) {
    typedef typename C2<T>::type T2;
    const int Tm = a.terms;
    const bool P = dealias_keep_b(g.q2, g.thr, b, g.n, i, j, k);
    const T kx = g.kv[i], ky = g.kv[j], kz = g.kv[k];
    const T sv = a.SV[idx];
    T2 fb;
    if (q < 3) {
        const T2 u = a.Y[q][idx];
        const bool diss = Tm & T_DISSIPATION, svo = Tm & T_SVISCOSITY;
        const T cf = diss && svo ? (a.tau + sv) : diss ? a.tau : svo ? sv : (T)0;
        fb = mk<T2>(cf * u.x, cf * u.y);
        if (Tm & T_DIFFUSION) {
            const T k2 = kx * kx + ky * ky + kz * kz;
            fb.x += a.D * k2 * u.x;
            fb.y += a.D * k2 * u.y;
        }
        const bool pres = Tm & T_PRESSURE, eint = Tm & T_E_INT;
        if (pres || eint) {
            T2 F1 = mk<T2>((T)0, (T)0);
            if (eint) {
                F1 = a.phihat[idx];
                if (pres) { const T pf = a.PF[idx]; F1.x *= pf; F1.y *= pf; }
            }
            if (pres) {
                const T2 s = a.Y[3][idx];
                F1.x += s.x / a.theta;
                F1.y += s.y / a.theta;
            }
            const T kc = q == 0 ? kx : q == 1 ? ky : kz;
            const T2 d = mul_ik(F1, kc);
            fb.x += d.x;
            fb.y += d.y;
        }
        if ((Tm & T_E_EXT) && P) {
            const T2 d = mul_ik(u, kx);
            fb.x += a.M * d.x;
            fb.y += a.M * d.y;
        }
    } else {
        const T2 s = a.Y[3][idx];
        const T cf = (Tm & T_SVISCOSITY) ? sv : (T)0;
        fb = mk<T2>(cf * s.x, cf * s.y);
        if (Tm & T_DIFFUSION) {
            const T k2 = kx * kx + ky * ky + kz * kz;
            fb.x += a.D * k2 * s.x;
            fb.y += a.D * k2 * s.y;
        }
        if ((Tm & T_E_EXT) && P) {
            const T2 d = mul_ik(s, kx);
            fb.x += a.M * d.x;
            fb.y += a.M * d.y;
        }
        if ((Tm & T_CONTINUITY) && P) {
            const T2 dx = mul_ik(a.Y[0][idx], kx);
            const T2 dy = mul_ik(a.Y[1][idx], ky);
            const T2 dz = mul_ik(a.Y[2][idx], kz);
            fb.x += dx.x; fb.y += dx.y;
            fb.x += dy.x; fb.y += dy.y;
            fb.x += dz.x; fb.y += dz.y;
        }
    }
    return fb;
}

// ------------------------------------ forward x pass + right-hand-side assembly
// For each of the four output fields the forward x transform of the y-passed
// product (or penalized) field is formed and combined per element:
//   penalization off: K_q = -(lin_q + F_q)        (rhs_standard.cpp:538-560)
//   penalization on : K_q = P(k) F_q              (the 2/3 filter after the
//                     physical-space penalization, rhs_standard.cpp:491-532)
// gridDim.x = number of column tiles; jobs[q].in = y-passed field, .out = K_q.
// PEN: the penalization form (a.terms has T_PENALIZATION), instantiated apart
// so that its registers do not carry the linear terms'.
template <typename T, int N, int V = 0, bool PEN = false>
__global__ void __launch_bounds__(Tile<T>::TC * PlanV<N, V>::P,
                                  (PEN ? PipeMinBlocks<T, N, V, 1, sizeof(T) == 4 ? 4 : 2, 64>::value : 1))
k_xfwd_assemble(const AxisJob *__restrict__ jobs, Geo<T> g, RhsArgs<T> a,
                const typename C2<T>::type *__restrict__ tw) {
    typedef typename C2<T>::type T2;
    constexpr int TC = Tile<T>::TC, P = PlanV<N, V>::P, E = N / P;
    extern __shared__ __align__(16) unsigned char kf_smem[];
    T2 *sm = reinterpret_cast<T2 *>(kf_smem);
    const int tile = blockIdx.x;
    const int c = threadIdx.x % TC, p = threadIdx.x / TC;
    const int n = g.n, nzc = g.nzc;
    const int col = tile * TC + c;
    const bool valid = col < n * nzc;
    const long rstride = (long)n * nzc;
    const int jj = col / nzc, kk = col - jj * nzc;
    const int b = valid ? dealias_bound(g.pb, jj, kk, nzc) : -2;
    for (int q = 0; q < 4; ++q) {
        const T2 *__restrict__ in = static_cast<const T2 *>(jobs[q].in);
        T2 *__restrict__ out = static_cast<T2 *>(jobs[q].out);
        T2 v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int row = reg_row<N, P, PlanV<N, V>::R1>(p, e);
            v[e] = valid ? in[col + row * rstride] : mk<T2>((T)0, (T)0);
        }
        PlanV<N, V>::template fft<T2, -1>(v, sm + c, StrideAddr{TC}, p, tw);
        if (valid) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int i = reg_row<N, P, PlanV<N, V>::RL>(p, e);
                const long idx = col + i * rstride;
                T2 F = v[e];
                T2 K;
                if constexpr (PEN) {
                    K = dealias_keep_b(g.q2, g.thr, b, N, i, jj, kk) ? F : mk<T2>((T)0, (T)0);
                } else {
                    T2 fb = lin_term(a, g, q, i, jj, kk, idx, b);
                    K = mk<T2>(-(fb.x + F.x), -(fb.y + F.y));
                }
                out[idx] = K;
            }
        }
        __syncthreads();
    }
}

}  // namespace kf
