// kf_fft.cuh -- register/shared-memory Stockham FFT engine for sm_100a.
//
// A length-N transform of one line is carried by P threads; each thread holds
// E = N/P complex values in registers.  Every stage s of radix R performs
// N/R butterflies (Stockham autosort, decimation in time): butterfly j reads
// x[j + t*N/R] (t < R), multiplies by W_N^(t*(j mod Ns)*N/(Ns*R)), runs an
// R-point DFT in registers and writes y[(j/Ns)*Ns*R + (j mod Ns) + t*Ns].
// Thread p owns butterflies j = p + b*P.  Stages exchange data through shared
// memory; the first stage reads its inputs straight from the caller's
// registers and the last stage leaves its outputs in registers, so that
//   input  v[b*R1 + t]  is element  p + b*P + t*N/R1,
//   output v[b*RL + t]  is element  p + b*P + t*N/RL.
// Twiddles W_N^m = exp(SIGN*2*pi*i*m/N) come from a per-N table (host-computed
// in long double), SIGN = -1 forward, +1 backward, as FFTW's r2c/c2r.
#pragma once

#include <cuda_runtime.h>

namespace kf {

template <typename T> struct C2;
template <> struct C2<double> { typedef double2 type; };
template <> struct C2<float> { typedef float2 type; };

template <typename T2> __device__ __forceinline__ T2 mk(decltype(T2::x) a, decltype(T2::x) b) {
    T2 r; r.x = a; r.y = b; return r;
}
template <typename T2> __device__ __forceinline__ T2 cadd(T2 a, T2 b) { return mk<T2>(a.x + b.x, a.y + b.y); }
template <typename T2> __device__ __forceinline__ T2 csub(T2 a, T2 b) { return mk<T2>(a.x - b.x, a.y - b.y); }
template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
    return mk<T2>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by SIGN*i :  (x + i y) * (SIGN i) = SIGN*(-y + i x)
template <int SIGN, typename T2> __device__ __forceinline__ T2 mul_si(T2 a) {
    return SIGN < 0 ? mk<T2>(a.y, -a.x) : mk<T2>(-a.y, a.x);
}
// multiply by exp(SIGN*2*pi*i*m/R) given cos, sin of 2*pi*m/R
template <int SIGN, typename T2>
__device__ __forceinline__ T2 rot(T2 a, double c, double s) {
    typedef decltype(T2::x) T;
    const T cc = (T)c, ss = (T)(SIGN * s);
    return mk<T2>(a.x * cc - a.y * ss, a.x * ss + a.y * cc);
}

// cos / sin of 2*pi*m/R for the composite register radices (literal values)
__host__ __device__ constexpr double kf_cos(int R, int m) {
    return R == 16 ? (m == 0 ? 1.0 : m == 1 ? 0.92387953251128675613 : m == 2 ? 0.70710678118654752440
                      : m == 3 ? 0.38268343236508977173 : m == 4 ? 0.0 : m == 5 ? -0.38268343236508977173
                      : m == 6 ? -0.70710678118654752440 : m == 7 ? -0.92387953251128675613 : m == 8 ? -1.0
                      : m == 9 ? -0.92387953251128675613 : m == 10 ? -0.70710678118654752440
                      : m == 11 ? -0.38268343236508977173 : m == 12 ? 0.0 : m == 13 ? 0.38268343236508977173
                      : m == 14 ? 0.70710678118654752440 : 0.92387953251128675613)
         : R == 12 ? (m == 0 ? 1.0 : m == 1 ? 0.86602540378443864676 : m == 2 ? 0.5 : m == 3 ? 0.0
                      : m == 4 ? -0.5 : m == 5 ? -0.86602540378443864676 : m == 6 ? -1.0
                      : m == 7 ? -0.86602540378443864676 : m == 8 ? -0.5 : m == 9 ? 0.0 : m == 10 ? 0.5
                      : 0.86602540378443864676)
         : R == 8 ? (m == 0 ? 1.0 : m == 1 ? 0.70710678118654752440 : m == 2 ? 0.0
                     : m == 3 ? -0.70710678118654752440 : m == 4 ? -1.0 : m == 5 ? -0.70710678118654752440
                     : m == 6 ? 0.0 : 0.70710678118654752440)
         : R == 6 ? (m == 0 ? 1.0 : m == 1 ? 0.5 : m == 2 ? -0.5 : m == 3 ? -1.0 : m == 4 ? -0.5 : 0.5)
         : 1.0;
}
__host__ __device__ constexpr double kf_sin(int R, int m) {
    // sin(2 pi m/R) = cos(2 pi (m - R/4)/R) for R divisible by 4; R = 6 spelled out
    return R == 6 ? (m == 0 ? 0.0 : m == 1 ? 0.86602540378443864676 : m == 2 ? 0.86602540378443864676
                     : m == 3 ? 0.0 : m == 4 ? -0.86602540378443864676 : -0.86602540378443864676)
                  : kf_cos(R, ((m - R / 4) % R + R) % R);
}

// ------------------------------------------------------------ register DFTs

template <int R, int SIGN> struct DFT;

template <int SIGN> struct DFT<2, SIGN> {
    template <typename T2> __device__ __forceinline__ static void run(T2 *a) {
        T2 a0 = a[0];
        a[0] = cadd(a0, a[1]);
        a[1] = csub(a0, a[1]);
    }
};

template <int SIGN> struct DFT<3, SIGN> {
    template <typename T2> __device__ __forceinline__ static void run(T2 *a) {
        typedef decltype(T2::x) T;
        const T h = (T)0.86602540378443864676;
        T2 t1 = cadd(a[1], a[2]);
        T2 t2 = mk<T2>(a[0].x - (T)0.5 * t1.x, a[0].y - (T)0.5 * t1.y);
        T2 d = csub(a[1], a[2]);
        // i*SIGN*h*d
        T2 s = mul_si<SIGN>(mk<T2>(h * d.x, h * d.y));
        a[0] = cadd(a[0], t1);
        a[1] = cadd(t2, s);
        a[2] = csub(t2, s);
    }
};

template <int SIGN> struct DFT<4, SIGN> {
    template <typename T2> __device__ __forceinline__ static void run(T2 *a) {
        T2 s0 = cadd(a[0], a[2]), d0 = csub(a[0], a[2]);
        T2 s1 = cadd(a[1], a[3]), d1 = mul_si<SIGN>(csub(a[1], a[3]));
        a[0] = cadd(s0, s1);
        a[1] = cadd(d0, d1);
        a[2] = csub(s0, s1);
        a[3] = csub(d0, d1);
    }
};

// R = R1 * R2 computed as a two-stage Stockham in registers
template <int R1, int R2, int SIGN> struct DFT2F {
    template <typename T2> __device__ __forceinline__ static void run(T2 *a) {
        constexpr int R = R1 * R2;
        T2 y[R];
#pragma unroll
        for (int j = 0; j < R2; ++j) {  // stage 1: radix R1, Ns = 1
            T2 b[R1];
#pragma unroll
            for (int t = 0; t < R1; ++t) b[t] = a[j + t * R2];
            DFT<R1, SIGN>::run(b);
#pragma unroll
            for (int t = 0; t < R1; ++t) y[j * R1 + t] = b[t];
        }
#pragma unroll
        for (int j = 0; j < R1; ++j) {  // stage 2: radix R2, Ns = R1, k = j
            T2 b[R2];
#pragma unroll
            for (int t = 0; t < R2; ++t) {
                T2 x = y[j + t * R1];
                const int m = (t * j) % R;
                b[t] = m == 0 ? x : rot<SIGN>(x, kf_cos(R, m), kf_sin(R, m));
            }
            DFT<R2, SIGN>::run(b);
#pragma unroll
            for (int t = 0; t < R2; ++t) a[j + t * R1] = b[t];
        }
    }
};

template <int SIGN> struct DFT<6, SIGN> : DFT2F<3, 2, SIGN> {};
template <int SIGN> struct DFT<8, SIGN> : DFT2F<2, 4, SIGN> {};
template <int SIGN> struct DFT<12, SIGN> : DFT2F<3, 4, SIGN> {};
template <int SIGN> struct DFT<16, SIGN> : DFT2F<4, 4, SIGN> {};

// ------------------------------------------------------------ stage engine

// Shared-memory addressing of element r of a line.
struct StrideAddr {  // columns interleaved: r * stride (+ the column offset in the base pointer)
    int s;
    __device__ __forceinline__ int operator()(int r) const { return r * s; }
};
struct PadAddr {  // one line contiguous, a pad word every 16: avoids the radix-16 scatter conflicts
    __device__ __forceinline__ int operator()(int r) const { return r + (r >> 4); }
};
template <int N> struct PadLen { static constexpr int value = N + N / 16 + 1; };

template <int... Rs> struct First;
template <int R, int... Rest> struct First<R, Rest...> { static constexpr int value = R; };
template <int... Rs> struct Last;
template <int R> struct Last<R> { static constexpr int value = R; };
template <int R, int R2, int... Rest> struct Last<R, R2, Rest...> { static constexpr int value = Last<R2, Rest...>::value; };

// Twiddle table W_N^m: in global memory (read through the read-only path) or
// staged in shared memory by a persistent kernel.
template <typename T2> __device__ __forceinline__ T2 tw_load(const T2 *__restrict__ tw, int m) { return __ldg(tw + m); }
template <typename T2> struct SharedTw {
    const T2 *p;
};
template <typename T2> __device__ __forceinline__ T2 tw_load(SharedTw<T2> tw, int m) { return tw.p[m]; }

// Stages of one line.  v: E registers; sm: this line's shared-memory column
// (element r at sm[r*stride]); tw: W_N table (global, read through L1, or a
// SharedTw).
template <typename T2, int N, int P, int SIGN, int Ns, int R, int... Rest>
struct Stages {
    static constexpr int E = N / P;
    static constexpr int NB = N / (P * R);
    static_assert(NB * P * R == N, "radix does not tile the line");
    template <typename A, typename TW>
    __device__ __forceinline__ static void run(T2 *v, T2 *sm, A addr, int p, TW tw) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = p + b * P;
            const int k = j % Ns;
            if (Ns > 1) {
#pragma unroll
                for (int t = 1; t < R; ++t) {
                    const int m = (t * k * (N / (Ns * R))) % N;
                    T2 w = tw_load(tw, m);
                    if (SIGN > 0) w.y = -w.y;
                    v[b * R + t] = cmul(v[b * R + t], w);
                }
            }
            DFT<R, SIGN>::run(v + b * R);
        }
        if constexpr (sizeof...(Rest) > 0) {
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int j = p + b * P;
                const int k = j % Ns;
                const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
                for (int t = 0; t < R; ++t) sm[addr(idxD + t * Ns)] = v[b * R + t];
            }
            __syncthreads();
            constexpr int R2 = First<Rest...>::value;
            constexpr int NB2 = N / (P * R2);
#pragma unroll
            for (int b = 0; b < NB2; ++b)
#pragma unroll
                for (int t = 0; t < R2; ++t) v[b * R2 + t] = sm[addr(p + b * P + t * (N / R2))];
            __syncthreads();
            Stages<T2, N, P, SIGN, Ns * R, Rest...>::run(v, sm, addr, p, tw);
        }
    }
};

template <typename T2, int N, int P, int SIGN, int... Rs, typename A, typename TW>
__device__ __forceinline__ void fft_line(T2 *v, T2 *sm, A addr, int p, TW tw) {
    Stages<T2, N, P, SIGN, 1, Rs...>::run(v, sm, addr, p, tw);
}

// Row index held by register q (= b*R + t) of thread p at the input of the
// first stage (R = first radix) or the output of the last stage (R = last radix).
template <int N, int P, int R>
__device__ __forceinline__ int reg_row(int p, int q) {
    return p + (q / R) * P + (q % R) * (N / R);
}

// Per-length launch plans: threads per line P and the radix sequence.
// Variant 0 is the default; variant 1 an alternative the autotuner can pick
// (kf_autotune): a different radix order and, where it allows, more threads
// per line with fewer registers each.
#define KF_PLAN(NN, V, PP, R1_, RL_, ...)                                                                   \
    template <> struct PlanV<NN, V> {                                                                       \
        static constexpr int P = PP;                                                                        \
        template <typename T2, int S, typename A, typename TW>                                              \
        __device__ static void fft(T2 *v, T2 *sm, A a, int p, TW tw) {                                      \
            fft_line<T2, NN, PP, S, __VA_ARGS__>(v, sm, a, p, tw);                                          \
        }                                                                                                   \
        static constexpr int R1 = R1_, RL = RL_;                                                            \
        static constexpr int radix[4] = {__VA_ARGS__};                                                      \
    };
template <int N, int V> struct PlanV;
KF_PLAN(16, 0, 4, 4, 4, 4, 4)
KF_PLAN(16, 1, 4, 4, 4, 4, 4)
KF_PLAN(32, 0, 4, 8, 4, 8, 4)
KF_PLAN(32, 1, 4, 4, 8, 4, 8)
KF_PLAN(64, 0, 8, 8, 8, 8, 8)
KF_PLAN(64, 1, 16, 4, 4, 4, 4, 4)
KF_PLAN(96, 0, 8, 6, 4, 6, 4, 4)
KF_PLAN(96, 1, 8, 4, 6, 4, 4, 6)
KF_PLAN(128, 0, 8, 16, 8, 16, 8)
KF_PLAN(128, 1, 16, 8, 4, 8, 4, 4)
KF_PLAN(256, 0, 16, 16, 16, 16, 16)
KF_PLAN(256, 1, 32, 8, 4, 8, 8, 4)
#undef KF_PLAN
template <int N> using Plan = PlanV<N, 0>;

}  // namespace kf
