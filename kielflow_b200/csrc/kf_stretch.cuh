// kf_stretch.cuh -- pointwise kernels of the right-hand side on sine-stretched
// axes (axis_CoSiSt, axis_SiSt.cpp).  There a derivative is the chain-rule
// form of OP_partial_derivative.cpp:104-136,
//   D_d F = r2c( m(x_d) * c2r( P i k_d F ) ),
// m = 1/dS of the axis after the 2/3 filter (OP_partial_derivative.cpp:60-80),
// so every derivative costs a transform pair; the transforms run as batched
// passes (kf_passes.cuh) and these kernels do the pointwise work between them.
#pragma once

#include "kf_passes.cuh"
#include "kf_types.cuh"

namespace kf {

// Linear spectral parts of FBuffer (no derivative; rhs_standard.cpp:119-140
// and the added diffusion) and the potential of the E-force/pressure term
// F1 = PF phi^ + s^/theta (rhs_standard.cpp:218-240), one thread per
// half-spectrum element.  Same order of operations as lin_term.
template <typename T>
__global__ void k_sl_lin(RhsArgs<T> a, Geo<T> g, typename C2<T>::type *l0, typename C2<T>::type *l1,
                         typename C2<T>::type *l2, typename C2<T>::type *l3, typename C2<T>::type *F1o) {
    typedef typename C2<T>::type T2;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long Nc = (long)g.n * g.n * g.nzc;
    if (idx >= Nc) return;
    const int k = (int)(idx % g.nzc);
    const long r = idx / g.nzc;
    const int j = (int)(r % g.n), i = (int)(r / g.n);
    const int Tm = a.terms;
    const T kx = g.kv[i], ky = g.kv[j], kz = g.kv[k];
    const T sv = a.SV[idx];
    T2 *o[3] = {l0, l1, l2};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const T2 u = a.Y[q][idx];
        const bool diss = Tm & T_DISSIPATION, svo = Tm & T_SVISCOSITY;
        const T cf = diss && svo ? (a.tau + sv) : diss ? a.tau : svo ? sv : (T)0;
        T2 fb = mk<T2>(cf * u.x, cf * u.y);
        if (Tm & T_DIFFUSION) {
            const T k2 = kx * kx + ky * ky + kz * kz;
            fb.x += a.D * k2 * u.x;
            fb.y += a.D * k2 * u.y;
        }
        o[q][idx] = fb;
    }
    const T2 s = a.Y[3][idx];
    {
        const T cf = (Tm & T_SVISCOSITY) ? sv : (T)0;
        T2 fb = mk<T2>(cf * s.x, cf * s.y);
        if (Tm & T_DIFFUSION) {
            const T k2 = kx * kx + ky * ky + kz * kz;
            fb.x += a.D * k2 * s.x;
            fb.y += a.D * k2 * s.y;
        }
        l3[idx] = fb;
    }
    T2 F1 = mk<T2>((T)0, (T)0);
    const bool pres = Tm & T_PRESSURE, eint = Tm & T_E_INT;
    if (eint) {
        F1 = a.phihat[idx];
        if (pres) {
            const T pf = a.PF[idx];
            F1.x *= pf;
            F1.y *= pf;
        }
    }
    if (pres) {
        F1.x += s.x / a.theta;
        F1.y += s.y / a.theta;
    }
    F1o[idx] = F1;
}

// The raw derivatives c2r(P i k_d F) times the metric of their direction, in
// place (OP_partial_derivative.cpp:125-127).  f[j] is a derivative along axis
// j % 3 (j = 3c + d for d_d u'_c, 9 + d for d_d s, 12 + d for d_d F1).
template <typename T> struct ScaleArgs {
    T *f[15];
    const T *met;
    int n;
    long N;
};

template <typename T>
__global__ void k_sl_scale(ScaleArgs<T> a) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.N) return;
    const int k = (int)(idx % a.n);
    const long r = idx / a.n;
    const int j = (int)(r % a.n), i = (int)(r / a.n);
    const T m[3] = {a.met[i], a.met[j], a.met[k]};
#pragma unroll
    for (int q = 0; q < 15; ++q) a.f[q][idx] = a.f[q][idx] * m[q % 3];
}

// Assembly of the right-hand side from the linear parts, the chain-rule
// derivatives dn[j] (spectral, numbered as ScaleArgs) and the transformed
// products pr (advection, continuity), in the reference's order of
// accumulation (rhs_standard.cpp:119-439) and sign (:538-560):
//   u_c: lin_c + D_c F1 + M D_x u'_c + r2c(u . grad u_c)
//   s  : lin_s + M D_x s + D_x u'_x + D_y u'_y + D_z u'_z + r2c(u . grad s)
template <typename T> struct AsmArgs {
    typedef typename C2<T>::type T2;
    const T2 *lin[4];
    const T2 *dn[15];
    const T2 *pr[4];  // nullptr without advection and continuity
    T2 *K[4];
    T M;
    int terms;
    long Nc;
};

template <typename T>
__global__ void k_sl_assemble(AsmArgs<T> a) {
    typedef typename C2<T>::type T2;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.Nc) return;
    const int Tm = a.terms;
    const bool force = (Tm & T_PRESSURE) || (Tm & T_E_INT);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        T2 fb = a.lin[q][idx];
        if (force) {
            const T2 d = a.dn[12 + q][idx];
            fb.x += d.x;
            fb.y += d.y;
        }
        if (Tm & T_E_EXT) {
            const T2 d = a.dn[3 * q][idx];
            fb.x += a.M * d.x;
            fb.y += a.M * d.y;
        }
        if (Tm & T_ADVECTION) {
            const T2 d = a.pr[q][idx];
            fb.x += d.x;
            fb.y += d.y;
        }
        a.K[q][idx] = mk<T2>(-fb.x, -fb.y);
    }
    T2 fb = a.lin[3][idx];
    if (Tm & T_E_EXT) {
        const T2 d = a.dn[9][idx];
        fb.x += a.M * d.x;
        fb.y += a.M * d.y;
    }
    if (Tm & T_CONTINUITY) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T2 d = a.dn[4 * c][idx];  // d_c u'_c
            fb.x += d.x;
            fb.y += d.y;
        }
        const T2 d = a.pr[3][idx];
        fb.x += d.x;
        fb.y += d.y;
    }
    a.K[3][idx] = mk<T2>(-fb.x, -fb.y);
}

// The 2/3 filter (OP_dealiasing.cpp:5-13) on four half spectra.
template <typename T>
__global__ void k_sl_dealias4(Geo<T> g, typename C2<T>::type *K0, typename C2<T>::type *K1,
                              typename C2<T>::type *K2, typename C2<T>::type *K3) {
    typedef typename C2<T>::type T2;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long Nc = (long)g.n * g.n * g.nzc;
    if (idx >= Nc) return;
    const int k = (int)(idx % g.nzc);
    const long r = idx / g.nzc;
    const int j = (int)(r % g.n), i = (int)(r / g.n);
    const T f = dealias_keep(g.q2, g.thr, i, j, k) ? (T)1 : (T)0;
    T2 *o[4] = {K0, K1, K2, K3};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        T2 x = o[q][idx];
        x.x *= f;
        x.y *= f;
        o[q][idx] = x;
    }
}

}  // namespace kf
