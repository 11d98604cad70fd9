// kf_pointwise.cuh -- physical-space products, Poisson source, RK4 stage updates.
#pragma once

#include "kf_passes.cuh"
#include "kf_types.cuh"

namespace kf {

// Physical-space nonlinear terms, one thread per grid point:
//   A_c = U_x d_x U_c + U_y d_y U_c + U_z d_z U_c   (rhs_standard.cpp:403-436)
//   B   = d_x s U_x + d_y s U_y + d_z s U_z          (rhs_standard.cpp:323-342)
// With penalization the masking form (effect_penalization.cpp:35) is applied to
// the physical right-hand side  r_q = c2r(-lin_q) - prod_q:
//   f_q = (1-H) r_q + H eta (q_d - q_fix),  q_fix = (-M, 0, 0, -10).
template <typename T> struct ProdArgs {
    const T *U[3];
    const T *dU[3][3];  // dU[c][d] = d_d U_c
    const T *ds[3];     // d_d s
    const T *rl[4];     // c2r(-lin_q)        (penalization only)
    const T *sd;        // c2r(P s^)           (penalization only)
    const T *H;         // mask               (penalization only)
    T *out[4];
    T M, eta;
    int terms;
    long N;
};

template <typename T>
__global__ void k_products(ProdArgs<T> a) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    const T ux = a.U[0][i], uy = a.U[1][i], uz = a.U[2][i];
    T pr[4];
    const bool adv = a.terms & T_ADVECTION, cont = a.terms & T_CONTINUITY;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        T s = (T)0;
        if (adv) {
            s = ux * a.dU[c][0][i];
            s += uy * a.dU[c][1][i];
            s += uz * a.dU[c][2][i];
        }
        pr[c] = s;
    }
    {
        T s = (T)0;
        if (cont) {
            s = a.ds[0][i] * ux;
            s += a.ds[1][i] * uy;
            s += a.ds[2][i] * uz;
        }
        pr[3] = s;
    }
    if (a.terms & T_PENALIZATION) {
        const T h = a.H[i];
        const T qd[4] = {ux, uy, uz, a.sd[i]};
        const T qfix[4] = {-a.M, (T)0, (T)0, (T)-10};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const T r = a.rl[q][i] - pr[q];
            a.out[q][i] = ((T)1 - h) * r + h * a.eta * (qd[q] - qfix[q]);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) a.out[q][i] = pr[q];
    }
}

// rl_q = -lin_q in k-space (penalization path).  Grid (ceil(nzc/32), n/8, n)
// of 32 x 8 blocks over (kz, j, i): no index division.  The four outputs of
// an element share its loads (state, phi^, tables); each is accumulated in the
// order of lin_term (kf_passes.cuh), so the values are those of lin_term.
template <typename T>
__global__ void __launch_bounds__(256) k_lin(RhsArgs<T> a, Geo<T> g, typename C2<T>::type *o0,
                                             typename C2<T>::type *o1, typename C2<T>::type *o2,
                                             typename C2<T>::type *o3) {
    typedef typename C2<T>::type T2;
    const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, i = blockIdx.z;
    if (k >= g.nzc || j >= g.n) return;
    const long idx = (long)k + (long)g.nzc * ((long)j + (long)i * g.n);
    const int Tm = a.terms;
    const bool P = dealias_keep(g.q2, g.thr, i, j, k);
    const T kx = g.kv[i], ky = g.kv[j], kz = g.kv[k];
    const T sv = a.SV[idx];
    const T2 u[3] = {a.Y[0][idx], a.Y[1][idx], a.Y[2][idx]};
    const T2 s = a.Y[3][idx];
    const bool diss = Tm & T_DISSIPATION, svo = Tm & T_SVISCOSITY;
    const bool pres = Tm & T_PRESSURE, eint = Tm & T_E_INT;
    // F1 = PF phi^ + s^/theta, the E-force/pressure potential (rhs_standard.cpp:218-248)
    T2 F1 = mk<T2>((T)0, (T)0);
    if (pres || eint) {
        if (eint) {
            F1 = a.phihat[idx];
            if (pres) { const T pf = a.PF[idx]; F1.x *= pf; F1.y *= pf; }
        }
        if (pres) {
            F1.x += s.x / a.theta;
            F1.y += s.y / a.theta;
        }
    }
    T2 *o[4] = {o0, o1, o2, o3};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const T cf = diss && svo ? (a.tau + sv) : diss ? a.tau : svo ? sv : (T)0;
        T2 fb = mk<T2>(cf * u[q].x, cf * u[q].y);
        if (Tm & T_DIFFUSION) {
            const T k2 = kx * kx + ky * ky + kz * kz;
            fb.x += a.D * k2 * u[q].x;
            fb.y += a.D * k2 * u[q].y;
        }
        if (pres || eint) {
            const T kc = q == 0 ? kx : q == 1 ? ky : kz;
            const T2 d = mul_ik(F1, kc);
            fb.x += d.x;
            fb.y += d.y;
        }
        if ((Tm & T_E_EXT) && P) {
            const T2 d = mul_ik(u[q], kx);
            fb.x += a.M * d.x;
            fb.y += a.M * d.y;
        }
        o[q][idx] = mk<T2>(-fb.x, -fb.y);
    }
    {
        const T cf = (Tm & T_SVISCOSITY) ? sv : (T)0;
        T2 fb = mk<T2>(cf * s.x, cf * s.y);
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
            const T2 dx = mul_ik(u[0], kx);
            const T2 dy = mul_ik(u[1], ky);
            const T2 dz = mul_ik(u[2], kz);
            fb.x += dx.x; fb.y += dx.y;
            fb.x += dy.x; fb.y += dy.y;
            fb.x += dz.x; fb.y += dz.y;
        }
        o[3][idx] = mk<T2>(-fb.x, -fb.y);
    }
}

// rho = exp(s_d) + n_d in FP64 (rhs_standard.cpp:108-111)
template <typename T>
__global__ void k_rho(const T *__restrict__ sd, const double *__restrict__ nd, double *__restrict__ rho, long N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) rho[i] = exp((double)sd[i]) + nd[i];
}

// RK4 stage combinations (RKO4.cpp:140-238), accumulated as
//   acc = k1; acc += 2 k2; acc += 2 k3;  y = y0 + dt/6 (acc + k4)
// mode 0: acc = K, ys = y0 + c K;  1: acc += 2K, ys = y0 + c K;  2: y0 += d (acc + K)
template <typename T>
__global__ void k_rk(typename C2<T>::type *__restrict__ y0, typename C2<T>::type *__restrict__ acc,
                     typename C2<T>::type *__restrict__ ys, const typename C2<T>::type *__restrict__ K,
                     T cdt, int mode, long M) {
    typedef typename C2<T>::type T2;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const T2 k = K[i];
    const T2 y = y0[i];
    if (mode == 0) {
        acc[i] = k;
        ys[i] = mk<T2>(y.x + cdt * k.x, y.y + cdt * k.y);
    } else if (mode == 1) {
        T2 a = acc[i];
        acc[i] = mk<T2>(a.x + (T)2 * k.x, a.y + (T)2 * k.y);
        ys[i] = mk<T2>(y.x + cdt * k.x, y.y + cdt * k.y);
    } else {
        T2 a = acc[i];
        y0[i] = mk<T2>(y.x + cdt * (a.x + k.x), y.y + cdt * (a.y + k.y));
    }
}

// x <- exp(x) (fn 0) or log(x) (fn 1) in place, evaluated in FP64: the
// density's linear <-> log scale (kielflow.cpp:172-182, 293-296)
template <typename T>
__global__ void k_explog(T *__restrict__ x, int fn, long N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double v = (double)x[i];
    x[i] = (T)(fn == 0 ? exp(v) : log(v));
}

// The real-space fields of an output file (IO.cpp save_field_imag and
// save_slice write iFFT of the spectra): u'_c, n = exp(s) from the c2r of the
// state, and phi, as FP64; all points (k0 < 0, o[q][id]) or the plane z
// index k0 only (o[q][j + n i]).
template <typename T>
__global__ void k_out_real(const T *__restrict__ ux, const T *__restrict__ uy, const T *__restrict__ uz,
                           const T *__restrict__ s, const double *__restrict__ phi, double *__restrict__ o0,
                           double *__restrict__ o1, double *__restrict__ o2, double *__restrict__ o3,
                           double *__restrict__ o4, int n, int k0, long M) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const long src = k0 >= 0 ? i * n + k0 : i;
    o0[i] = (double)ux[src];
    o1[i] = (double)uy[src];
    o2[i] = (double)uz[src];
    o3[i] = exp((double)s[src]);
    o4[i] = phi[src];
}

// rho = n_background + n_d (the frontend's Poisson source)
__global__ void k_add_const(double *__restrict__ out, const double *__restrict__ in, double a, long N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = a + in[i];
}

// frontend.cpp:245-248: the Boltzmann ion density n = exp(-theta phi)
template <typename T>
__global__ void k_boltzmann(T *__restrict__ out, const double *__restrict__ phi, double theta, long N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = (T)exp(-theta * phi[i]);
}

// X *= f elementwise over a half spectrum (dealiasing_undesignated with a
// precomputed filter table, operations.hpp:20-46)
template <typename T>
__global__ void k_filter(typename C2<T>::type *__restrict__ X, const T *__restrict__ f, long Nc) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nc) return;
    typename C2<T>::type x = X[i];
    const T w = f[i];
    x.x *= w;
    x.y *= w;
    X[i] = x;
}

// FP64 <-> bulk precision conversion of interleaved complex / real arrays
template <typename T>
__global__ void k_from_f64(T *__restrict__ dst, const double *__restrict__ src, long M) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) dst[i] = (T)src[i];
}
template <typename T>
__global__ void k_to_f64(double *__restrict__ dst, const T *__restrict__ src, long M) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) dst[i] = (double)src[i];
}

}  // namespace kf
