// kf_types.cuh -- argument blocks shared by the kernels and the host driver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include "kf_fft.cuh"

namespace kf {

// Multipliers applied to a spectral element as it is loaded by a pass.
enum Mul : int {
    MUL_NONE = 0,   // 1
    MUL_P = 1,      // 2/3 dealiasing mask P(k)            (x pass only: needs i, j, k)
    MUL_P_IK = 2,   // P(k) * i k_axis                     (x pass only)
    MUL_IK = 3,     // i k_axis  (k of the pass's own axis)
    MUL_HALF = 4,   // z c2r only: 1/2 for 0 < kz < n/2 (the half-spectrum weight of a transpose)
};

// Term bits (runtime form of rhs_standard.hpp:22-30 plus the added terms).
enum Term : int {
    T_POISSON = 1 << 0, T_DISSIPATION = 1 << 1, T_SVISCOSITY = 1 << 2, T_E_INT = 1 << 3,
    T_PRESSURE = 1 << 4, T_E_EXT = 1 << 5, T_CONTINUITY = 1 << 6, T_ADVECTION = 1 << 7,
    T_PENALIZATION = 1 << 8, T_DIFFUSION = 1 << 9,
};

// One batched 1-D transform along x or y: in -> out with a load multiplier.
struct AxisJob {
    const void *in;
    void *out;
    int mul;
    int pad_;
};

// One z-axis real transform pair: two real rows <-> one complex line.
// c2r: half spectra inA/inB (multiplied by mulA/mulB) -> real rows outA/outB;
// r2c: real rows inA/inB -> half spectra outA/outB.  inB == nullptr: single row.
struct ZJob {
    const void *inA, *inB;
    void *outA, *outB;
    int mulA, mulB;
};

// Grid geometry and axis tables, valid for all three axes of the cubic box.
template <typename T> struct Geo {
    int n, nzc;
    const T *kv;       // k_val_at(i), i < n                        (axis_EqSt.cpp:57-61)
    const double *q2;  // pow(k_val_at(i)/k_val_at(n/2), 2.), i < n  (OP_dealiasing.hpp:24-28)
    double thr;        // smallest double s with sqrt(s) >= 2/3 (see dealias_threshold)
    const int *pb;     // per (j, kz) column: the 2/3 rule along i as a bound (dealias_bounds), or nullptr
};

// sqrt is correctly rounded and monotone, so sqrt(s) < 2/3 holds exactly when
// s < thr for the smallest double thr with sqrt(thr) >= 2/3: the 2/3 rule of
// rhs_standard.cpp:22 on |k~| (OP_dealiasing.hpp:28) without a square root.
inline double dealias_threshold() {
    const double c = 2. / 3.;
    double s = c * c;
    while (!(std::sqrt(s) < c)) s = std::nextafter(s, 0.);
    while (std::sqrt(s) < c) s = std::nextafter(s, 1.);
    return s;
}

// 2/3 rule of rhs_standard.cpp:22 on the exact |k~|^2 = (q2[i] + q2[j]) + q2[k].
__device__ __forceinline__ bool dealias_keep(const double *__restrict__ q2, double thr, int i, int j, int k) {
    return __dadd_rn(__dadd_rn(q2[i], q2[j]), q2[k]) < thr;
}

// The 2/3 rule along the x axis of one (j, kz) column as a bound: keep(i) ==
// (min(i, n - i) <= b), with b from the host table dealias_bounds (which checks
// that equivalence for every i of the column and stores -2 where it does not
// hold); -2 or no table: the exact sum of dealias_keep per element.
__device__ __forceinline__ int dealias_bound(const int *__restrict__ pb, int jj, int kk, int nzc) {
    return pb ? pb[jj * nzc + kk] : -2;
}
__device__ __forceinline__ bool dealias_keep_b(const double *__restrict__ q2, double thr, int b, int n, int i, int j,
                                               int k) {
    if (b >= -1) return (i <= n / 2 ? i : n - i) <= b;
    return dealias_keep(q2, thr, i, j, k);
}

// Everything the spectral linear terms and the assembly need.
template <typename T> struct RhsArgs {
    typedef typename C2<T>::type T2;
    const T2 *Y[4];     // stage input: u'_x, u'_y, u'_z, s  (half spectra)
    const T2 *phihat;   // r2c(phi), unnormalised
    const T *SV;        // spectral-viscosity table field_SV (rhs_standard.cpp:57-71), cut applied
    const T *PF;        // phi filter exp(-2000 |k~_Q1|^15) (operations.hpp:20-46)
    T tau, theta, M, D;
    int terms;
};

}  // namespace kf
