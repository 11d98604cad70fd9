"""Seeded synthetic inputs for the kielflow time step (host side, numpy).

The reference starts from HDF5 files written by its frontend
(``src/frontend/frontend.cpp:133-198``; loaded at ``kielflow.cpp:156-163``).
Here the initial state is built in memory from a seed so that every arm (the
CUDA path, the CPU oracle, the reference compiled on the CPU) gets the same
bits:

* box: ``axis_CoEqSt(-L/2, L, n)`` on each axis (``axis_EqSt.cpp:52-55``),
  L = 2*pi*4 Debye lengths;
* noise: ``eps(x) = sum_m 1e-3 (g1 cos(2 pi m.x/L) + g2 sin(2 pi m.x/L))`` over
  the half space of integer wave vectors 0 < |m| <= 4, with g1, g2 standard
  normal draws from SplitMix64 (Steele, Lea & Flood 2014) through the
  Box-Muller transform, one stream per field;
* state: ``s = ln n = ln(1 + eps_n)`` (the reference evolves ln n,
  ``kielflow.cpp:172-182``) and the velocity perturbation ``u' = eps_u`` (the
  mean flow M e_x enters only through M d/dx, ``rhs_standard.cpp:279-311``);
* dust: ``fkt3d_Gauss(Q, sigma, sigma, sigma)`` at the box centre
  (``masks.hpp:351-366``); penalization mask ``H = [r < radius]``.

Spectral fields use the reference's half-spectrum layout (``field_imag``,
``field_imag.cpp:16,23``): complex128 arrays of shape (n, n, n//2 + 1), C order,
FFTW's unnormalised forward convention.
"""
from __future__ import annotations

import math

import numpy as np

L_DEFAULT = 2.0 * math.pi * 4.0
_MASK64 = (1 << 64) - 1


def val_at(i: int, n: int, L: float, m: float = 0.0) -> float:
    """Position of index i (-1 <= i <= n): ``axis_CoEqSt::val_at`` = l0 + i*(L/N)
    for m == 0, else ``axis_CoSiSt::val_at`` (axis_SiSt.cpp:93-116), the
    periodic extension of S(l0 + L i/N) with S(x) = x - m sin(2 pi x/L)."""
    l0 = -0.5 * L
    if m == 0.0:
        return l0 + i * (L / n)
    shift = 0
    if i < 0:
        while True:
            shift += 1
            if not i + shift * n < 0:
                break
    if i >= n:
        while True:
            shift -= 1
            if not i + shift * n >= n - 1:
                break
    pi = math.acos(-1.0)
    x = l0 + L * float(i + shift * n) / n
    return (x - m * math.sin(2.0 * pi * x / L)) - shift * L


def axis_values(n: int, L: float, m: float = 0.0) -> np.ndarray:
    """val_at(i) for i < n (axis_CoEqSt, or axis_CoSiSt for m > 0)."""
    return np.array([val_at(i, n, L, m) for i in range(n)], dtype=np.float64)


def frontend_stretch(L: float) -> float:
    """The stretching the reference's frontend uses, m = L (1 - 0.3) / (2 pi)
    (frontend.cpp:285-287): cells at the box centre are 0.3 h wide."""
    return L * (1.0 - 0.3) / (2.0 * math.acos(-1.0))


def k_values(n: int, L: float) -> np.ndarray:
    """``axis_CoEqSt::k_val_at`` (axis_EqSt.cpp:57-61); the Nyquist index n/2
    carries +pi n / L."""
    pi = math.acos(-1.0)
    return np.array([(2.0 * pi * i / L) if i <= n // 2 else (2.0 * pi * (i - n) / L)
                     for i in range(n)], dtype=np.float64)


class SplitMix64:
    """SplitMix64 generator (published constants), 53-bit uniforms."""

    def __init__(self, seed: int, stream: int):
        self.state = (seed * 0x9E3779B97F4A7C15 + (stream + 1) * 0xD1B54A32D192ED03) & _MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / 9007199254740992.0)

    def normal_pair(self) -> tuple[float, float]:
        u1 = 1.0 - self.uniform()  # (0, 1]
        u2 = self.uniform()
        r = math.sqrt(-2.0 * math.log(u1))
        return r * math.cos(2.0 * math.pi * u2), r * math.sin(2.0 * math.pi * u2)


def noise_modes(kmax: int = 4):
    """Integer wave vectors m with 0 < |m| <= kmax in the half space
    (mx > 0) or (mx == 0 and my > 0) or (mx == my == 0 and mz > 0), in
    lexicographic order."""
    out = []
    for mx in range(-kmax, kmax + 1):
        for my in range(-kmax, kmax + 1):
            for mz in range(-kmax, kmax + 1):
                r2 = mx * mx + my * my + mz * mz
                if r2 == 0 or r2 > kmax * kmax:
                    continue
                if mx > 0 or (mx == 0 and my > 0) or (mx == 0 and my == 0 and mz > 0):
                    out.append((mx, my, mz))
    return out


def noise_spectrum(n: int, seed: int, stream: int, amp: float = 1e-3, kmax: int = 4) -> np.ndarray:
    """Half spectrum H with ``numpy.fft.irfftn(H, (n,n,n)) == eps`` exactly in
    exact arithmetic (the box origin -L/2 only flips the sign of odd modes)."""
    if n < 2 * kmax + 2:
        raise ValueError("grid too small for the noise band")
    N = float(n) ** 3
    H = np.zeros((n, n, n // 2 + 1), dtype=np.complex128)
    rng = SplitMix64(seed, stream)
    for (mx, my, mz) in noise_modes(kmax):
        g1, g2 = rng.normal_pair()
        a, b = amp * g1, amp * g2
        sgn = -1.0 if (abs(mx) + abs(my) + abs(mz)) % 2 else 1.0
        plus = N * sgn * complex(a, -b) / 2.0   # coefficient of e^{+i psi}
        minus = N * sgn * complex(a, b) / 2.0   # coefficient of e^{-i psi}
        if mz > 0:
            H[mx % n, my % n, mz] += plus
        elif mz < 0:
            H[(-mx) % n, (-my) % n, -mz] += minus
        else:
            H[mx % n, my % n, 0] += plus
            H[(-mx) % n, (-my) % n, 0] += minus
    return H


def initial_state(n: int, seed: int = 0, amp: float = 1e-3, kmax: int = 4):
    """(FUx, FUy, FUz, Fs): spectral u' (noise) and s = ln(1 + noise)."""
    Hu = [noise_spectrum(n, seed, q, amp, kmax) for q in range(3)]
    eps_n = np.fft.irfftn(noise_spectrum(n, seed, 3, amp, kmax), s=(n, n, n), axes=(0, 1, 2))
    s = np.log1p(eps_n)
    Fs = np.fft.rfftn(s)
    return Hu[0], Hu[1], Hu[2], Fs


def gauss_charge(n: int, L: float, Q: float, sigma: float, m: float = 0.0) -> np.ndarray:
    """``fkt3d_Gauss(Q, sigma, sigma, sigma)`` sampled on the grid
    (masks.hpp:351-366, filled as field_real::fill, field_real.cpp:78-95)."""
    pi = math.acos(-1.0)
    A = Q / (math.pow(math.sqrt(pi), 3.0) * sigma * sigma * sigma)
    x = axis_values(n, L, m)
    X = (x / sigma) ** 2
    e = -X[:, None, None] - X[None, :, None] - X[None, None, :]
    return A * np.exp(e)


def sphere_mask(n: int, L: float, radius: float, m: float = 0.0) -> np.ndarray:
    x = axis_values(n, L, m)
    r2 = x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2
    return (r2 < radius * radius).astype(np.float64)


def cfl_dt(state, n: int, L: float, M: float, cfl: float = 0.2, m: float = 0.0) -> float:
    """dt = cfl * h_min / max(|M + u'_x|, |u'_y|, |u'_z|) from the initial
    state, then held fixed (the reference's RK4 keeps dt_ fixed,
    RKO4.cpp:41-47); h_min = h (1 - 2 pi m / L) on a stretched axis."""
    h = L / n * (1.0 - 2.0 * math.acos(-1.0) * m / L)
    ux = np.fft.irfftn(state[0], s=(n, n, n), axes=(0, 1, 2))
    uy = np.fft.irfftn(state[1], s=(n, n, n), axes=(0, 1, 2))
    uz = np.fft.irfftn(state[2], s=(n, n, n), axes=(0, 1, 2))
    vmax = max(np.abs(M + ux).max(), np.abs(uy).max(), np.abs(uz).max())
    return float(cfl * h / vmax)
