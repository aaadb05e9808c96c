"""Independent dense formulas used by the ported reference tests.

These restate the reference's own test oracles (not its production code):
  * tests/parallel_correctness.cpp:53-107  -- dense H0, V1, V2, dV/dt built from
    the 3j/Ylm formulas, evaluated here with sympy's exact 3j and scipy's Ylm;
  * tests/SphericalAbsorptionReference.hpp:19-89 -- the s-wave sink from the
    addition theorem, integrating in the distance from the black hole.
They work on any object exposing the reference's public members (the oracle or
the GPU drop-in): Nr, n_modes, modes, r, dr, mu, M1, M2, q, R1, R2, theta,
Omega, counter, P, l_max.
"""
from __future__ import annotations

import functools
import math

import numpy as np
from numpy.polynomial.legendre import leggauss
from scipy.special import eval_legendre, sph_harm_y


@functools.lru_cache(maxsize=None)
def _w3j(a, b, c, d, e, f):
    from sympy import N
    from sympy.physics.wigner import wigner_3j
    return float(N(wigner_3j(a, b, c, d, e, f), 25))


def equatorial_plm(l, m):
    """gsl_sf_legendre_sphPlm(l, |m|, 0) with the reference's sign flip for odd negative m."""
    y = float(np.real(sph_harm_y(l, abs(m), np.pi / 2, 0.0)))
    if m < 0 and abs(m) % 2:
        y = -y
    return y


def angular(l, m, l1, m1, ls):
    ms = m1 - m
    pref = (1.0 if m1 % 2 == 0 else -1.0) * math.sqrt((2 * l + 1) * (2 * l1 + 1) * (2 * ls + 1) / (4 * math.pi))
    return pref * _w3j(ls, l1, l, 0, 0, 0) * _w3j(ls, l1, l, -ms, m1, -m) * equatorial_plm(ls, ms)


def dense_reference(cn, time, ramp_periods, smear=None, absorb=False):
    """Dense H0, V1, V2, dVdt (and the sink) of tests/parallel_correctness.cpp:53-107."""
    n, Nr = cn.n_modes, cn.Nr
    size = n * Nr
    h0 = np.zeros((size, size), complex)
    v1 = np.zeros_like(h0)
    v2 = np.zeros_like(h0)
    dvdt = np.zeros_like(h0)
    P = cn.P
    ramp_x = time / (ramp_periods * P) if ramp_periods > 0 else 0.0
    ramp = 3 * ramp_x ** 2 - 2 * ramp_x ** 3 if time < ramp_periods * P else 1.0
    abs_ramp = 1.0
    if time < ramp_periods * P:
        abs_ramp = 0.0
    elif time < (ramp_periods + 1) * P:
        x = (time - ramp_periods * P) / P
        abs_ramp = 3 * x * x - 2 * x ** 3
    r = np.asarray(cn.r)
    dr = cn.dr
    for j, (l, m) in enumerate(cn.modes):
        for i in range(1, Nr - 1):
            row = j * Nr + i
            h0[row, row] = (2 / (dr * dr) + l * (l + 1) / (r[i] * r[i])) / (2 * cn.mu)
            h0[row, row - 1] = h0[row, row + 1] = -1 / (2 * cn.mu * dr * dr)
        for k, (l1, m1) in enumerate(cn.modes):
            ms = m1 - m
            for ls in range(abs(l1 - l), l1 + l + 1):
                if abs(ms) > ls:
                    continue
                a = angular(l, m, l1, m1, ls)
                if a == 0.0:
                    continue
                phase = np.exp(1j * ms * cn.theta)
                ri = r[1:Nr - 1]
                rad1 = np.minimum(ri, cn.R1) ** ls / np.maximum(ri, cn.R1) ** (ls + 1)
                rad2 = np.minimum(ri, cn.R2) ** ls / np.maximum(ri, cn.R2) ** (ls + 1)
                common = -cn.mu * (cn.M1 + cn.M2) * 4 * np.pi / (2 * ls + 1) * a * phase
                e1 = common / (1 + cn.q) * rad1
                e2 = common * (1.0 if ms % 2 == 0 else -1.0) * cn.q / (1 + cn.q) * rad2
                rows = j * Nr + np.arange(1, Nr - 1)
                cols = k * Nr + np.arange(1, Nr - 1)
                v1[rows, cols] += e1
                v2[rows, cols] += e2
                dvdt[rows, cols] += (e1 + ramp * e2) * (-1.0 if cn.counter else 1.0) * 1j * ms * cn.Omega
    out = dict(h0=h0, v1=v1, v2=v2, dvdt=dvdt, ramp=ramp, abs_ramp=abs_ramp)
    if absorb:
        out["absorption"] = sink_reference(cn, smear, abs_ramp)
    return out


def absorption_moments(cn, smear, body):
    """Legendre moments of one body's kernel in distance space (SphericalAbsorptionReference.hpp:19-45)."""
    Nr, lmax = cn.Nr, cn.l_max
    mom = np.zeros((2 * lmax + 1, Nr))
    width = smear * (cn.M1 if body == 1 else cn.M2)
    d = cn.R1 if body == 1 else cn.R2
    if width < cn.dr or width <= 0:
        return mom
    xg, wg = leggauss(256)
    r = np.asarray(cn.r)
    for i in range(1, Nr - 1):
        ri = r[i]
        low, high = abs(ri - d), min(width, ri + d)
        if d < 1e-8 * width:
            if ri < width:
                mom[0, i] = 4 * np.pi * np.exp(-1 / (1 - ri * ri / (width * width)))
        elif low < high:
            s = (high - low) / 2 * xg + (high + low) / 2
            w = (high - low) / 2 * wg
            u = np.clip((ri * ri + d * d - s * s) / (2 * ri * d), -1, 1)
            ker = 2 * np.pi / (ri * d) * w * s * np.exp(-1 / (1 - s * s / (width * width)))
            for l in range(2 * lmax + 1):
                mom[l, i] = np.sum(ker * eval_legendre(l, u))
    norm = np.sum(cn.dr * r[1:Nr - 1] ** 2 * mom[0, 1:Nr - 1])
    if norm > 0:
        mom /= norm
    return mom


def swave_projector_reference(cn, smear, body):
    mom = absorption_moments(cn, smear, body)
    phi = cn.theta + (0.0 if body == 1 else np.pi)
    v = np.zeros(cn.Nr * cn.n_modes, complex)
    r = np.asarray(cn.r)
    for j, (l, m) in enumerate(cn.modes):
        direction = np.conj(np.real(sph_harm_y(l, abs(m), np.pi / 2, 0.0)) * (-1.0 if (m < 0 and abs(m) % 2) else 1.0)
                            * np.exp(1j * m * phi))
        v[j * cn.Nr + 1:(j + 1) * cn.Nr - 1] = r[1:cn.Nr - 1] * mom[l, 1:cn.Nr - 1] * direction
    return v


def sink_reference(cn, smear, ramp):
    size = cn.Nr * cn.n_modes
    g = np.zeros((size, size), complex)
    for body in (1, 2):
        mass = cn.M1 if body == 1 else cn.M2
        v = swave_projector_reference(cn, smear, body)
        g += 16 * np.pi * mass * mass * ramp * cn.dr * np.outer(v, v.conj())
    return g


def read_modesbin(path, modes):
    """MODESBIN reader (include/InitialData.hpp:18-34): missing modes are zero, extras ignored."""
    import struct
    with open(path, "rb") as f:
        if f.read(8) != b"MODESBIN":
            raise RuntimeError("not a MODESBIN file")
        (version,) = struct.unpack("<i", f.read(4))
        if version != 1:
            raise RuntimeError("unsupported MODESBIN version")
        nr, count = struct.unpack("<qq", f.read(16))
        stored = {}
        for _ in range(count):
            l, m = struct.unpack("<ii", f.read(8))
            re = np.frombuffer(f.read(8 * nr), "<f8")
            im = np.frombuffer(f.read(8 * nr), "<f8")
            stored[(l, m)] = re + 1j * im
    psi = np.zeros(nr * len(modes), complex)
    for j, lm in enumerate(modes):
        if tuple(lm) in stored:
            psi[j * nr:(j + 1) * nr] = stored[tuple(lm)]
    return psi
