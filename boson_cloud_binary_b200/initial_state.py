"""Synthetic initial states of the shapes the benchmark configurations name.

``hydrogenic_on_primary`` projects a hydrogenic (n, l, m) state of the primary
(mass M1, Bohr radius 1/(mu^2 M1)), centred on the primary at x = +R1 in the
centre-of-mass frame, onto the solver's (l, m) modes:
    U_lm(r) = r * int Y_lm^*(Omega) psi_nlm(r Omega - R1 e_x) dOmega,
by Gauss-Legendre quadrature in cos(theta) and the trapezoidal rule in phi.
This is the state the reference's initial_states/get_initial_state_COM_fast.py
writes to a MODESBIN file (there by translation matrices); the test suite pins
the two against each other on a fixture written by that script.
The returned stack is mode-major (j*Nr + i) and normalised to sum |U|^2 dr = 1.
"""
from __future__ import annotations

import math

import numpy as np
from numpy.polynomial.legendre import leggauss
from scipy.special import eval_genlaguerre, sph_harm_y


def _ylm(l, m, theta, phi):
    """Y_lm with the Condon-Shortley phase, negative m from Y_{l,-m} = (-1)^m conj(Y_{l,|m|})."""
    if m >= 0:
        return sph_harm_y(l, m, theta, phi)
    return (-1) ** (-m) * np.conj(sph_harm_y(l, -m, theta, phi))


def radial_hydrogen(n, l, r, a0):
    rho = 2.0 * r / (n * a0)
    norm = math.sqrt((2.0 / (n * a0)) ** 3 * math.factorial(n - l - 1) / (2 * n * math.factorial(n + l)))
    return norm * np.exp(-rho / 2) * rho ** l * eval_genlaguerre(n - l - 1, 2 * l + 1, rho)


def hydrogenic_on_primary(r, modes, mu, q, R, n=2, l=1, m=1, M1=1.0, n_theta=None, n_phi=None,
                          chunk=2048):
    r = np.asarray(r, float)
    l_max = max(lm[0] for lm in modes)
    n_theta = n_theta or max(48, 2 * (l_max + l) + 16)
    n_phi = n_phi or 2 * n_theta
    a0 = 1.0 / (mu * mu * M1)
    R1 = q / (1.0 + q) * R
    x, w = leggauss(n_theta)
    theta = np.arccos(x)
    phi = 2 * np.pi * np.arange(n_phi) / n_phi
    TH, PH = np.meshgrid(theta, phi, indexing="ij")
    weights = (w[:, None] * (2 * np.pi / n_phi)) * np.ones_like(PH)
    # conj(Y_j) * weight on the angular grid, shape (modes, n_theta * n_phi)
    ystar = np.stack([np.conj(_ylm(lj, mj, TH, PH)) * weights for (lj, mj) in modes]).reshape(len(modes), -1)
    st, ct = np.sin(TH).ravel(), np.cos(TH).ravel()
    cp, sp = np.cos(PH).ravel(), np.sin(PH).ravel()
    out = np.zeros((len(modes), r.size), complex)
    for s in range(0, r.size, chunk):
        rr = r[s:s + chunk, None]
        dx = rr * st * cp - R1
        dy = rr * st * sp
        dz = rr * ct
        d = np.sqrt(dx * dx + dy * dy + dz * dz)
        th_b = np.arccos(np.clip(np.where(d > 0, dz / np.where(d > 0, d, 1), 1.0), -1, 1))
        ph_b = np.arctan2(dy, dx)
        psi = radial_hydrogen(n, l, d, a0) * _ylm(l, m, th_b, ph_b)
        out[:, s:s + chunk] = (psi @ ystar.T).T * r[s:s + chunk]
    out[:, 0] = 0.0
    out[:, -1] = 0.0
    flat = out.reshape(-1)
    dr = r[1] - r[0]
    return flat / math.sqrt(np.vdot(flat, flat).real * dr)
