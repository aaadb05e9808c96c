"""The oracle's restatements of the three GSL routines and of the coupling cache,
pinned against golden tables from sympy / scipy / numpy (tests/golden/make_golden.py)."""
import os

import numpy as np

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_wigner3j_matches_sympy_exact():
    g = np.load(os.path.join(GOLD, "special.npz"))
    got = np.array([O.wigner3j(*map(int, a)) for a in g["w3j_args"]])
    ref = g["w3j"]
    assert np.array_equal(got == 0, ref == 0)
    nz = ref != 0
    assert np.max(np.abs(got[nz] - ref[nz]) / np.abs(ref[nz])) < 4e-16


def test_equatorial_legendre_matches_scipy():
    g = np.load(os.path.join(GOLD, "special.npz"))
    got = np.array([O.sph_plm_equator(int(l), int(m)) for l, m in g["ylm_lm"]])
    assert np.max(np.abs(got - g["ylm"])) < 2e-15


def test_gauss_legendre_matches_numpy():
    g = np.load(os.path.join(GOLD, "special.npz"))
    x, w = O.gauss_legendre(128, 0.0, 1.0)
    assert np.max(np.abs(x - g["gl128_x"])) < 1e-15
    assert np.max(np.abs(w - g["gl128_w"])) < 5e-15  # numpy's own weights carry ~3e-15
    assert abs(w.sum() - 1.0) < 1e-14


def test_coupling_cache_matches_exact_gaunt():
    c = np.load(os.path.join(GOLD, "coupling_l4.npz"))
    cn = O.OracleCNM(16, 10.0, 1.0, 0.0, 4, 0.2, 0.0, 0.1, 0.0, 30.0, False, False, 10, 0.0, 2.0)
    cn.initialize()
    rows, cols, ls, ang = cn.coupling_terms()
    assert np.array_equal(rows, c["rows"]) and np.array_equal(cols, c["cols"])
    assert np.array_equal(ls, c["l_star"])
    assert np.max(np.abs(ang - c["angular"])) < 1e-15
