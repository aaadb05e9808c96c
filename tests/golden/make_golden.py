"""Generate the golden fixtures under tests/golden/.

Run once in a container that has the reference checkout and sympy/scipy:

    python tests/golden/make_golden.py /path/to/reference

Outputs (all small, committed):
  special.npz        Wigner 3j symbols (sympy, exact), normalised associated
                     Legendre values at the equator (scipy) and 128-point
                     Gauss-Legendre nodes on [0, 1] (numpy): the three GSL
                     routines the reference calls (gsl_sf_coupling_3j,
                     gsl_sf_legendre_sphPlm, gsl_integration_glfixed).
  coupling_l4.npz    The reference's coupling cache (pair order, l*, angular
                     coefficient) for l_max = 4, evaluated with sympy's exact
                     3j and Ylm (formula of
                     src/CrankNicolsonModes_hamiltonian.cpp:68-104).
  state_211_*.modesbin  MODESBIN initial states written by the reference's own
                     generator initial_states/get_initial_state_COM_fast.py
                     (a 2p hydrogenic cloud on the primary), on small grids.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def special(out):
    from sympy import Rational, N
    from sympy.physics.wigner import wigner_3j
    from scipy.special import sph_harm_y

    rng = np.random.default_rng(1)
    args, vals = [], []
    # every 3j the coupling cache needs for l_max <= 4, and a random sample up to l* = 32
    for l in range(0, 5):
        for l1 in range(0, 5):
            for ls in range(abs(l - l1), l + l1 + 1):
                for m in range(-l, l + 1):
                    for m1 in range(-l1, l1 + 1):
                        ms = m1 - m
                        if abs(ms) > ls:
                            continue
                        args.append((2 * ls, 2 * l1, 2 * l, -2 * ms, 2 * m1, -2 * m))
    while len(args) < 4000:
        l = int(rng.integers(0, 17))
        l1 = int(rng.integers(0, 17))
        ls = int(rng.integers(abs(l - l1), l + l1 + 1))
        m = int(rng.integers(-l, l + 1))
        m1 = int(rng.integers(-l1, l1 + 1))
        ms = m1 - m
        if abs(ms) > ls:
            continue
        args.append((2 * ls, 2 * l1, 2 * l, -2 * ms, 2 * m1, -2 * m))
        args.append((2 * ls, 2 * l1, 2 * l, 0, 0, 0))
    for a in args:
        v = wigner_3j(Rational(a[0], 2), Rational(a[1], 2), Rational(a[2], 2),
                      Rational(a[3], 2), Rational(a[4], 2), Rational(a[5], 2))
        vals.append(float(N(v, 30)))
    lm, ylm = [], []
    for l in range(0, 33):
        for m in range(0, l + 1):
            lm.append((l, m))
            ylm.append(float(np.real(sph_harm_y(l, m, np.pi / 2, 0.0))))
    x, w = np.polynomial.legendre.leggauss(128)
    np.savez(out, w3j_args=np.array(args, np.int32), w3j=np.array(vals),
             ylm_lm=np.array(lm, np.int32), ylm=np.array(ylm),
             gl128_x=(x + 1) / 2, gl128_w=w / 2)


def coupling(out, l_max=4):
    from sympy import Rational, N, sqrt, pi, Ynm, Symbol
    from sympy.physics.wigner import wigner_3j

    modes = [(l, m) for l in range(l_max + 1) for m in range(-l, l + 1) if (l - m) % 2 == 0]
    rows, cols, lss, ang = [], [], [], []
    for j, (l, m) in enumerate(modes):
        for k, (l1, m1) in enumerate(modes):
            ms = m1 - m
            for ls in range(abs(l1 - l), l1 + l + 1):
                if abs(ms) > ls or (l + l1 + ls) % 2:
                    continue
                w1 = wigner_3j(ls, l1, l, 0, 0, 0)
                w2 = wigner_3j(ls, l1, l, -ms, m1, -m)
                # Y_{l*,|m*|}(pi/2, 0) with the Condon-Shortley phase, sign-flipped for odd negative m*
                y = Ynm(ls, abs(ms), pi / 2, 0).expand(func=True)
                if ms < 0 and abs(ms) % 2:
                    y = -y
                pref = (1 if m1 % 2 == 0 else -1) * sqrt(Rational((2 * l + 1) * (2 * l1 + 1) * (2 * ls + 1), 4) / pi)
                a = N(pref * w1 * w2 * y, 30)
                if a != 0:
                    rows.append(j)
                    cols.append(k)
                    lss.append(ls)
                    ang.append(float(a))
    np.savez(out, l_max=l_max, rows=np.array(rows, np.int32), cols=np.array(cols, np.int32),
             l_star=np.array(lss, np.int32), angular=np.array(ang))


CONFIG = """
[grid]
N = {N}
L = {L}
[binary]
q = {q}
R = {R}
[atom]
mu = {mu}
n = 2
l = 1
m = 1
M_c = 0.01
[simulation]
dt = 1.0
num_steps = 11
save_every = 5
l_max = {l_max}
r_ex = 50.0
epsilon = 0.0
absorption = false
evolve_orbit = false
"""


def states(reference):
    script = os.path.join(reference, "initial_states", "get_initial_state_COM_fast.py")
    cases = [dict(N=256, L=128.0, q=0.1, R=30.0, mu=0.2, l_max=4),
             dict(N=320, L=160.0, q=0.5, R=50.0, mu=0.25, l_max=8)]
    for c in cases:
        name = "state_211_N{N}_L{L:g}_q{q:g}_R{R:g}_mu{mu:g}_l{l_max}.modesbin".format(**c)
        with tempfile.TemporaryDirectory() as tmp:
            cfg = os.path.join(tmp, "config.toml")
            with open(cfg, "w") as f:
                f.write(CONFIG.format(**c))
            subprocess.run([sys.executable, script, "--config", cfg, "--output",
                            os.path.join(HERE, name)], check=True, cwd=tmp)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else None
    special(os.path.join(HERE, "special.npz"))
    coupling(os.path.join(HERE, "coupling_l4.npz"))
    if ref:
        states(ref)
