"""Mixed-precision path: the tensor-core coupling apply and the defect-correction solve.

The low-precision operator (complex64 state, fp16 Gaunt and radial-weight products on
the tensor cores, fp32 accumulation) is checked three ways: against a numpy emulation of
the same rounding (fp16 significands, exact products, fp32-level sums) to 2e-5 of the
operator's norm, against the fp64 operator of the same handle (the fp16 error budget,
3e-3 of |V x|, 2e-5 of |A x|), and the mixed step against the fp64 step.  Tolerances
are relative 2-norms.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def f16(a):
    """Round to the fp16 significand (11 bits) with an unbounded exponent: the kernel scales
    both operands by powers of two into fp16's range, so only the significand rounds."""
    m, e = np.frexp(np.asarray(a, np.float64))
    return np.ldexp(np.rint(m * 2048.0) / 2048.0, e)


def make(precision, l_max=12, N=2000, L=200.0, mu=0.25, q=0.5, R=50.0, dt=0.5, absorption=True, t_factor=3.0):
    from boson_cloud_binary_b200 import CrankNicolsonModes
    from boson_cloud_binary_b200.initial_state import hydrogenic_on_primary
    cn = CrankNicolsonModes(N, L, dt, 0.0, l_max, mu, 0.01, q, 0.0, R, False, absorption, 10 ** 9, 2.0, 2.0,
                            precision=precision)
    cn.set_initial_state_full(hydrogenic_on_primary(cn.r, cn.modes, mu, q, R))
    cn.evolve_orbit = True
    cn.steps_per_period = cn.P / dt
    cn.initialize()
    cn.build_damping_mask(0.85, 1.0, 6)
    cn.run(10 ** 9, 0.75 * L)
    t0 = t_factor * cn.P
    cn.t_i = t0
    cn.refresh(t0)
    return cn


def emulate_v(cn, x):
    """fp16 emulation of the tensor-core coupling V x (the handle's current operator)."""
    from oracle import oracle as O
    n, N = cn.n_modes, cn.Nr
    orc = O.OracleCNM(N, cn.L, cn.dt, 0.0, cn.l_max, cn.mu, 0.01, cn.q, 0.0, cn.R, False, False, 10 ** 9, 2.0, 2.0)
    orc.set_initial_state_full(np.zeros(n * N, complex))
    orc.initialize()   # builds the coupling cache
    rows, cols, ls, ang = orc.coupling_terms()
    K = 2 * cn.l_max + 1
    G = np.zeros((K, n, n))
    for r_, c_, l_, a_ in zip(rows, cols, ls, ang):
        G[l_, r_, c_] += a_ * 4 * math.pi / (2 * l_ + 1)
    r = cn.r
    R1, R2, q, Mt = cn.R1, cn.R2, cn.q, cn.M1 + cn.M2
    hh = np.zeros((K, N))
    for l in range(K):
        f1 = 1 / (1 + q) * np.minimum(r, R1) ** l / np.maximum(r, R1) ** (l + 1)
        f2 = q / (1 + q) * np.minimum(r, R2) ** l / np.maximum(r, R2) ** (l + 1)
        hh[l] = -cn.mu * Mt * (f1 + (-1) ** l * f2)
    hh[:, 0] = hh[:, -1] = 0.0
    m = np.array([mm for _, mm in cn.modes])
    th = np.float32(cn.theta)
    ph = np.exp(1j * (m * th).astype(np.float32)).astype(np.complex64)
    X = np.asarray(x, np.complex64).reshape(n, N)
    Z = ph[:, None] * X
    Zr = np.concatenate([Z.real, Z.imag], axis=1).astype(np.float32)
    h2 = np.concatenate([hh, hh], axis=1).astype(np.float32)
    acc = np.zeros((n, 2 * N), np.float64)
    for l in range(K):
        acc += f16(G[l]) @ f16(h2[l][None, :] * Zr)
    w = acc[:, :N] + 1j * acc[:, N:]
    return (np.conj(ph)[:, None].astype(np.complex128) * w).reshape(-1)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("l_max", [4, 8, 12])
def test_tc_apply_against_emulation_and_fp64(l_max):
    cn = make("mixed", l_max=l_max, N=1200, L=120.0)
    rng = np.random.default_rng(l_max)
    x = cn.psi + 1e-2 * np.linalg.norm(cn.psi) / math.sqrt(cn.size) * (
        rng.standard_normal(cn.size) + 1j * rng.standard_normal(cn.size))
    v_tc = cn.apply_lowp("V", x)
    v64 = cn.apply("V", x)
    v_em = emulate_v(cn, x)
    assert rel(v_tc, v_em) < 2e-5
    assert rel(v_tc, v64) < 3e-3
    a_tc = cn.apply_lowp("A", x)
    a64 = cn.apply("A", x)
    assert rel(a_tc, a64) < 2e-5
    h_tc = cn.apply_lowp("H", x)
    h64 = cn.apply("H", x)
    assert rel(h_tc, h64) < 1e-3


def test_tc_apply_sinks_match_fp64():
    cn = make("mixed", l_max=8, N=1200, L=120.0)
    assert cn.absorption_sink_active()
    x = cn.psi
    a_tc = cn.apply_lowp("A_full", x)
    a64 = cn.apply("A_full", x)
    assert rel(a_tc, a64) < 2e-5
    # the sink part alone, A_full - A (both outputs are rounded to complex64 at the scale
    # of |A x|, so the difference is compared on that scale)
    d_tc = a_tc - cn.apply_lowp("A", x)
    d64 = a64 - cn.apply("A", x)
    assert np.linalg.norm(d64) > 0.0
    assert np.linalg.norm(d_tc - d64) < 1e-6 * np.linalg.norm(a64)


@pytest.mark.parametrize("l_max,N,L", [(8, 2000, 200.0), (12, 2000, 200.0)])
def test_mixed_steps_match_fp64(l_max, N, L):
    """Ten steps of the mixed solve against the fp64 solve at tolerance 1e-14 from the same
    state: U_lm within 1e-10, cloud mass (mu dr sum |U|^2) within 1e-12, R within 1e-12."""
    a = make("mixed", l_max=l_max, N=N, L=L)
    b = make("fp64", l_max=l_max, N=N, L=L)
    a.tolerance = 1e-12
    b.tolerance = 1e-14
    b.psi = a.psi
    for k in range(1, 11):
        da = a.step(k)
        db = b.step(k)
        passes, fp64_applies, res = a.mixed_info()
        assert res <= 1e-12
        assert passes == 2, (k, a.mixed_trace())
    pa, pb = a.psi, b.psi
    assert rel(pa, pb) < 1e-10
    ma = a.mu * a.dr * np.sum(np.abs(pa) ** 2)
    mb = b.mu * b.dr * np.sum(np.abs(pb) ** 2)
    assert abs(ma - mb) / mb < 1e-12
    assert abs(da["R"] - db["R"]) / db["R"] < 1e-12
    assert abs(da["energy"] - db["energy"]) / abs(db["energy"]) < 1e-9
