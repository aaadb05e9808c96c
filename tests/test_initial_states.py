"""displaced_100_state (src/DisplacedAtom.cpp:12-76): the mode projection of a displaced
hydrogenic 1s state.  The known-answer checks of the reference's tests/isolated_bh.cpp
(check_projection) run on the oracle and on the device generator: the centred state
equals the analytic 2 r e^{-r/a0} / a0^{3/2} to 1e-13 with no higher modes, the continuum
norm is 1 to 1e-5, and the translated state reconstructed on the x axis at x = +-5
matches e^{-|x - x_bh|/a0} / sqrt(pi a0^3) to 1e-5 relative.  The device generator
matches the oracle to 1e-12."""
import numpy as np
import pytest

from oracle.oracle import displaced_100_state as oracle_state
from oracle.oracle import sph_plm_equator


def _modes(lmax):
    return [(l, m) for l in range(lmax + 1) for m in range(-l, l + 1) if (l - m) % 2 == 0]


def _device_state(*args):
    from boson_cloud_binary_b200 import displaced_100_state
    return displaced_100_state(*args)


IMPLS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


@pytest.mark.parametrize("kind", IMPLS)
def test_projection_known_answers(kind):
    gen = oracle_state if kind == "oracle" else _device_state
    mu, a0 = 0.5, 4.0
    r = np.linspace(0.0, 40.0, 257)
    modes = _modes(12)
    centred = gen(r, modes, mu, 0.0)
    i = np.arange(1, len(r) - 1)
    assert np.max(np.abs(centred[i] - 2 * r[i] * np.exp(-r[i] / a0) / a0 ** 1.5)) < 1e-13
    assert np.linalg.norm(centred[len(r):]) == 0.0
    assert abs(np.vdot(centred, centred).real * (r[1] - r[0]) - 1) < 1e-5
    for offset in (-2.0, 2.0):
        state = gen(r, modes, mu, offset)
        for x in (-5.0, 5.0):
            k = 32  # r = 5
            rec = 0.0
            for j, (l, m) in enumerate(modes):
                y = sph_plm_equator(l, abs(m))
                if m < 0 and abs(m) % 2:
                    y = -y
                if x < 0 and abs(m) % 2:
                    y = -y
                rec += state[j * len(r) + k] * y / r[k]
            expected = np.exp(-abs(x - offset) / a0) / np.sqrt(np.pi * a0 ** 3)
            assert abs(rec - expected) < 1e-5 * expected


def test_invalid_parameters_rejected():
    r = np.linspace(0.0, 10.0, 11)
    with pytest.raises(ValueError):
        oracle_state(r, _modes(2), -1.0, 0.0)
    with pytest.raises(ValueError):
        oracle_state(r[::-1].copy(), _modes(2), 0.5, 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("offset", [0.0, 3.0, -7.5])
def test_device_generator_matches_oracle(offset):
    r = np.linspace(0.0, 120.0, 2001)
    modes = _modes(8)
    want = oracle_state(r, modes, 0.3, offset)
    got = _device_state(r, modes, 0.3, offset)
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)
    with pytest.raises(ValueError):
        _device_state(r, modes, 0.0, offset)


@pytest.mark.gpu
@pytest.mark.parametrize("n,l,m,lmax", [(2, 1, 1, 8), (3, 2, 2, 10), (3, 2, -2, 6), (2, 1, -1, 4), (1, 0, 0, 4)])
def test_device_hydrogenic_state_matches_host_generator(n, l, m, lmax):
    """The device projection of a translated hydrogenic (n, l, m) state (the state of the
    reference's initial_states/get_initial_state_COM_fast.py) against the host generator of
    the benchmark (scipy spherical harmonics and Laguerre polynomials) on the same
    quadrature, to 1e-12 relative.  (States with l - m odd are odd in z and have no weight on
    the solver's modes, which all have l - m even.)"""
    from boson_cloud_binary_b200 import hydrogenic_state
    from boson_cloud_binary_b200.initial_state import hydrogenic_on_primary
    modes = _modes(lmax)
    r = np.linspace(0.0, 120.0, 600)
    mu, q, R = 0.3, 0.5, 30.0
    dev = hydrogenic_state(r, modes, mu, q, R, n=n, l=l, m=m)
    host = hydrogenic_on_primary(r, modes, mu, q, R, n=n, l=l, m=m)
    assert np.linalg.norm(dev - host) / np.linalg.norm(host) < 1e-12


def test_gaussian_state_is_the_reference_profile():
    """initial_states/get_initial_state_gaussian.py: U_00 = sqrt(4 pi) r exp(-r^2/(2 sigma^2)),
    normalised by the trapezoidal rule, every other mode zero."""
    from boson_cloud_binary_b200.cnm import gaussian_state
    r = np.linspace(0.0, 200.0, 2001)
    modes = _modes(4)
    u = gaussian_state(r, modes, 10.0).reshape(len(modes), -1)
    assert np.count_nonzero(np.abs(u[1:]).sum(axis=1)) == 0
    assert abs(np.trapezoid(np.abs(u[0]) ** 2, x=r) - 1.0) < 1e-14
    ref = np.sqrt(4 * np.pi) * r * np.exp(-0.5 * (r / 10.0) ** 2)
    assert np.allclose(u[0] / u[0][10], ref / ref[10], rtol=1e-14, atol=0)
