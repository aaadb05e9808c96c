"""Ports of the reference's absorber and boundary tests against the oracle and the GPU drop-in:
tests/spherical_absorption.cpp, tests/fixed_orbit_absorption.cpp, tests/orbital_ramp.cpp and
tests/flux_time_alignment.cpp (tolerances as in the reference)."""
import numpy as np
import pytest
from numpy.polynomial.legendre import leggauss
from scipy.special import sph_harm_y

from impls import IMPLS, make
from reference_formulas import swave_projector_reference


# ----------------------------------------------------------------------------- spherical_absorption.cpp

def direct_angular_projection(cn, i, width):
    """int K Y_j^* dOmega at r_i by direct quadrature in COM polar angles (spherical_absorption.cpp:43-69)."""
    nt, nphi = 512, 1024
    u, w = leggauss(nt)
    phi = 2 * np.pi * np.arange(nphi) / nphi
    U, PHI = np.meshgrid(u, phi, indexing="ij")
    W = np.repeat(w[:, None], nphi, axis=1) * (2 * np.pi / nphi)
    ri = cn.r[i]
    x = ri * np.sqrt(1 - U * U) * np.cos(PHI) - cn.R1 * np.cos(cn.theta)
    y = ri * np.sqrt(1 - U * U) * np.sin(PHI) - cn.R1 * np.sin(cn.theta)
    z = ri * U
    s2 = (x * x + y * y + z * z) / (width * width)
    inside = s2 < 1
    ker = np.where(inside, np.exp(-1 / (1 - np.where(inside, s2, 0.5))), 0.0)
    out = np.zeros(cn.n_modes, complex)
    for j, (l, m) in enumerate(cn.modes):
        theta_pol = np.arccos(U)
        y_lm = sph_harm_y(l, abs(m), theta_pol, 0.0).real * (-1.0 if (m < 0 and abs(m) % 2) else 1.0)
        out[j] = np.sum(W * ker * y_lm * np.exp(-1j * m * PHI))
    return out


def verify_geometry(cn, smear, direct):
    width = smear * cn.M1
    g = 16 * np.pi * cn.M1 ** 2 * cn.dr
    assert cn.absorption_sink_active()
    assert cn.sink_strength(2) == 0.0, "unresolved secondary must not absorb"
    ref = swave_projector_reference(cn, smear, 1)
    rng = np.random.default_rng(7)
    for _ in range(3):
        x = rng.normal(size=ref.size) + 1j * rng.normal(size=ref.size)
        want = g * np.vdot(ref, x) * ref
        assert np.linalg.norm(cn.apply_sink(x) - want) < 1e-10 * np.linalg.norm(want)
    assert abs(cn.sink_strength(1) - g * np.vdot(ref, ref).real) < 1e-10 * cn.sink_strength(1)
    v = cn.sink_vector(1)
    j00 = cn.modes.index((0, 0))
    j11 = cn.modes.index((1, 1)) if (1, 1) in cn.modes else -1
    r = np.asarray(cn.r)
    volume, centroid = 0.0, 0.0j
    for i in range(1, cn.Nr - 1):
        volume += np.sqrt(4 * np.pi) * cn.dr * r[i] * v[j00 * cn.Nr + i].real
        if j11 >= 0:
            centroid -= np.sqrt(8 * np.pi / 3) * cn.dr * r[i] ** 2 * np.conj(v[j11 * cn.Nr + i])
        for j in range(cn.n_modes):
            if abs(r[i] - cn.R1) >= width:
                assert abs(v[j * cn.Nr + i]) < 1e-13, "support outside the radius"
            if cn.R1 == 0 and j != j00:
                assert abs(v[j * cn.Nr + i]) < 1e-13, "central absorber is not isotropic"
    assert abs(volume - 1) < 1e-12
    assert abs(centroid / volume - cn.R1 * np.exp(1j * cn.theta)) < 2e-4
    if direct:
        i = max(1, int(round(cn.R1 / cn.dr)))
        actual = np.array([v[j * cn.Nr + i] / r[i] for j in range(cn.n_modes)])
        quad = direct_angular_projection(cn, i, width)
        scale = actual[j00].real / quad[j00].real
        assert np.linalg.norm(actual - scale * quad) / np.linalg.norm(actual) < 2e-8
    return v


@pytest.mark.parametrize("kind", IMPLS)
@pytest.mark.parametrize("radius,smear,counter,lmax", [
    (0.0, 8, False, 3), (1e-10, 8, True, 3), (90 * 0.01 / 1.01, 8, True, 3), (12.0, 3, False, 3),
    (90 * 0.01 / 1.01, 8, True, 12)])
def test_spherical_absorber_geometry(kind, radius, smear, counter, lmax):
    cn = make(kind, 129, 32, 1, 0, lmax, 0.2, 0, 0.01, 0, 90, counter, True, 100, 0, smear)
    cn.evolve_orbit = False
    cn.R1 = radius
    cn.theta = 0.73
    cn.set_initial_state_full(np.zeros(cn.Nr * cn.n_modes))
    cn.initialize()
    cn.run(1, 20)
    cn.dt = cn.P
    cn.step(1)
    before = verify_geometry(cn, smear, radius > 0 and lmax <= 3)
    th0 = cn.theta
    cn.dt = cn.P / 7
    cn.step(2)
    after = cn.sink_vector(1)
    ang = cn.theta - th0
    ms = np.repeat([m for (_, m) in cn.modes], cn.Nr)
    assert np.max(np.abs(after - before * np.exp(-1j * ms * ang))) < 1e-12, "absorber did not rotate"
    cn.R1 = cn.R1 + 0.4
    cn.M1 = 1.1
    cn.step(3)
    verify_geometry(cn, smear, False)


# ----------------------------------------------------------------------------- fixed_orbit_absorption.cpp

def fixed_orbit_case(kind, absorb, smear, q, radius, ramp_periods, expect_loss):
    cn = make(kind, 65, 64.0, 1.0, 0.0, 0, 0.2, 0.1, q, 0.0, radius, True, absorb, 100, ramp_periods, smear)
    cn.evolve_orbit = False
    cn.dt = cn.P / 16
    dt, period, r1, r2 = cn.dt, cn.P, cn.R1, cn.R2
    init = np.zeros(cn.Nr)
    i = np.arange(1, cn.Nr - 1)
    init[i] = np.sin(np.pi * i / (cn.Nr - 1))
    cn.set_initial_state_full(init)
    cn.initialize()
    cn.run(1, 40.0)
    n0 = np.vdot(cn.psi, cn.psi).real
    assert cn.sink_strength(1) + cn.sink_strength(2) == 0.0
    total, last_sink = 0.0, 0.0
    for k in range(1, 41):
        prev = cn.psi
        d = cn.step(k)
        cur = cn.psi
        assert np.all(np.isfinite(cur))
        assert (cn.R == radius and cn.M1 == 1.0 and cn.M2 == q and cn.R1 == r1 and cn.R2 == r2
                and cn.P == period and cn.dt == dt)
        loss = np.vdot(prev, prev).real - np.vdot(cur, cur).real
        assert loss >= -1e-10 * n0
        total += loss
        mid = 0.5 * (prev + cur)
        assert abs(loss - dt * np.vdot(mid, cn.apply_sink(mid)).real) < 1e-9 * n0
        sink = cn.sink_strength(1) + cn.sink_strength(2)
        if d["t"] <= ramp_periods * period:
            assert sink == 0.0
        if d["t"] >= (ramp_periods + 1) * period and last_sink > 0.0:
            assert abs(sink - last_sink) < 1e-12
        if d["t"] >= (ramp_periods + 1) * period:
            last_sink = sink
    assert cn.phase > 0 and cn.theta < 0 and abs(cn.phase + cn.theta) < 1e-12
    if ramp_periods == 0.0:
        assert abs(cn.phase - 40 * dt * cn.Omega_0) < 1e-12
    if expect_loss:
        assert total > 1e-4 * n0 and last_sink > 0.0
        if q != 1.0:
            off, on = (2, 1) if q < 1.0 else (1, 2)
            assert cn.sink_strength(off) == 0.0 and cn.sink_strength(on) > 0.0
    else:
        assert abs(total) < 1e-9 * n0 and last_sink == 0.0
    return cn.psi


@pytest.mark.parametrize("kind", IMPLS)
def test_fixed_orbit_absorption(kind):
    control = fixed_orbit_case(kind, False, 4.0, 1.0, 20.0, 0.0, False)
    fixed_orbit_case(kind, True, 4.0, 1.0, 20.0, 0.0, True)
    fixed_orbit_case(kind, True, 4.0, 1.0, 20.0, 1.0, True)
    for smear in (0.0, 0.5):
        unresolved = fixed_orbit_case(kind, True, smear, 1.0, 20.0, 0.0, False)
        assert np.linalg.norm(unresolved - control) < 1e-10 * np.linalg.norm(control)
    fixed_orbit_case(kind, True, 4.0, 0.1, 22.0, 0.0, True)
    fixed_orbit_case(kind, True, 0.4, 10.0, 22.0, 0.0, True)
    fixed_orbit_case(kind, True, 4.0, 1.0, 200.0, 0.0, False)


# ----------------------------------------------------------------------------- orbital_ramp.cpp

def check_close(actual, expected):
    assert abs(actual - expected) <= 1e-11 * max(1.0, abs(expected)), (actual, expected)


def set_radius(cn, radius):
    cn.R = radius
    cn.R1 = cn.M2 / (cn.M1 + cn.M2) * radius
    cn.R2 = cn.M1 / (cn.M1 + cn.M2) * radius
    cn.Omega = np.sqrt((cn.M1 + cn.M2) / radius ** 3)
    cn.P = 2 * np.pi / cn.Omega


def smoothstep(x):
    return 0.0 if x <= 0 else 1.0 if x >= 1 else 3 * x * x - 2 * x ** 3


def expected_radius(cn, duration, ramp=1.0):
    return cn.R - (64.0 / 5.0) * cn.M1 * cn.M2 * (cn.M1 + cn.M2) / cn.R ** 3 * duration * ramp


def prepare(cn):
    cn.set_initial_state_full(np.zeros(cn.Nr * cn.n_modes))
    cn.initialize()
    cn.run(1, 100.0)


def potential_gap(cn, weight):
    """max over probes of |(V - (V1 + weight V2)) x| relative to |V x|."""
    rng = np.random.default_rng(11)
    x = rng.normal(size=cn.Nr * cn.n_modes) + 1j * rng.normal(size=cn.Nr * cn.n_modes)
    vx = cn.apply("V", x)
    return np.linalg.norm(vx - cn.apply("V1", x) - weight * cn.apply("V2", x)), np.linalg.norm(vx)


@pytest.mark.parametrize("kind", IMPLS)
@pytest.mark.parametrize("absorb", [False, True])
def test_expanding_orbit(kind, absorb):
    cn = make(kind, 64, 200.0, 200.0, 0.1, 0, 0.2, 0.0, 0.25, 0.0, 50.0, False, absorb, 100, 5.0, 15.0)
    P0 = cn.P
    ramp_end = 5 * P0
    prepare(cn)
    cn.dt = ramp_end + 0.1 * P0
    d1 = cn.step(1)
    set_radius(cn, 80.0)
    cn.dt = 0.1 * P0
    assert 5 * cn.P > d1["t"] + cn.dt
    ramp = smoothstep((d1["t"] + cn.dt - ramp_end) / P0)
    expected = expected_radius(cn, cn.dt, ramp)
    cn.step(2)
    check_close(cn.R, expected)
    gap, _ = potential_gap(cn, 1.0)
    assert gap < 1e-13
    partial = cn.sink_strength(1)
    if absorb:
        assert partial > 0
    cn.dt = P0
    cn.step(3)
    set_radius(cn, 80.0)
    for k in range(4, 9):
        cn.dt = 0.05 * P0
        nxt = expected_radius(cn, cn.dt)
        cn.step(k)
        check_close(cn.R, nxt)
        gap, _ = potential_gap(cn, 1.0)
        assert gap < 1e-13
        if absorb and k == 4:
            check_close(partial, cn.sink_strength(1) * smoothstep(0.2))


@pytest.mark.parametrize("kind", IMPLS)
def test_crossing_step(kind):
    cn = make(kind, 32, 200.0, 200.0, 0.1, 0, 0.2, 0.0, 0.25, 0.0, 50.0, False, False, 100, 5.0, 15.0)
    P0 = cn.P
    prepare(cn)
    cn.dt = 4.9 * P0
    cn.step(1)
    check_close(cn.R, 50.0)
    cn.dt = 0.2 * P0
    expected = expected_radius(cn, 0.1 * P0, smoothstep((5.1 * P0 - 5 * P0) / P0))
    d = cn.step(2)
    check_close(cn.R, expected)
    check_close(d["t"], 5.1 * P0)


@pytest.mark.parametrize("kind", IMPLS)
@pytest.mark.parametrize("ramp_potential", [True, False])
def test_frequency_only_ramp(kind, ramp_potential):
    cn = make(kind, 32, 200.0, 200.0, 0.1, 2, 0.2, 0.0, 0.25, 0.0, 50.0, False, False, 100, 5.0, 15.0)
    cn.ramp_secondary_potential = ramp_potential
    P0 = cn.P
    prepare(cn)
    gap, vn = potential_gap(cn, 0.0 if ramp_potential else 1.0)
    assert gap < 1e-13 * max(1.0, vn)
    cn.dt = 2.0 * P0
    cn.step(1)
    s = smoothstep(0.4)
    check_close(cn.Omega, cn.Omega_0 * s)
    gap, vn = potential_gap(cn, s if ramp_potential else 1.0)
    assert gap < 1e-13 * max(1.0, vn)
    check_close(cn.R, 50.0)
    cn.dt = 4.0 * P0
    cn.step(2)
    gap, vn = potential_gap(cn, 1.0)
    assert gap < 1e-13 * max(1.0, vn)


@pytest.mark.parametrize("kind", IMPLS)
def test_zero_ramp_fixed_orbit(kind):
    cn = make(kind, 32, 200.0, 20.0, 0.1, 0, 0.2, 0.0, 0.25, 0.0, 50.0, True, False, 100, 0.0, 15.0)
    cn.evolve_orbit = False
    prepare(cn)
    check_close(cn.Omega, cn.Omega_0)
    cn.step(1)
    cn.step(2)
    check_close(cn.R, 50.0)
    assert cn.phase > 0 and cn.theta < 0


# ----------------------------------------------------------------------------- flux_time_alignment.cpp

@pytest.mark.parametrize("kind", IMPLS)
@pytest.mark.parametrize("mask", [False, True])
def test_flux_time_alignment(kind, mask):
    cn = make(kind, 129, 64, 2, 0.1, 3, 0.2, 0.1, 0.2, 0, 12, False, True, 1, 0.02, 4)
    cn.evolve_orbit = False
    init = np.zeros(cn.Nr * cn.n_modes, complex)
    for m in range(cn.n_modes):
        i = np.arange(cn.Nr)
        init[m * cn.Nr + i] = np.sin(np.pi * i / (cn.Nr - 1)) / (1 + m) * np.exp(1j * (0.15 * i + 0.3 * m))
    init /= np.linalg.norm(init)
    cn.set_initial_state_full(init)
    cn.initialize()
    cn.build_cap(0.75, 0.02, 3)
    if mask:
        cn.build_damping_mask(0.3, 3, 2)
    cn.run(1, 42.5)
    rng = np.random.default_rng(2)
    x = rng.normal(size=init.size) + 1j * rng.normal(size=init.size)
    assert np.linalg.norm(cn.apply("H", x) - cn.apply("H0", x) - cn.apply("V", x) - cn.apply("CAP", x)) < 1e-12 * np.linalg.norm(x)
    k_ex = int(np.floor(42.5 / cn.dr))
    r = np.asarray(cn.r)
    for step in range(1, 5):
        cn.dt = 3.1 if step % 2 == 0 else 2.0
        d = cn.step(step)
        psi = cn.psi
        deriv = cn.schrodinger_rhs(psi)
        vpsi = cn.apply("V", psi)
        sel = (np.arange(psi.size) % cn.Nr) <= k_ex
        expected_dv = np.sum(np.conj(deriv[sel]) * vpsi[sel]).real * cn.dr
        assert abs(d["dV_bin_dt"] - expected_dv) <= 2e-11 * max(1e-10, abs(expected_dv))
        assert abs(d["t"] - cn.t[step]) <= 2e-11 * max(1e-10, abs(d["t"]))
        for m in range(cn.n_modes):
            c = m * cn.Nr + k_ex
            dU = (psi[c + 1] - psi[c - 1]) / (2 * cn.dr) - psi[c] / r[k_ex]
            want = (np.conj(deriv[c]) * dU).real / cn.mu
            assert abs(d["energy_flux"][m] - want) <= 2e-11 * max(1e-10, abs(want))
