"""Port of the reference's tests/physics.cpp against the oracle and the GPU drop-in.

Conservation laws, known eigenstates, symmetries, orbital decay, accretion and the
outer-boundary absorbers, with the reference's tolerances.  Operator properties
are checked through applications on probe vectors, so the matrix-free GPU path
is tested the same way as the assembled oracle.
"""
import numpy as np
import pytest

from impls import IMPLS, make


class Setup:
    def __init__(self, **kw):
        self.Nr, self.L, self.dt, self.epsilon = 65, 64.0, 2.0, 0.0
        self.l_max, self.mu, self.M_c, self.q, self.R = 2, 0.2, 0.1, 0.5, 20.0
        self.counter, self.absorption, self.ramp_periods, self.smear = False, False, 0.0, 4.0
        self.__dict__.update(kw)


def build(kind, s):
    return make(kind, s.Nr, s.L, s.dt, s.epsilon, s.l_max, s.mu, s.M_c, s.q, 0.0, s.R, s.counter,
                s.absorption, 1000, s.ramp_periods, s.smear)


def mode_index(cn, l, m):
    return cn.modes.index((l, m)) if (l, m) in cn.modes else -1


def generic_state(cn):
    """Smooth, complex, mode-dependent unit-norm state vanishing at both ends (physics.cpp:41-56)."""
    psi = np.zeros(cn.Nr * cn.n_modes, complex)
    r = np.asarray(cn.r)
    i = np.arange(1, cn.Nr - 1)
    for j, (l, m) in enumerate(cn.modes):
        width, centre = 6.0 + 1.5 * l, 18.0 + 2.0 * m
        weight = (1.0 / (1.0 + l)) * np.exp(1j * (0.7 * m + 0.3 * l))
        x = (r[i] - centre) / width
        psi[j * cn.Nr + i] = weight * np.exp(-x * x) * np.sin(np.pi * i / (cn.Nr - 1)) * np.exp(1j * 0.05 * r[i])
    return psi / np.sqrt(np.vdot(psi, psi).real * cn.dr)


def mirror(cn, psi):
    """y -> -y: U'_{l,m} = (-1)^m U_{l,-m} (physics.cpp:58-69)."""
    out = np.zeros_like(psi)
    for j, (l, m) in enumerate(cn.modes):
        k = mode_index(cn, l, -m)
        assert k >= 0
        out[j * cn.Nr:(j + 1) * cn.Nr] = (1.0 if m % 2 == 0 else -1.0) * psi[k * cn.Nr:(k + 1) * cn.Nr]
    return out


def cloud_mass(cn, psi):
    return cn.mu * cn.dr * np.vdot(psi, psi).real


def close(actual, expected, tol):
    return abs(actual - expected) <= tol * max(1.0, abs(expected))


@pytest.mark.parametrize("kind", IMPLS)
def test_hamiltonian_and_sink_are_hermitian(kind):
    s = Setup(l_max=4, absorption=True)
    cn = build(kind, s)
    cn.set_initial_state_full(generic_state(cn))
    cn.initialize()
    cn.run(1, 40)
    for k in range(1, 4):
        cn.step(k)
    rng = np.random.default_rng(3)
    interior = np.ones(cn.Nr * cn.n_modes)
    for j in range(cn.n_modes):
        interior[j * cn.Nr] = interior[j * cn.Nr + cn.Nr - 1] = 0
    for op in ("H", "dVdt"):
        for _ in range(3):
            a = (rng.normal(size=interior.size) + 1j * rng.normal(size=interior.size)) * interior
            b = (rng.normal(size=interior.size) + 1j * rng.normal(size=interior.size)) * interior
            ab = np.vdot(a, cn.apply(op, b))
            ba = np.vdot(b, cn.apply(op, a))
            scale = np.linalg.norm(a) * np.linalg.norm(cn.apply(op, b)) + 1e-300
            assert abs(ab - np.conj(ba)) < 1e-12 * scale, f"{op} is not Hermitian"
    a = generic_state(cn)
    b = mirror(cn, a)
    ab = np.vdot(a, cn.apply_sink(b))
    ba = np.vdot(b, cn.apply_sink(a))
    assert abs(ab - np.conj(ba)) < 1e-12 * (1 + abs(ab)), "Sink is not Hermitian"
    assert np.vdot(a, cn.apply_sink(a)).real >= 0 and np.vdot(b, cn.apply_sink(b)).real >= 0


@pytest.mark.parametrize("kind", IMPLS)
def test_unitarity_without_absorption(kind):
    s = Setup(l_max=4, ramp_periods=0.2)
    cn = build(kind, s)
    cn.evolve_orbit = False
    cn.set_initial_state_full(generic_state(cn))
    cn.initialize()
    cn.run(1, 40)
    norm0 = np.vdot(cn.psi, cn.psi).real
    for k in range(1, 31):
        cn.step(k)
        assert close(np.vdot(cn.psi, cn.psi).real, norm0, 1e-9), f"Norm changed at step {k}"
    assert cn.last_solver_residual <= 1e-9


@pytest.mark.parametrize("kind", IMPLS)
@pytest.mark.parametrize("n,l", [(1, 0), (2, 1)])
def test_hydrogen_eigenstates(kind, n, l):
    s = Setup(Nr=513, L=80.0, mu=0.5, l_max=2, dt=0.5, M_c=0.5)
    cn = build(kind, s)
    cn.configure_isolated_black_hole(0.0)
    a0 = 1.0 / (s.mu * s.mu)
    psi = np.zeros(cn.Nr * cn.n_modes, complex)
    j = mode_index(cn, l, l)
    r = np.asarray(cn.r)
    psi[j * cn.Nr:(j + 1) * cn.Nr] = r * np.exp(-r / a0) if n == 1 else r * r * np.exp(-r / (2 * a0))
    psi /= np.sqrt(np.vdot(psi, psi).real * cn.dr)
    cn.set_initial_state_full(psi)
    cn.initialize()
    initial = cn.psi
    norm = np.vdot(initial, initial).real
    energy = np.vdot(initial, cn.apply("H", initial)).real / norm
    exact = -s.mu ** 3 / (2.0 * n * n)
    assert close(energy, exact, 2e-3 * abs(exact) / max(1.0, abs(exact))), "Hydrogenic energy"
    cn.run(1, 60)
    steps = 40
    for k in range(1, steps + 1):
        cn.step(k)
    overlap = np.vdot(initial, cn.psi) / norm
    assert abs(overlap) > 1 - 1e-4, "Hydrogenic eigenstate is not stationary"
    expected_phase = -2.0 * steps * np.arctan(energy * s.dt / 2.0)
    assert close(np.remainder(np.angle(overlap) - expected_phase + np.pi, 2 * np.pi) - np.pi, 0.0, 1e-3)
    # tests/physics.cpp:167 forms |psi|^2 - |psi_j|^2; the mass outside mode j is
    # summed directly here, since the difference of two rounded sums can be one ulp
    # of the norm even when every other mode is exactly zero
    p = np.array(cn.psi)
    p[j * cn.Nr:(j + 1) * cn.Nr] = 0.0
    leaked = np.vdot(p, p).real
    assert leaked < 1e-20 * norm, "Spherical potential coupled different (l, m) modes"


def jacobi_drift(kind, counter, per_period):
    s = Setup(l_max=4, counter=counter)
    cn = build(kind, s)
    cn.evolve_orbit = False
    cn.dt = cn.P / per_period
    cn.set_initial_state_full(generic_state(cn))
    cn.initialize()
    cn.run(1, 40)
    ms = np.repeat([m for (_, m) in cn.modes], cn.Nr)

    def expectation(jacobi):
        psi = cn.psi
        lz = np.sum(ms * np.abs(psi) ** 2)
        energy = np.vdot(psi, cn.apply("H", psi)).real
        return (energy - ((-1.0 if counter else 1.0) * cn.Omega * lz if jacobi else 0.0)) * cn.dr

    steps = 2 * per_period
    cn.step(1)
    j0, e0 = expectation(True), expectation(False)
    drift = energy_change = 0.0
    for k in range(2, steps + 1):
        cn.step(k)
        drift = max(drift, abs(expectation(True) - j0) / abs(j0))
        energy_change = max(energy_change, abs(expectation(False) - e0) / abs(e0))
    assert energy_change > 20 * drift, "Rotating potential did no work on the cloud"
    return drift


@pytest.mark.slow
@pytest.mark.parametrize("kind", IMPLS)
@pytest.mark.parametrize("counter", [False, True])
def test_jacobi_constant_on_fixed_orbit(kind, counter):
    coarse = jacobi_drift(kind, counter, 200)
    fine = jacobi_drift(kind, counter, 800)
    assert coarse < 1e-3
    assert fine < coarse / 3


@pytest.mark.parametrize("kind", IMPLS)
def test_co_counter_mirror_symmetry(kind):
    s = Setup(l_max=3, absorption=True, ramp_periods=0.3)
    co = build(kind, s)
    s.counter = True
    ctr = build(kind, s)
    for cn in (co, ctr):
        cn.evolve_orbit = False
    initial = generic_state(co)
    co.set_initial_state_full(initial)
    ctr.set_initial_state_full(mirror(ctr, initial))
    co.initialize()
    ctr.initialize()
    co.run(1, 40)
    ctr.run(1, 40)
    for k in range(1, 41):
        co.step(k)
        ctr.step(k)
    assert abs(co.theta + ctr.theta) < 1e-12
    err = np.linalg.norm(mirror(co, co.psi) - ctr.psi) / np.linalg.norm(co.psi)
    assert err < 1e-7, f"Counter-rotating run is not the mirror image ({err})"
    assert np.linalg.norm(co.psi - ctr.psi) > 1e-3 * np.linalg.norm(co.psi)


@pytest.mark.parametrize("kind", IMPLS)
def test_probability_flux_continuity(kind):
    s = Setup(l_max=4)
    cn = build(kind, s)
    cn.evolve_orbit = False
    cn.dt = cn.P / 64
    cn.set_initial_state_full(generic_state(cn))
    cn.initialize()
    r_ex = 30.0
    k = int(np.floor(r_ex / cn.dr))
    cn.run(1, r_ex)
    r = np.asarray(cn.r)

    def inner_mass(psi):
        tot = 0.0
        for j in range(cn.n_modes):
            seg = psi[j * cn.Nr:j * cn.Nr + k]
            tot += np.vdot(seg, seg).real + 0.5 * abs(psi[j * cn.Nr + k]) ** 2
        return cn.mu * cn.dr * tot

    def flux(psi):
        tot = 0.0
        for j in range(cn.n_modes):
            c = j * cn.Nr + k
            dU = (psi[c + 1] - psi[c - 1]) / (2 * cn.dr) - psi[c] / r[k]
            tot += (np.conj(psi[c]) * dU).imag
        return tot

    largest = 0.0
    for step in range(1, 41):
        prev = cn.psi
        d = cn.step(step)
        cur = cn.psi
        change = inner_mass(cur) - inner_mass(prev)
        predicted = -cn.dt * flux(0.5 * (prev + cur))
        largest = max(largest, abs(predicted))
        assert abs(change - predicted) < 1e-8 * cloud_mass(cn, prev)
        # the flux diagnostic of the step is the per-mode flux of the end state
        assert abs(np.sum(d["flux"]) - flux(cur)) < 1e-12 * max(1.0, abs(flux(cur)))
    assert largest > 1e-6 * s.M_c


@pytest.mark.parametrize("kind", IMPLS)
def test_gravitational_wave_inspiral(kind):
    s = Setup(q=1.0, R=16.0, M_c=1e-12, l_max=0)
    cn = build(kind, s)
    cn.evolve_orbit = True
    cn.steps_per_period = 200
    P0 = cn.P
    cn.dt = P0 / 200
    cn.set_initial_state_full(generic_state(cn))
    cn.initialize()
    cn.run(1, 40)
    steps = 600
    R_ref, t_ref = s.R, 0.0

    def ramp(t):
        x = min(max(t / P0, 0.0), 1.0)
        return 3 * x * x - 2 * x ** 3

    def f(t, R):
        return -ramp(t) * (64.0 / 5.0) * 2.0 / (R ** 3)

    R4_start = t_start = 0.0
    t_end = 0.0
    for step in range(1, steps + 1):
        d = cn.step(step)
        t_end = d["t"]
        sub = 20
        h = (t_end - t_ref) / sub
        for _ in range(sub):
            k1 = f(t_ref, R_ref)
            k2 = f(t_ref + h / 2, R_ref + h * k1 / 2)
            k3 = f(t_ref + h / 2, R_ref + h * k2 / 2)
            k4 = f(t_ref + h, R_ref + h * k3)
            R_ref += h * (k1 + 2 * k2 + 2 * k3 + k4) / 6
            t_ref += h
        t_ref = t_end
        assert close(cn.R, R_ref, 2e-3)
        assert close(cn.Omega, np.sqrt(2.0 / cn.R ** 3), 1e-12)
        assert close(cn.R1, cn.R / 2, 1e-12)
        assert close(cn.dt, cn.P / 200, 1e-12)
        if t_end > 1.5 * P0 and t_start == 0:
            t_start, R4_start = t_end, cn.R ** 4
    assert cn.R < s.R - 0.5
    expected_R4 = R4_start - (256.0 / 5.0) * 2.0 * (t_end - t_start)
    assert close(cn.R ** 4, expected_R4, 5e-3)


@pytest.mark.parametrize("kind", IMPLS)
def test_accretion_balances_absorbed_mass(kind):
    s = Setup(q=1.0, R=20.0, l_max=2, M_c=0.05, absorption=True)
    cn = build(kind, s)
    cn.evolve_orbit = True
    cn.steps_per_period = 16
    cn.dt = cn.P / 16
    cn.set_initial_state_full(generic_state(cn))
    cn.initialize()
    cn.run(1, 40)
    total0 = cloud_mass(cn, cn.psi) + cn.M1 + cn.M2
    cloud0 = cloud_mass(cn, cn.psi)
    for k in range(1, 41):
        cn.step(k)
        assert close(cloud_mass(cn, cn.psi) + cn.M1 + cn.M2, total0, 1e-10)
        assert close(cn.q, cn.M2 / cn.M1, 1e-14)
    assert cloud0 - cloud_mass(cn, cn.psi) > 1e-3 * cloud0
    assert cn.M1 > 1 and cn.M2 > 1


@pytest.mark.parametrize("kind", IMPLS)
def test_damping_mask_acts_outside_only(kind):
    s = Setup()
    plain, masked = build(kind, s), build(kind, s)
    for cn in (plain, masked):
        cn.evolve_orbit = False
        cn.set_initial_state_full(generic_state(cn))
        cn.initialize()
    masked.build_damping_mask(0.75, 3.0, 2)
    plain.run(1, 30)
    masked.run(1, 30)
    plain.step(1)
    masked.step(1)
    edge = int(np.floor(0.75 * s.L / plain.dr))
    r = np.asarray(plain.r)
    pp, pm = plain.psi, masked.psi
    for j in range(plain.n_modes):
        for i in range(plain.Nr):
            f = 1.0 if i < edge else np.exp(-3.0 * ((r[i] - 0.75 * s.L) / (0.25 * s.L)) ** 2)
            k = j * plain.Nr + i
            assert abs(pm[k] - f * pp[k]) < 1e-14 * (1 + abs(pp[k]))
    assert np.vdot(pm, pm).real < np.vdot(pp, pp).real


@pytest.mark.parametrize("kind", IMPLS)
def test_complex_absorbing_potential(kind):
    s = Setup(Nr=129, L=128)
    plain, absorbing = build(kind, s), build(kind, s)
    for cn in (plain, absorbing):
        cn.evolve_orbit = False
        cn.set_initial_state_full(generic_state(cn))
        cn.initialize()
    absorbing.build_cap(0.8, 0.5, 2)
    plain.run(1, 40)
    absorbing.run(1, 40)
    # H_cap - H_plain is the diagonal CAP: probe with unit vectors on a few rows
    edge = int(np.floor(0.8 * s.L / plain.dr))
    rng = np.random.default_rng(5)
    x = rng.normal(size=plain.Nr * plain.n_modes) + 1j * rng.normal(size=plain.Nr * plain.n_modes)
    diff = absorbing.apply("H", x) - plain.apply("H", x)
    capdiag = absorbing.apply("CAP", np.ones_like(x))
    assert np.allclose(diff, capdiag * x, rtol=0, atol=1e-12 * np.abs(x).max() * max(1, np.abs(capdiag).max()))
    idx = np.arange(capdiag.size) % s.Nr
    assert np.all(capdiag[idx < edge] == 0), "CAP acts inside its start radius"
    assert np.all(np.isfinite(capdiag.imag)) and np.all(capdiag.imag <= 0) and np.all(capdiag.real == 0)
    assert np.abs(capdiag).max() > 0
    for k in range(1, 21):
        prev = absorbing.psi
        absorbing.step(k)
        cur = absorbing.psi
        mid = 0.5 * (prev + cur)
        predicted = 2 * absorbing.dt * np.vdot(mid, capdiag * mid).imag
        change = np.vdot(cur, cur).real - np.vdot(prev, prev).real
        pn = np.vdot(prev, prev).real
        assert change <= 1e-12 * pn, "CAP increased the norm"
        assert abs(change - predicted) < 1e-9 * pn, "CAP norm balance violated"
