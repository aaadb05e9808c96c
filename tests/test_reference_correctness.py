"""Port of the reference's tests/parallel_correctness.cpp against the oracle and the GPU drop-in.

For five scenarios (plain / absorbing + evolving orbit / absorbing counter-rotating
with CAP and mask / orbital ramp / vanishing cloud) it checks, after one CN step:
  * the operators against the independent dense formulas (1e-12 absolute, Frobenius),
    through operator applications on probe vectors so the matrix-free GPU path is
    checked the same way as the assembled oracle;
  * the sink against the addition-theorem construction (1e-10 relative);
  * the state against a dense LU solve of the CN system (1e-8 at the reference's
    BiCGSTAB tolerance 1e-10, and 1e-12 with both sides at tolerance 1e-14);
  * the accepted residual (<= 1e-9) and thread-count invariance (1e-13).
"""
import numpy as np
import pytest

from impls import IMPLS, make, set_threads
from reference_formulas import dense_reference

NR, DT, SMEAR = 32, 0.2, 10.0


def setup(kind, scenario, tol=None):
    absorb = scenario in (1, 2)
    initial_period = 2 * np.pi / np.sqrt(1.2 / 30.0 ** 3)
    ramp_periods = 2 * DT / initial_period if scenario == 3 else 0.0
    cn = make(kind, NR, 120.0, DT, 0.1, 3, 0.2, 1e-20 if scenario == 4 else 0.01, 0.2, 0.0, 30.0,
              scenario == 2, absorb, 10, ramp_periods, SMEAR)
    if tol is not None:
        cn.tolerance = tol
    cn.evolve_orbit = absorb
    cn.theta = 0.3
    cn.Omega = cn.Omega_0
    i = np.arange(NR * cn.n_modes)
    init = np.where((i % NR == 0) | (i % NR == NR - 1), 0, (0.1 + 0.001 * i) * np.exp(1j * 0.1 * i))
    init = init / np.linalg.norm(init)
    cn.set_initial_state_full(init)
    cn.initialize()
    return cn, ramp_periods, absorb


def apply_err(cn, op, dense, rng, trials=3):
    """max over probes of ||(M_impl - M_dense) x|| / ||x|| (a lower bound of the 2-norm gap)."""
    worst = 0.0
    for _ in range(trials):
        x = rng.normal(size=dense.shape[0]) + 1j * rng.normal(size=dense.shape[0])
        worst = max(worst, np.linalg.norm(cn.apply(op, x) - dense @ x) / np.linalg.norm(x))
    return worst


def run_scenario(kind, scenario, tol=None):
    rng = np.random.default_rng(scenario)
    cn, ramp_periods, absorb = setup(kind, scenario, tol)
    first = dense_reference(cn, 0.0, ramp_periods)
    assert apply_err(cn, "H0", first["h0"], rng) < 1e-12, "Stationary Hamiltonian mismatch"
    assert apply_err(cn, "V1", first["v1"], rng) < 1e-12, "Initial potential mismatch"
    if scenario == 2:
        cn.build_cap(0.8, 0.01, 3)
        cn.build_damping_mask(0.8, 0.01, 3)
    old_theta, old_omega = cn.theta, cn.Omega
    cn.theta = cn.theta + (-1.0 if cn.counter else 1.0) * cn.Omega * DT
    if DT < ramp_periods * cn.P:
        x = DT / (ramp_periods * cn.P)
        cn.Omega = cn.Omega_0 * (3 * x * x - 2 * x ** 3)
    nxt = dense_reference(cn, DT, ramp_periods, SMEAR, absorb)
    x = DT / (ramp_periods * cn.P) if ramp_periods > 0 else 1.0
    companion = 3 * x * x - 2 * x ** 3 if x < 1 else 1.0
    h = nxt["h0"] + nxt["v1"] + companion * nxt["v2"]
    if scenario == 2:
        r = np.asarray(cn.r)
        start = int(np.floor(cn.L * 0.8 / cn.dr))
        capd = np.zeros(NR * cn.n_modes, complex)
        for j in range(cn.n_modes):
            for i in range(max(start, 0), NR):
                capd[j * NR + i] = -1j * 0.01 * ((r[i] - cn.L * 0.8) / (r[i] - cn.L * 0.2)) ** 3
        h = h + np.diag(capd)
    h_full = h - 0.5j * nxt["absorption"] if absorb else h
    ident = np.eye(h.shape[0])
    a = ident + 1j * (DT / 2) * h_full
    rhs = (ident - 1j * (DT / 2) * h_full) @ cn.psi
    expected = np.linalg.solve(a, rhs)
    if scenario == 2:
        start = int(np.floor(cn.L * 0.8 / cn.dr))
        r = np.asarray(cn.r)
        for j in range(cn.n_modes):
            for i in range(start, NR):
                expected[j * NR + i] *= np.exp(-0.01 * ((r[i] - cn.L * 0.8) / (cn.L * 0.2)) ** 3)
    cn.theta, cn.Omega = old_theta, old_omega
    cn.run(2, 60.0)
    cn.step(1)
    assert apply_err(cn, "V1", nxt["v1"], rng) < 1e-12, "V1 reference mismatch"
    assert apply_err(cn, "V2", nxt["v2"], rng) < 1e-12, "V2 reference mismatch"
    assert apply_err(cn, "dVdt", nxt["dvdt"], rng) < 1e-12, "Potential derivative mismatch"
    assert apply_err(cn, "H", h, rng) < 1e-12, "Full Hamiltonian reference mismatch"
    if absorb:
        assert np.linalg.norm(nxt["absorption"]) > 0, "Fixture's absorber is not resolved"
        probe = expected
        want = nxt["absorption"] @ probe
        assert np.linalg.norm(cn.apply_sink(probe) - want) <= 1e-10 * np.linalg.norm(want)
    err = np.linalg.norm(cn.psi - expected) / np.linalg.norm(expected)
    assert cn.last_solver_residual <= 1e-9
    return cn.psi, err


@pytest.mark.parametrize("kind", IMPLS)
@pytest.mark.parametrize("scenario", range(5))
def test_cn_step_matches_dense_solve(kind, scenario):
    psi, err = run_scenario(kind, scenario)
    assert err < 1e-8, "CN differs from independent dense solve"


@pytest.mark.parametrize("kind", IMPLS)
@pytest.mark.parametrize("scenario", range(5))
def test_cn_step_tight_tolerance(kind, scenario):
    # Both sides converged far below the reference's 1e-10 BiCGSTAB tolerance.
    psi, err = run_scenario(kind, scenario, tol=1e-14)
    assert err < 1e-12, f"tight-tolerance CN step differs from dense LU by {err:.2e}"


@pytest.mark.parametrize("scenario", range(5))
def test_thread_count_invariance(scenario):
    set_threads("oracle", 1)
    serial, _ = run_scenario("oracle", scenario)
    set_threads("oracle", 4)
    parallel, _ = run_scenario("oracle", scenario)
    set_threads("oracle", 0)
    assert np.linalg.norm(serial - parallel) / np.linalg.norm(serial) < 1e-13
