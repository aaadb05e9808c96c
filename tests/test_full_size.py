"""Size-independent properties at the full sizes of the reference's benchmark
configurations (the oracle cannot assemble these operators in host memory):
Hermiticity of H, A + B = 2 (A = 1 + i dt H/2, B = 1 - i dt H/2), unitarity of a CN step
without sinks, and the solve's own acceptance residual.  Sizes: 45 modes x 20000
nodes (l_max 8), 91 modes x 40000 (l_max 12), 153 modes x 65536 (l_max 16)."""
import numpy as np
import pytest

CASES = [
    # Nr, L, l_max, mu, q, R, dt
    (20000, 2000.0, 8, 0.25, 0.5, 50.0, 0.5),
    (40000, 4000.0, 12, 0.25, 0.5, 50.0, 0.5),
    (65536, 6000.0, 16, 0.3, 1.0, 60.0, 0.25),
]


def _solver(Nr, L, l_max, mu, q, R, dt, absorption):
    from boson_cloud_binary_b200 import CrankNicolsonModes
    cn = CrankNicolsonModes(Nr, L, dt, 0.0, l_max, mu, 0.01, q, 0.0, R, False, absorption, 10**6, 0.0, 2.0)
    rng = np.random.default_rng(Nr)
    r = np.asarray(cn.r)
    prof = r * r * np.exp(-r / 40.0)
    psi = np.zeros(cn.Nr * cn.n_modes, complex)
    for j in range(cn.n_modes):
        psi[j * Nr:(j + 1) * Nr] = prof * (rng.normal() + 1j * rng.normal())
    psi[::Nr] = 0
    psi[Nr - 1::Nr] = 0
    cn.set_initial_state_full(psi / np.sqrt(np.vdot(psi, psi).real * cn.dr))
    cn.evolve_orbit = False
    cn.theta = 0.7
    cn.initialize()
    return cn


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=["n45_N20000", "n91_N40000", "n153_N65536"])
def test_full_size_operator_identities(case):
    cn = _solver(*case, absorption=False)
    n = cn.Nr * cn.n_modes
    rng = np.random.default_rng(1)
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    y = rng.normal(size=n) + 1j * rng.normal(size=n)
    for v in (x, y):
        v[::cn.Nr] = 0
        v[cn.Nr - 1::cn.Nr] = 0
    hx, hy = cn.apply("H", x), cn.apply("H", y)
    lhs, rhs = np.vdot(x, hy), np.vdot(hx, y)
    assert abs(lhs - rhs) <= 1e-12 * np.linalg.norm(x) * np.linalg.norm(hy), "H is not Hermitian"
    ax, bx = cn.apply("A", x), cn.apply("B", x)
    assert np.linalg.norm(ax + bx - 2 * x) <= 1e-14 * np.linalg.norm(ax), "A + B != 2"


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=["n45_N20000", "n91_N40000", "n153_N65536"])
def test_full_size_unitary_step(case):
    cn = _solver(*case, absorption=False)
    cn.run(4, 0.9 * case[1])
    n0 = np.vdot(cn.psi, cn.psi).real
    for k in range(1, 3):
        cn.step(k)
        assert cn.last_solver_residual <= 1e-9
    n1 = np.vdot(cn.psi, cn.psi).real
    # BiCGSTAB stops at a relative residual of 1e-10 per step
    assert abs(n1 - n0) <= 1e-9 * n0, f"norm changed by {abs(n1 - n0) / n0:.3e}"
