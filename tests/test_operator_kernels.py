"""The two operator kernels -- the one specialised at compile time for l_max <= 8 and
the generic plan-driven one -- apply the same operators (H, A, B, rhs, V with sinks and
CAP) to rounding, and both match the oracle's assembled sparse matrices."""
import numpy as np
import pytest

from impls import make


@pytest.mark.gpu
@pytest.mark.parametrize("l_max", [1, 3, 4, 6, 8])
def test_specialised_and_generic_operator_kernels_agree(l_max):
    args = (300, 60.0, 0.5, 0.0, l_max, 0.3, 0.01, 0.4, 0.0, 12.0, False, True, 10, 0.0, 2.0)
    cn = make("gpu", *args)
    orc = make("oracle", *args)
    for c in (cn, orc):
        c.theta = 0.37
        c.evolve_orbit = False
        n = c.Nr * c.n_modes
        rng = np.random.default_rng(l_max)
        psi = rng.normal(size=n) + 1j * rng.normal(size=n)
        c.set_initial_state_full(psi)
        c.initialize()
        c.build_cap(0.8, 1.0, 2)
        c.run(2, 50.0)
    rng = np.random.default_rng(7)
    x = rng.normal(size=cn.Nr * cn.n_modes) + 1j * rng.normal(size=cn.Nr * cn.n_modes)
    for op in ("H", "V", "A", "B", "A_full", "schrodinger_rhs", "H0", "dVdt"):
        cn.set_operator_kernel(True)
        ys = cn.apply(op, x)
        cn.set_operator_kernel(False)
        yg = cn.apply(op, x)
        yo = orc.apply(op, x)
        scale = np.linalg.norm(yo)
        assert scale > 0.0, op
        assert np.linalg.norm(ys - yg) <= 1e-13 * scale, f"{op}: kernels differ"
        assert np.linalg.norm(ys - yo) <= 1e-12 * scale, f"{op}: specialised kernel vs oracle"
    cn.set_operator_kernel(True)


@pytest.mark.gpu
@pytest.mark.parametrize("l_max", [3, 8])
def test_specialised_and_generic_diagnostics_agree(l_max):
    """One step's diagnostics (energies, fluxes, norms, p_bin, dV/dt) from the specialised
    diagnostics pass and from the generic one, on the same state and operators."""
    args = (400, 60.0, 0.5, 0.0, l_max, 0.3, 0.01, 0.4, 0.0, 12.0, False, True, 10, 0.0, 2.0)
    out = []
    for specialised in (True, False):
        cn = make("gpu", *args)
        cn.set_operator_kernel(specialised)
        cn.theta = 0.37
        cn.evolve_orbit = True
        n = cn.Nr * cn.n_modes
        rng = np.random.default_rng(l_max)
        psi = rng.normal(size=n) + 1j * rng.normal(size=n)
        psi[::cn.Nr] = 0
        psi[cn.Nr - 1::cn.Nr] = 0
        cn.set_initial_state_full(psi / np.linalg.norm(psi))
        cn.initialize()
        cn.run(3, 45.0)
        out.append([cn.step(1), cn.step(2)])
    for d_s, d_g in zip(*out):
        for key in ("energy", "p_bin_inst", "dV_bin_dt", "R", "Omega"):
            assert abs(d_s[key] - d_g[key]) <= 1e-11 * max(1.0, abs(d_g[key])), key
        for key in ("flux", "energy_flux", "norms", "energies"):
            a, b = np.asarray(d_s[key]), np.asarray(d_g[key])
            assert np.linalg.norm(a - b) <= 1e-11 * max(1e-300, np.linalg.norm(b)) + 1e-300, key


@pytest.mark.gpu
@pytest.mark.parametrize("precision,l_max", [("fp64", 12), ("mixed", 8)])
def test_autotuner_choices_keep_the_operator(precision, l_max, tmp_path):
    """The autotuner's timed search changes launch plans only: the operator (and, for a
    mixed handle, the step) computed after tuning, after re-applying the choices from its
    JSON cache, and with the creation-time plan agree to rounding."""
    from boson_cloud_binary_b200 import CrankNicolsonModes
    from boson_cloud_binary_b200 import hydrogenic_state
    args = (800, 80.0, 0.5, 0.0, l_max, 0.3, 0.01, 0.5, 0.0, 15.0, False, True, 10, 0.0, 2.0)
    cn = CrankNicolsonModes(*args, precision=precision)
    cn.set_initial_state_full(hydrogenic_state(cn.r, cn.modes, 0.3, 0.5, 15.0))
    cn.evolve_orbit = False
    cn.tolerance = 1e-12
    cn.initialize()
    cn.run(10, 60.0)
    rng = np.random.default_rng(3)
    x = rng.normal(size=cn.Nr * cn.n_modes) + 1j * rng.normal(size=cn.Nr * cn.n_modes)
    y0 = cn.apply("A", x)
    cache = str(tmp_path / "tune.json")
    t1 = cn.autotune(cache_file=cache)
    assert not t1["cached"] and 1 <= t1["apply_groups"] <= 8
    assert (t1["tc_stages"] >= 2) if precision == "mixed" else (t1["tc_stages"] == 0)
    y1 = cn.apply("A", x)
    t2 = cn.autotune(cache_file=cache)
    assert t2["cached"] and t2["apply_groups"] == t1["apply_groups"] and t2["tc_stages"] == t1["tc_stages"]
    y2 = cn.apply("A", x)
    scale = np.linalg.norm(y0)
    assert np.linalg.norm(y1 - y0) <= 1e-13 * scale and np.linalg.norm(y2 - y0) <= 1e-13 * scale
    cn.set_tuning(0, 0)
    assert np.linalg.norm(cn.apply("A", x) - y0) <= 1e-13 * scale
    cn.set_tuning(t1["apply_groups"], t1["tc_stages"])
    if precision == "mixed":
        cn.step(1)   # (rebuilds the operators: apply("A") changes after it)
        assert cn.mixed_info()[2] <= 1e-12
