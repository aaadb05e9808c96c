"""Batched sweep (cnm_batch_*): independent binaries of different sizes, stepped
together with their device work interleaved, reproduce the same binaries stepped one
by one -- bit for bit, since every reduction has a fixed order."""
import numpy as np
import pytest

CASES = [
    # Nx, L, dt, eps, l_max, mu, M_c, q, a, R, counter, absorption, save_every, ramp, smear
    (300, 60.0, 0.5, 0.0, 2, 0.3, 0.01, 0.5, 0.0, 12.0, False, True, 100, 0.0, 2.0),
    (500, 80.0, 0.5, 0.0, 4, 0.2, 0.01, 0.2, 0.0, 20.0, True, True, 100, 0.0, 2.0),
    (420, 50.0, 0.25, 0.0, 3, 0.25, 0.01, 1.0, 0.0, 15.0, False, False, 100, 0.0, 2.0),
]


def _setup(cn, seed):
    rng = np.random.default_rng(seed)
    n = cn.Nr * cn.n_modes
    psi = rng.normal(size=n) + 1j * rng.normal(size=n)
    psi[::cn.Nr] = 0
    psi[cn.Nr - 1::cn.Nr] = 0
    cn.set_initial_state_full(psi / np.linalg.norm(psi))
    cn.evolve_orbit = True
    cn.theta = 0.2 * seed
    cn.initialize()
    cn.run(5, 0.7 * cn.L)


@pytest.mark.gpu
def test_batch_matches_single_binaries():
    from boson_cloud_binary_b200 import Batch, CrankNicolsonModes
    batch = Batch(CASES)
    singles = [CrankNicolsonModes(*c) for c in CASES]
    for i, (cb, cs) in enumerate(zip(batch.binaries, singles)):
        _setup(cb, i + 1)
        _setup(cs, i + 1)
    for k in range(1, 5):
        diags = batch.step(k)
        for i, cs in enumerate(singles):
            d = cs.step(k)
            for key in ("t", "R", "energy", "p_bin_inst", "residual", "iterations"):
                assert diags[i][key] == d[key], (i, k, key)
    for cb, cs in zip(batch.binaries, singles):
        assert np.array_equal(cb.psi, cs.psi)


MIXED_CASES = [
    (600, 60.0, 0.5, 0.0, 4, 0.3, 0.01, 0.5, 0.0, 12.0, False, True, 100, 0.0, 2.0),
    (900, 90.0, 0.5, 0.0, 6, 0.25, 0.01, 0.3, 0.0, 20.0, False, True, 100, 0.0, 2.0),
    (700, 70.0, 0.5, 0.0, 8, 0.3, 0.01, 1.0, 0.0, 15.0, True, True, 100, 0.0, 2.0),
]


def _setup_smooth(cn, c):
    from boson_cloud_binary_b200 import hydrogenic_state
    cn.set_initial_state_full(hydrogenic_state(cn.r, cn.modes, c[5], c[7], c[9]))
    cn.evolve_orbit = True
    cn.steps_per_period = cn.P / c[2]
    cn.tolerance = 1e-12
    cn.initialize()
    cn.run(10 ** 9, 0.7 * cn.L)


@pytest.mark.gpu
def test_mixed_batch_matches_single_binaries():
    """The same for mixed-precision binaries: the tensor-core apply draws its tiles from a
    counter, so which CTA runs a tile changes from launch to launch, but its reductions are
    summed per tile in a fixed order and the results stay bit for bit reproducible."""
    from boson_cloud_binary_b200 import Batch, CrankNicolsonModes
    batch = Batch(MIXED_CASES, precision="mixed")
    singles = [CrankNicolsonModes(*c, precision="mixed") for c in MIXED_CASES]
    for c, cb, cs in zip(MIXED_CASES, batch.binaries, singles):
        _setup_smooth(cb, c)
        _setup_smooth(cs, c)
    for k in range(1, 5):
        diags = batch.step(k)
        for i, cs in enumerate(singles):
            d = cs.step(k)
            assert cs.mixed_info()[0] >= 1
            for key in ("t", "R", "energy", "p_bin_inst", "residual", "iterations"):
                assert diags[i][key] == d[key], (i, k, key)
    for cb, cs in zip(batch.binaries, singles):
        assert np.array_equal(cb.psi, cs.psi)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_handles_of_different_degrees_coexist(precision):
    """Kernel attributes (dynamic shared memory limits) are process-wide: a handle created
    after another one of a different l_max must not leave the first one unable to launch.
    l_max 10 uses the generic operator and diagnostics kernels, l_max 4 the specialised ones."""
    from boson_cloud_binary_b200 import CrankNicolsonModes
    big = (600, 60.0, 0.5, 0.0, 10, 0.3, 0.01, 0.5, 0.0, 12.0, False, True, 100, 0.0, 2.0)
    small = (600, 60.0, 0.5, 0.0, 4, 0.3, 0.01, 0.5, 0.0, 12.0, False, True, 100, 0.0, 2.0)
    a = CrankNicolsonModes(*big, precision=precision)
    _setup_smooth(a, big)
    b = CrankNicolsonModes(*small, precision=precision)
    _setup_smooth(b, small)
    for k in range(1, 3):
        a.step(k)
        b.step(k)
    assert np.isfinite(np.abs(a.psi)).all() and np.isfinite(np.abs(b.psi)).all()
