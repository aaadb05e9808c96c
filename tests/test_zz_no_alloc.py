"""cnm_radial_solve_noalloc against the handle's own preconditioner solve.

The no-allocation entry point exists for callers that cannot call cudaMalloc
(a host code that owns a fixed, pre-reserved device arena, a driver launching
from a region where allocation is forbidden, a plug-in handed device pointers
only).  They pass device buffers for the diagonal, the right-hand side and the
result; the pivots live in the library's fixed device array.  This test builds a
small binary through the ordinary handle API, reads the diagonal and the
off-diagonal of its sparse CN operator A back through cnm_apply, and checks
that two consecutive no-allocation solves reproduce cnm_apply(CNM_OP_PRECOND)
on two different right-hand sides.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, as the other FP64 parity tests at tight tolerance


def _solver():
    from boson_cloud_binary_b200 import CrankNicolsonModes
    cn = CrankNicolsonModes(96, 120.0, 0.2, 0.1, 3, 0.2, 0.01, 0.2, 0.0, 30.0, False, True, 10, 0.0, 10.0)
    cn.theta = 0.3
    cn.Omega = cn.Omega_0
    i = np.arange(96 * cn.n_modes)
    init = np.where((i % 96 == 0) | (i % 96 == 95), 0, (0.1 + 0.001 * i) * np.exp(1j * 0.1 * i))
    cn.set_initial_state_full(init / np.linalg.norm(init))
    cn.initialize()
    cn.build_cap(0.8, 0.01, 3)
    cn.run(2, 60.0)
    return cn


def _diag_and_off(cn):
    """Diagonal of A from comb probes (every third node of one mode), off-diagonal from one probe."""
    Nr, n = cn.Nr, cn.n_modes
    diag = np.zeros(Nr * n, complex)
    for j in range(n):
        for p in range(3):
            e = np.zeros(Nr * n, complex)
            e[j * Nr + np.arange(p, Nr, 3)] = 1.0
            y = cn.apply("A", e)
            idx = j * Nr + np.arange(p, Nr, 3)
            diag[idx] = y[idx]
    e = np.zeros(Nr * n, complex)
    e[5] = 1.0
    off = cn.apply("A", e)[6]
    return diag, off


def test_noalloc_radial_solve_matches_handle_preconditioner():
    import torch
    from boson_cloud_binary_b200.cnm import CNM_EINVAL, CNM_OK, load_library

    lib = load_library()
    fn = lib.cnm_radial_solve_noalloc
    fn.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                   C.c_void_p]
    fn.restype = C.c_int
    cn = _solver()
    Nr, n = cn.Nr, cn.n_modes
    diag, off = _diag_and_off(cn)
    dev = torch.device("cuda:0")
    d_diag = torch.from_numpy(diag.view(np.float64).copy()).to(dev)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(17)
    for call in range(2):   # two calls in a row share (and reuse) the library's scratch
        b = rng.normal(size=Nr * n) + 1j * rng.normal(size=Nr * n)
        want = cn.apply("precond", b)
        d_b = torch.from_numpy(b.view(np.float64).copy()).to(dev)
        d_x = torch.full_like(d_b, float("nan"))
        torch.cuda.synchronize(dev)
        rc = fn(d_diag.data_ptr(), off.real, off.imag, Nr, n, d_b.data_ptr(), d_x.data_ptr(), stream.cuda_stream)
        assert rc == CNM_OK, f"call {call}: status {rc}"
        got = d_x.cpu().numpy().view(np.complex128)
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < TOL, f"call {call}: no-allocation solve differs from the handle's by {err:.2e}"
    # a problem larger than the fixed scratch is refused before any GPU work
    big_nr = (1 << 20) // n + 1
    rc = fn(d_diag.data_ptr(), off.real, off.imag, big_nr, n, d_b.data_ptr(), d_x.data_ptr(), stream.cuda_stream)
    assert rc == CNM_EINVAL


def _thomas_reference(diag, off, b, Nr, n):
    """Host solve of the same per-mode tridiagonal systems (scipy banded LU)."""
    from scipy.linalg import solve_banded
    x = np.zeros(Nr * n, complex)
    for j in range(n):
        d = diag[j * Nr:(j + 1) * Nr]
        ab = np.zeros((3, Nr), complex)
        ab[1] = d
        up = np.full(Nr - 1, off, complex)
        lo = np.full(Nr - 1, off, complex)
        up[0] = 0.0      # row 0 has no upper neighbour term
        lo[-1] = 0.0     # row Nr-1 has no lower neighbour term
        ab[0, 1:] = up
        ab[2, :-1] = lo
        x[j * Nr:(j + 1) * Nr] = solve_banded((1, 1), ab, b[j * Nr:(j + 1) * Nr])
    return x


def test_noalloc_multichunk_solve_and_dominance_check():
    """Nr = 7000 spans four 2048-node chunks, so the warm-up windows between chunks are
    exercised: a CN-like block (diag 1 + i (2 kappa + V), off -i kappa) matches a host banded
    solve to 1e-12 on two calls in a row; a block that is not diagonally dominant enough for
    the windows is refused with CNM_EDEVICE, not solved inexactly."""
    import torch
    from boson_cloud_binary_b200.cnm import CNM_EDEVICE, CNM_OK, load_library

    lib = load_library()
    fn = lib.cnm_radial_solve_noalloc
    fn.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                   C.c_void_p]
    fn.restype = C.c_int
    Nr, n, kappa = 7000, 2, 50.0
    rng = np.random.default_rng(3)
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    off = -1j * kappa
    i = np.arange(Nr)
    good = np.concatenate([1.0 + 1j * (2 * kappa + 0.3 * np.sin(0.01 * i + j)) for j in range(n)])
    good[[0, Nr - 1, Nr, 2 * Nr - 1]] = 1.0
    d_diag = torch.from_numpy(good.view(np.float64).copy()).to(dev)
    for call in range(2):
        b = rng.normal(size=Nr * n) + 1j * rng.normal(size=Nr * n)
        want = _thomas_reference(good, off, b, Nr, n)
        d_b = torch.from_numpy(b.view(np.float64).copy()).to(dev)
        d_x = torch.full_like(d_b, float("nan"))
        torch.cuda.synchronize(dev)
        rc = fn(d_diag.data_ptr(), off.real, off.imag, Nr, n, d_b.data_ptr(), d_x.data_ptr(), stream.cuda_stream)
        assert rc == CNM_OK, f"call {call}: status {rc}"
        got = d_x.cpu().numpy().view(np.complex128)
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < TOL, f"call {call}: multi-chunk solve differs from the banded solve by {err:.2e}"
    # |diag| only slightly above 2 |off|: the sweeps contract too slowly for the windows
    weak = np.concatenate([1e-3 + 1j * (2.0005 * kappa) * np.ones(Nr) for _ in range(n)])
    d_weak = torch.from_numpy(weak.view(np.float64).copy()).to(dev)
    torch.cuda.synchronize(dev)
    rc = fn(d_weak.data_ptr(), off.real, off.imag, Nr, n, d_b.data_ptr(), d_x.data_ptr(), stream.cuda_stream)
    assert rc == CNM_EDEVICE
