"""ctypes binding of the CPU oracle (oracle/cnm_oracle.cpp).

Test infrastructure only: the parity tests, the smoke check and the benchmark's
CPU-baseline leg use this module as the checker.  The object mirrors the public
surface of the reference class CrankNicolsonModes
(include/CrankNicolsonModes.hpp:60-239) closely enough that ported reference
tests read like the originals: scalar members are attributes, ``psi`` is a
complex numpy vector (mode-major, entry j*Nr+i), and errors raise the same
exception types (invalid_argument -> ValueError, logic_error -> RuntimeError
subclass LogicError, runtime_error -> RuntimeError).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_cnm.so")
_lib = None

# Operators accepted by apply()/dense().
OPS = {"H": 0, "H0": 1, "V": 2, "V1": 3, "V2": 4, "dVdt": 5, "A": 6, "B": 7,
       "sink": 8, "schrodinger_rhs": 9, "A_full": 10, "CAP": 11}

_SCALARS = ("R", "R1", "R2", "M1", "M2", "q", "theta", "phase", "Omega", "Omega_0", "P",
            "dt", "dr", "L", "mu", "M_c", "epsilon", "t_i", "p_bin", "steps_per_period",
            "last_solver_residual", "tolerance", "accept_residual", "initial_period",
            "ramp_factor")
_FLAGS = ("evolve_orbit", "ramp_secondary_potential", "use_block_preconditioner")


class LogicError(RuntimeError):
    """std::logic_error raised by the oracle."""


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ with OpenMP) if needed."""
    src = os.path.join(_HERE, "cnm_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        d, i, p, dp, ip = C.c_double, C.c_int, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_create.restype = p
        L.orc_create.argtypes = [i, d, d, d, i, d, d, d, d, d, i, i, i, d, d]
        L.orc_destroy.argtypes = [p]
        L.orc_last_error.restype = C.c_char_p
        L.orc_set_threads.argtypes = [i]
        L.orc_set_threads.restype = i
        L.orc_n_modes.argtypes = [p]
        L.orc_modes.argtypes = [p, ip, ip]
        L.orc_grid.argtypes = [p, dp]
        for f in ("orc_set_initial_state_full", "orc_set_psi"):
            getattr(L, f).argtypes = [p, dp, C.c_int64]
        L.orc_get_psi.argtypes = [p, dp]
        L.orc_initialize.argtypes = [p]
        L.orc_configure_isolated_black_hole.argtypes = [p, d]
        L.orc_build_damping_mask.argtypes = [p, d, d, i]
        L.orc_build_cap.argtypes = [p, d, d, i]
        L.orc_set_power_average_orbits.argtypes = [p, d]
        L.orc_set_flag.argtypes = [p, C.c_char_p, i]
        L.orc_get_int.argtypes = [p, C.c_char_p]
        L.orc_get_scalar.argtypes = [p, C.c_char_p, dp]
        L.orc_set_scalar.argtypes = [p, C.c_char_p, d]
        L.orc_prepare_run.argtypes = [p, i, d]
        L.orc_refresh.argtypes = [p, d]
        L.orc_step.argtypes = [p, i, dp]
        L.orc_apply.argtypes = [p, i, dp, dp]
        L.orc_dense.argtypes = [p, i, dp]
        L.orc_sink_strength.argtypes = [p, i]
        L.orc_sink_strength.restype = d
        L.orc_sink_vector.argtypes = [p, i, dp]
        L.orc_coupling_terms.argtypes = [p, ip, ip, ip, dp]
        L.orc_multipoles.argtypes = [p, i, dp]
        L.orc_wigner3j.argtypes = [i] * 6
        L.orc_wigner3j.restype = d
        L.orc_sph_plm_equator.argtypes = [i, i]
        L.orc_sph_plm_equator.restype = d
        L.orc_gauss_legendre.argtypes = [i, d, d, dp, dp]
        _lib = L
    return _lib


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(rc):
    if rc == 0:
        return
    msg = lib().orc_last_error().decode()
    if rc == 1:
        raise ValueError(msg)
    if rc == 2:
        raise LogicError(msg)
    raise RuntimeError(msg)


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


def wigner3j(tj1, tj2, tj3, tm1, tm2, tm3) -> float:
    return lib().orc_wigner3j(tj1, tj2, tj3, tm1, tm2, tm3)


def sph_plm_equator(l: int, m: int) -> float:
    return lib().orc_sph_plm_equator(l, m)


def gauss_legendre(n: int, a: float = 0.0, b: float = 1.0):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauss_legendre(n, a, b, _dptr(x), _dptr(w))
    return x, w


class Diag(dict):
    """One step's diagnostic record (the values step() writes to its files)."""


class OracleCNM:
    """CPU restatement of CrankNicolsonModes with the reference's constructor."""

    def __init__(self, Nx, L, dt, epsilon, l_max, mu, M_c, q, a, R, counter, absorption,
                 save_every, ramp_periods, epsilon_smear, config_file=None):
        h = lib().orc_create(int(Nx), float(L), float(dt), float(epsilon), int(l_max), float(mu),
                             float(M_c), float(q), float(a), float(R), int(bool(counter)),
                             int(bool(absorption)), int(save_every), float(ramp_periods),
                             float(epsilon_smear))
        if not h:
            raise ValueError(lib().orc_last_error().decode())
        object.__setattr__(self, "_h", h)
        n = lib().orc_n_modes(h)
        l = np.zeros(n, np.int32)
        m = np.zeros(n, np.int32)
        lib().orc_modes(h, l.ctypes.data_as(C.POINTER(C.c_int)), m.ctypes.data_as(C.POINTER(C.c_int)))
        object.__setattr__(self, "n_modes", n)
        object.__setattr__(self, "modes", [(int(a_), int(b_)) for a_, b_ in zip(l, m)])
        object.__setattr__(self, "Nr", int(Nx))
        r = np.zeros(int(Nx))
        lib().orc_grid(h, _dptr(r))
        object.__setattr__(self, "r", r)
        object.__setattr__(self, "l_max", int(l_max))
        object.__setattr__(self, "counter", bool(counter))
        object.__setattr__(self, "t", [])

    def __del__(self):
        h = self.__dict__.get("_h")
        if h and _lib is not None:
            _lib.orc_destroy(h)
            self.__dict__["_h"] = None

    # scalar members ---------------------------------------------------------
    def __getattr__(self, name):
        if name in _SCALARS:
            out = C.c_double()
            _check(lib().orc_get_scalar(self._h, name.encode(), C.byref(out)))
            return out.value
        if name in _FLAGS or name in ("last_solver_iterations", "idx_ex", "sink_active", "n_pairs"):
            return lib().orc_get_int(self._h, name.encode())
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in _SCALARS:
            _check(lib().orc_set_scalar(self._h, name.encode(), float(value)))
        elif name in _FLAGS:
            _check(lib().orc_set_flag(self._h, name.encode(), int(bool(value))))
        elif name == "max_iterations":
            _check(lib().orc_set_flag(self._h, b"max_iterations", int(value)))
        else:
            object.__setattr__(self, name, value)

    @property
    def size(self):
        return self.Nr * self.n_modes

    @property
    def psi(self):
        out = np.zeros(2 * self.size)
        lib().orc_get_psi(self._h, _dptr(out))
        return out.view(np.complex128).copy()

    @psi.setter
    def psi(self, value):
        v = np.ascontiguousarray(np.asarray(value, np.complex128)).view(np.float64)
        _check(lib().orc_set_psi(self._h, _dptr(v), self.size))

    # reference methods ---------------------------------------------------------
    def set_initial_state_full(self, psi0):
        v = np.ascontiguousarray(np.asarray(psi0, np.complex128))
        _check(lib().orc_set_initial_state_full(self._h, _dptr(v.view(np.float64)), v.size))

    def initialize(self):
        _check(lib().orc_initialize(self._h))

    def configure_isolated_black_hole(self, x):
        _check(lib().orc_configure_isolated_black_hole(self._h, float(x)))

    def build_damping_mask(self, f, W, n):
        _check(lib().orc_build_damping_mask(self._h, float(f), float(W), int(n)))

    def build_cap(self, f, W, n):
        _check(lib().orc_build_cap(self._h, float(f), float(W), int(n)))

    def set_power_average_orbits(self, n):
        _check(lib().orc_set_power_average_orbits(self._h, float(n)))

    def run(self, n_steps, r_ex):
        """run() without the output folder: extraction radius, t = 0, operator refresh."""
        _check(lib().orc_prepare_run(self._h, int(n_steps), float(r_ex)))
        self.t = [0.0]

    def refresh(self, time):
        _check(lib().orc_refresh(self._h, float(time)))

    def step(self, step_id):
        n = self.n_modes
        out = np.zeros(12 + 4 * n)
        _check(lib().orc_step(self._h, int(step_id), _dptr(out)))
        d = Diag(R=out[0], theta=out[1], Omega=out[2], M1=out[3], q=out[4], t=out[5], energy=out[6],
                 p_bin=out[7], p_bin_inst=out[8], dV_bin_dt=out[9], residual=out[10],
                 iterations=int(out[11]), energy_flux=out[12:12 + n].copy(),
                 flux=out[12 + n:12 + 2 * n].copy(), norms=out[12 + 2 * n:12 + 3 * n].copy(),
                 energies=out[12 + 3 * n:12 + 4 * n].copy())
        while len(self.t) <= step_id:
            self.t.append(0.0)
        self.t[step_id] = d["t"]
        return d

    def should_stop(self):
        return lib().orc_get_int(self._h, b"should_stop") == 1

    def apply(self, op, x):
        x = np.ascontiguousarray(np.asarray(x, np.complex128))
        y = np.zeros(2 * self.size)
        _check(lib().orc_apply(self._h, OPS[op], _dptr(x.view(np.float64)), _dptr(y)))
        return y.view(np.complex128).copy()

    def apply_sink(self, x):
        return self.apply("sink", x)

    def schrodinger_rhs(self, x):
        return self.apply("schrodinger_rhs", x)

    def dense(self, op):
        n = self.size
        out = np.zeros(2 * n * n)
        _check(lib().orc_dense(self._h, OPS[op], _dptr(out)))
        return out.view(np.complex128).reshape(n, n)

    def sink_strength(self, body):
        return lib().orc_sink_strength(self._h, int(body))

    def absorption_sink_active(self):
        return bool(self.sink_active)

    def sink_vector(self, body):
        out = np.zeros(2 * self.size)
        lib().orc_sink_vector(self._h, int(body), _dptr(out))
        return out.view(np.complex128).copy()

    def multipoles(self, body):
        out = np.zeros((2 * self.l_max + 1) * self.Nr)
        lib().orc_multipoles(self._h, int(body), _dptr(out))
        return out.reshape(2 * self.l_max + 1, self.Nr)

    def coupling_terms(self):
        n = lib().orc_coupling_terms(self._h, None, None, None, None)
        rows = np.zeros(n, np.int32)
        cols = np.zeros(n, np.int32)
        ls = np.zeros(n, np.int32)
        ang = np.zeros(n)
        ip = C.POINTER(C.c_int)
        lib().orc_coupling_terms(self._h, rows.ctypes.data_as(ip), cols.ctypes.data_as(ip),
                                 ls.ctypes.data_as(ip), _dptr(ang))
        return rows, cols, ls, ang


def displaced_100_state(r, modes, mu, x_bh):
    """displaced_100_state (src/DisplacedAtom.cpp:12-76) on the CPU: the mode projection
    of a hydrogenic 1s state centred at x_bh on the x axis (complex, n_modes x Nr)."""
    r = np.ascontiguousarray(np.asarray(r, float))
    l = np.array([a for a, _ in modes], np.int32)
    m = np.array([b for _, b in modes], np.int32)
    out = np.zeros(2 * len(r) * len(modes))
    ip = C.POINTER(C.c_int)
    rc = lib().orc_displaced_100_state(_dptr(r), len(r), l.ctypes.data_as(ip), m.ctypes.data_as(ip), len(modes),
                                       C.c_double(mu), C.c_double(x_bh), _dptr(out))
    if rc != 0:
        raise ValueError(lib().orc_last_error().decode())
    return out.view(np.complex128)
