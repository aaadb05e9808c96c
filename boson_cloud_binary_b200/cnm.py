"""Python binding of the B200 Crank-Nicolson step (libcnm_gpu.so, include/cnm_gpu.h).

``CrankNicolsonModes`` mirrors the public surface of the reference class
(include/CrankNicolsonModes.hpp:60-239): the constructor takes the same
arguments, scalar members (R, R1, theta, Omega, dt, ...) are attributes that
read and write the device-side solver, ``psi`` is the mode-major complex128
state, and ``step``/``run``/``initialize``/``build_cap``/``build_damping_mask``/
``apply_sink``/``schrodinger_rhs``/``sink_strength`` keep their meaning.
Errors raise the Python counterparts of the reference's exceptions:
std::invalid_argument -> ValueError, std::logic_error -> LogicError,
std::runtime_error -> SolveError.

There is no CPU fallback: if the CUDA library cannot be loaded or no GPU is
present the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcnm_gpu.so")

CNM_OK, CNM_EINVAL, CNM_ELOGIC, CNM_ESOLVE, CNM_ECUDA, CNM_ENOMEM, CNM_EDEVICE = range(7)

OPS = {"H": 0, "H0": 1, "V": 2, "V1": 3, "V2": 4, "dVdt": 5, "A": 6, "B": 7, "sink": 8,
       "schrodinger_rhs": 9, "A_full": 10, "CAP": 11, "precond": 12}


class LogicError(RuntimeError):
    """std::logic_error of the reference."""


class SolveError(RuntimeError):
    """std::runtime_error of the reference (the CN solve failed)."""


class CudaError(RuntimeError):
    """CUDA failure, or the CUDA library is unavailable."""


class cnm_params(C.Structure):
    _fields_ = [("Nr", C.c_int32), ("L", C.c_double), ("dt", C.c_double), ("epsilon", C.c_double),
                ("l_max", C.c_int32), ("mu", C.c_double), ("M_c", C.c_double), ("q", C.c_double),
                ("a", C.c_double), ("R", C.c_double), ("counter", C.c_int32), ("absorption", C.c_int32),
                ("save_every", C.c_int32), ("ramp_periods", C.c_double), ("epsilon_smear", C.c_double),
                ("precision", C.c_int32)]


class cnm_scalars(C.Structure):
    _fields_ = [("t", C.c_double), ("theta", C.c_double), ("phase", C.c_double), ("Omega", C.c_double),
                ("Omega_0", C.c_double), ("P", C.c_double), ("R", C.c_double), ("R1", C.c_double),
                ("R2", C.c_double), ("M1", C.c_double), ("M2", C.c_double), ("q", C.c_double),
                ("dt", C.c_double), ("p_bin", C.c_double), ("steps_per_period", C.c_double),
                ("evolve_orbit", C.c_int32), ("ramp_secondary_potential", C.c_int32),
                ("use_block_preconditioner", C.c_int32), ("last_solver_iterations", C.c_int32),
                ("last_solver_residual", C.c_double), ("tolerance", C.c_double),
                ("max_iterations", C.c_int32), ("accept_residual", C.c_double)]


class cnm_diag(C.Structure):
    _fields_ = [("R", C.c_double), ("theta", C.c_double), ("Omega", C.c_double), ("M1", C.c_double),
                ("q", C.c_double), ("t", C.c_double), ("energy", C.c_double), ("p_bin", C.c_double),
                ("p_bin_inst", C.c_double), ("dV_bin_dt", C.c_double), ("residual", C.c_double),
                ("iterations", C.c_int32)]


# Exported entry points of include/cnm_gpu.h, checked by the CPU test suite.
EXPORTS = ("cnm_create", "cnm_destroy", "cnm_last_error", "cnm_create_error", "cnm_n_modes", "cnm_modes",
           "cnm_grid", "cnm_coupling_info", "cnm_get_scalars", "cnm_set_scalars", "cnm_set_initial_state_full", "cnm_set_state",
           "cnm_get_state", "cnm_configure_isolated_black_hole", "cnm_initialize",
           "cnm_set_power_average_orbits", "cnm_build_damping_mask", "cnm_build_cap", "cnm_prepare_run",
           "cnm_refresh", "cnm_step", "cnm_should_stop", "cnm_apply", "cnm_sink_strength", "cnm_sink_active",
           "cnm_sink_vector", "cnm_save_checkpoint", "cnm_load_checkpoint", "cnm_replay_power_average", "cnm_select_device", "cnm_set_profiling", "cnm_kernel_times", "cnm_timer_start", "cnm_timer_stop",
           "cnm_plan_info", "cnm_measure_fp64_peak", "cnm_set_operator_kernel",
           "cnm_batch_create", "cnm_batch_size", "cnm_batch_handle", "cnm_batch_step", "cnm_batch_destroy",
           "cnm_displaced_100_state", "cnm_apply_lowp", "cnm_mixed_info", "cnm_mixed_trace", "cnm_launch_count", "cnm_tc_blocks",
           "cnm_hydrogenic_state", "cnm_autotune", "cnm_set_tuning", "cnm_device_name")

def displaced_100_state(r, modes, mu, x_bh):
    """displaced_100_state (src/DisplacedAtom.cpp:12-76) on the device: the mode projection
    of a hydrogenic 1s state centred at x_bh on the x axis, complex n_modes x Nr."""
    L = load_library()
    r = np.ascontiguousarray(np.asarray(r, float))
    l = np.array([a for a, _ in modes], np.int32)
    m = np.array([b for _, b in modes], np.int32)
    out = np.zeros(2 * len(r) * len(modes))
    rc = L.cnm_displaced_100_state(_dptr(r), len(r), l.ctypes.data_as(C.POINTER(C.c_int32)),
                                   m.ctypes.data_as(C.POINTER(C.c_int32)), len(modes), float(mu), float(x_bh),
                                   _dptr(out))
    if rc != CNM_OK:
        msg = L.cnm_create_error().decode()
        raise ValueError(msg) if rc == CNM_EINVAL else CudaError(msg)
    return out.view(np.complex128)


def hydrogenic_state(r, modes, mu, q, R, n=2, l=1, m=1, M1=1.0, n_theta=None, n_phi=None):
    """cnm_hydrogenic_state: the mode projection of the hydrogenic (n, l, m) state of the
    primary (mass M1, centred at x = R1 = q R / (1 + q)) computed on the device, complex
    n_modes x Nr, normalised to sum |U|^2 dr = 1 (the reference's
    initial_states/get_initial_state_COM_fast.py state; the quadrature defaults follow
    initial_state.hydrogenic_on_primary)."""
    L = load_library()
    r = np.ascontiguousarray(np.asarray(r, float))
    lmax = max(a for a, _ in modes)
    n_theta = n_theta or max(48, 2 * (lmax + l) + 16)
    n_phi = n_phi or 2 * n_theta
    ls = np.array([a for a, _ in modes], np.int32)
    ms = np.array([b for _, b in modes], np.int32)
    out = np.zeros(2 * len(r) * len(modes))
    rc = L.cnm_hydrogenic_state(_dptr(r), len(r), ls.ctypes.data_as(C.POINTER(C.c_int32)),
                                ms.ctypes.data_as(C.POINTER(C.c_int32)), len(modes), float(mu), float(M1),
                                float(q) / (1.0 + float(q)) * float(R), int(n), int(l), int(m), int(n_theta),
                                int(n_phi), _dptr(out))
    if rc != CNM_OK:
        msg = L.cnm_create_error().decode()
        raise ValueError(msg) if rc == CNM_EINVAL else CudaError(msg)
    return out.view(np.complex128)


def gaussian_state(r, modes, sigma):
    """The reference's spherical Gaussian initial state (initial_states/get_initial_state_gaussian.py):
    U_00 = sqrt(4 pi) r exp(-r^2 / (2 sigma^2)), every other mode zero, normalised on the grid
    by the trapezoidal rule, complex n_modes x Nr."""
    r = np.asarray(r, float)
    out = np.zeros((len(modes), r.size), complex)
    j00 = [i for i, lm in enumerate(modes) if tuple(lm) == (0, 0)]
    if not j00 or not sigma > 0:
        raise ValueError("the Gaussian state needs the (0, 0) mode and sigma > 0")
    u = np.sqrt(4 * np.pi) * r * np.exp(-0.5 * (r / sigma) ** 2)
    out[j00[0]] = u / np.sqrt(np.trapezoid(np.abs(u) ** 2, x=r))
    return out.reshape(-1)


def measure_fp64_peak():
    """FP64 FMA throughput of the current device, TFLOP/s (cnm_measure_fp64_peak)."""
    L = load_library()
    v = C.c_double()
    rc = L.cnm_measure_fp64_peak(C.byref(v))
    if rc != CNM_OK:
        raise CudaError(L.cnm_create_error().decode())
    return v.value


PRECISIONS = {"fp64": 0, "mixed": 1}

KERNELS = {"apply": 0, "precond_solve": 1, "precond_factor": 2, "diagnostics": 3, "tc_apply": 4,
           "precond_solve32": 5}

_lib = None


def load_library():
    """Load libcnm_gpu.so (built by boson_cloud_binary_b200/Makefile); raise if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CudaError(f"CUDA extension not built: {LIB_PATH} is missing (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    p, i32, d = C.c_void_p, C.c_int32, C.c_double
    dp = C.POINTER(C.c_double)
    L.cnm_create.argtypes = [C.POINTER(cnm_params), C.POINTER(p)]
    L.cnm_destroy.argtypes = [p]
    L.cnm_last_error.argtypes = [p]
    L.cnm_last_error.restype = C.c_char_p
    L.cnm_create_error.restype = C.c_char_p
    L.cnm_n_modes.argtypes = [p, C.POINTER(i32)]
    L.cnm_modes.argtypes = [p, C.POINTER(i32), C.POINTER(i32)]
    L.cnm_grid.argtypes = [p, dp]
    L.cnm_coupling_info.argtypes = [p, C.POINTER(i32), C.POINTER(i32)]
    L.cnm_get_scalars.argtypes = [p, C.POINTER(cnm_scalars)]
    L.cnm_set_scalars.argtypes = [p, C.POINTER(cnm_scalars)]
    for f in ("cnm_set_initial_state_full", "cnm_set_state", "cnm_get_state"):
        getattr(L, f).argtypes = [p, dp, C.c_int64]
    L.cnm_configure_isolated_black_hole.argtypes = [p, d]
    L.cnm_initialize.argtypes = [p]
    L.cnm_set_power_average_orbits.argtypes = [p, d]
    L.cnm_build_damping_mask.argtypes = [p, d, d, i32]
    L.cnm_build_cap.argtypes = [p, d, d, i32]
    L.cnm_prepare_run.argtypes = [p, i32, d]
    L.cnm_refresh.argtypes = [p, d]
    L.cnm_step.argtypes = [p, i32, C.POINTER(cnm_diag), dp, dp, dp, dp]
    L.cnm_should_stop.argtypes = [p, C.POINTER(i32)]
    L.cnm_apply.argtypes = [p, i32, dp, dp]
    L.cnm_apply_lowp.argtypes = [p, i32, dp, dp]
    L.cnm_mixed_info.argtypes = [p, C.POINTER(i32), C.POINTER(i32), dp]
    L.cnm_mixed_trace.argtypes = [p, dp]
    L.cnm_launch_count.argtypes = [p, C.POINTER(C.c_int64)]
    L.cnm_tc_blocks.argtypes = [p, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    L.cnm_sink_strength.argtypes = [p, i32, dp]
    L.cnm_sink_active.argtypes = [p, C.POINTER(i32)]
    L.cnm_sink_vector.argtypes = [p, i32, dp]
    L.cnm_save_checkpoint.argtypes = [p, i32, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
    L.cnm_load_checkpoint.argtypes = [p, i32, C.c_void_p, C.c_int64, C.POINTER(i32)]
    L.cnm_replay_power_average.argtypes = [p, dp, dp, dp, i32]
    L.cnm_select_device.argtypes = [i32]
    L.cnm_set_profiling.argtypes = [p, i32]
    L.cnm_kernel_times.argtypes = [p, i32, dp, C.POINTER(C.c_int64)]
    L.cnm_timer_start.argtypes = [p]
    L.cnm_timer_stop.argtypes = [p, dp]
    L.cnm_plan_info.argtypes = [p, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    L.cnm_autotune.argtypes = [p, C.POINTER(i32), C.POINTER(i32)]
    L.cnm_set_tuning.argtypes = [p, i32, i32]
    L.cnm_device_name.argtypes = [C.c_char_p, i32]
    L.cnm_measure_fp64_peak.argtypes = [dp]
    L.cnm_set_operator_kernel.argtypes = [p, i32]
    L.cnm_batch_create.argtypes = [C.POINTER(cnm_params), i32, C.POINTER(C.c_void_p)]
    L.cnm_batch_size.argtypes = [p, C.POINTER(i32)]
    L.cnm_batch_handle.argtypes = [p, i32, C.POINTER(C.c_void_p)]
    L.cnm_batch_step.argtypes = [p, i32, C.c_void_p]
    L.cnm_batch_destroy.argtypes = [p]
    L.cnm_displaced_100_state.argtypes = [dp, i32, C.POINTER(i32), C.POINTER(i32), i32, C.c_double, C.c_double, dp]
    L.cnm_hydrogenic_state.argtypes = [dp, i32, C.POINTER(i32), C.POINTER(i32), i32, C.c_double, C.c_double,
                                       C.c_double, i32, i32, i32, i32, i32, dp]
    _lib = L
    return L


def select_device(device: int) -> None:
    """Make `device` current (for one-process-per-GPU runs) before creating solvers."""
    lib = load_library()
    if lib.cnm_select_device(int(device)) != CNM_OK:
        raise CudaError(lib.cnm_create_error().decode())


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


_SCALAR_FIELDS = {f for f, _ in cnm_scalars._fields_}
_BOOL_FIELDS = {"evolve_orbit", "ramp_secondary_potential", "use_block_preconditioner"}


class Diag(dict):
    """One step's diagnostics: the values step() appends to the run's text files."""


class CrankNicolsonModes:
    """B200 drop-in of the reference's CrankNicolsonModes.

    ``precision="fp64"`` (default) is the complex128 drop-in; ``precision="mixed"`` solves
    each step by defect correction with complex64 inner iterations on the tensor-core
    coupling apply and fp64 residuals, stopping at the relative residual ``tolerance``."""

    def __init__(self, Nx, L, dt, epsilon, l_max, mu, M_c, q, a, R, counter, absorption, save_every,
                 ramp_periods, epsilon_smear, config_file=None, _handle=None, precision="fp64"):
        lib = load_library()
        if _handle is None:
            prm = cnm_params(int(Nx), float(L), float(dt), float(epsilon), int(l_max), float(mu), float(M_c),
                             float(q), float(a), float(R), int(bool(counter)), int(bool(absorption)),
                             int(save_every), float(ramp_periods), float(epsilon_smear),
                             PRECISIONS[precision])
            h = C.c_void_p()
            rc = lib.cnm_create(C.byref(prm), C.byref(h))
            if rc != CNM_OK:
                msg = lib.cnm_create_error().decode()
                if rc == CNM_EINVAL:
                    raise ValueError(msg)
                raise CudaError(msg)
            self.__dict__["_owned"] = True
        else:
            h = _handle   # a binary of a Batch: the batch owns and destroys it
            self.__dict__["_owned"] = False
        self.__dict__["_h"] = h
        self.__dict__["_lib"] = lib
        self.__dict__["precision"] = precision
        n = C.c_int32()
        lib.cnm_n_modes(h, C.byref(n))
        l = np.zeros(n.value, np.int32)
        m = np.zeros(n.value, np.int32)
        lib.cnm_modes(h, l.ctypes.data_as(C.POINTER(C.c_int32)), m.ctypes.data_as(C.POINTER(C.c_int32)))
        r = np.zeros(int(Nx))
        lib.cnm_grid(h, _dptr(r))
        self.__dict__.update(n_modes=n.value, modes=[(int(x), int(y)) for x, y in zip(l, m)], Nr=int(Nx),
                             r=r, l_max=int(l_max), counter=bool(counter), L=float(L), mu=float(mu),
                             M_c=float(M_c), epsilon=float(epsilon), dr=float(L) / (int(Nx) - 1),
                             save_every=int(save_every), a=float(a), t=[], config_file=config_file)

    def __del__(self):
        h = self.__dict__.get("_h")
        if h and self.__dict__.get("_owned", True):
            self._lib.cnm_destroy(h)
        self.__dict__["_h"] = None

    def _check(self, rc):
        if rc == CNM_OK:
            return
        msg = self._lib.cnm_last_error(self._h).decode()
        if rc == CNM_EINVAL:
            raise ValueError(msg)
        if rc == CNM_ELOGIC:
            raise LogicError(msg)
        if rc == CNM_ESOLVE:
            raise SolveError(msg)
        raise CudaError(msg)

    # ---- scalar members ------------------------------------------------------------
    def _scalars(self):
        s = cnm_scalars()
        self._check(self._lib.cnm_get_scalars(self._h, C.byref(s)))
        return s

    def __getattr__(self, name):
        if name == "t_i":
            return self._scalars().t
        if name in _SCALAR_FIELDS:
            v = getattr(self._scalars(), name)
            return bool(v) if name in _BOOL_FIELDS else v
        if name == "sink_active":
            a = C.c_int32()
            self._check(self._lib.cnm_sink_active(self._h, C.byref(a)))
            return bool(a.value)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        key = "t" if name == "t_i" else name
        if key in _SCALAR_FIELDS and not (name == "t"):
            s = self._scalars()
            setattr(s, key, type(getattr(s, key))(value) if not isinstance(getattr(s, key), int)
                    else int(value))
            self._check(self._lib.cnm_set_scalars(self._h, C.byref(s)))
        else:
            self.__dict__[name] = value

    @property
    def size(self):
        return self.Nr * self.n_modes

    @property
    def psi(self):
        out = np.zeros(2 * self.size)
        self._check(self._lib.cnm_get_state(self._h, _dptr(out), self.size))
        return out.view(np.complex128).copy()

    @psi.setter
    def psi(self, value):
        v = np.ascontiguousarray(np.asarray(value, np.complex128))
        self._check(self._lib.cnm_set_state(self._h, _dptr(v.view(np.float64)), v.size))

    # ---- reference methods -------------------------------------------------------------
    def set_initial_state_full(self, psi0):
        v = np.ascontiguousarray(np.asarray(psi0, np.complex128))
        self._check(self._lib.cnm_set_initial_state_full(self._h, _dptr(v.view(np.float64)), v.size))

    def initialize(self):
        self._check(self._lib.cnm_initialize(self._h))

    def configure_isolated_black_hole(self, x):
        self._check(self._lib.cnm_configure_isolated_black_hole(self._h, float(x)))

    def set_power_average_orbits(self, n):
        self._check(self._lib.cnm_set_power_average_orbits(self._h, float(n)))

    def build_damping_mask(self, f, W, n):
        self._check(self._lib.cnm_build_damping_mask(self._h, float(f), float(W), int(n)))

    def build_cap(self, f, W, n):
        self._check(self._lib.cnm_build_cap(self._h, float(f), float(W), int(n)))

    def run(self, n_steps, r_ex):
        """The computational part of run(): extraction radius, t = 0, operator refresh.

        (The text output of a run -- diagnostic files, snapshots, checkpoints -- is written by
        the C++ drop-in class in host/.)"""
        self._check(self._lib.cnm_prepare_run(self._h, int(n_steps), float(r_ex)))
        self.__dict__["t"] = [0.0]

    def refresh(self, time):
        self._check(self._lib.cnm_refresh(self._h, float(time)))

    def step(self, step_id):
        n = self.n_modes
        d = cnm_diag()
        ef, fl, nm, en = (np.zeros(n) for _ in range(4))
        self._check(self._lib.cnm_step(self._h, int(step_id), C.byref(d), _dptr(ef), _dptr(fl), _dptr(nm),
                                       _dptr(en)))
        out = Diag({f: getattr(d, f) for f, _ in cnm_diag._fields_})
        out.update(energy_flux=ef, flux=fl, norms=nm, energies=en)
        t = self.__dict__["t"]
        while len(t) <= step_id:
            t.append(0.0)
        t[step_id] = d.t
        return out

    def coupling_info(self):
        """(number of coupled mode pairs, number of Gaunt terms) of the coupling cache."""
        a, b = C.c_int32(), C.c_int32()
        self._check(self._lib.cnm_coupling_info(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def should_stop(self):
        s = C.c_int32()
        self._check(self._lib.cnm_should_stop(self._h, C.byref(s)))
        return bool(s.value)

    def apply(self, op, x):
        x = np.ascontiguousarray(np.asarray(x, np.complex128))
        y = np.zeros(2 * self.size)
        self._check(self._lib.cnm_apply(self._h, OPS[op], _dptr(x.view(np.float64)), _dptr(y)))
        return y.view(np.complex128).copy()

    def apply_lowp(self, op, x):
        """The mixed path's complex64 tensor-core operator (op in H, V, A, A_full)."""
        x = np.ascontiguousarray(np.asarray(x, np.complex128))
        y = np.zeros(2 * self.size)
        self._check(self._lib.cnm_apply_lowp(self._h, OPS[op], _dptr(x.view(np.float64)), _dptr(y)))
        return y.view(np.complex128).copy()

    def mixed_info(self):
        """(passes, fp64 operator applications, final relative residual) of the last mixed step."""
        p, f, r = C.c_int32(), C.c_int32(), C.c_double()
        self._check(self._lib.cnm_mixed_info(self._h, C.byref(p), C.byref(f), C.byref(r)))
        return p.value, f.value, r.value

    def tc_blocks(self):
        """(padded mode count, non-zero 16-column Gaunt slices per multipole, highest multipole
        every tile runs, nodes per tile) of a mixed handle."""
        kp, lc_min, nt = C.c_int32(), C.c_int32(), C.c_int32()
        nb = np.zeros(2 * self.l_max + 1, np.int32)
        self._check(self._lib.cnm_tc_blocks(self._h, C.byref(kp), nb.ctypes.data_as(C.POINTER(C.c_int32)),
                                            C.byref(lc_min), C.byref(nt)))
        return kp.value, nb, lc_min.value, nt.value

    def launch_count(self):
        """Kernels launched by this handle so far (cnm_launch_count)."""
        v = C.c_int64()
        self._check(self._lib.cnm_launch_count(self._h, C.byref(v)))
        return v.value

    def mixed_trace(self):
        """Last residual check of the mixed solve (see cnm_mixed_trace)."""
        out = np.zeros(6)
        self._check(self._lib.cnm_mixed_trace(self._h, _dptr(out)))
        return dict(zip(("res_tc", "est", "res64", "d_cal", "d_last", "ratio"), out.tolist()))

    def apply_sink(self, x):
        return self.apply("sink", x)

    def schrodinger_rhs(self, x):
        return self.apply("schrodinger_rhs", x)

    def sink_strength(self, body):
        out = C.c_double()
        self._check(self._lib.cnm_sink_strength(self._h, int(body), C.byref(out)))
        return out.value

    def absorption_sink_active(self):
        return self.sink_active

    def sink_vector(self, body):
        out = np.zeros(2 * self.size)
        self._check(self._lib.cnm_sink_vector(self._h, int(body), _dptr(out)))
        return out.view(np.complex128).copy()

    # ---- checkpoints --------------------------------------------------------------------
    def save_checkpoint(self, step_id):
        """The bytes of checkpoint.bin for step_id (reference layout GMCKPT01)."""
        n = C.c_int64()
        self._check(self._lib.cnm_save_checkpoint(self._h, int(step_id), None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        self._check(self._lib.cnm_save_checkpoint(self._h, int(step_id), buf, n.value, C.byref(n)))
        return buf.raw[:n.value]

    def load_checkpoint(self, step_id, blob):
        """Restore from checkpoint bytes; False (state untouched) if they do not match."""
        ok = C.c_int32()
        self._check(self._lib.cnm_load_checkpoint(self._h, int(step_id), blob, len(blob), C.byref(ok)))
        return bool(ok.value)

    # ---- measurement hooks ------------------------------------------------------------
    def set_profiling(self, on=True):
        self._check(self._lib.cnm_set_profiling(self._h, int(bool(on))))

    def kernel_times(self, name):
        """(total device milliseconds, launches) of one hot kernel class since profiling began."""
        ms = C.c_double()
        n = C.c_int64()
        self._check(self._lib.cnm_kernel_times(self._h, KERNELS[name], C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def timer_start(self):
        self._check(self._lib.cnm_timer_start(self._h))

    def set_operator_kernel(self, specialised):
        """Select the operator kernel specialised for l_max <= 8 (True, default) or the
        generic plan-driven one (False)."""
        self._check(self._lib.cnm_set_operator_kernel(self._h, int(bool(specialised))))

    def autotune(self, cache_file=None):
        """Timed search of the launch plans (cnm_autotune): the operator kernel's row groups and,
        on a mixed handle, the tensor-core apply's Gaunt stages.  With `cache_file` (JSON) the
        choices are looked up by device, precision and shape and stored after a search.
        Returns {"apply_groups", "tc_stages", "cached"}."""
        import json
        key = None
        cache = {}
        if cache_file:
            dev = C.create_string_buffer(256)
            self._lib.cnm_device_name(dev, 256)
            key = f"{dev.value.decode()}|{self.precision}|l{self.l_max}|n{self.n_modes}|N{self.Nr}"
            if os.path.exists(cache_file):
                with open(cache_file) as f:
                    cache = json.load(f)
            if key in cache:
                c = cache[key]
                self._check(self._lib.cnm_set_tuning(self._h, int(c["apply_groups"]), int(c["tc_stages"])))
                return dict(c, cached=True)
        g, st = C.c_int32(), C.c_int32()
        self._check(self._lib.cnm_autotune(self._h, C.byref(g), C.byref(st)))
        out = {"apply_groups": g.value, "tc_stages": st.value}
        if key is not None:
            cache[key] = out
            with open(cache_file, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
        return dict(out, cached=False)

    def set_tuning(self, apply_groups=0, tc_stages=0):
        """Apply launch-plan choices (cnm_set_tuning; 0 = the creation-time plan)."""
        self._check(self._lib.cnm_set_tuning(self._h, int(apply_groups), int(tc_stages)))

    def plan_info(self):
        """Launch plan chosen for this device: {scan_per, scan_cluster, apply_groups,
        apply_weights_in_smem} (see cnm_plan_info)."""
        v = [C.c_int32() for _ in range(4)]
        self._check(self._lib.cnm_plan_info(self._h, *[C.byref(x) for x in v]))
        return dict(zip(("scan_per", "scan_cluster", "apply_groups", "apply_weights_in_smem"), (x.value for x in v)))

    def timer_stop(self):
        """Device milliseconds on the solver's stream since timer_start()."""
        ms = C.c_double()
        self._check(self._lib.cnm_timer_stop(self._h, C.byref(ms)))
        return ms.value


class Batch:
    """Independent binaries stepped together (cnm_batch_*): ``Batch([args0, args1, ...])``
    with the constructor arguments of CrankNicolsonModes per binary.  ``binaries[i]`` is a
    CrankNicolsonModes view of binary i for set-up and read-out; ``step(k)`` advances all
    of them by one step and returns their step diagnostics (scalars only)."""

    def __init__(self, arg_lists, precision="fp64"):
        lib = load_library()
        n = len(arg_lists)
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        prms = (cnm_params * n)()
        for i, a in enumerate(arg_lists):
            (Nx, L, dt, epsilon, l_max, mu, M_c, q, aa, R, counter, absorption, save_every,
             ramp_periods, epsilon_smear) = a[:15]
            prms[i] = cnm_params(int(Nx), float(L), float(dt), float(epsilon), int(l_max), float(mu), float(M_c),
                                 float(q), float(aa), float(R), int(bool(counter)), int(bool(absorption)),
                                 int(save_every), float(ramp_periods), float(epsilon_smear), PRECISIONS[precision])
        b = C.c_void_p()
        rc = lib.cnm_batch_create(prms, n, C.byref(b))
        if rc != CNM_OK:
            msg = lib.cnm_create_error().decode()
            raise ValueError(msg) if rc == CNM_EINVAL else CudaError(msg)
        self._lib, self._b = lib, b
        self.binaries = []
        for i, a in enumerate(arg_lists):
            h = C.c_void_p()
            lib.cnm_batch_handle(b, i, C.byref(h))
            self.binaries.append(CrankNicolsonModes(*a[:15], _handle=h, precision=precision))

    def step(self, step_id):
        n = len(self.binaries)
        diags = (cnm_diag * n)()
        rc = self._lib.cnm_batch_step(self._b, int(step_id), C.cast(diags, C.c_void_p))
        if rc != CNM_OK:
            errs = []
            for i, c in enumerate(self.binaries):
                msg = self._lib.cnm_last_error(c._h)
                if msg:
                    errs.append(f"binary {i}: {msg.decode()}")
            raise SolveError(f"batch step {step_id} failed (status {rc}): " + "; ".join(errs))
        out = []
        for i, c in enumerate(self.binaries):
            d = diags[i]
            out.append({f: getattr(d, f) for f, _ in cnm_diag._fields_})
            t = c.__dict__["t"]
            while len(t) <= step_id:
                t.append(0.0)
            t[step_id] = d.t
        return out

    def __del__(self):
        b = getattr(self, "_b", None)
        if b:
            for c in self.binaries:
                c.__dict__["_h"] = None
            self._lib.cnm_batch_destroy(b)
            self._b = None
