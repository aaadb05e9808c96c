"""B200-native Crank-Nicolson step of CrankNicolsonModes (rdellamonica/boson-cloud-binary).

The compute path is libcnm_gpu.so (hand-written sm_100a CUDA behind the C ABI
in include/cnm_gpu.h); this package is its Python binding.
"""
from .cnm import (Batch, CrankNicolsonModes, CudaError, LogicError, SolveError, LIB_PATH, EXPORTS,  # noqa: F401
                  load_library, select_device, measure_fp64_peak, displaced_100_state, hydrogenic_state,
                  gaussian_state)
