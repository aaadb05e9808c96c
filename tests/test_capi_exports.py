"""CPU checks of the C-ABI library: it loads, exports every entry point that
include/cnm_gpu.h declares, and the Python binding refuses to run without a GPU
instead of falling back to the CPU."""
import ctypes
import os
import re

import pytest

import boson_cloud_binary_b200 as pkg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^[a-z_ *]+?\b(cnm_[a-z0-9_]+)\s*\(", text, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_entry_point():
    lib = ctypes.CDLL(pkg.LIB_PATH)
    names = declared_entry_points()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(pkg.EXPORTS) <= set(names)


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.CudaError):
        pkg.CrankNicolsonModes(32, 120.0, 0.2, 0.1, 3, 0.2, 0.01, 0.2, 0.0, 30.0, False, True, 10, 0.0, 10.0)
