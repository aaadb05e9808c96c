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
            with open(os.path.join(ROOT, "include", h)) as f:
                text = f.read()
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


def test_batched_sweep_list_is_its_seed0_draw():
    """bench_c4_binaries.json (the 64 binaries of the batched sweep) is the seed-0 draw of
    bench.c4_binaries, and holds the sweep's ranges."""
    import bench
    binaries = bench.c4_load()
    assert len(binaries) == 64
    for b in binaries:
        assert 0.05 <= b["q"] <= 1.0 and 20.0 <= b["R"] <= 80.0
        assert b["mu"] in (0.1, 0.15, 0.2, 0.3) and b["l_max"] in (4, 6, 8, 10)
        assert 4000 <= b["Nr"] <= 32000 and b["L"] == b["Nr"] / 10.0 and b["dt"] == 0.5
