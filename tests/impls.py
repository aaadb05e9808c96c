"""Factories for the two implementations the ported reference tests run against.

``oracle``: the CPU FP64 restatement (oracle/), the checker.
``gpu``: the product, boson_cloud_binary_b200.CrankNicolsonModes, which calls the
CUDA kernels through the C-ABI library (include/cnm_gpu.h).
Both take the reference constructor's arguments
(include/CrankNicolsonModes.hpp:84) and expose its public members.
"""
import pytest

IMPLS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


def make(kind, *args, **kw):
    if kind == "oracle":
        from oracle.oracle import OracleCNM
        return OracleCNM(*args)
    from boson_cloud_binary_b200 import CrankNicolsonModes
    return CrankNicolsonModes(*args, **kw)


def set_threads(kind, n):
    if kind == "oracle":
        from oracle import oracle as O
        O.set_threads(n)
