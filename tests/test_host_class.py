"""The C++ drop-in class over the C ABI (boson_cloud_binary_b200/host), driven by
tests/host_check.cpp through the scenarios of the reference's tests/restart.cpp: resume
from the checkpoint (the folder byte-identical to an uninterrupted run, also after a
crash mid-write), resume from the diagnostics alone and from an earlier snapshot
(diagnostics within 2e-4), refusal of a foreign or empty folder; plus the MODESBIN
reader."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK = os.path.join(ROOT, "boson_cloud_binary_b200", "cnm_host_check")


def test_host_check_binary_built():
    assert os.path.exists(CHECK), "build the package (make -C boson_cloud_binary_b200) first"


def test_output_queue_order_bound_and_drain():
    """The background writer of the C++ class (host/cnm_output_queue.hpp), on the CPU:
    posting order kept, drain complete, at most two snapshot jobs in flight, failures
    reported without stopping the queue."""
    check = os.path.join(ROOT, "boson_cloud_binary_b200", "cnm_output_queue_check")
    assert os.path.exists(check), "build the package (make -C boson_cloud_binary_b200) first"
    res = subprocess.run([check], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "output_queue_check: OK" in res.stdout


@pytest.mark.gpu
def test_host_class_run_and_resume(tmp_path):
    res = subprocess.run([CHECK, str(tmp_path)], capture_output=True, text=True, timeout=600)
    print(res.stdout)
    print(res.stderr)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "host_check: OK" in res.stdout
