"""The multi-GPU path of bench.py is replicas only: every rank advances its own binary, the
timed region is bracketed by barriers, the time is the maximum over the ranks and the
throughput counts every rank's units.  These checks run that aggregation with world size 2
on the gloo backend (CPU processes, no GPU): one rank slower than the other, the slowest
rank's time wins, and the job's units are the sum."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    ms_local = 10.0 * (rank + 1)          # rank 1 is the slow one
    dist.barrier()
    ms = bench.reduce_max(ms_local, dist, "cpu")
    units, value = bench.whole_job(1000, ms, ws)
    out[rank] = (ms, units, value)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_two_ranks():
    import torch.multiprocessing as mp
    ws = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(ws, port, out), nprocs=ws, start_method="spawn", join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for rank in (0, 1):
        ms, units, value = res[rank]
        assert ms == 20.0                 # the slower rank's time on every rank
        assert units == 2000              # both replicas' units
        assert value == pytest.approx(2000 / 0.020)


def test_single_process_aggregation_is_identity():
    import bench
    assert bench.reduce_max(3.5, None, "cpu") == 3.5
    assert bench.whole_job(500, 5.0, 1) == (500, 500 / 0.005)
