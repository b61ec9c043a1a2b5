"""bench.py's N-GPU path runs independent replicas (the engine does not
shard spins across GPUs): every rank times its own copy of the workload and
the job's time is the slowest rank's.  Checked here with two gloo ranks on
the CPU: both ranks see the maximum, and the whole-job throughput counts
the units of both."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, results):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms_local = 10.0 + 5.0 * rank  # rank 1 is the slow one
        value, ms_max = bench.replica_throughput(ms_local, 1e12, ws, device="cpu")
        dist.barrier()
        results[rank] = (value, ms_max)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    results = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    assert results[0] == results[1]
    value, ms_max = results[0]
    assert ms_max == 15.0
    assert value == pytest.approx(2 * 1e12 / 0.015)


def test_single_rank_needs_no_process_group():
    import bench
    value, ms_max = bench.replica_throughput(20.0, 1e12, 1, device="cpu")
    assert ms_max == 20.0 and value == pytest.approx(5e13)
