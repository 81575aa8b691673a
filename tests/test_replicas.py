"""The multi-GPU bench runs independent replicas (one process per GPU); its
only exchange is the timing: every rank's elapsed time, the maximum taken
over ranks, and the whole-job rate from it. Exercised here with two gloo
ranks on the CPU (the GPU run uses NCCL for the same calls)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ms = bench.reduce_max(10.0 * (rank + 1), dist)  # rank 1 is the slow one
    dist.barrier()
    out.put((rank, ms, bench.replica_value(ms, 5, world)))
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [20.0, 20.0]
    assert got[0][2] == pytest.approx(2 * 5 / 0.020)


def test_single_process_keeps_its_own_time():
    import bench
    assert bench.reduce_max(12.5) == 12.5
    assert bench.replica_value(12.5, 10, 1) == pytest.approx(800.0)
