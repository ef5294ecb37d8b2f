"""Multi-GPU runs of the query path are replicas (no data-path collective): each rank searches
its own batch on its own copy of the index; the job's throughput is the total queries over the
slowest rank's time. Exercised here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        ms = [2.0, 3.0][rank]  # per-rank step time of its own batch
        value = bench.replica_throughput(10_000, ms, world)
        bench.barrier(world)
        out[rank] = value
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_report_total_over_slowest():
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == out[1] == pytest.approx(2 * 10_000 / 3.0e-3)
