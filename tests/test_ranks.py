"""The bench's host logic on CPU: two gloo ranks (the replicas of bench.py
--gpus 2) reduce their timings with a max and their work with a sum, the way
the NCCL run does; the reference arm's replica count follows the host's
cores and memory."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    times = [[3.0, 10.0], [5.0, 7.0]][rank]
    cells = [[100.0], [250.0]][rank]
    mx, sm = bench.over_ranks(dist, times, cells, "cpu")
    out[rank] = (mx, sm)
    dist.barrier()
    dist.destroy_process_group()


def test_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            assert out[r] == ([5.0, 10.0], [350.0])


def test_over_ranks_single_process():
    import bench
    assert bench.over_ranks(None, [1.5, 2.0], [3.0], "cpu") == ([1.5, 2.0], [3.0])


def test_reference_arm_replica_count():
    """The reference arm runs one whole-domain replica per core, bounded by
    host memory (about 6 GB per 2048 x 1024 replica) and by 16."""
    import bench
    assert bench.reference_replicas(16, 196e9, 2048, 1024) == 16
    assert bench.reference_replicas(64, 196e9, 2048, 1024) == 16
    assert bench.reference_replicas(64, 30e9, 2048, 1024) == 5
    assert bench.reference_replicas(8, None, 2048, 1024) == 8
    assert bench.reference_replicas(8, 1e9, 2048, 1024) == 1
    assert bench.reference_replicas(0, None, 256, 128) == 1
