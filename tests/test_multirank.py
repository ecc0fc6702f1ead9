"""CPU, world_size 2 over gloo: the multi-GPU path of bench.py runs replicas
(no data-path collective); its only exchange is the max over ranks of the
step time, and the whole-job rate counts every rank's units."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow replica
    m = bench.max_over_ranks(local_ms, world)
    v = bench.replica_throughput(world, 1e9, 10, m)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, m, v))


def test_replica_timing_takes_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, v in out:
        assert m == pytest.approx(150.0)
        assert v == pytest.approx(2 * 1e9 * 10 / 0.150)


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(42.0, 1) == 42.0
    assert bench.replica_throughput(1, 10.0, 5, 1000.0) == pytest.approx(50.0)
