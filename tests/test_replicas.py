"""Multi-GPU form of the path: replicas.  Every rank runs its own solve, the
job time is the slowest rank's, and the reported throughput is the units of
all ranks over that time.  Two gloo ranks on the CPU exercise the reduction
the benchmark uses (bench.replica_throughput)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    local_ms = [1000.0, 1500.0][rank]
    ms, value = bench.replica_throughput(local_ms, 3, world, dist, "cpu")
    out.put((rank, ms, value))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_throughput_takes_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value in res:
        assert ms == pytest.approx(1500.0)
        assert value == pytest.approx(2 * 3 / 1.5)


def test_single_rank_needs_no_process_group():
    import bench
    ms, value = bench.replica_throughput(500.0, 2, 1, None)
    assert ms == 500.0 and value == pytest.approx(4.0)
