"""bench.py's multi-GPU plumbing on CPU: two gloo ranks stand in for two
GPUs.  Each GPU runs an independent replica (no collective on the data
path); the job's throughput is every rank's units over the slowest rank's
time, which all ranks agree on."""
import datetime
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ranks = bench.Ranks(dist, "cpu")
    ranks.barrier()
    # rank r simulated 1000 (r + 1) atoms for 10 steps in 5 + r ms
    value, ms = bench.replica_rate(1000 * (rank + 1), 10, 5.0 + rank, ranks)
    q.put((rank, value, ms))
    ranks.barrier()
    dist.destroy_process_group()


def test_replica_rate_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, ms in out:
        assert ms == pytest.approx(6.0)                       # the slower rank
        assert value == pytest.approx(3000 * 10 / 6.0e-3)     # all atoms / max time


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.Ranks()
    ranks.barrier()
    value, ms = bench.replica_rate(24000, 100, 40.0, ranks)
    assert ms == 40.0 and value == pytest.approx(24000 * 100 / 0.04)
