"""bench.py's N > 1 host logic on CPU: world_size-2 gloo ranks (127.0.0.1)
combine their timings as the driver expects (max device time over ranks, sum
of voxel updates)."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms, upd = bench.job_totals(100.0 + 50.0 * rank, 1000 * (rank + 1), world, "cpu")
    q.put((rank, ms, upd))
    dist.barrier()
    dist.destroy_process_group()


def test_job_totals_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 150.0, 3000.0), (1, 150.0, 3000.0)]


def test_job_totals_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_totals(12.5, 7, 1, "cpu") == (12.5, 7.0)


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
