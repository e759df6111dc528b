"""Multi-process logic of bench.py on CPU (gloo, world size 2): every rank times its own
replica, the job time is the max over ranks and the rate counts all replicas."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    local_ms = 100.0 + 50.0 * rank
    m = bench.max_over_ranks(local_ms)
    bench.barrier()
    rate = bench.whole_job_rate(1000, 10, m / 1e3, world)
    out.put((rank, m, rate, bench.dist_env()[:2]))
    dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, rate, env in res:
        assert m == 150.0
        assert rate == pytest.approx(1000 * 10 * 2 / 0.15)
        assert env == (rank, 2)


def test_single_process_defaults():
    import bench

    assert bench.max_over_ranks(3.5) == 3.5
    # 3 N_p state fields + p' in and out + 8 grid/base-state fields, 4 bytes each
    assert bench.bytes_per_cell_stage(8) == 136
    assert bench.bytes_per_cell_stage(6) == 112
