"""Multi-rank (replicas) host logic of bench.py on CPU: world_size 2 over gloo on 127.0.0.1.

The DGEMM path does not shard across GPUs ("replicas only"); what bench.py does across ranks is
take the slowest rank's time (all-reduce MAX), report whole-job throughput as world x per-rank
work / that time, and run the reference arm on rank 0 alone.
"""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    slowest = bench.reduce_max(10.0 + 5.0 * rank, dist)
    tput = bench.job_throughput(2.0e12, world, slowest)

    class Args:
        size, phi, steps, warmup = 64, 0, 1, 3

    # non-zero ranks leave the reference arm without doing work or printing
    ran = None
    if rank != 0:
        bench.run_reference(Args())
        ran = "returned"
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, slowest, tput, ran))


def test_two_rank_replicas_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank reports the slowest rank's time and the whole-job throughput of both replicas
    assert [r[1] for r in res] == [15.0, 15.0]
    assert all(abs(r[2] - 2 * 2.0e12 / 15e-3 / 1e12) < 1e-9 for r in res)
    assert res[1][3] == "returned"


def _failing_worker(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    import bench

    if rank == 1:
        out.put((rank, "failed"))
        raise SystemExit(3)  # this rank fails between steps, before the max-over-ranks reduction
    try:
        bench.reduce_max(1.0, dist)
        out.put((rank, "no error"))
    except Exception as e:  # the survivor learns of it from the collective: an error, not a hang
        out.put((rank, "error " + type(e).__name__))


def test_failed_rank_ends_the_others_collective_with_an_error():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert res[1] == "failed" and procs[1].exitcode == 3
    assert res[0].startswith("error"), res[0]
    assert procs[0].exitcode == 0


def test_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.reduce_max(3.5) == 3.5
    assert bench.job_throughput(1e12, 1, 1000.0) == 1.0
