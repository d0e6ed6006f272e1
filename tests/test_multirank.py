"""The N > 1 path of bench.py on the CPU: two `gloo` ranks.

`bench.py --gpus N` runs N independent replicas (one process per GPU, no
data-path collective); the job's figures are the slowest rank's times and
the sums of the units every rank processed (`over_ranks`).  Here two CPU
processes with the gloo backend run that reduction with different
per-rank values, and the reference arm's rank 1 returns without work.
"""
import multiprocessing as mp
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    import datetime

    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    times, counts = bench.over_ranks([10.0 + rank, 3.0 * (rank + 1)],
                                     [1000 * (rank + 1), 7 + rank], world, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, times, counts))


def test_over_ranks_takes_the_slowest_time_and_sums_the_units():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, times, counts in results:
        assert times == [11.0, 6.0]
        assert counts == [3000, 15]


def test_over_ranks_is_the_identity_at_one_rank():
    sys.path.insert(0, REPO)
    import bench
    assert bench.over_ranks([2.5], [41], 1, device="cpu") == ([2.5], [41])


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, REPO)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.run_reference(bench.parse_args(["--impl", "reference", "--gpus", "2"])) is None
