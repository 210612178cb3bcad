"""The ensemble's split over ranks, on two gloo processes (CPU): every run
goes to exactly one rank, the particle counts are balanced, and the timing
taken is the slowest rank's (bench.max_over_ranks)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from ctca_b200 import ensemble


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cases = ensemble.ensemble_cases(512)
        mine = ensemble.split_runs(cases, world, rank)
        load = sum(ensemble.particles(cases[i]) for i in mine)
        t = bench.max_over_ranks(world, 1.0 + rank)  # this rank's "time"
        q.put((rank, mine, load, t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_split_over_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    runs = [i for _, mine, _, _ in out for i in mine]
    assert sorted(runs) == list(range(512))          # each run once
    loads = [load for _, _, load, _ in out]
    assert max(loads) - min(loads) <= max(ensemble.particles(c) for c in ensemble.ensemble_cases(512))
    assert all(t == float(world) for _, _, _, t in out)  # the slowest rank's time on every rank


def test_split_single_rank_takes_everything():
    cases = ensemble.ensemble_cases(16)
    assert ensemble.split_runs(cases, 1, 0) == list(range(16))
