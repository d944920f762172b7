"""The multi-GPU protocol of the bench (independent replicas, one process per GPU) on the host:
two ranks over gloo join the group, seed their replicas by rank, meet at the barriers, agree
on the slowest rank's time, and report the whole-job rate of weak scaling; a rank that never
joins makes the others fail within the group's timeout instead of hanging."""
from __future__ import annotations

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

from hnanosolver_b200 import replicas  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r = replicas.ranks_from_env()
    replicas.start(r, "gloo", timeout_s=30)
    replicas.barrier(r)
    slowest = replicas.max_over_ranks(r, times[rank])
    replicas.barrier(r)
    out.put((rank, r.world, replicas.seed_of(r), slowest, replicas.aggregate_rate(r, 1000, 4, slowest)))
    replicas.finish(r)


def test_two_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    times = [12.5, 20.0]  # ms of the timed region on each rank
    procs = [ctx.Process(target=_rank_main, args=(rk, 2, port, times, out)) for rk in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == 2 for g in got)
    assert [g[2] for g in got] == [0, 1]  # each replica its own seed
    assert all(g[3] == 20.0 for g in got)  # max over ranks, on every rank
    assert all(g[4] == pytest.approx(2 * 1000 * 4 / 0.020) for g in got)  # all ranks' units / slowest time


def _lonely_main(port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0", WORLD_SIZE="2", LOCAL_RANK="0")
    r = replicas.ranks_from_env()
    try:
        replicas.start(r, "gloo", timeout_s=3)
        replicas.barrier(r)
        out.put("joined")
    except Exception as e:  # the peer never joins: an error, not a hang
        out.put(type(e).__name__)


def test_missing_rank_fails_within_the_timeout():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    p = ctx.Process(target=_lonely_main, args=(_free_port(), out))
    p.start()
    msg = out.get(timeout=120)
    p.join(timeout=60)
    if p.is_alive():
        p.kill()
    assert msg != "joined"


def test_one_rank_needs_no_group():
    r = replicas.Ranks(0, 1, 0)
    replicas.start(r)  # no process group for a single replica
    replicas.barrier(r)
    assert replicas.max_over_ranks(r, 7.0) == 7.0
    assert replicas.aggregate_rate(r, 100, 2, 1000.0) == pytest.approx(200.0)
    replicas.finish(r)
