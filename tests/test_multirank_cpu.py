"""World-size-2 gloo test of bench.py's multi-GPU plumbing on CPU: the
barrier, the max-over-ranks timing and the whole-job throughput (replicas,
weak scaling).  Each rank contributes a different elapsed time; every rank
must see the maximum and compute the same aggregate."""
from __future__ import annotations

import os

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench

    r = bench.Ranks(world, backend="gloo")
    try:
        r.barrier()
        t = 1.0 + rank  # rank 1 is the slower one
        tmax = r.max(t)
        agg = bench.aggregate(tmax, cells=1000, steps=10, world=world)
        out[rank] = (tmax, agg["value"], agg["ms_per_step"])
    finally:
        r.close()


def test_two_rank_max_over_ranks_and_aggregate():
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1]
    tmax, value, ms = out[0]
    assert tmax == pytest.approx(2.0)
    assert value == pytest.approx(1000 * 10 * 2 / 2.0 / 1e9)
    assert ms == pytest.approx(200.0)


def test_aggregate_single_rank():
    import bench

    agg = bench.aggregate(0.5, cells=128**4, steps=100, world=1)
    assert agg["value"] == pytest.approx(128**4 * 100 / 0.5 / 1e9)
    assert agg["ms_per_step"] == pytest.approx(5.0)
