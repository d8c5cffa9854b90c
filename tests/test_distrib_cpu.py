"""CPU tests of the multi-GPU decomposition logic (p3-miniapps_b200/distrib.py).

* partition of the vy planes and of ensemble members;
* the slab time loop with its two exchanges (rho all-reduce, halo
  send/recv) driven over real torch.distributed ranks (world size 2, gloo)
  and over LocalComm (1 to 4 ranks in one process), with the CPU oracle
  standing in for the GPU stages (tests/slab_cpu.py), checked against the
  oracle's one-domain run: the decomposition must reproduce the undivided
  time loop (f and the energy/mass history) to FP64 rounding.

The GPU stages themselves are checked in tests/test_slab_gpu.py."""
from __future__ import annotations

import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import ROOT
from oracle.oracle import IC_LANDAU_SUM, Restatement

N = (8, 6, 8, 12)
MINP = (0.0, 0.0, -6.0, -6.0)
MAXP = (4 * math.pi, 4 * math.pi, 6.0, 6.0)
DT, IDCASE, STEPS = 0.125, 10, 4


def _distrib(pkg):
    import importlib

    return importlib.import_module(pkg.__name__ + ".distrib")


@pytest.fixture(scope="module")
def reference():
    ora = Restatement(N, MINP, MAXP, DT, IDCASE)
    f0 = ora.init_case(IC_LANDAU_SUM, amp=0.05, k=0.5)
    f, nrj, mass, _, _ = ora.run(f0, STEPS)
    return f0, f, nrj, mass


def test_partition_vy(pkg):
    d = _distrib(pkg)
    for nvy in (12, 30, 128):
        for world in range(1, 9):
            if world > nvy:
                continue
            parts = d.partition_vy(nvy, world)
            assert len(parts) == world
            assert parts[0][0] == 0
            for (a, n), (b, _) in zip(parts, parts[1:]):
                assert a + n == b
            assert parts[-1][0] + parts[-1][1] == nvy
            sizes = [n for _, n in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        d.partition_vy(3, 4)


def test_halo_width_and_views(pkg):
    d = _distrib(pkg)
    assert d.halo_for_shift(0.0) == 3 and d.halo_for_shift(0.99) == 3
    assert d.halo_for_shift(1.0) == 4 and d.halo_for_shift(-2.5) == 5
    assert d.neighbours(0, 4) == (3, 1) and d.neighbours(3, 4) == (2, 0) and d.neighbours(0, 1) == (0, 0)
    f = torch.arange(10 * 2).reshape(10, 2)  # nloc 6, halo 2
    lh, rh, first, last = d.halo_views(f, 6, 2)
    assert lh[:, 0].tolist() == [0, 2] and rh[:, 0].tolist() == [16, 18]
    assert first[:, 0].tolist() == [4, 6] and last[:, 0].tolist() == [12, 14]
    assert all(v.is_contiguous() for v in (lh, rh, first, last))


def test_partition_members_balanced_and_deterministic(pkg):
    d = _distrib(pkg)
    rng = np.random.default_rng(5)
    members = [tuple(int(v) for v in rng.choice([16, 24, 32, 48], 4)) for _ in range(256)]
    for world in (1, 2, 3, 8):
        parts = d.partition_members(members, world)
        assert parts == d.partition_members(members, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(members)))
        loads = [sum(math.prod(members[i]) for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(math.prod(m) for m in members)


def _slab_runs(pkg, world, halo, f0):
    from slab_cpu import CpuSlabContext

    d = _distrib(pkg)
    runs = []
    for ivy0, nloc in d.partition_vy(N[3], world):
        ctx = CpuSlabContext(N, MINP, MAXP, DT, IDCASE, ivy0, nloc, halo)
        run = d.SlabRun(ctx, DT)
        ctx.set_owned_from_global(run.state, f0)
        runs.append(run)
    return runs


def _gather(runs):
    f = np.concatenate([r.ctx.owned(r.state).numpy() for r in runs], axis=0)
    nrj = np.array([runs[0].ctx.nrj[i] for i in range(STEPS + 1)])
    mass = np.array([runs[0].ctx.mass[i] for i in range(STEPS + 1)])
    for r in runs[1:]:  # every rank solved the same field
        assert [r.ctx.nrj[i] for i in range(STEPS + 1)] == nrj.tolist()
    return f, nrj, mass


@pytest.mark.parametrize("world,halo", [(1, 3), (2, 3), (3, 4), (4, 3)])
def test_local_ranks_match_one_domain(pkg, reference, world, halo):
    f0, f_ref, nrj_ref, mass_ref = reference
    runs = _slab_runs(pkg, world, halo, f0)
    _distrib(pkg).run_local(runs, STEPS)
    f, nrj, mass = _gather(runs)
    assert np.abs(f - f_ref).max() < 1e-13 * np.abs(f_ref).max()
    assert np.abs(nrj - nrj_ref).max() < 1e-12
    assert np.abs(mass - mass_ref).max() < 1e-12


def test_local_ranks_detect_divergence(pkg, reference):
    """Ranks whose step sequences differ are an error, not a hang."""
    d = _distrib(pkg)
    f0 = reference[0]
    runs = _slab_runs(pkg, 2, 3, f0)
    with pytest.raises(RuntimeError):
        d.LocalComm().serve(runs, [runs[0].steps(1, 2), runs[1].steps(1, 1)])


def _gloo_worker(rank, world, port, halo, out):
    import sys

    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    import __graft_entry__ as ge

    pkg = ge.load_package()
    d = _distrib(pkg)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        from slab_cpu import CpuSlabContext

        ora = Restatement(N, MINP, MAXP, DT, IDCASE)
        f0 = ora.init_case(IC_LANDAU_SUM, amp=0.05, k=0.5)
        ivy0, nloc = d.partition_vy(N[3], world)[rank]
        ctx = CpuSlabContext(N, MINP, MAXP, DT, IDCASE, ivy0, nloc, halo)
        run = d.SlabRun(ctx, DT)
        ctx.set_owned_from_global(run.state, f0)
        comm = d.TorchComm()
        assert (comm.rank, comm.world) == (rank, world)
        d.run_distributed(run, comm, STEPS)
        out[rank] = (ivy0, ctx.owned(run.state).numpy().copy(), [ctx.nrj[i] for i in range(STEPS + 1)],
                     [ctx.mass[i] for i in range(STEPS + 1)], comm.halo_bytes)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,halo", [(2, 3), (3, 4)])
def test_gloo_ranks_match_one_domain(reference, world, halo):
    f0, f_ref, nrj_ref, mass_ref = reference
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, halo, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    parts = sorted(out[r] for r in range(world))
    f = np.concatenate([p[1] for p in parts], axis=0)
    assert np.abs(f - f_ref).max() < 1e-13 * np.abs(f_ref).max()
    for p in parts:
        assert np.abs(np.array(p[2]) - nrj_ref).max() < 1e-12
        assert np.abs(np.array(p[3]) - mass_ref).max() < 1e-12
        # Two halos of `halo` planes per step, FP64.
        assert p[4] == STEPS * 2 * halo * N[0] * N[1] * N[2] * 8
