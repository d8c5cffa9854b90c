"""Batched ensemble (vlp4d_ensemble_*): members of uneven grids advanced in
one persistent launch, against the single-run path member by member;
replays of the captured graph; the autotuner; the batched-ensemble
configuration (256 members, N per dimension from {16, 24, 32, 48}, 50 steps)."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _single_run(pkg, torch, m, nsteps):
    """The same member through a Context (FP32 f) and vlp4d_steps."""
    v = pkg.vlp4d
    dom = m.domain(nsteps + 1)
    with pkg.Context(dom, "f32") as ctx:
        a, b = ctx.empty_f(), ctx.empty_f()
        ctx.init_case(a, v.IC_LANDAU_SUM, m.amp, m.k)
        ctx.field_rho(a)
        ctx.field_poisson()
        ctx.diags_compute(0)
        if nsteps:
            ctx.steps(a, b, 1, nsteps)
        else:
            b.copy_(a)
        nrj, _ = ctx.diags_read(nsteps + 1)
        return b.clone(), nrj


def _members(pkg, dims, nsteps_dt=0.1):
    out = []
    for i, n in enumerate(dims):
        k = 0.5 if i % 2 == 0 else 0.3
        L = 2 * math.pi / k
        out.append(pkg.EnsembleMember(list(n), [0, 0, -6, -6], [L, L, 6, 6], nsteps_dt, 0.02 + 0.01 * i, k))
    return out


# (10, 12, 16, 14): rows that are not a multiple of four floats (the scalar
# plane sweeps); (16, 15, 12, 10): an odd number of rows (one-row y items).
DIMS = [(16, 24, 32, 16), (24, 16, 16, 32), (32, 32, 24, 24), (16, 16, 16, 16), (48, 24, 16, 24),
        (24, 48, 48, 16), (8, 12, 20, 10), (40, 16, 24, 36), (10, 12, 16, 14), (16, 15, 12, 10)]


def test_members_match_single_runs(pkg, cuda):
    torch = cuda
    nsteps = 6
    members = _members(pkg, DIMS)
    with pkg.Ensemble(members, nsteps) as ens:
        ens.run()
        ens.check()
        for i, m in enumerate(members):
            f, nrj = ens.read(i)
            f_ref, nrj_ref = _single_run(pkg, torch, m, nsteps)
            scale = float(f_ref.abs().max())
            assert float((f - f_ref).abs().max()) <= 2e-6 * scale, i
            assert np.abs(nrj - nrj_ref).max() < 1e-6, (i, nrj, nrj_ref)


def test_graph_replays_are_bit_identical(pkg, cuda):
    torch = cuda
    members = _members(pkg, DIMS[:5])
    with pkg.Ensemble(members, 4) as ens:
        ens.run()
        ens.check()
        first = [ens.read(i) for i in range(len(members))]
        ens.set_tiles(128, 16, 1)  # another schedule: a different tile order
        ens.run()
        ens.run()
        ens.check()
        for i in range(len(members)):
            f, nrj = ens.read(i)
            assert torch.equal(f, first[i][0])
            assert np.array_equal(nrj, first[i][1])


def test_autotuner_writes_csv_and_keeps_best(pkg, cuda, tmp_path):
    members = _members(pkg, DIMS)
    csv = tmp_path / "tiles.csv"
    with pkg.Ensemble(members, 3) as ens:
        best = ens.autotune(2, str(csv))
        rows = [line.split(",") for line in csv.read_text().splitlines()[1:]]
        assert len(rows) >= 12
        times = {(int(r[0]), int(r[1]), int(r[2])): float(r[4]) for r in rows}
        assert best in times and times[best] == min(times.values())
        ens.run()
        ens.check()


def test_batched_ensemble_configuration(pkg, cuda):
    """256 members, N per dimension from {16, 24, 32, 48}, amp ~ U[0.01, 0.1],
    k in {0.3, 0.5}, 50 steps of dt 0.1, FP32 f, one persistent launch."""
    torch = cuda
    nsteps = 50
    members = pkg.landau_ensemble_members(256)
    with pkg.Ensemble(members, nsteps) as ens:
        ens.run()
        ens.check()
        rng = np.random.default_rng(3)
        for i in rng.choice(len(members), 3, replace=False):
            f, nrj = ens.read(int(i))
            assert bool(torch.isfinite(f).all())
            f_ref, nrj_ref = _single_run(pkg, torch, members[int(i)], nsteps)
            assert float((f - f_ref).abs().max()) <= 1e-5 * float(f_ref.abs().max())
            assert np.abs(nrj - nrj_ref).max() < 1e-5


def test_idle_limit_runs_out_then_ensemble_recovers(pkg, cuda):
    """The persistent kernel's wait for work, made to run out: with a limit
    of one cycle, every CTA that finds no free tile on its first look flags
    the timeout and leaves (there is always such a CTA: at the end, while
    the last member finishes).  The CTAs that kept finding work complete the
    run, vlp4d_ensemble_check reports VLP4D_ERR_TIMEOUT, and a run with the
    default limit then gives results bit-identical to a fresh ensemble's."""
    torch = cuda
    members = _members(pkg, DIMS[:4])
    nsteps = 3
    with pkg.Ensemble(members, nsteps) as ens:
        ens.set_idle_limit(1)
        ens.run()
        with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
            ens.check()
        assert e.value.code == pkg.vlp4d.ERR_TIMEOUT
        ens.set_idle_limit(0)
        ens.run()
        ens.check()
        after = [ens.read(i) for i in range(len(members))]
    with pkg.Ensemble(members, nsteps) as fresh:
        fresh.run()
        fresh.check()
        for i in range(len(members)):
            f, nrj = fresh.read(i)
            assert torch.equal(f, after[i][0])
            assert np.array_equal(nrj, after[i][1])
    with pkg.Ensemble(members, nsteps) as ens:
        for bad in (-1, 4_000_000_001):
            with pytest.raises(pkg.vlp4d.Vlp4dError):
                ens.set_idle_limit(bad)


def test_rows_per_tile_do_not_change_results(pkg, cuda):
    """The x/y stages batch the vy rows of small members into tiles of about
    VLP4D_ENS_TILE_CELLS cells; one row per tile and the default give the
    same f and energy history bit for bit (each row's moment is summed in
    ivx order whatever the tile)."""
    import os

    torch = cuda
    members = _members(pkg, DIMS)
    res = []
    for cells in ("1", ""):
        if cells:
            os.environ["VLP4D_ENS_TILE_CELLS"] = cells
        try:
            with pkg.Ensemble(members, 4) as ens:
                ens.run()
                ens.check()
                res.append([ens.read(i) for i in range(len(members))])
        finally:
            os.environ.pop("VLP4D_ENS_TILE_CELLS", None)
    for (f1, n1), (f2, n2) in zip(*res):
        assert torch.equal(f1, f2)
        assert np.array_equal(n1, n2)
