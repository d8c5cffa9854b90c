"""GPU tests of the vy-slab contexts (vlp4d_ctx_create_slab) and of the slab
time loop (distrib.SlabRun) through the C ABI.

* One rank (the whole run as one slab with its own halos, TorchComm with no
  process group) is bit-identical to vlp4d_steps on an ordinary context,
  FP64 and FP32: the slab kernels read the halo planes where the periodic
  kernels wrap, with the same taps, weights and summation orders.
* Two to four ranks run in one process (LocalComm: halos copied between the
  ranks' buffers, rho summed in rank order) on the fused and on the generic
  kernels, even and uneven cuts, and reproduce the undivided run to FP64
  rounding (the rho sums add the ranks' moments in a different order).
* The single-stage entry points of a slab context equal the ordinary
  context's on the owned planes (bit for bit), the initial condition uses
  the global vy index, and a vy shift wider than the halo is reported as
  VLP4D_ERR_RANGE without reading outside the buffer.

Several ranks on one GPU run one after another in one process: no kernel
waits for another rank's."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _d(pkg):
    return importlib.import_module(pkg.__name__ + ".distrib")


def _reference_run(pkg, dom, dtype, steps, f0=None):
    """Initial field + `steps` steps of vlp4d_steps on an ordinary context:
    (final f as FP64, energy history, mass history)."""
    import torch

    with pkg.Context(dom, dtype) as ctx:
        fa, fb = ctx.empty_f(), ctx.empty_f()
        if f0 is None:
            ctx.init_case(fa, pkg.vlp4d.IC_LANDAU_SUM, 0.05, 0.5)
        else:
            fa.copy_(f0)
        ctx.field_rho(fa)
        ctx.field_poisson()
        ctx.diags_compute(0)
        ctx.steps(fa, fb, 1, steps)
        nrj, mass = ctx.diags_read(steps + 1)
        torch.cuda.synchronize()
        return fb.double(), nrj, mass


def _slab_runs(pkg, dom, dtype, world, halo):
    d = _d(pkg)
    runs = []
    for ivy0, nloc in d.partition_vy(dom.nxmax[3], world):
        ctx = pkg.Context(dom, dtype, slab=(ivy0, nloc, halo))
        run = d.SlabRun(ctx, dom.dt)
        ctx.init_case(run.state, pkg.vlp4d.IC_LANDAU_SUM, 0.05, 0.5)
        runs.append(run)
    return runs


def _gather(runs, steps):
    import torch

    f = torch.cat([r.ctx.owned(r.state).double() for r in runs], dim=0)
    hist = [r.ctx.diags_read(steps + 1) for r in runs]
    for r in runs:
        r.ctx.check()
    for h in hist[1:]:  # every rank solved the same field
        assert np.array_equal(h[0], hist[0][0]) and np.array_equal(h[1], hist[0][1])
    return f, hist[0][0], hist[0][1]


def _close(runs):
    for r in runs:
        r.ctx.close()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_one_rank_slab_bit_identical_to_time_loop(pkg, cuda, dtype):
    d = _d(pkg)
    steps = 6
    dom = pkg.landau_domain(32, dt=0.125, nbiter=steps)
    f_ref, nrj_ref, mass_ref = _reference_run(pkg, dom, dtype, steps)
    runs = _slab_runs(pkg, dom, dtype, 1, 4)
    try:
        comm = d.TorchComm()
        assert comm.world == 1
        d.run_distributed(runs[0], comm, steps)
        f, nrj, mass = _gather(runs, steps)
        assert bool((f == f_ref).all())
        assert np.array_equal(nrj, nrj_ref) and np.array_equal(mass, mass_ref)
    finally:
        _close(runs)


@pytest.mark.parametrize("kernels", ["fused", "generic"])
@pytest.mark.parametrize("world,halo,n", [(2, 3, (32, 32, 32, 32)), (3, 4, (32, 24, 32, 30)),
                                          (4, 3, (16, 16, 16, 32))])
def test_local_ranks_match_undivided_run_f64(pkg, cuda, monkeypatch, kernels, world, halo, n):
    monkeypatch.setenv("VLP4D_KERNELS", kernels)
    steps = 5
    dom = pkg.landau_domain(n, dt=0.125, nbiter=steps)
    f_ref, nrj_ref, mass_ref = _reference_run(pkg, dom, "f64", steps)
    runs = _slab_runs(pkg, dom, "f64", world, halo)
    try:
        _d(pkg).run_local(runs, steps)
        f, nrj, mass = _gather(runs, steps)
        assert float((f - f_ref).abs().max()) < 1e-13 * float(f_ref.abs().max())
        assert np.abs(nrj - nrj_ref).max() < 1e-11
        assert np.abs(mass - mass_ref).max() < 1e-12
    finally:
        _close(runs)


def test_local_ranks_match_undivided_run_f32(pkg, cuda):
    """FP32 f: the joined x/y/x/y pass on every slab; equal to the undivided
    FP32 time loop to FP32 rounding of the moment's summation order."""
    steps = 8
    dom = pkg.landau_domain(32, dt=0.125, nbiter=steps)
    f_ref, nrj_ref, _ = _reference_run(pkg, dom, "f32", steps)
    runs = _slab_runs(pkg, dom, "f32", 4, 3)
    try:
        _d(pkg).run_local(runs, steps)
        f, nrj, _ = _gather(runs, steps)
        assert float((f - f_ref).abs().max()) < 1e-6 * float(f_ref.abs().max())
        assert np.abs(np.exp(2 * (nrj - nrj_ref)) - 1).max() < 1e-6
    finally:
        _close(runs)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_slab_stage_entry_points_match_ordinary_context(pkg, cuda, dtype):
    """x, y, vx sweeps and the moment on the owned planes, the vy sweep from
    filled halos, the joined x/y/x/y pass and the initial condition, each
    against the ordinary context on the same planes (bit for bit; the moment
    is the owned planes' share of rho)."""
    import torch

    dom = pkg.landau_domain((32, 16, 32, 24), dt=0.25, nbiter=2)
    ivy0, nloc, halo = 8, 10, 4
    with pkg.Context(dom, dtype) as full, pkg.Context(dom, dtype, slab=(ivy0, nloc, halo)) as sl:
        f = full.empty_f()
        full.init_case(f, pkg.vlp4d.IC_LANDAU_SUM, 0.05, 0.5)
        g = sl.empty_f()
        sl.init_case(g, pkg.vlp4d.IC_LANDAU_SUM, 0.05, 0.5)
        assert torch.equal(sl.owned(g), f[ivy0:ivy0 + nloc])
        # The field of the whole state on both contexts.
        full.field_rho(f)
        full.field_poisson()
        sl.rho.copy_(full.rho)  # any field will do: the same one on both
        sl.ex.copy_(full.ex)
        sl.ey.copy_(full.ey)
        g[:halo].copy_(f[ivy0 - halo:ivy0])
        g[halo + nloc:].copy_(f[ivy0 + nloc:ivy0 + nloc + halo])
        out_f, out_g = full.empty_f(), sl.empty_f()
        for name, dt in (("advect_x", 0.3), ("advect_y", 0.3), ("advect_vx", 0.5), ("advect_vy", 0.5),
                         ("advect_xy", 0.3), ("advect_vxvy", 0.5), ("advect_xyxy", 0.3)):
            getattr(full, name)(f, out_f, dt)
            getattr(sl, name)(g, out_g, dt)
            torch.cuda.synchronize()
            assert torch.equal(sl.owned(out_g), out_f[ivy0:ivy0 + nloc]), name
        sl.check()
        full.check()


def test_halo_too_narrow_is_reported(pkg, cuda):
    """A vy shift of several cells with a three-plane halo: the fused and the
    generic slab sweeps clamp their reads to the buffer and report
    VLP4D_ERR_RANGE through vlp4d_check; the context stays usable."""
    import os

    import torch

    dom = pkg.landau_domain(32, dt=0.125, nbiter=2)
    for kernels in ("fused", "generic"):
        os.environ["VLP4D_KERNELS"] = kernels
        try:
            with pkg.Context(dom, "f64", slab=(0, 16, 3)) as sl:
                g, out = sl.empty_f(), sl.empty_f()
                g.fill_(1.0)
                sl.ey.fill_(0.0)
                sl.ex.fill_(0.0)
                sl.ey[5, 7] = 40.0  # dt * Ey / dvy = 13 cells for one column
                # The v tables are built from Ex/Ey by the vy sweep itself.
                sl.advect_vy(g, out, 0.125)
                with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
                    sl.check()
                assert e.value.code == pkg.vlp4d.ERR_RANGE and "halo" in str(e.value)
                sl.ey.fill_(0.0)
                sl.advect_vy(g, out, 0.125)
                sl.check()
                assert bool((sl.owned(out) == 1.0).all())
        finally:
            del os.environ["VLP4D_KERNELS"]
    torch.cuda.synchronize()


def test_slab_context_rejects_whole_run_entry_points(pkg, cuda):
    dom = pkg.landau_domain(16, dt=0.125, nbiter=2)
    with pkg.Context(dom, "f64", slab=(0, 8, 3)) as sl:
        a, b = sl.empty_f(), sl.empty_f()
        for call in (lambda: sl.step(a, b, 1), lambda: sl.steps(a, b, 1, 1)):
            with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
                call()
            assert e.value.code == pkg.vlp4d.ERR_UNSUPPORTED
    for bad in ((0, 8, 2), (0, 8, 9), (10, 8, 3), (-1, 4, 3)):
        with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
            pkg.Context(dom, "f64", slab=bad)
        assert e.value.code == pkg.vlp4d.ERR_INVALID_ARG
