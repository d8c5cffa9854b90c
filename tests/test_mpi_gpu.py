"""GPU parity of the vlp4d_mpi entry points (one process, FP64) against the
restated reference (oracle/vlp4d_mpi_oracle.c, itself bit-identical to the
reference's own OpenMP vlp4d_mpi build) and the fixtures made from it.

Tolerances.  The reference-facing entry points (halo fill, both spline
prefilters, advect_2D_xy, advect_4D) round every product and sum separately
in the reference's order, so they are compared bit for bit.  The field solve
uses cuFFT (1e-12 relative to max|E|).  vlp4d_mpi_step fuses the sequence
and uses FMA and its own summation orders; a step then differs from the
reference at the level of FP64 rounding amplified by the interpolation
(checked at 1e-12 of max|f| per step for a few steps).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle.oracle import IC_SLD10, IC_TSI20_MPI, MpiRestatement, interior

pytestmark = pytest.mark.gpu

FOUR_PI = 4 * np.pi
CASES = [
    ((16, 12, 10, 14), (0, 0, -9, -9), (FOUR_PI, FOUR_PI, 9, 9), 0.05, 10, IC_SLD10),
    ((12, 16, 20, 10), (0, 0, -8, -8), (10 * np.pi, 10 * np.pi, 8, 8), 0.1, 20, IC_TSI20_MPI),
    ((10, 12, 10, 11), (0, 0, -6, -6), (FOUR_PI, FOUR_PI, 6, 6), 0.1, 10, IC_SLD10),
]
IDS = ["sld10", "tsi20", "small"]


def _dom(pkg, n, minp, maxp, dt, idcase, nbiter):
    return pkg.Domain(list(n), list(map(float, minp)), list(map(float, maxp)), float(dt), nbiter, idcase)


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=torch.float64)


def _host(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_entry_points_bit_identical(pkg, cuda, case):
    torch = cuda
    n, minp, maxp, dt, idcase, ic = case
    rest = MpiRestatement(n, minp, maxp, dt, idcase)
    f0 = rest.init_halo(ic)
    with pkg.Context(_dom(pkg, n, minp, maxp, dt, idcase, 4), "f64") as ctx:
        f = _dev(torch, f0)
        ctx.mpi_halo_fill(f)
        h = rest.halo_fill(f0)
        assert np.array_equal(_host(f), h)
        ctx.mpi_spline_xy(f)
        cxy = rest.spline_xy(h)
        assert np.array_equal(_host(f), cxy)
        tmp = ctx.mpi_empty()
        ctx.mpi_advect_2d(f, tmp, 0.5 * dt)
        half, err = rest.advect_2d(cxy, 0.5 * dt)
        assert err == 0
        assert np.array_equal(_host(tmp), cxy)
        assert np.array_equal(_host(f), half)
        ctx.mpi_field(f)
        phi, ex, ey = rest.field_poisson(rest.field_rho_halo(half))
        escale = max(np.abs(ex).max(), np.abs(ey).max())
        assert np.abs(_host(ctx.ex) - ex).max() <= 1e-12 * escale
        assert np.abs(_host(ctx.ey) - ey).max() <= 1e-12 * escale
        # The 4D stages, driven by the oracle's field so they can be exact.
        ctx.ex.copy_(_dev(torch, ex))
        ctx.ey.copy_(_dev(torch, ey))
        c = _dev(torch, cxy)
        ctx.mpi_spline_vxvy(c)
        c4 = rest.spline_vxvy(cxy)
        assert np.array_equal(_host(c), c4)
        ctx.mpi_advect_4d(c, tmp, dt)
        fnew, err = rest.advect_4d(c4, ex, ey)
        assert err == 0
        assert np.array_equal(_host(tmp), c4)
        assert np.array_equal(_host(c), fnew)
        ctx.check()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_step_matches_oracle(pkg, cuda, case):
    torch = cuda
    n, minp, maxp, dt, idcase, ic = case
    nsteps = 4
    rest = MpiRestatement(n, minp, maxp, dt, idcase)
    f0 = rest.init_halo(ic)
    fr, diags, _, _ = rest.run_mpi(f0, nsteps)
    with pkg.Context(_dom(pkg, n, minp, maxp, dt, idcase, nsteps), "f64") as ctx:
        fn, fnp1 = _dev(torch, f0), ctx.mpi_empty()
        out = ctx.mpi_run(fn, fnp1, nsteps)
        ctx.check()
        got = interior(_host(out))
        want = interior(fr)
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
        nrj, mass = ctx.diags_read()
        nrjx, nrjy, l2 = ctx.diags_read_ext()
    np.testing.assert_allclose(nrj, diags[:, 0], rtol=0, atol=1e-11)
    np.testing.assert_allclose(nrjx, diags[:, 1], rtol=1e-11)
    np.testing.assert_allclose(nrjy, diags[:, 2], rtol=1e-11)
    np.testing.assert_allclose(l2, diags[:, 4], rtol=1e-12)
    # mass is the sum of phi: rounding noise around zero.
    assert np.abs(mass - diags[:, 3]).max() < 1e-9


def test_run_matches_reference_fixture(pkg, cuda):
    """12 steps against the reference's own nrj.out / l2norm.out history
    (tests/golden/mpi_stages_small.npz, 13 printed digits)."""
    torch = cuda
    g = golden("mpi_stages_small.npz")
    n, minp, maxp, dt = tuple(int(v) for v in g["n"]), tuple(g["minp"]), tuple(g["maxp"]), float(g["dt"])
    steps = int(g["run_nrj"].shape[0]) - 1
    rest = MpiRestatement(n, minp, maxp, dt, 10)
    with pkg.Context(_dom(pkg, n, minp, maxp, dt, 10, steps), "f64") as ctx:
        fn, fnp1 = _dev(torch, rest.init_halo(IC_SLD10)), ctx.mpi_empty()
        out = ctx.mpi_run(fn, fnp1, steps)
        ctx.check()
        nrj, _ = ctx.diags_read()
        nrjx, nrjy, l2 = ctx.diags_read_ext()
        final = _host(out)
    np.testing.assert_allclose(nrj, g["run_nrj"][:, 1], rtol=1e-11)
    np.testing.assert_allclose(nrjx, g["run_nrj"][:, 2], rtol=1e-11)
    np.testing.assert_allclose(nrjy, g["run_nrj"][:, 3], rtol=1e-11)
    np.testing.assert_allclose(l2, g["run_l2norm"][:, 1], rtol=1e-12)
    # Sampled grid points of the final state.
    pos, val = g["run_pos"], g["run_val"]
    inner = np.zeros(final.shape, dtype=bool)
    inner[3:-3, 3:-3, 3:-3, 3:-3] = True
    sel = inner.reshape(-1)[pos]
    got = final.reshape(-1)[pos[sel]]
    assert np.abs(got - val[sel]).max() <= 1e-11 * np.abs(val[sel]).max()


def test_larger_grid_steps(pkg, cuda):
    """32^4 (the 4D pass with several x and y blocks and plane groups)."""
    torch = cuda
    n, minp, maxp, dt = (32, 32, 32, 32), (0, 0, -6, -6), (FOUR_PI, FOUR_PI, 6, 6), 0.05
    rest = MpiRestatement(n, minp, maxp, dt, 10)
    f0 = rest.init_halo(IC_SLD10)
    fr, diags, _, _ = rest.run_mpi(f0, 3)
    with pkg.Context(_dom(pkg, n, minp, maxp, dt, 10, 3), "f64") as ctx:
        fn, fnp1 = _dev(torch, f0), ctx.mpi_empty()
        out = ctx.mpi_run(fn, fnp1, 3)
        ctx.check()
        got = interior(_host(out))
        _, _, l2 = ctx.diags_read_ext()
    want = interior(fr)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    np.testing.assert_allclose(l2, diags[:, 4], rtol=1e-12)


def test_range_error_reported_and_context_usable(pkg, cuda):
    """A time step whose feet leave the spline's range: the reference exits
    ("Time step is too large"); here vlp4d_check reports VLP4D_ERR_RANGE and
    the context keeps working."""
    torch = cuda
    n, minp, maxp = (12, 12, 12, 12), (0, 0, -9, -9), (FOUR_PI, FOUR_PI, 9, 9)
    rest = MpiRestatement(n, minp, maxp, 0.05, 10)
    f0 = rest.init_halo(IC_SLD10)
    from importlib import import_module

    vl = import_module(pkg.__name__ + ".vlp4d")
    with pkg.Context(_dom(pkg, n, minp, maxp, 0.8, 10, 2), "f64") as ctx:
        fn, fnp1 = _dev(torch, f0), ctx.mpi_empty()
        ctx.mpi_step(fn, fnp1, 1)
        with pytest.raises(vl.Vlp4dError) as e:
            ctx.check()
        assert e.value.code == vl.ERR_RANGE
    with pkg.Context(_dom(pkg, n, minp, maxp, 0.05, 10, 2), "f64") as ctx:
        fn, fnp1 = _dev(torch, f0), ctx.mpi_empty()
        ctx.mpi_step(fn, fnp1, 1)
        ctx.check()


def test_argument_checks(pkg, cuda):
    torch = cuda
    from importlib import import_module

    vl = import_module(pkg.__name__ + ".vlp4d")
    small = _dom(pkg, (8, 12, 12, 12), (0, 0, -6, -6), (FOUR_PI, FOUR_PI, 6, 6), 0.05, 10, 1)
    with pkg.Context(small, "f64") as ctx:
        a, b = ctx.mpi_empty(), ctx.mpi_empty()
        with pytest.raises(vl.Vlp4dError) as e:
            ctx.mpi_step(a, b, 1)
        assert e.value.code == vl.ERR_INVALID_ARG
    ok = _dom(pkg, (12, 12, 12, 12), (0, 0, -6, -6), (FOUR_PI, FOUR_PI, 6, 6), 0.05, 10, 1)
    with pkg.Context(ok, "f32") as ctx:
        a = torch.zeros(ctx.mpi_shape, dtype=torch.float64, device="cuda")
        b = torch.zeros_like(a)
        with pytest.raises(vl.Vlp4dError) as e:
            ctx.mpi_step(a, b, 1)
        assert e.value.code == vl.ERR_UNSUPPORTED
    with pkg.Context(ok, "f64") as ctx:
        a = ctx.mpi_empty()
        with pytest.raises(vl.Vlp4dError) as e:
            ctx.mpi_step(a, a, 1)
        assert e.value.code == vl.ERR_INVALID_ARG


def test_fused_step_matches_entry_point_sequence_64(pkg, cuda):
    """At 64^4 (beyond what the CPU checker covers quickly) the fused step
    against the reference-order entry points on the GPU, which are
    bit-identical to the reference stage by stage: three steps on the SLD10
    deck geometry, states within 1e-12 of max|f| and equal diagnostics."""
    torch = cuda
    n, L, dt, steps = 64, 12.56637112, 0.01, 3
    dom = _dom(pkg, (n,) * 4, (0, 0, -9, -9), (L, L, 9, 9), dt, 10, steps)
    with pkg.Context(dom, "f64") as ctx:
        # SLD10 initial condition on the device (Init.cpp:228-247).
        dx = [(dom.max_phy[k] - dom.min_phy[k]) / n for k in range(4)]
        ar = lambda k: dom.min_phy[k] + torch.arange(n, dtype=torch.float64, device="cuda") * dx[k]
        x, y, vx, vy = ar(0), ar(1), ar(2), ar(3)
        f0 = ctx.mpi_empty()
        f0[3:-3, 3:-3, 3:-3, 3:-3] = (torch.exp(-0.5 * (vy[:, None] ** 2 + vx[None, :] ** 2)) / (2 * np.pi))[
            :, :, None, None] * (1 + 0.05 * torch.cos(0.5 * y)[:, None] * torch.cos(0.5 * x)[None, :])[None, None]
        # Fused.
        a, b = f0.clone(), ctx.mpi_empty()
        fused = ctx.mpi_run(a, b, steps)
        ctx.check()
        nrj_f, _ = ctx.diags_read()
        _, _, l2_f = ctx.diags_read_ext()
        got = fused[3:-3, 3:-3, 3:-3, 3:-3].clone()
        del a, b, fused
        # Reference order.
        fn, fnp1, tmp = f0.clone(), ctx.mpi_empty(), ctx.mpi_empty()
        ctx.mpi_field(fn)
        ctx.diags_compute(0)
        ctx.mpi_l2norm(fn, 0)
        for it in range(1, steps + 1):
            ctx.mpi_halo_fill(fn)
            ctx.mpi_spline_xy(fn)
            fnp1.copy_(fn)
            ctx.mpi_advect_2d(fn, tmp, 0.5 * dt)
            ctx.mpi_field(fn)
            ctx.mpi_spline_vxvy(fnp1)
            ctx.mpi_advect_4d(fnp1, fn, dt)
            ctx.mpi_field(fnp1)
            ctx.diags_compute(it)
            ctx.mpi_l2norm(fnp1, it)
            fn, fnp1 = fnp1, fn
        ctx.check()
        nrj_r, _ = ctx.diags_read()
        _, _, l2_r = ctx.diags_read_ext()
        want = fn[3:-3, 3:-3, 3:-3, 3:-3]
        err = float((got - want).abs().max() / want.abs().max())
    assert err <= 1e-12
    np.testing.assert_allclose(nrj_f, nrj_r, rtol=0, atol=1e-11)
    np.testing.assert_allclose(l2_f, l2_r, rtol=1e-12)


@pytest.mark.parametrize("deck", ["sld10_mpi_12", "tsi20_mpi_32x10"])
def test_decks_match_reference_main(pkg, cuda, deck):
    """The fused step on the decks the reference's own vlp4d_mpi main() ran
    (nrj.out / l2norm.out in tests/golden, 13 printed digits)."""
    torch = cuda
    from conftest import GOLDEN

    dom = pkg.Domain.from_deck(GOLDEN / "decks" / f"{deck}.dat")
    ic = IC_SLD10 if dom.idcase == 10 else IC_TSI20_MPI
    rest = MpiRestatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, dom.idcase)
    with pkg.Context(dom, "f64") as ctx:
        fn, fnp1 = _dev(torch, rest.init_halo(ic)), ctx.mpi_empty()
        ctx.mpi_run(fn, fnp1, dom.nbiter)
        ctx.check()
        nrj, _ = ctx.diags_read()
        nrjx, nrjy, l2 = ctx.diags_read_ext()
    ref = np.loadtxt(GOLDEN / f"{deck}_nrj.out")
    ref_l2 = np.loadtxt(GOLDEN / f"{deck}_l2norm.out")
    np.testing.assert_allclose(nrj, ref[:, 1], rtol=1e-11)
    np.testing.assert_allclose(nrjx, ref[:, 2], rtol=1e-11)
    np.testing.assert_allclose(nrjy, ref[:, 3], rtol=1e-11)
    np.testing.assert_allclose(l2, ref_l2[:, 1], rtol=1e-12)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_init_case_matches_reference(pkg, cuda, case):
    """vlp4d_mpi_init_case against the restated initcase (Init.cpp:126-277):
    the same formulas, device exp/sin/cos against the host's (a few ulps)."""
    torch = cuda
    n, minp, maxp, dt, idcase, ic = case
    rest = MpiRestatement(n, minp, maxp, dt, idcase)
    want = rest.init_halo(ic)
    with pkg.Context(_dom(pkg, n, minp, maxp, dt, idcase, 1), "f64") as ctx:
        f = torch.full(ctx.mpi_shape, 7.0, dtype=torch.float64, device="cuda")
        ctx.mpi_init_case(f)
        got = _host(f)
    assert np.abs(got - want).max() <= 1e-15 * np.abs(want).max()
    assert np.array_equal(got == 0, want == 0)


@pytest.mark.parametrize("deck", ["sld10_mpi_12", "tsi20_mpi_32x10"])
@pytest.mark.parametrize("mode", ["fused", "staged"])
def test_driver_matches_reference_main(cuda, deck, mode, tmp_path):
    """The vlp4d_mpi driver (p3-miniapps_b200/cpp/vlp4d_mpi_main.cpp, the flow of
    Vlp4d.cpp on the C ABI) writes nrj.out and l2norm.out that match the
    reference's own main() on the same deck."""
    import shutil
    import subprocess

    from conftest import GOLDEN, ROOT

    exe = ROOT / "p3-miniapps_b200" / "_build" / "vlp4d_mpi_b200"
    if not exe.exists():
        pytest.fail(f"{exe} missing: build with make -C p3-miniapps_b200")
    shutil.copy(GOLDEN / "decks" / f"{deck}.dat", tmp_path / "deck.dat")
    args = [str(exe), "-f", "deck.dat"] + (["--staged"] if mode == "staged" else [])
    res = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr + res.stdout
    got, got_l2 = np.loadtxt(tmp_path / "nrj.out"), np.loadtxt(tmp_path / "l2norm.out")
    ref, ref_l2 = np.loadtxt(GOLDEN / f"{deck}_nrj.out"), np.loadtxt(GOLDEN / f"{deck}_l2norm.out")
    assert got.shape == ref.shape and got_l2.shape == ref_l2.shape
    assert np.array_equal(got[:, 0], ref[:, 0])
    np.testing.assert_allclose(got[:, 1:4], ref[:, 1:4], rtol=1e-11)
    np.testing.assert_allclose(got_l2[:, 1], ref_l2[:, 1], rtol=1e-12)
    assert "MainLoop" in res.stdout and ("advec4D" in res.stdout) == (mode == "staged")
