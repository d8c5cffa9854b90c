"""GPU parity of every C-ABI entry point against the reference's own outputs
(tests/golden, produced by the reference's OpenMP build) and the live CPU
oracle (oracle/vlp4d_oracle.c).

Tolerances (FP64 path).  The CUDA kernels evaluate the foot of the
characteristic once per swept line instead of once per cell; the reference's
per-cell foot differs from the line's by the rounding of x_i - disp, i.e.
|d_i - d_0| <= ~1e-13 cells, so one sweep may differ from the reference by
at most ~1e-13 * max|f|.  Single stages are checked at 1e-12 * max|f|; the
FP64 field solve (cuFFT vs FFTW) at 1e-12 relative to max|E|.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle.oracle import IC_LANDAU_SUM, IC_SLD10, IC_TSI20, IC_TWO_STREAM, Restatement

pytestmark = pytest.mark.gpu

STAGE_TOL = 1e-12


def _dom_from(pkg, g, nbiter=4):
    return pkg.Domain(list(map(int, g["n"])), list(map(float, g["minp"])), list(map(float, g["maxp"])),
                      float(g["dt"]), nbiter, int(g["idcase"]))


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def _host(t):
    return t.detach().double().cpu().numpy()


def _maxrel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", ["landau8", "odd", "thin"])
def test_stages_match_reference_golden_f64(pkg, cuda, name):
    torch = cuda
    g = golden(f"stages_{name}.npz")
    dom = _dom_from(pkg, g)
    dt = dom.dt
    with pkg.Context(dom, "f64") as ctx:
        f0 = _dev(torch, g["f0"], torch.float64)
        out = ctx.empty_f()
        ctx.advect_x(f0, out, 0.5 * dt)
        assert _maxrel(_host(out), g["x_half"]) < STAGE_TOL
        ctx.advect_y(f0, out, 0.5 * dt)
        assert _maxrel(_host(out), g["y_half"]) < STAGE_TOL
        ctx.field_rho(f0)
        assert _maxrel(_host(ctx.rho), g["rho"]) < 1e-14
        ctx.field_poisson()
        escale = max(np.abs(g["ex"]).max(), np.abs(g["ey"]).max())
        assert np.abs(_host(ctx.ex) - g["ex"]).max() < 1e-12 * escale + 1e-17
        assert np.abs(_host(ctx.ey) - g["ey"]).max() < 1e-12 * escale + 1e-17
        assert np.abs(_host(ctx.rho) - g["phi"]).max() < 1e-12 * max(np.abs(g["phi"]).max(), 1e-3)
        ctx.ex.copy_(_dev(torch, g["ex_in"], torch.float64))
        ctx.ey.copy_(_dev(torch, g["ey_in"], torch.float64))
        ctx.advect_vx(f0, out, dt)
        assert _maxrel(_host(out), g["vx_full"]) < STAGE_TOL
        ctx.advect_vy(f0, out, dt)
        assert _maxrel(_host(out), g["vy_full"]) < STAGE_TOL


@pytest.mark.parametrize("name", ["landau8", "odd", "thin"])
def test_fused_step_matches_reference_onetimestep_f64(pkg, cuda, name):
    torch = cuda
    g = golden(f"stages_{name}.npz")
    dom = _dom_from(pkg, g)
    with pkg.Context(dom, "f64") as ctx:
        f0 = _dev(torch, g["f0"], torch.float64)
        nxt = ctx.empty_f()
        ctx.step(f0, nxt, 1)
        nrj, mass = ctx.diags_read(2)
        assert _maxrel(_host(nxt), g["step1"]) < 1e-12
        assert abs(nrj[1] - float(g["step1_nrj"])) < 1e-10
        assert abs(mass[1] - float(g["step1_mass"])) < 1e-12


@pytest.mark.parametrize("name", ["landau8", "odd", "thin"])
def test_fused_pairs_equal_1d_sequence(pkg, cuda, name):
    torch = cuda
    g = golden(f"stages_{name}.npz")
    dom = _dom_from(pkg, g)
    dt = dom.dt
    for dtype, tol in (("f64", 1e-13), ("f32", 2e-6)):
        with pkg.Context(dom, dtype) as ctx:
            f0 = _dev(torch, g["f0"], ctx.torch_dtype)
            a, b = ctx.empty_f(), ctx.empty_f()
            ctx.advect_x(f0, a, 0.5 * dt)
            ctx.advect_y(a, b, 0.5 * dt)
            fused = ctx.empty_f()
            ctx.advect_xy(f0, fused, 0.5 * dt)
            assert _maxrel(_host(fused), _host(b)) < tol
            ctx.ex.copy_(_dev(torch, g["ex_in"], torch.float64))
            ctx.ey.copy_(_dev(torch, g["ey_in"], torch.float64))
            ctx.advect_vx(f0, a, dt)
            ctx.advect_vy(a, b, dt)
            ctx.advect_vxvy(f0, fused, dt)
            assert _maxrel(_host(fused), _host(b)) < tol


def test_landau32_run_matches_reference_history(pkg, cuda):
    """Benchmark configuration 1 (32^4, dt 0.125, 80 steps) through vlp4d_run
    with host buffers, against the reference's nrj.out and final f."""
    torch = cuda
    g = golden("run_landau32.npz")
    steps = int(g["steps"])
    dom = pkg.Domain(list(map(int, g["n"])), list(map(float, g["minp"])), list(map(float, g["maxp"])),
                     float(g["dt"]), steps, 10)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, 10)
    f0 = ora.init_case(IC_LANDAU_SUM, amp=0.05, k=0.5)
    with pkg.Context(dom, "f64") as ctx:
        fn, fnp1 = ctx.empty_f(), ctx.empty_f()
        fout = torch.empty(dom.shape4, dtype=torch.float64).pin_memory()
        nrj, mass = ctx.run(torch.from_numpy(f0).pin_memory(), steps, fn, fnp1, f_out_host=fout)
        f = fout.numpy()
    n = dom.nxmax
    assert np.abs(nrj - g["nrj"]).max() < 1e-9
    assert np.abs(mass - g["mass"]).max() < 1e-12
    assert np.abs(f[n[3] // 2, :, 0, :] - g["fxvx"]).max() < 1e-11
    assert np.abs(f.sum(axis=(0, 1)) - g["fsum_v"]).max() < 1e-9
    # Relative electric-energy error W = exp(2 nrj).
    w_err = np.abs(np.exp(2 * (nrj - g["nrj"])) - 1).max()
    assert w_err < 1e-8


def test_f32_storage_energy_error_landau32(pkg, cuda):
    """FP32-stored f with FP64 field solve and diagnostics against the FP64
    reference history over the 80 steps of configuration 1 (32^4).

    The relative error W32/W64 - 1 is largest at the deep minima of the field
    energy (steps 30 and 48, where W is ~1/100 of its neighbours); there even
    FP32 storage with exact FP64 arithmetic reaches ~1e-5 at 32^4 (a CPU
    emulation of the scheme gives 1.0e-5), so this test bounds the error at
    steps where W is below 1% of its maximum by 4e-5, elsewhere by 1e-5, and
    relative to the largest energy by 3e-7.  The 1e-5 target itself is stated at 128^4, where FP32
    noise is lower: see test_f32_energy_error_landau128."""
    torch = cuda
    g = golden("run_landau32.npz")
    steps = int(g["steps"])
    dom = pkg.Domain(list(map(int, g["n"])), list(map(float, g["minp"])), list(map(float, g["maxp"])),
                     float(g["dt"]), steps, 10)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, 10)
    f0 = ora.init_case(IC_LANDAU_SUM, amp=0.05, k=0.5)
    with pkg.Context(dom, "f32") as ctx:
        fn, fnp1 = ctx.empty_f(), ctx.empty_f()
        nrj, mass = ctx.run(torch.from_numpy(f0.astype(np.float32)), steps, fn, fnp1)
    w32, w64 = np.exp(2 * nrj), np.exp(2 * g["nrj"])
    rel = np.abs(w32 / w64 - 1)
    deep = w64 < 1e-2 * w64.max()
    assert rel[deep].max() < 4e-5, rel[deep].max()
    assert rel[~deep].max() < 1e-5, rel[~deep].max()
    assert np.abs(w32 - w64).max() / w64.max() < 3e-7
    assert np.abs(mass - g["mass"]).max() < 1e-6


_LANDAU128 = {}


def _landau128(pkg, dtype, api):
    """Landau 128^4, dt 0.1, 100 steps from the sum-form initial condition:
    (energy history, final f as FP64, this library's kernel launches of the
    100 steps).  api "steps" is the time loop vlp4d_steps (in FP32 the
    joined k_plane_xyxy pass between steps, the path the benchmark times);
    api "step" is 100 vlp4d_step calls (three passes each).  Cached per
    (dtype, api) for the tests of this module."""
    key = (dtype, api)
    if key in _LANDAU128:
        return _LANDAU128[key]
    import torch

    dom = pkg.landau_domain(128, dt=0.1, nbiter=100)
    with pkg.Context(dom, dtype) as ctx:
        fa, fb = ctx.empty_f(), ctx.empty_f()
        ctx.init_case(fa, pkg.vlp4d.IC_LANDAU_SUM, 0.05, 0.5)
        ctx.field_rho(fa)
        ctx.field_poisson()
        ctx.diags_compute(0)
        torch.cuda.synchronize()
        l0 = pkg.vlp4d.kernel_launches()
        if api == "steps":
            ctx.steps(fa, fb, 1, 100)
            cur = fb
        else:
            cur, nxt = fa, fb
            for it in range(1, 101):
                ctx.step(cur, nxt, it)
                cur, nxt = nxt, cur
        torch.cuda.synchronize()
        launches = pkg.vlp4d.kernel_launches() - l0
        hist = ctx.diags_read(101)[0]
        final = cur.double()
        del fa, fb, cur
    torch.cuda.empty_cache()
    _LANDAU128[key] = (hist, final, launches)
    return _LANDAU128[key]


def _check_f32_against_f64(h32, f32, h64, f64):
    w32, w64 = np.exp(2 * h32), np.exp(2 * h64)
    rel = np.abs(w32 / w64 - 1)
    assert rel.max() < 1e-5, (rel.max(), int(rel.argmax()))
    df = (f32 - f64).abs().max().item()
    assert df < 1e-5 * f64.abs().max().item(), df
    return rel.max(), df


def test_f32_energy_error_landau128(pkg, cuda):
    """The FP32-storage criterion on configuration 2 (Landau 128^4, dt 0.1,
    100 steps) for the three-pass step: relative electric-energy error of
    FP32 f against the FP64 path (itself checked against the reference at
    small sizes) at most 1e-5 over the whole history, and the max-norm
    error of the final f at most 1e-5 of max|f|."""
    h64, f64, _ = _landau128(pkg, "f64", "step")
    h32, f32, _ = _landau128(pkg, "f32", "step")
    _check_f32_against_f64(h32, f32, h64, f64)


def test_f32_energy_error_landau128_time_loop(pkg, cuda):
    """The same criterion for the path the headline throughput is measured
    on: vlp4d_steps with FP32 f, whose passes between steps apply the two
    x/y half steps as the composed 11-tap stencils of k_plane_xyxy, against
    FP64 vlp4d_step calls (the three-pass step, pinned to the reference at
    small sizes).  The joined path must have run: it launches one x/y pass
    fewer per step than 100 vlp4d_step calls.  The FP64 time loop (joined as
    well, k_plane_xyxy64) equals the FP64 step calls to FP64 rounding."""
    try:
        h64s, f64s, _ = _landau128(pkg, "f64", "step")
        h64, f64, _ = _landau128(pkg, "f64", "steps")
        assert np.abs(np.exp(2 * (h64 - h64s)) - 1).max() < 1e-11
        assert float((f64 - f64s).abs().max()) < 1e-12 * float(f64s.abs().max())
        h32, f32, launches_joined = _landau128(pkg, "f32", "steps")
        _, _, launches_3pass = _landau128(pkg, "f32", "step")
        assert launches_joined <= launches_3pass - 95, (launches_joined, launches_3pass)
        _check_f32_against_f64(h32, f32, h64s, f64s)
    finally:
        _LANDAU128.clear()


def test_init_cases(pkg, cuda):
    torch = cuda
    g = golden("initcases.npz")
    n = list(map(int, g["n"]))
    for name, ic in (("sld10", IC_SLD10), ("tsi20", IC_TSI20)):
        dom = pkg.Domain(n, list(map(float, g[name + "_minp"])), list(map(float, g[name + "_maxp"])), 0.125, 1, ic)
        with pkg.Context(dom, "f64") as ctx:
            f = ctx.empty_f()
            ctx.init_case(f, ic)
            assert _maxrel(_host(f), g[name]) < 4e-15
    dom = pkg.landau_domain((12, 10, 8, 6))
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, 10)
    for ic, kw in ((IC_LANDAU_SUM, dict(amp=0.05, k=0.5)), (IC_TWO_STREAM, dict(amp=0.001, k=0.2, u=2.4))):
        with pkg.Context(dom, "f64") as ctx:
            f = ctx.empty_f()
            ctx.init_case(f, ic, **kw)
            assert _maxrel(_host(f), ora.init_case(ic, **kw)) < 4e-15


def test_large_and_zero_shifts(pkg, cuda):
    """Lines with zero displacement (vx = 0 at ivx = N/2, E = 0), negative
    displacements of several box widths and shifts of exactly one cell,
    against the oracle.  The reference (and so the oracle) is defined only for
    displacements disp <= box width (advection.hpp:120: a larger positive disp
    makes fmod negative and the tap index go below zero), so every positive
    displacement here stays inside the box."""
    torch = cuda
    n = (16, 12, 16, 10)
    dom = pkg.Domain(list(n), [0.0, 0.0, -6.0, -6.0], [2.0, 3.0, 6.0, 6.0], 0.7, 2, 10)
    ora = Restatement(n, dom.min_phy, dom.max_phy, dom.dt, 10)
    f0 = ora.init_case(IC_TWO_STREAM, amp=0.2, k=np.pi, u=1.3)
    rng = np.random.default_rng(11)
    ex = rng.normal(size=ora.shape2) * 20.0
    ey = np.zeros(ora.shape2)
    ey[:, ::3] = -(6.0 - -6.0) / 10  # exactly one cell at dt = 1
    with pkg.Context(dom, "f64") as ctx:
        fd = _dev(torch, f0, torch.float64)
        out = ctx.empty_f()
        # x box 2.0, y box 3.0, |v| <= 6: |dt| <= 1/3 keeps dt*v inside both boxes;
        # dt = 1/6 moves the vx = 0.75 line by exactly one x cell (0.125).
        for dt in (0.3, -0.3, 1.0 / 6.0):
            ctx.advect_x(fd, out, dt)
            assert _maxrel(_host(out), ora.advect_x(f0, dt)) < STAGE_TOL
            ctx.advect_y(fd, out, dt)
            assert _maxrel(_host(out), ora.advect_y(f0, dt)) < STAGE_TOL
        ctx.ex.copy_(_dev(torch, -np.abs(ex), torch.float64))
        ctx.ey.copy_(_dev(torch, ey, torch.float64))
        for dt in (0.7, 1.0):
            ctx.advect_vx(fd, out, dt)
            assert _maxrel(_host(out), ora.advect_vx(f0, -np.abs(ex), dt)) < STAGE_TOL
            ctx.advect_vy(fd, out, dt)
            assert _maxrel(_host(out), ora.advect_vy(f0, ey, dt)) < STAGE_TOL


def test_shift_beyond_reference_range_is_periodic(pkg, cuda):
    """Displacements larger than the box (undefined in the reference, whose
    tap index goes negative) wrap periodically: shifting by disp + L equals
    shifting by disp."""
    torch = cuda
    n = (16, 8, 8, 8)
    L = 2.0
    dom = pkg.Domain(list(n), [0.0, 0.0, -1.0, -1.0], [L, L, 1.0, 1.0], 0.1, 2, 10)
    ora = Restatement(n, dom.min_phy, dom.max_phy, dom.dt, 10)
    f0 = ora.init_case(IC_LANDAU_SUM, amp=0.3, k=np.pi)
    ex_small = np.full(ora.shape2, 0.37)
    with pkg.Context(dom, "f64") as ctx:
        fd = _dev(torch, f0, torch.float64)
        a, b = ctx.empty_f(), ctx.empty_f()
        ctx.ex.copy_(_dev(torch, ex_small, torch.float64))
        ctx.advect_vx(fd, a, 1.0)
        ctx.ex.copy_(_dev(torch, ex_small + 3 * 2.0, torch.float64))
        ctx.advect_vx(fd, b, 1.0)
        assert _maxrel(_host(b), _host(a)) < 1e-12


@pytest.mark.parametrize("rows,cols", [(16, 32), (15, 30), (129, 67)])
@pytest.mark.parametrize("dtype", ["float32", "float64", "complex128"])
def test_transpose_kat(pkg, cuda, rows, cols, dtype):
    """tests/thrust/test_transpose.cpp:5-79: a(j, i) = 0.12 i + 0.5 j on
    (rows x cols), forward then backward, eps 1e-8 (here exact)."""
    torch = cuda
    j, i = np.meshgrid(np.arange(rows), np.arange(cols), indexing="xy")
    a = (i * 0.12 + j * 0.5).astype(np.float64)  # shape (cols, rows): column-major (rows x cols)
    if dtype == "complex128":
        a = a + 1j * (a * 2 - 1)
    ta = torch.from_numpy(a.astype(dtype)).cuda()
    d = torch.empty((rows, cols), dtype=ta.dtype, device="cuda")
    pkg.vlp4d.transpose(ta, d)
    assert np.array_equal(d.cpu().numpy(), a.astype(dtype).T)
    b = torch.empty_like(ta)
    pkg.vlp4d.transpose(d, b)
    assert np.array_equal(b.cpu().numpy(), a.astype(dtype))


def test_diags_save_and_fxvx_formats(pkg, cuda, tmp_path):
    torch = cuda
    dom = pkg.landau_domain(8, dt=0.125, nbiter=2)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, 10)
    f0 = ora.init_case(IC_LANDAU_SUM)
    with pkg.Context(dom, "f64") as ctx:
        fn = _dev(torch, f0, torch.float64)
        ctx.field_rho(fn)
        ctx.field_poisson()
        ctx.diags_compute(0)
        ctx.diags_save(tmp_path / "nrj.out")
        ctx.print_fxvx(fn, tmp_path / "fxvx.csv")
    rows = np.loadtxt(tmp_path / "nrj.out", ndmin=2)
    assert rows.shape == (3, 3)
    rho = ora.field_rho(f0)
    phi, ex, ey = ora.field_poisson(rho)
    nrj, mass = ora.diags(phi, ex, ey)
    assert abs(rows[0, 1] - nrj) < 1e-11 and abs(rows[0, 2] - mass) < 1e-12
    line = (tmp_path / "nrj.out").read_text().splitlines()[0]
    assert line == "%17.13e %17.13e %17.13e" % (0.0, rows[0, 1], rows[0, 2])
    csv = np.loadtxt(tmp_path / "fxvx.csv", delimiter=",")
    # "%20.13le" keeps 14 significant digits.
    assert np.allclose(csv, f0[dom.nxmax[3] // 2, :, 0, :], rtol=1e-13, atol=0)


def test_invalid_iter_rejected(pkg, cuda):
    dom = pkg.landau_domain(8, nbiter=2)
    with pkg.Context(dom, "f64") as ctx:
        with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
            ctx.diags_compute(3)
        assert e.value.code == pkg.vlp4d.ERR_INVALID_ARG
        f = ctx.empty_f()
        with pytest.raises(pkg.vlp4d.Vlp4dError):
            ctx.step(f, f, 1)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_mpi_diagnostics_match_oracle(pkg, cuda, dtype):
    """nrjx/nrjy (recorded by vlp4d_diags_compute) and the L2 norm of f
    (vlp4d_diags_l2norm) against the oracle's restatement of the vlp4d_mpi
    diagnostics, over three fused steps."""
    torch = cuda
    n, nsteps = (16, 12, 20, 16), 3
    dom = pkg.Domain(list(n), [0.0, 0.0, -6.0, -6.0], [4 * np.pi, 4 * np.pi, 6.0, 6.0], 0.125, nsteps, 110)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, 110)
    v = pkg.vlp4d
    with pkg.Context(dom, dtype) as ctx:
        a, b = ctx.empty_f(), ctx.empty_f()
        ctx.init_case(a, v.IC_LANDAU_SUM, 0.05, 0.5)
        ctx.field_rho(a)
        ctx.field_poisson()
        ctx.diags_compute(0)
        ctx.diags_l2norm(a, 0)
        ref = [(ora.diags_mpi(ctx.ex.cpu().numpy(), ctx.ey.cpu().numpy()), ora.l2norm(a.double().cpu().numpy()))]
        for it in range(1, nsteps + 1):
            ctx.step(a, b, it)
            ctx.diags_l2norm(b, it)
            ref.append((ora.diags_mpi(ctx.ex.cpu().numpy(), ctx.ey.cpu().numpy()), ora.l2norm(b.double().cpu().numpy())))
            a, b = b, a
        nrjx, nrjy, l2 = ctx.diags_read_ext(nsteps + 1)
    for it, ((rx, ry), rl) in enumerate(ref):
        assert abs(nrjx[it] - rx) <= 1e-13 * rx and abs(nrjy[it] - ry) <= 1e-13 * ry, it
        assert abs(l2[it] - rl) <= 1e-13 * rl, it
