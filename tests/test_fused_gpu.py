"""The bandwidth-optimised fused kernels (x/y plane pass, v-slab pass, fused
moment) against the generic per-cell kernels, entry point by entry point, and
against the CPU oracle.  Contexts created with VLP4D_KERNELS=fused refuse to
fall back, so a passing test proves the fused kernels ran."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle.oracle import IC_LANDAU_SUM, IC_TWO_STREAM, Restatement

pytestmark = pytest.mark.gpu

# (nx, ny, nvx, nvy): shapes the fused kernels accept, including chunked
# planes (ny > R), a plane thinner than the stencil (ny = 4), several vy
# segments (nvy > 32) and non-square grids.
SHAPES = [(8, 8, 8, 8), (16, 4, 16, 4), (32, 32, 32, 32), (64, 48, 16, 64), (128, 64, 32, 40)]


def _ctx(pkg, dom, dtype, kernels, xyxy=""):
    saved = {k: os.environ.get(k) for k in ("VLP4D_KERNELS", "VLP4D_XYXY")}
    os.environ["VLP4D_KERNELS"] = kernels
    os.environ["VLP4D_XYXY"] = xyxy
    try:
        return pkg.Context(dom, dtype)
    finally:
        for k, v in saved.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def _dom(pkg, n, dt=0.2):
    return pkg.Domain(list(n), [0.0, 0.0, -6.0, -6.0], [4 * np.pi, 4 * np.pi, 6.0, 6.0], dt, 6, 10)


def _fields(torch, n, seed, scale):
    rng = np.random.default_rng(seed)
    ex = rng.normal(size=(n[1], n[0])) * scale
    ey = rng.normal(size=(n[1], n[0])) * scale
    return ex, ey


def _rel(a, b):
    a = a.double()
    b = b.double()
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("n", SHAPES)
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_fused_entry_points_match_generic(pkg, cuda, n, dtype):
    torch = cuda
    dom = _dom(pkg, n)
    tol = 1e-14 if dtype == "f64" else 2e-7
    ex, ey = _fields(torch, n, 5, 3.0)  # large E: vy offsets spread over several cells
    with _ctx(pkg, dom, dtype, "fused") as fz, _ctx(pkg, dom, dtype, "generic") as gn:
        f0 = fz.empty_f()
        fz.init_case(f0, IC_TWO_STREAM, 0.2, 0.5, 2.0)
        for c in (fz, gn):
            c.ex.copy_(torch.from_numpy(ex))
            c.ey.copy_(torch.from_numpy(ey))
        a, b = fz.empty_f(), gn.empty_f()
        for name, dt in (("advect_x", 0.1), ("advect_y", -0.1), ("advect_xy", 0.1),
                         ("advect_vx", 0.2), ("advect_vy", 0.2), ("advect_vxvy", 0.2)):
            getattr(fz, name)(f0, a, dt)
            getattr(gn, name)(f0, b, dt)
            assert _rel(a, b) < tol, (name, _rel(a, b))
        fz.check()


@pytest.mark.parametrize("n", SHAPES)
def test_fused_step_matches_generic_and_oracle(pkg, cuda, n):
    """Three fused steps (plane pass with the moment in its epilogue, field
    solve, v-slab pass, plane pass) against the generic path and against the
    FP64 CPU oracle."""
    torch = cuda
    dom = _dom(pkg, n, dt=0.125)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, 10)
    f0 = ora.init_case(IC_LANDAU_SUM, amp=0.05, k=0.5)
    steps = 3
    f_ref, nrj_ref, mass_ref, _, _ = ora.run(f0, steps)
    results = {}
    for kernels in ("fused", "generic"):
        with _ctx(pkg, dom, "f64", kernels) as ctx:
            fn, fnp1 = ctx.empty_f(), ctx.empty_f()
            nrj, mass = ctx.run(torch.from_numpy(f0), steps, fn, fnp1)
            results[kernels] = (fn.cpu().numpy(), nrj, mass)
    ff, nf, mf = results["fused"]
    fg, ng, mg = results["generic"]
    assert np.abs(ff - fg).max() <= 1e-13 * np.abs(fg).max()
    assert np.abs(nf - ng).max() < 1e-11
    assert np.abs(ff - f_ref).max() <= 1e-12 * np.abs(f_ref).max()
    assert np.abs(nf - nrj_ref).max() < 1e-10
    assert np.abs(mf - mass_ref).max() < 1e-12


def test_fused_moment_matches_generic_moment(pkg, cuda):
    """The moment accumulated in the plane pass's epilogue (FP64 shared
    memory, one partial per plane group) gives the same mid-step diagnostics
    as the generic path's separate field_rho reduction."""
    torch = cuda
    dom = _dom(pkg, (128, 64, 32, 40), dt=0.125)
    for dtype, tol in (("f64", 1e-12), ("f32", 1e-6)):
        with _ctx(pkg, dom, dtype, "fused") as fz, _ctx(pkg, dom, dtype, "generic") as gn:
            f0 = fz.empty_f()
            fz.init_case(f0, IC_LANDAU_SUM, 0.05, 0.5)
            a, b = fz.empty_f(), gn.empty_f()
            fz.step(f0.clone(), a, 1)
            gn.step(f0.clone(), b, 1)
            na, ma = fz.diags_read(2)
            nb, mb = gn.diags_read(2)
            assert abs(na[1] - nb[1]) < tol and abs(ma[1] - mb[1]) < tol


@pytest.mark.parametrize("n", [(12, 10, 14, 10), (16, 12, 20, 16)])
def test_fused_only_mode_rejects_unsupported_shape(pkg, cuda, n):
    # nvx = 14: no v-slab configuration; nvx = 20 in FP64: 16 columns x 5
    # row groups = 80 threads, not whole warps.
    dom = _dom(pkg, n)
    with _ctx(pkg, dom, "f64", "fused") as ctx:
        f, g = ctx.empty_f(), ctx.empty_f()
        ctx.init_case(f, IC_LANDAU_SUM)
        ctx.advect_xy(f, g, 0.1)  # the plane pass accepts nx = 12
        with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
            ctx.advect_vx(f, g, 0.1)
        assert e.value.code == pkg.vlp4d.ERR_UNSUPPORTED


def test_unaligned_buffers_fall_back_to_generic(pkg, cuda):
    torch = cuda
    n = (32, 32, 32, 32)
    dom = _dom(pkg, n)
    with pkg.Context(dom, "f32") as ctx:
        cells = dom.cells
        buf = torch.empty(cells + 1, dtype=torch.float32, device="cuda")
        f = buf[1:]  # 4-byte aligned only
        ctx.init_case(f, IC_LANDAU_SUM)
        out_u = torch.empty(cells + 1, dtype=torch.float32, device="cuda")[1:]
        out_a = ctx.empty_f()
        ctx.advect_xy(f, out_u, 0.1)
        ctx.advect_xy(f.clone(), out_a, 0.1)
        assert _rel(out_u, out_a.reshape(-1)) < 2e-7


@pytest.mark.parametrize("n", SHAPES)
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("xyxy", ["0", "1"])
def test_steps_bit_identical_to_single_steps(pkg, cuda, n, dtype, xyxy):
    """vlp4d_steps runs the last x/y half step of each step and the first of
    the next as two passes (VLP4D_XYXY=0), every sweep the same operation in
    the same order and precision as vlp4d_step: K steps equal K calls of
    vlp4d_step bit for bit, diagnostics included.  With VLP4D_XYXY=1 the two
    half steps are one pass of the composed 11-tap stencils, equal in exact
    arithmetic: the results agree to rounding."""
    torch = cuda
    K = 4
    dom = pkg.Domain(list(n), [0.0, 0.0, -6.0, -6.0], [4 * np.pi, 4 * np.pi, 6.0, 6.0], 0.125, K + 1, 10)
    with _ctx(pkg, dom, dtype, "fused", xyxy) as ctx:
        f0 = ctx.empty_f()
        ctx.init_case(f0, IC_LANDAU_SUM, 0.05, 0.5)
        a, b = f0.clone(), ctx.empty_f()
        for it in range(1, K + 1):
            ctx.step(a, b, it)
            a, b = b, a
        single = a.clone()
        nrj1, mass1 = ctx.diags_read(K + 1)
        c, d = f0.clone(), ctx.empty_f()
        ctx.steps(c, d, 1, K)
        nrj2, mass2 = ctx.diags_read(K + 1)
        if xyxy == "0":
            assert torch.equal(d, single)
            assert np.array_equal(nrj1[1:], nrj2[1:]) and np.array_equal(mass1[1:], mass2[1:])
        else:
            tol = 1e-13 if dtype == "f64" else 2e-6
            assert _rel(d, single) < tol
            assert np.abs(nrj1[1:] - nrj2[1:]).max() < (1e-11 if dtype == "f64" else 1e-6)


@pytest.mark.parametrize("n", [(16, 4, 16, 4), (32, 32, 32, 32), (12, 10, 14, 10)])
def test_steps_generic_and_oracle(pkg, cuda, n):
    """The fused time loop against the generic kernels' separate passes and
    against the FP64 CPU oracle (shapes include ones the fused passes decline)."""
    torch = cuda
    K = 3
    dom = pkg.Domain(list(n), [0.0, 0.0, -6.0, -6.0], [4 * np.pi, 4 * np.pi, 6.0, 6.0], 0.125, K + 1, 10)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, 10)
    f0 = ora.init_case(IC_LANDAU_SUM, amp=0.05, k=0.5)
    f_ref, nrj_ref, _, _, _ = ora.run(f0, K)
    outs = {}
    for kernels in ("", "generic"):
        with _ctx(pkg, dom, "f64", kernels) as ctx:
            a = torch.from_numpy(f0).cuda()
            b = ctx.empty_f()
            ctx.field_rho(a)
            ctx.field_poisson()
            ctx.diags_compute(0)
            ctx.steps(a, b, 1, K)
            outs[kernels] = (b.cpu().numpy(), ctx.diags_read(K + 1)[0])
    for f, nrj in outs.values():
        assert np.abs(f - f_ref).max() <= 1e-12 * np.abs(f_ref).max()
        assert np.abs(nrj - nrj_ref).max() < 1e-10


@pytest.mark.parametrize("n", SHAPES + [(12, 10, 14, 10)])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_advect_xyxy_matches_two_xy_passes(pkg, cuda, n, dtype):
    """vlp4d_advect_xyxy (one pass of the composed 11-tap stencils) against
    vlp4d_advect_xy twice, to rounding; the moment it leaves in rho against
    field_rho of the result."""
    torch = cuda
    dom = _dom(pkg, n)
    for kernels in ("", "generic"):
        with _ctx(pkg, dom, dtype, kernels) as ctx:
            f0 = ctx.empty_f()
            ctx.init_case(f0, IC_TWO_STREAM, 0.2, 0.5, 2.0)
            a, b, c = ctx.empty_f(), ctx.empty_f(), ctx.empty_f()
            ctx.advect_xy(f0, a, 0.15)
            ctx.advect_xy(a, b, 0.15)
            ctx.field_rho(b)
            rho_sep = ctx.rho.clone()
            if kernels == "generic":
                with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
                    ctx.advect_xyxy(f0, c, 0.15)
                assert e.value.code == pkg.vlp4d.ERR_UNSUPPORTED
                continue
            ctx.advect_xyxy(f0, c, 0.15)
            rho_one = ctx.rho.clone()
            assert _rel(c, b) < (1e-13 if dtype == "f64" else 2e-6), kernels
            assert float((rho_one - rho_sep).abs().max()) <= (1e-13 if dtype == "f64" else 1e-6) * float(
                rho_sep.abs().max())
            ctx.check()


# Odd shapes: thin planes (ny below the stencil span), row widths that are
# not powers of two (runtime-width paths), vx extents that give partial or
# no v-slab configurations, tiny vy extents.
ODD_SHAPES = [(4, 3, 8, 2), (8, 5, 12, 6), (12, 7, 24, 11), (20, 9, 40, 6), (36, 6, 16, 9), (24, 16, 8, 3)]


@pytest.mark.parametrize("n", ODD_SHAPES)
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_odd_shapes_default_path_matches_generic(pkg, cuda, n, dtype):
    """Two steps and a two-step time loop on the default path (fused kernels
    where the shape allows, generic otherwise) against the generic kernels."""
    torch = cuda
    dom = pkg.Domain(list(n), [0.0, 0.0, -6.0, -6.0], [4 * np.pi, 4 * np.pi, 6.0, 6.0], 0.125, 4, 110)
    res = {}
    for kernels in ("", "generic"):
        with _ctx(pkg, dom, dtype, kernels) as ctx:
            f0 = ctx.empty_f()
            ctx.init_case(f0, IC_LANDAU_SUM, 0.05, 0.5)
            ctx.field_rho(f0)
            ctx.field_poisson()
            a, b = f0.clone(), ctx.empty_f()
            ctx.step(a, b, 1)
            ctx.step(b, a, 2)
            c, d = f0.clone(), ctx.empty_f()
            ctx.steps(c, d, 1, 2)
            ctx.check()
            res[kernels] = (a.clone(), d.clone())
    tol = 1e-12 if dtype == "f64" else 2e-6
    assert _rel(res[""][0], res["generic"][0]) < tol
    assert _rel(res[""][1], res["generic"][1]) < tol
