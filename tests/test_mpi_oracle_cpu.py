"""CPU checks of the vlp4d_mpi oracle: the C restatement of the one-process
vlp4d_mpi step against the reference's own OpenMP build and against the
committed fixtures made from it.

The reference build (oracle/_ref/libvlp4d_mpi_ref.so) exists only where the
reference tree is present; the fixture checks run everywhere.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import IC_SLD10, IC_TSI20_MPI, MpiReference, MpiRestatement, interior

GOLDEN = Path(__file__).resolve().parent / "golden"
FOUR_PI = 4 * np.pi

need_ref = pytest.mark.skipif(not MpiReference.available(), reason="reference vlp4d_mpi build absent")

CASES = [
    # (n, minp, maxp, dt, idcase, initial condition)
    ((16, 12, 10, 14), (0, 0, -9, -9), (FOUR_PI, FOUR_PI, 9, 9), 0.05, 10, IC_SLD10),
    ((12, 16, 20, 10), (0, 0, -8, -8), (10 * np.pi, 10 * np.pi, 8, 8), 0.1, 20, IC_TSI20_MPI),
]


@need_ref
@pytest.mark.parametrize("case", CASES, ids=["sld10", "tsi20"])
def test_stages_bit_identical_to_reference(case):
    n, minp, maxp, dt, idcase, ic = case
    rest = MpiRestatement(n, minp, maxp, dt, idcase)
    ref = MpiReference(n, minp, maxp, dt, nbiter=4, idcase=idcase)
    f = rest.init_halo(ic)
    assert np.array_equal(ref.get_f(0), f)
    ref.exchange_halo(0)
    f = rest.halo_fill(f)
    assert np.array_equal(ref.get_f(0), f)
    ref.spline_xy(0)
    cxy = rest.spline_xy(f)
    assert np.array_equal(ref.get_f(0), cxy)
    ref.set_f(1, cxy)
    ref.advect_2d(0, 0.5 * dt)
    half, err = rest.advect_2d(cxy, 0.5 * dt)
    assert err == 0
    assert np.array_equal(ref.get_f(0), half)
    ref.field(0)
    phi, ex, ey = rest.field_poisson(rest.field_rho_halo(half))
    assert np.array_equal(ref.get_field(1), ex)
    assert np.array_equal(ref.get_field(2), ey)
    assert np.array_equal(ref.get_field(0), phi)  # rho_ holds phi after the solve
    ref.spline_vxvy(1)
    c4 = rest.spline_vxvy(cxy)
    assert np.array_equal(ref.get_f(1), c4)
    ref.advect_4d(1, 0, dt)
    fnew, err = rest.advect_4d(c4, ex, ey)
    assert err == 0
    assert np.array_equal(ref.get_f(1), fnew)
    ref.close()


@need_ref
@pytest.mark.parametrize("case", CASES, ids=["sld10", "tsi20"])
def test_run_matches_reference(case):
    """Five steps through the reference's main loop: the state bit for bit,
    the diagnostics to the 13 digits nrj.out / l2norm.out keep."""
    n, minp, maxp, dt, idcase, ic = case
    steps = 5
    rest = MpiRestatement(n, minp, maxp, dt, idcase)
    ref = MpiReference(n, minp, maxp, dt, nbiter=steps, idcase=idcase)
    ref.run(steps)
    f, diags, _, _ = rest.run_mpi(rest.init_halo(ic), steps)
    assert np.array_equal(interior(ref.get_f(0)), interior(f))
    nrj, l2 = ref.diags()
    # nrj.out columns: t, nrj, nrjx, nrjy, mass.  mass is the sum of phi
    # (zero mean), i.e. rounding noise whose value depends on the reduction
    # order; compare it absolutely.
    np.testing.assert_allclose(nrj[:, 1:4], diags[:, 0:3], rtol=1e-12, atol=0)
    np.testing.assert_allclose(nrj[:, 4], diags[:, 3], rtol=0, atol=1e-10)
    np.testing.assert_allclose(l2[:, 1], diags[:, 4], rtol=1e-12, atol=0)
    ref.close()


def _digest_check(prefix, g, a):
    flat = np.ascontiguousarray(a).reshape(-1)
    assert np.array_equal(flat[g[f"{prefix}_pos"]], g[f"{prefix}_val"]), prefix
    assert np.array_equal(a[0, 3, 0, :], g[f"{prefix}_line"]), prefix
    np.testing.assert_allclose(flat.sum(), g[f"{prefix}_sum"], rtol=1e-13, atol=1e-15, err_msg=prefix)
    np.testing.assert_allclose((flat * flat).sum(), g[f"{prefix}_sq"], rtol=1e-13, err_msg=prefix)


def test_restatement_matches_fixtures():
    """The stage digests and the run history the reference's vlp4d_mpi
    produced (tests/golden/mpi_stages_small.npz, make_golden.py)."""
    g = np.load(GOLDEN / "mpi_stages_small.npz")
    n, minp, maxp, dt = tuple(g["n"]), tuple(g["minp"]), tuple(g["maxp"]), float(g["dt"])
    rest = MpiRestatement(n, minp, maxp, dt, 10)
    f = rest.init_halo(IC_SLD10)
    _digest_check("init", g, f)
    f = rest.halo_fill(f)
    _digest_check("halo", g, f)
    cxy = rest.spline_xy(f)
    _digest_check("spline_xy", g, cxy)
    half, err = rest.advect_2d(cxy, 0.5 * dt)
    assert err == 0
    _digest_check("advect_2d", g, half)
    phi, ex, ey = rest.field_poisson(rest.field_rho_halo(half))
    assert np.array_equal(ex, g["ex"]) and np.array_equal(ey, g["ey"]) and np.array_equal(phi, g["phi"])
    c4 = rest.spline_vxvy(cxy)
    _digest_check("spline_vxvy", g, c4)
    fnew, err = rest.advect_4d(c4, ex, ey)
    assert err == 0
    _digest_check("advect_4d", g, fnew)
    steps = int(g["run_nrj"].shape[0]) - 1
    f, diags, _, _ = rest.run_mpi(rest.init_halo(IC_SLD10), steps)
    np.testing.assert_allclose(g["run_nrj"][:, 1:4], diags[:, 0:3], rtol=1e-12, atol=0)
    np.testing.assert_allclose(g["run_l2norm"][:, 1], diags[:, 4], rtol=1e-12, atol=0)
    # The interior of the final state (the halo holds 4D spline coefficients
    # in the reference and is not part of the state).
    flat = np.ascontiguousarray(f).reshape(-1)
    pos, val = g["run_pos"], g["run_val"]
    inner = np.zeros(f.shape, dtype=bool)
    inner[3:-3, 3:-3, 3:-3, 3:-3] = True
    sel = inner.reshape(-1)[pos]
    assert sel.any()
    assert np.array_equal(flat[pos[sel]], val[sel])


def test_spline_interpolates_grid_values():
    """With dt = 0 the 2D spline evaluation returns the grid values
    (c[i-1] + 4 c[i] + c[i+1]) / 6 = f[i]: exact up to the truncated boundary
    sums (alpha^9 ~ 7e-6 of the line's scale) and rounding."""
    n, minp, maxp = (16, 16, 10, 10), (0, 0, -6, -6), (FOUR_PI, FOUR_PI, 6, 6)
    rest = MpiRestatement(n, minp, maxp, 0.1, 10)
    f = rest.init_halo(IC_SLD10)
    g, err = rest.advect_2d(rest.spline_xy(rest.halo_fill(f)), 0.0)
    assert err == 0
    scale = np.abs(interior(f)).max()
    assert np.abs(interior(g) - interior(f)).max() < 1e-5 * scale


def test_halo_fill_periodic_images_and_outer_sums():
    """Inner halo layers are periodic images; an outer-layer point in one
    dimension holds sum_j alpha^j f at the periodic continuation."""
    n, minp, maxp = (10, 11, 12, 10), (0, 0, -6, -6), (FOUR_PI, FOUR_PI, 6, 6)
    rest = MpiRestatement(n, minp, maxp, 0.1, 10)
    rng = np.random.default_rng(3)
    f = rest.empty_halo()
    interior(f)[...] = rng.normal(size=interior(f).shape)
    h = rest.halo_fill(f)
    inner = interior(f)
    # periodic images (layers -2..-1 and n..n+1 of x, other coords interior)
    for cx in (-2, -1, n[0], n[0] + 1):
        assert np.array_equal(h[3:-3, 3:-3, 3:-3, cx + 3], inner[:, :, :, cx % n[0]])
    # outer x layer: left = sum_{j=1..8} alpha^j f(n-2-j), right = sum alpha^j f(1+j)
    alpha = np.sqrt(3.0) - 2.0
    left = sum(alpha ** j * inner[:, :, :, (n[0] - 2 - j) % n[0]] for j in range(1, 9))
    right = sum(alpha ** j * inner[:, :, :, (1 + j) % n[0]] for j in range(1, 9))
    np.testing.assert_allclose(h[3:-3, 3:-3, 3:-3, 0], left, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(h[3:-3, 3:-3, 3:-3, -1], right, rtol=1e-13, atol=1e-15)


def _read_deck(path):
    """Values after each ':' of a reference deck (Init.cpp:12-90 order)."""
    vals = [line.split(":", 1)[1].strip() for line in Path(path).read_text().splitlines() if ":" in line]
    n = [int(v) for v in vals[0:4]]
    mm = [float(v) for v in vals[4:12]]
    minp, maxp = mm[0::2], mm[1::2]
    return n, minp, maxp, int(vals[12]), float(vals[13]), int(vals[14])


@pytest.mark.parametrize("deck", ["sld10_mpi_12", "tsi20_mpi_32x10"])
def test_restatement_matches_reference_main_decks(deck):
    """nrj.out and l2norm.out written by the reference's own vlp4d_mpi
    main() (Vlp4d.cpp, one process) on two small decks."""
    n, minp, maxp, case, dt, steps = _read_deck(GOLDEN / "decks" / f"{deck}.dat")
    ic = IC_SLD10 if case == 10 else IC_TSI20_MPI
    rest = MpiRestatement(n, minp, maxp, dt, case)
    _, diags, _, _ = rest.run_mpi(rest.init_halo(ic), steps)
    nrj = np.loadtxt(GOLDEN / f"{deck}_nrj.out")
    l2 = np.loadtxt(GOLDEN / f"{deck}_l2norm.out")
    np.testing.assert_allclose(nrj[:, 1:4], diags[:, 0:3], rtol=1e-12, atol=0)
    np.testing.assert_allclose(l2[:, 1], diags[:, 4], rtol=1e-12, atol=0)
