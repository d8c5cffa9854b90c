"""CPU tests of the oracle: the plain-C restatement against the reference's
golden outputs, the reference build itself (when present), the FFTW-subset
shim against numpy.fft, and properties of the Lagrange-5 weights."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle.oracle import IC_LANDAU_SUM, IC_SLD10, IC_TSI20, IC_TWO_STREAM, Reference, Restatement

STAGES = ("landau8", "odd", "thin")


def _rest(g):
    return Restatement(tuple(g["n"]), tuple(g["minp"]), tuple(g["maxp"]), float(g["dt"]), int(g["idcase"]))


@pytest.mark.parametrize("name", STAGES)
def test_restatement_matches_reference_stages(name):
    """Each stage of the restatement equals the reference's output bit for bit
    (same operation order), except reductions, which match to rounding."""
    g = golden(f"stages_{name}.npz")
    R = _rest(g)
    dt = float(g["dt"])
    f0 = g["f0"]
    assert np.array_equal(R.advect_x(f0, 0.5 * dt), g["x_half"])
    assert np.array_equal(R.advect_y(f0, 0.5 * dt), g["y_half"])
    assert np.array_equal(R.advect_vx(f0, g["ex_in"], dt), g["vx_full"])
    assert np.array_equal(R.advect_vy(f0, g["ey_in"], dt), g["vy_full"])
    rho = R.field_rho(f0)
    assert np.array_equal(rho, g["rho"])
    phi, ex, ey = R.field_poisson(rho)
    scale = max(np.abs(g["ex"]).max(), 1e-300)
    assert np.abs(phi - g["phi"]).max() <= 1e-13 * max(np.abs(g["phi"]).max(), 1.0)
    assert np.abs(ex - g["ex"]).max() <= 1e-13 * scale + 1e-18
    assert np.abs(ey - g["ey"]).max() <= 1e-13 * max(np.abs(g["ey"]).max(), scale) + 1e-18


@pytest.mark.parametrize("name", STAGES)
def test_restatement_one_step(name):
    g = golden(f"stages_{name}.npz")
    R = _rest(g)
    fn = g["f0"].copy()
    fnp1 = np.zeros_like(fn)
    rho, ex, ey = R.empty2(), R.empty2(), R.empty2()
    import ctypes as C

    nrj, mass = C.c_double(), C.c_double()
    R.L.orc_step(C.byref(R.d), fn, fnp1, rho, ex, ey, C.byref(nrj), C.byref(mass))
    assert np.abs(fn - g["step1"]).max() <= 1e-14 * np.abs(g["step1"]).max()
    assert abs(nrj.value - float(g["step1_nrj"])) <= 1e-12
    assert abs(mass.value - float(g["step1_mass"])) <= 1e-12


def test_restatement_landau32_history():
    """Benchmark configuration 1 (32^4, 80 steps): energy/mass history and
    final-f slices of the restatement against the reference's Diags output."""
    g = golden("run_landau32.npz")
    n = tuple(g["n"])
    R = Restatement(n, tuple(g["minp"]), tuple(g["maxp"]), float(g["dt"]), 10)
    f0 = R.init_case(IC_LANDAU_SUM, amp=0.05, k=0.5)
    f, nrj, mass, _, _ = R.run(f0, int(g["steps"]))
    assert np.abs(nrj - g["nrj"]).max() < 1e-10
    assert np.abs(mass - g["mass"]).max() < 1e-12
    assert np.abs(f[n[3] // 2, :, 0, :] - g["fxvx"]).max() < 1e-12
    assert np.abs(f.sum(axis=(0, 1)) - g["fsum_v"]).max() < 1e-10


def test_restatement_initcases_match_reference():
    g = golden("initcases.npz")
    n = tuple(g["n"])
    for name, ic in (("sld10", IC_SLD10), ("tsi20", IC_TSI20)):
        R = Restatement(n, tuple(g[name + "_minp"]), tuple(g[name + "_maxp"]), 0.125, ic)
        assert np.array_equal(R.init_case(ic), g[name])


def test_landau_damping_rate():
    """Physics check on the golden history: the 32^4 Landau run (k = 0.5)
    damps at the Vlasov dispersion-relation rate gamma ~ -0.153 (Landau root
    of 1 + (1 + z Z(z)) / k^2 = 0, z = w / (k sqrt 2))."""
    from scipy.special import wofz

    k = 0.5

    def disp(w):
        z = w / (k * np.sqrt(2))
        Z = 1j * np.sqrt(np.pi) * wofz(z)
        return 1 + (1 + z * Z) / k**2

    from scipy.optimize import fsolve

    sol = fsolve(lambda p: [disp(p[0] + 1j * p[1]).real, disp(p[0] + 1j * p[1]).imag], [1.4, -0.15])
    gamma = sol[1]
    assert abs(gamma + 0.1533) < 2e-3
    g = golden("run_landau32.npz")
    t, nrj = g["t"], g["nrj"]
    # Fit the envelope through the local maxima of log|E|.
    peaks = [i for i in range(1, len(nrj) - 1) if nrj[i] > nrj[i - 1] and nrj[i] >= nrj[i + 1]]
    slope = np.polyfit(t[peaks], nrj[peaks], 1)[0]
    assert abs(slope - gamma) < 0.02, (slope, gamma)


def test_lag_basis_properties():
    R = Restatement((8, 8, 8, 8), (0, 0, -6, -6), (1, 1, 6, 6), 0.1)
    for px in np.linspace(2.0, 3.0, 17):
        c = R.lag_basis(px)
        assert abs(c.sum() - 1.0) < 1e-14
    assert np.allclose(R.lag_basis(2.0), [0, 0, 1, 0, 0, 0], atol=0)
    # The reference's LAG_ORDER 5 weights (advect.hpp:69-87) reproduce
    # polynomials of degree <= 4 exactly on the six nodes 0..5, but not x^5:
    # they are a quintic blend, not the classical 6-point Lagrange basis.
    nodes = np.arange(6.0)
    for deg in range(5):
        for px in (2.0, 2.3, 2.71, 2.999):
            assert abs(R.lag_basis(px) @ nodes**deg - px**deg) < 1e-12 * max(1, px**deg)
    assert abs(R.lag_basis(2.3) @ nodes**5 - 2.3**5) > 0.1


def test_restatement_fft_matches_numpy():
    R = Restatement((8, 8, 8, 8), (0, 0, -6, -6), (1, 1, 6, 6), 0.1)
    rng = np.random.default_rng(7)
    for ny, nx in ((12, 16), (10, 14), (16, 8), (4, 16), (24, 48)):
        a = rng.normal(size=(ny, nx))
        h = R.rfft2(a)
        assert np.abs(h - np.fft.rfft2(a)).max() < 1e-12
        assert np.abs(R.irfft2(h, nx) / (nx * ny) - a).max() < 1e-13


def test_fft_kat_golden():
    """The reference's own FFT round-trip case (tests/openmp/test_fft.cpp,
    eps 1e-8) through Impl::FFT on the FFTW-subset shim, pinned to numpy."""
    g = golden("fft_kat.npz")
    assert np.abs(g["back"] - g["u"]).max() < 1e-8
    assert np.abs(g["hat"] - np.fft.rfft2(g["u"])).max() < 1e-12


@pytest.mark.skipif(not Reference.available(), reason="reference build (oracle/_ref) not present")
def test_reference_fft_shim_matches_numpy():
    rng = np.random.default_rng(3)
    for nb, ny, nx in ((1, 12, 16), (2, 16, 16), (3, 10, 6), (1, 48, 24)):
        a = rng.normal(size=(nb, ny, nx))
        h = Reference.rfft2(a)
        assert np.abs(h - np.fft.rfft2(a)).max() < 1e-12
        assert np.abs(Reference.irfft2(h, nx) / (nx * ny) - a).max() < 1e-13


@pytest.mark.skipif(not Reference.available(), reason="reference build (oracle/_ref) not present")
def test_reference_and_restatement_agree_live():
    """A fresh random case (not a fixture): the two CPU checkers agree."""
    n, minp, maxp, dt = (10, 6, 8, 12), (0, 0, -5, -7), (7.0, 5.0, 5, 7), 0.3
    R = Restatement(n, minp, maxp, dt, 10)
    F = Reference(n, minp, maxp, dt, nbiter=3, idcase=10)
    f0 = R.init_case(IC_TWO_STREAM, amp=0.1, k=0.9, u=1.5)
    F.set_f(0, f0)
    F.run(3)
    d = F.diags()
    f, nrj, mass, _, _ = R.run(f0, 3)
    assert np.abs(F.get_f(0) - f).max() < 1e-14
    assert np.abs(d[:, 1] - nrj).max() < 1e-12


def test_mpi_diagnostics_restatement():
    """orc_diags_mpi / orc_l2norm against their definitions
    (miniapps/vlp4d_mpi/thrust/Diags.cpp:63-64, 68-92)."""
    L = 4 * np.pi
    o = Restatement((8, 6, 10, 8), [0, 0, -6, -6], [L, L, 6, 6], 0.125, 110)
    rng = np.random.default_rng(2)
    ex, ey = rng.normal(size=o.shape2), rng.normal(size=o.shape2)
    f = rng.normal(size=o.shape4)
    dx = o.dx
    nx, ny = o.diags_mpi(ex, ey)
    assert abs(nx - np.sqrt(0.5 * (ex ** 2).sum() * dx[0] * dx[1])) < 1e-14 * nx
    assert abs(ny - np.sqrt(0.5 * (ey ** 2).sum() * dx[0] * dx[1])) < 1e-14 * ny
    l2 = o.l2norm(f)
    assert abs(l2 - np.sqrt((f ** 2).sum() * np.prod(dx))) < 1e-13 * l2
