"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Runs the reference's OpenMP vlp4d (miniapps/vlp4d/openmp, compiled from its
sources into oracle/_ref/libvlp4d_ref.so by oracle/Makefile and driven by
oracle/ref_driver.cpp) on small seeded inputs and stores what it computes:

* ``stages_<name>.npz``: for one domain, f0 and the output of every stage
  the reference exposes, each from the same input f0 / fields:
  advect_1D_x/y (dt/2), field_rho, field_poisson (phi, Ex, Ey),
  advect_1D_vx/vy (dt) with seeded E fields, and one full onetimestep
  plus the Diags line it records.
* ``run_landau32.npz``: benchmark configuration 1 (32^4 Landau, sum-form
  initial condition, x,y in [0,4pi), v in [-6,6], dt 0.125, 80 steps): the
  nrj/mass history of Diags::save and slices of the final f.
* ``initcases.npz``: the reference's own testcaseSLD10/TSI20 initial
  conditions on a small deck-like domain.
* ``fft_kat.npz``: the reference's FFT round-trip case
  (tests/openmp/test_fft.cpp:7-71) through its Impl::FFT wrapper.
* ``<deck>_nrj.out``: nrj.out written by the reference's own driver
  (oracle/_ref/vlp4d_ref) on the small decks in decks/.
* ``<deck>_nrj.out`` / ``<deck>_l2norm.out`` for the vlp4d_mpi decks
  ``sld10_mpi_12`` and ``tsi20_mpi_32x10``: written by the reference's own
  vlp4d_mpi driver (oracle/_ref/vlp4d_mpi_ref, main() of
  miniapps/vlp4d_mpi/openmp/Vlp4d.cpp, one process).
* ``mpi_stages_small.npz``: the reference's OpenMP vlp4d_mpi
  (miniapps/vlp4d_mpi/openmp, one process, oracle/_ref/libvlp4d_mpi_ref.so
  driven by oracle/ref_mpi_driver.cpp) on a 10x12x10x11 grid: digests of
  the halo exchange, both spline prefilters, advect_2D_xy, the field,
  advect_4D and one onetimestep (sum, sum of squares, the values at 400
  seeded positions of the halo-extended array and one full x line through
  the outer halo layers), plus the nrj.out / l2norm.out history of 12 steps.

Usage (needs the reference tree, which only the build container has):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import (IC_LANDAU_SUM, IC_SLD10, IC_TWO_STREAM, MpiReference, MpiRestatement,  # noqa: E402
                           Reference, Restatement, build)

OUT = Path(__file__).resolve().parent
FOUR_PI = 4 * np.pi


def stage_dump(name, n, minp, maxp, dt, ic, idcase=10, seed=0, amp=0.05, k=0.5, u=2.4, e_scale=0.5):
    rest = Restatement(n, minp, maxp, dt, idcase)
    f0 = rest.init_case(ic, amp=amp, k=k, u=u)
    rng = np.random.default_rng(seed)
    ex = rng.normal(size=rest.shape2) * e_scale
    ey = rng.normal(size=rest.shape2) * e_scale
    ref = Reference(n, minp, maxp, dt, nbiter=4, idcase=idcase)
    out = {"n": np.array(n), "minp": np.array(minp), "maxp": np.array(maxp), "dt": np.array(dt),
           "idcase": np.array(idcase), "f0": f0, "ex_in": ex, "ey_in": ey}
    ref.set_f(0, f0)
    ref.advect_x(0, 1, 0.5 * dt)
    out["x_half"] = ref.get_f(1)
    ref.advect_y(0, 1, 0.5 * dt)
    out["y_half"] = ref.get_f(1)
    ref.field_rho(0)
    out["rho"] = ref.get_field(0)
    ref.field_poisson()
    out["phi"], out["ex"], out["ey"] = ref.get_field(0), ref.get_field(1), ref.get_field(2)
    ref.set_field(1, ex)
    ref.set_field(2, ey)
    ref.advect_vx(0, 1, dt)
    out["vx_full"] = ref.get_f(1)
    ref.advect_vy(0, 1, dt)
    out["vy_full"] = ref.get_f(1)
    # One complete onetimestep from f0 (its field solve overwrites the E above).
    ref.set_f(0, f0)
    ref.onetimestep(1)
    out["step1"] = ref.get_f(0)
    d = ref.diags()
    out["step1_nrj"], out["step1_mass"] = d[1, 1], d[1, 2]
    ref.close()
    np.savez_compressed(OUT / f"stages_{name}.npz", **out)
    print(f"stages_{name}: {n}")


def landau32():
    n, minp, maxp, dt, steps = (32, 32, 32, 32), (0, 0, -6, -6), (FOUR_PI, FOUR_PI, 6, 6), 0.125, 80
    rest = Restatement(n, minp, maxp, dt, 10)
    f0 = rest.init_case(IC_LANDAU_SUM, amp=0.05, k=0.5)
    ref = Reference(n, minp, maxp, dt, nbiter=steps, idcase=10)
    ref.set_f(0, f0)
    ref.run(steps)
    d = ref.diags()
    f = ref.get_f(0)
    ref.close()
    np.savez_compressed(
        OUT / "run_landau32.npz", n=np.array(n), minp=np.array(minp), maxp=np.array(maxp), dt=np.array(dt),
        steps=np.array(steps), t=d[:, 0], nrj=d[:, 1], mass=d[:, 2],
        fxvx=f[n[3] // 2, :, 0, :],           # f(ix, iy=0, ivx, ivy=nvy/2), the print_fxvx slice
        fxy=f[n[3] // 2, n[2] // 2, :, :],      # f(ix, iy, ivx=nvx/2, ivy=nvy/2)
        fsum_v=f.sum(axis=(0, 1)),              # sum over (ivy, ivx) of f(ix, iy, ., .)
        fnorm2=np.array(float((f * f).sum())))
    print("run_landau32: nrj[0], nrj[-1] =", d[0, 1], d[-1, 1])


def initcases():
    n = (12, 10, 16, 14)
    out = {}
    for name, idc, minp, maxp in (("sld10", 10, (0, 0, -9, -9), (12.56637112, 12.56637112, 9, 9)),
                                  ("tsi20", 20, (0, 0, -9, -9), (25.13274122871834590, 25.13274122871834590, 9, 9))):
        ref = Reference(n, minp, maxp, 0.125, nbiter=1, idcase=idc)
        ref.initcase(0)
        out[name] = ref.get_f(0)
        out[name + "_minp"], out[name + "_maxp"] = np.array(minp), np.array(maxp)
        ref.close()
    out["n"] = np.array(n)
    np.savez_compressed(OUT / "initcases.npz", **out)
    print("initcases:", n)


def fft_kat():
    """The reference's FFT round-trip test case (tests/openmp/test_fft.cpp:7-71),
    16x16x2 batched, plus its forward spectrum for an independent check."""
    nx, ny, nz = 16, 16, 2
    ix = np.arange(nx) / nx
    iy = np.arange(ny) / ny
    u = np.sin(ix[None, :] * 2 * np.pi) + np.cos(iy[:, None] * 3 * np.pi)
    u3 = np.stack([u] * nz)
    hat = Reference.rfft2(u3)
    back = Reference.irfft2(hat / (nx * ny), nx)
    np.savez_compressed(OUT / "fft_kat.npz", u=u3, hat=hat, back=back)
    print("fft_kat: round-trip err", float(np.abs(back - u3).max()))


def write_deck(path, n, mins, maxs, case, dt, steps, freq, fxvx):
    """An input deck in the reference's format (import(), init.cpp:12-82):
    the value after each colon, in a fixed order."""
    names = ["x", "y", "vx", "vy"]
    lines = ["# vlp4d input deck; the parser reads the value after each colon, in this order"]
    lines += [f"grid points along {nm} : {v}" for nm, v in zip(names, n)]
    for nm, a, b in zip(names, mins, maxs):
        lines += [f"lower bound of {nm} : {a}", f"upper bound of {nm} : {b}"]
    lines += [f"test case (10 Landau, 20 two-beam) : {case}", f"time step : {dt}", f"number of steps : {steps}",
              f"diagnostic frequency : {freq}", f"write fxvx slices : {fxvx}"]
    Path(path).write_text("\n".join(lines) + "\n")


def deck_runs():
    """The reference's own driver (oracle/_ref/vlp4d_ref, main() of
    miniapps/vlp4d/openmp/vlp4d.cpp) on two small decks; keeps its nrj.out."""
    import shutil
    import subprocess
    import tempfile

    from oracle.oracle import REFERENCE_EXE

    decks = OUT / "decks"
    write_deck(decks / "sld10_16.dat", [16] * 4, ["0.", "0.", "-9.", "-9."], ["12.56637112"] * 2 + ["9.", "9."],
               10, 0.125, 20, 4, 0)
    write_deck(decks / "tsi20_32x4.dat", [32, 4, 32, 4], ["0.", "0.", "-9.", "-9."],
               ["25.13274122871834590"] * 2 + ["9.", "9."], 20, 0.125, 20, 4, 1)
    for name in ("sld10_16", "tsi20_32x4"):
        with tempfile.TemporaryDirectory() as d:
            (Path(d) / "data" / "vlp4d").mkdir(parents=True)
            shutil.copy(decks / f"{name}.dat", Path(d) / "deck.dat")
            subprocess.run([str(REFERENCE_EXE), "deck.dat"], cwd=d, check=True, capture_output=True,
                           env={"OMP_NUM_THREADS": "4", "PATH": "/usr/bin:/bin"})
            shutil.copy(Path(d) / "nrj.out", OUT / f"{name}_nrj.out")
        print("deck run:", name)


MPI_SMALL = dict(n=(10, 12, 10, 11), minp=(0, 0, -6, -6), maxp=(FOUR_PI, FOUR_PI, 6, 6), dt=0.1, steps=12)


def mpi_digest(a, seed):
    """sum, sum of squares, 400 values at seeded flat positions, and the x
    line at (iy, ivx, ivy) = (-3, 0, -3) of a halo-extended array."""
    flat = np.ascontiguousarray(a).reshape(-1)
    pos = np.random.default_rng(seed).choice(flat.size, 400, replace=False)
    return {"sum": np.array(flat.sum()), "sq": np.array((flat * flat).sum()), "pos": pos,
            "val": flat[pos], "line": np.array(a[0, 3, 0, :])}


def mpi_stages():
    c = MPI_SMALL
    n, dt = c["n"], c["dt"]
    ref = MpiReference(n, c["minp"], c["maxp"], dt, nbiter=c["steps"], idcase=10)
    out = {"n": np.array(n), "minp": np.array(c["minp"]), "maxp": np.array(c["maxp"]), "dt": np.array(dt)}
    stages = {}
    stages["init"] = ref.get_f(0)
    ref.exchange_halo(0)
    stages["halo"] = ref.get_f(0)
    ref.spline_xy(0)
    stages["spline_xy"] = ref.get_f(0)
    ref.set_f(1, stages["spline_xy"])
    ref.advect_2d(0, 0.5 * dt)
    stages["advect_2d"] = ref.get_f(0)
    ref.field(0)
    out["phi"], out["ex"], out["ey"] = ref.get_field(0), ref.get_field(1), ref.get_field(2)
    ref.spline_vxvy(1)
    stages["spline_vxvy"] = ref.get_f(1)
    ref.advect_4d(1, 0, dt)
    stages["advect_4d"] = ref.get_f(1)
    for i, (k, v) in enumerate(stages.items()):
        for dk, dv in mpi_digest(v, 100 + i).items():
            out[f"{k}_{dk}"] = dv
    ref.close()
    # A run through the reference's main loop (Vlp4d.cpp:30-49).
    ref = MpiReference(n, c["minp"], c["maxp"], dt, nbiter=c["steps"], idcase=10)
    ref.run(c["steps"])
    nrj, l2 = ref.diags()
    out["run_nrj"], out["run_l2norm"] = nrj, l2
    for dk, dv in mpi_digest(ref.get_f(0), 200).items():
        out[f"run_{dk}"] = dv
    ref.close()
    np.savez_compressed(OUT / "mpi_stages_small.npz", **out)
    print("mpi_stages_small:", n)


def mpi_deck_runs():
    """The reference's own vlp4d_mpi driver on two small decks (every
    dimension at least 10); keeps its nrj.out and l2norm.out."""
    import shutil
    import subprocess
    import tempfile

    exe = ROOT / "oracle" / "_ref" / "vlp4d_mpi_ref"
    decks = OUT / "decks"
    write_deck(decks / "sld10_mpi_12.dat", [12] * 4, ["0.", "0.", "-9.", "-9."], ["12.56637112"] * 2 + ["9.", "9."],
               10, 0.05, 20, 4, 0)
    write_deck(decks / "tsi20_mpi_32x10.dat", [32, 10, 32, 10], ["0.", "0.", "-9.", "-9."],
               ["25.13274122871834590"] * 2 + ["9.", "9."], 20, 0.05, 20, 4, 0)
    for name in ("sld10_mpi_12", "tsi20_mpi_32x10"):
        with tempfile.TemporaryDirectory() as d:
            shutil.copy(decks / f"{name}.dat", Path(d) / "deck.dat")
            subprocess.run([str(exe), "-f", "deck.dat"], cwd=d, check=True, capture_output=True,
                           env={"OMP_NUM_THREADS": "4", "PATH": "/usr/bin:/bin"})
            shutil.copy(Path(d) / "nrj.out", OUT / f"{name}_nrj.out")
            shutil.copy(Path(d) / "l2norm.out", OUT / f"{name}_l2norm.out")
        print("mpi deck run:", name)


def main():
    build(reference=True)
    if not Reference.available():
        raise SystemExit("reference build unavailable")
    stage_dump("landau8", (8, 8, 8, 8), (0, 0, -6, -6), (FOUR_PI, FOUR_PI, 6, 6), 0.125, IC_LANDAU_SUM)
    stage_dump("odd", (12, 10, 14, 10), (0, 0, -6, -6), (FOUR_PI, FOUR_PI, 6, 6), 0.125, IC_LANDAU_SUM, seed=1)
    stage_dump("thin", (16, 4, 16, 4), (0, 0, -9, -9), (25.13274122871834590, 25.13274122871834590, 9, 9), 0.125,
               IC_TWO_STREAM, idcase=20, seed=2, amp=0.05, k=0.25, u=2.4)
    landau32()
    initcases()
    fft_kat()
    deck_runs()
    if MpiReference.available():
        mpi_stages()
        mpi_deck_runs()


if __name__ == "__main__":
    main()
