"""The two-stream configuration: 64 x 64 x 128 x 128, x, y in [0, 10 pi),
v in [-8, 8), dt 0.05, 400 steps, f0 = (1 + 0.001 cos 0.2x + 0.001 cos 0.2y)
* 1/2 [M(vx - 2.4) + M(vx + 2.4)] M(vy); FP32 f / FP64 fields against the
FP64 path, and a reduced grid of the same case against the CPU oracle."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.oracle import IC_TWO_STREAM, Restatement

pytestmark = pytest.mark.gpu

L = 10 * math.pi


def _dom(pkg, n, nbiter):
    return pkg.Domain(list(n), [0.0, 0.0, -8.0, -8.0], [L, L, 8.0, 8.0], 0.05, nbiter, 120)


def _run(pkg, torch, dom, dtype, nsteps):
    v = pkg.vlp4d
    with pkg.Context(dom, dtype) as ctx:
        a, b = ctx.empty_f(), ctx.empty_f()
        ctx.init_case(a, v.IC_TWO_STREAM, 0.001, 0.2, 2.4)
        ctx.field_rho(a)
        ctx.field_poisson()
        ctx.diags_compute(0)
        ctx.steps(a, b, 1, nsteps)
        nrj, mass = ctx.diags_read(nsteps + 1)
        return b.double().cpu(), nrj


def test_two_stream_fp32_against_fp64(pkg, cuda):
    torch = cuda
    nsteps = 400
    dom = _dom(pkg, (64, 64, 128, 128), nsteps)
    f64, e64 = _run(pkg, torch, dom, "f64", nsteps)
    f32, e32 = _run(pkg, torch, dom, "f32", nsteps)
    w64, w32 = np.exp(2 * e64), np.exp(2 * e32)
    rel = np.abs(w32 - w64) / w64
    print("two-stream FP32 vs FP64: energy rel max %.3e, final %.3e, f max abs %.3e (max f %.3e), growth %.1f"
          % (rel.max(), rel[-1], float((f32 - f64).abs().max()), float(f64.abs().max()), w64[-1] / w64[0]))
    # The instability grows: the field energy rises more than tenfold by T = 20.
    assert w64[-1] > 10 * w64[:10].max()
    # Measured on B200: 8.2e-5 (energy), 1.5e-5 of max|f| (f).
    assert rel.max() < 5e-4, rel.max()
    assert float((f32 - f64).abs().max()) < 1e-4 * float(f64.abs().max())


def test_two_stream_reduced_grid_matches_oracle(pkg, cuda):
    torch = cuda
    n, nsteps = (16, 16, 32, 32), 12
    dom = _dom(pkg, n, nsteps)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, 120)
    f0 = ora.init_case(IC_TWO_STREAM, amp=0.001, k=0.2, u=2.4)
    f_ref, nrj_ref, _, _, _ = ora.run(f0, nsteps)
    f, nrj = _run(pkg, torch, dom, "f64", nsteps)
    assert np.abs(f.numpy() - f_ref).max() <= 1e-12 * np.abs(f_ref).max()
    assert np.abs(nrj - nrj_ref).max() < 1e-9
