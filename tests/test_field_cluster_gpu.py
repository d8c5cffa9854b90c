"""GPU tests of the cluster field solve (k_field_cluster, csrc/field_cluster.cu)
against the cuFFT path of the same entry point (VLP4D_FIELD=cufft): the
mode-wise solve is shared, the transforms differ only in rounding, so phi,
Ex and Ey agree to FP64 rounding of the transforms.  Shapes: the powers of
two of the benchmark configurations (Stockham passes), and a row count that
is not a power of two (direct DFT along y), rows and columns of lengths
48, 96, 40 (direct DFTs along x, along both); cases 10 (rho - 1) and 110."""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(pkg, dom, rho, use_cufft):
    import torch

    if use_cufft:
        os.environ["VLP4D_FIELD"] = "cufft"
    try:
        with pkg.Context(dom, "f64") as ctx:
            ctx.rho.copy_(rho)
            ctx.field_poisson()
            torch.cuda.synchronize()
            ctx.check()
            return ctx.rho.clone(), ctx.ex.clone(), ctx.ey.clone()
    finally:
        os.environ.pop("VLP4D_FIELD", None)


@pytest.mark.parametrize("nxy", [(128, 128), (64, 64), (32, 16), (16, 8), (64, 128), (32, 24), (48, 48), (96, 64), (40, 16)])
@pytest.mark.parametrize("idcase", [10, 110])
def test_cluster_solve_matches_cufft(pkg, cuda, nxy, idcase):
    torch = cuda
    nx, ny = nxy
    dom = pkg.landau_domain((nx, ny, 8, 8), dt=0.1, nbiter=1, idcase=idcase)
    gen = torch.Generator().manual_seed(nx * 1000 + ny + idcase)
    # A smooth density with modes along both axes plus noise: every mode of
    # the spectrum is populated.
    x = torch.arange(nx, dtype=torch.float64) * (2 * np.pi / nx)
    y = torch.arange(ny, dtype=torch.float64) * (2 * np.pi / ny)
    rho = (1.0 + 0.05 * torch.cos(x)[None, :] + 0.03 * torch.sin(2 * y)[:, None]
           + 1e-3 * torch.rand((ny, nx), generator=gen, dtype=torch.float64)).cuda()
    got = _solve(pkg, dom, rho, False)
    ref = _solve(pkg, dom, rho, True)
    for name, a, b in zip(("phi", "ex", "ey"), got, ref):
        scale = float(b.abs().max())
        assert scale > 0
        assert float((a - b).abs().max()) <= 1e-13 * scale, (name, float((a - b).abs().max()), scale)


def test_uniform_density_has_no_field(pkg, cuda):
    torch = cuda
    dom = pkg.landau_domain((128, 128, 8, 8), dt=0.1, nbiter=1)
    with pkg.Context(dom, "f64") as ctx:
        ctx.rho.fill_(1.0)
        ctx.field_poisson()
        torch.cuda.synchronize()
        assert float(ctx.ex.abs().max()) < 1e-14 and float(ctx.ey.abs().max()) < 1e-14
        assert float(ctx.rho.abs().max()) < 1e-14  # phi of rho - 1 = 0
