"""vlp4d_field_rho_noalloc: the velocity moment for callers that cannot
allocate device memory (their device memory belongs to their own allocator,
or their loop must not pay cudaMalloc/cudaFree), so cannot create a context.

Checked through the C ABI against the context-based vlp4d_field_rho on the
same inputs, on two calls in a row (the built-in scratch keeps the previous
call's contents; each call must be correct regardless), for FP64 and FP32
f, and the size limit of the built-in scratch.  This file is collected last
so that a run stopping at the first failure has run every other test."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _moment_with_context(pkg, dom, dtype, f):
    with pkg.Context(dom, dtype) as ctx:
        ctx.field_rho(f)
        return ctx.rho.clone()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_noalloc_moment_matches_context_moment_twice(pkg, cuda, dtype):
    torch = cuda
    tdt = torch.float64 if dtype == "f64" else torch.float32
    shapes = [(32, 24, 16, 20), (64, 64, 32, 32)]  # two calls in a row, different sizes
    for n in shapes:
        dom = pkg.landau_domain(n)
        g = torch.Generator(device="cuda").manual_seed(7 + n[0])
        f = torch.rand(dom.shape4, device="cuda", dtype=torch.float64, generator=g).to(tdt)
        ref = _moment_with_context(pkg, dom, dtype, f)
        rho = torch.full(dom.shape2, float("nan"), device="cuda", dtype=torch.float64)
        dvx, dvy = dom.dx[2], dom.dx[3]
        pkg.vlp4d.field_rho_noalloc(f, rho, dom.nxmax, dvx, dvy)
        torch.cuda.synchronize()
        err = float((rho - ref).abs().max() / ref.abs().max())
        assert err < 1e-14, (n, err)


def test_noalloc_rejects_grid_beyond_scratch(pkg, cuda):
    torch = cuda
    f = torch.zeros(8, device="cuda", dtype=torch.float64)
    rho = torch.zeros(8, device="cuda", dtype=torch.float64)
    with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
        pkg.vlp4d.field_rho_noalloc(f, rho, (1024, 1024, 1, 1), 1.0, 1.0)
    assert e.value.code == pkg.vlp4d.ERR_INVALID_ARG
    assert "scratch" in str(e.value)
