"""vlp4d_field_rho_noalloc: the velocity moment for callers that cannot
allocate device memory (their device memory belongs to their own allocator,
or their loop must not pay cudaMalloc/cudaFree), so cannot create a context.

Checked through the C ABI against the context-based vlp4d_field_rho on the
same inputs.  Both run the same two-level reduction with the same number of
plane groups and the same fixed summation order, so the results must be
bit-identical.  The calls go large grid, small grid, large grid on one
device: the built-in scratch keeps the previous call's contents, and each
call must be correct whatever a larger or smaller earlier call left there.
FP64 and FP32 f; the size limit of the built-in scratch; the argument
checks of the Python wrapper.  This file is collected last so that a run
stopping at the first failure has run every other test."""
from __future__ import annotations

import ctypes as C

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
    shapes = [(64, 64, 32, 32), (32, 24, 16, 20), (64, 64, 32, 32)]  # large, small, large again
    for i, n in enumerate(shapes):
        dom = pkg.landau_domain(n)
        g = torch.Generator(device="cuda").manual_seed(7 + 13 * i + n[0])
        f = torch.rand(dom.shape4, device="cuda", dtype=torch.float64, generator=g).to(tdt)
        ref = _moment_with_context(pkg, dom, dtype, f)
        rho = torch.full(dom.shape2, float("nan"), device="cuda", dtype=torch.float64)
        pkg.vlp4d.field_rho_noalloc(f, rho, dom.nxmax, dom.dx[2], dom.dx[3])
        torch.cuda.synchronize()
        assert torch.equal(rho, ref), (n, float((rho - ref).abs().max()))


def test_noalloc_rejects_grid_beyond_scratch(pkg, cuda):
    """The C entry point refuses nx*ny above its built-in scratch before it
    touches any buffer (called directly through ctypes with small buffers)."""
    torch = cuda
    f = torch.zeros(8, device="cuda", dtype=torch.float64)
    rho = torch.zeros(8, device="cuda", dtype=torch.float64)
    L = pkg.vlp4d.lib()
    rc = L.vlp4d_field_rho_noalloc(C.c_void_p(f.data_ptr()), pkg.vlp4d.F64, 1024, 1024, 1, 1, 1.0, 1.0,
                                   C.c_void_p(rho.data_ptr()), None)
    assert rc == pkg.vlp4d.ERR_INVALID_ARG
    assert b"scratch" in L.vlp4d_last_error()


def test_noalloc_wrapper_checks_tensors(pkg, cuda):
    torch = cuda
    dom = pkg.landau_domain((8, 8, 8, 8))
    f = torch.zeros(dom.shape4, device="cuda", dtype=torch.float32)
    rho = torch.zeros(dom.shape2, device="cuda", dtype=torch.float64)
    nxmax, dvx, dvy = dom.nxmax, dom.dx[2], dom.dx[3]
    bad = [
        (f.half(), rho),                       # element type the C side would misread
        (f.cpu(), rho),                        # host memory
        (f.transpose(0, 3), rho),              # not contiguous
        (f[:4], rho),                          # fewer elements than nxmax says
        (f, rho.float()),                      # rho must be FP64
        (f, rho[:4]),                          # rho too small
    ]
    for fa, ra in bad:
        with pytest.raises(ValueError):
            pkg.vlp4d.field_rho_noalloc(fa, ra, nxmax, dvx, dvy)
