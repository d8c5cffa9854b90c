"""Failure detection on the GPU without a GPU fault: a bounded device wait
that nothing completes gives up after its limit and the host sees
VLP4D_ERR_TIMEOUT; the context stays usable afterwards."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(pkg, cuda):
    torch = cuda
    v = pkg.vlp4d
    dom = pkg.landau_domain(16, dt=0.125, nbiter=4, idcase=110)
    with pkg.Context(dom, "f64") as ctx:
        f, g = ctx.empty_f(), ctx.empty_f()
        ctx.init_case(f, v.IC_LANDAU_SUM, 0.05, 0.5)
        ref_in = f.clone()
        ctx.selftest_wait_timeout(2_000_000)  # about a millisecond
        with pytest.raises(v.Vlp4dError) as e:
            ctx.check()
        assert e.value.code == v.ERR_TIMEOUT
        ctx.check()  # the error word was cleared
        # The context still computes: a step equals a step on a fresh context.
        ctx.field_rho(f)
        ctx.field_poisson()
        ctx.step(f, g, 1)
        with pkg.Context(dom, "f64") as fresh:
            a, b = ref_in.clone(), fresh.empty_f()
            fresh.field_rho(a)
            fresh.field_poisson()
            fresh.step(a, b, 1)
        assert torch.equal(g, b)


def test_wait_limit_is_validated(pkg, cuda):
    v = pkg.vlp4d
    dom = pkg.landau_domain(8, nbiter=1)
    with pkg.Context(dom, "f32") as ctx:
        for bad in (-1, 5_000_000_000):
            with pytest.raises(v.Vlp4dError) as e:
                ctx.selftest_wait_timeout(bad)
            assert e.value.code == v.ERR_INVALID_ARG
        ctx.selftest_wait_timeout(0)
        with pytest.raises(v.Vlp4dError):
            ctx.check()
