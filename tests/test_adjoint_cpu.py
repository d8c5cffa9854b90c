"""The FP64 CPU adjoint (oracle/vlp4d_adjoint.c) checked on its own: the
Lagrange-weight derivative against finite differences, every stage transpose
by the dot-product identity <A x, y> = <x, A^T y>, the E-derivative of the
v stages and the whole checkpoint-free run gradient against central finite
differences of the restated forward map."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import IC_LANDAU_SUM, Restatement

L_BOX = 4 * np.pi


def _ora(n=(8, 6, 10, 8), dt=0.125, idcase=110):
    return Restatement(n, [0, 0, -6, -6], [L_BOX, L_BOX, 6, 6], dt, idcase)


@pytest.mark.parametrize("px", [2.0, 2.1, 2.5, 2.77, 2.999])
def test_lag_basis_derivative(px):
    o = _ora()
    h = 1e-6
    fd = (o.lag_basis(px + h) - o.lag_basis(px - h)) / (2 * h)
    assert np.abs(fd - o.lag_basis_deriv(px)).max() < 1e-8
    assert abs(o.lag_basis_deriv(px).sum()) < 1e-13  # the weights sum to one for every px


def test_stage_transposes():
    o = _ora()
    rng = np.random.default_rng(3)
    x, y = rng.normal(size=o.shape4), rng.normal(size=o.shape4)
    for dt in (0.3, -0.7, 5.0):
        assert abs(np.vdot(o.advect_x(x, dt), y) - np.vdot(x, o.advect_x_T(y, dt))) < 1e-11
        assert abs(np.vdot(o.advect_y(x, dt), y) - np.vdot(x, o.advect_y_T(y, dt))) < 1e-11
    ex, ey = rng.normal(size=o.shape2) * 2, rng.normal(size=o.shape2) * 2
    lt, _ = o.advect_vx_T(y, x, ex, 0.2)
    assert abs(np.vdot(o.advect_vx(x, ex, 0.2), y) - np.vdot(x, lt)) < 1e-11
    lt, _ = o.advect_vy_T(y, x, ey, 0.2)
    assert abs(np.vdot(o.advect_vy(x, ey, 0.2), y) - np.vdot(x, lt)) < 1e-11
    r, gx, gy = rng.normal(size=o.shape2), rng.normal(size=o.shape2), rng.normal(size=o.shape2)
    _, fx, fy = o.field_poisson(r)
    assert abs(np.vdot(fx, gx) + np.vdot(fy, gy) - np.vdot(r, o.field_poisson_T(gx, gy))) < 1e-12


def test_v_stage_field_derivative():
    o = _ora()
    rng = np.random.default_rng(4)
    x, y = rng.normal(size=o.shape4), rng.normal(size=o.shape4)
    e, u = rng.normal(size=o.shape2) * 2, rng.normal(size=o.shape2)
    h = 1e-6
    for adv, adj in ((o.advect_vx, o.advect_vx_T), (o.advect_vy, o.advect_vy_T)):
        _, g = adj(y, x, e, 0.2)
        fd = (np.vdot(adv(x, e + h * u, 0.2), y) - np.vdot(adv(x, e - h * u, 0.2), y)) / (2 * h)
        assert abs(fd - np.vdot(g, u)) < 1e-6 * max(1.0, abs(fd))


@pytest.mark.parametrize("idcase", [110, 10])
def test_run_gradient_matches_finite_differences(idcase):
    o = _ora(idcase=idcase)
    f0 = o.init_case(IC_LANDAU_SUM, 0.05, 0.5)
    nsteps = 3
    J, grad = o.adjoint_run(f0, nsteps)

    def J_of(f):
        for _ in range(nsteps):
            f = o.step(f)
        return o.energy(f)

    assert abs(J - J_of(f0)) <= 1e-14 * J
    rng = np.random.default_rng(5)
    h = 1e-4
    for _ in range(2):
        u = rng.normal(size=o.shape4) * f0
        fd = (J_of(f0 + h * u) - J_of(f0 - h * u)) / (2 * h)
        assert abs(np.vdot(grad, u) - fd) <= 1e-7 * abs(fd)
