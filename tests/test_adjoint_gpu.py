"""Reverse mode on the GPU (vlp4d_adjoint_*, vlp4d_step_adjoint,
vlp4d_energy_grad) against the FP64 CPU adjoint of the oracle, against
central finite differences of the GPU forward map, FP32 against FP64, and
through the torch.autograd binding."""
from __future__ import annotations

import math
import os

import numpy as np
import pytest

from oracle.oracle import IC_LANDAU_SUM, Restatement

pytestmark = pytest.mark.gpu

L_BOX = 4 * np.pi


def _dom(pkg, n, dt=0.125, nbiter=8, idcase=110):
    return pkg.Domain(list(n), [0.0, 0.0, -6.0, -6.0], [L_BOX, L_BOX, 6.0, 6.0], dt, nbiter, idcase)


def _ctx(pkg, dom, dtype, kernels=""):
    old = os.environ.get("VLP4D_KERNELS")
    os.environ["VLP4D_KERNELS"] = kernels
    try:
        return pkg.Context(dom, dtype)
    finally:
        if old is None:
            del os.environ["VLP4D_KERNELS"]
        else:
            os.environ["VLP4D_KERNELS"] = old


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


# Shapes the fused kernels take, shapes they decline (generic path), thin planes.
SHAPES = [((8, 8, 8, 8), ""), ((16, 4, 16, 4), ""), ((12, 10, 14, 10), ""), ((16, 16, 16, 16), "generic"),
          ((32, 16, 32, 24), "")]


@pytest.mark.parametrize("n,kernels", SHAPES)
def test_step_adjoint_matches_cpu_adjoint(pkg, cuda, n, kernels):
    torch = cuda
    dom = _dom(pkg, n)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, dom.idcase)
    f0 = ora.init_case(IC_LANDAU_SUM, 0.05, 0.5)
    f1 = ora.step(f0)  # a state with a nonzero field
    rng = np.random.default_rng(11)
    lam = rng.normal(size=ora.shape4)
    ref = ora.step_adjoint(f1, lam)
    with _ctx(pkg, dom, "f64", kernels) as ctx, pkg.Adjoint(ctx, 1, 1) as adj:
        out = ctx.empty_f()
        adj.step_adjoint(torch.from_numpy(f1).cuda(), torch.from_numpy(lam).cuda(), out)
        assert _rel(out.cpu().numpy(), ref) < 1e-11
        J, g = ora.energy_grad(f1)
        lam_d = ctx.empty_f()
        Jd = adj.energy_grad(torch.from_numpy(f1).cuda(), lam_d)
        assert abs(Jd - J) <= 1e-12 * J
        assert _rel(lam_d.cpu().numpy(), g) < 1e-11
        ctx.check()


@pytest.mark.parametrize("every", [1, 3, 8, 0])
def test_checkpointed_run_gradient_matches_cpu_adjoint(pkg, cuda, every):
    """every = 0: the forward run stores every step's stage input and field,
    the reverse run recomputes nothing."""
    torch = cuda
    n, nsteps = (16, 8, 16, 12), 7
    dom = _dom(pkg, n, nbiter=nsteps)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, dom.idcase)
    f0 = ora.init_case(IC_LANDAU_SUM, 0.05, 0.5)
    J_ref, g_ref = ora.adjoint_run(f0, nsteps)
    with _ctx(pkg, dom, "f64") as ctx, pkg.Adjoint(ctx, nsteps, every) as adj:
        J = adj.forward(torch.from_numpy(f0).cuda())
        g = adj.backward().cpu().numpy()
    assert abs(J - J_ref) <= 1e-11 * J_ref
    assert _rel(g, g_ref) < 1e-10


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_store_all_run_equals_one_segment_run(pkg, cuda, dtype):
    """every = 0 runs the forward sweep of a single checkpoint segment
    (every = nsteps) and stores what that segment's recomputation would
    store: J, the final state and the gradient are bit-identical."""
    torch = cuda
    n, nsteps = (32, 16, 32, 24), 9
    dom = _dom(pkg, n, nbiter=nsteps)
    res = []
    for every in (nsteps, 0):
        with pkg.Context(dom, dtype) as ctx, pkg.Adjoint(ctx, nsteps, every) as adj:
            f0 = ctx.empty_f()
            ctx.init_case(f0, IC_LANDAU_SUM, 0.05, 0.5)
            fN = ctx.empty_f()
            for _ in range(2):  # the second call through the cached graphs
                J = adj.forward(f0, fN)
                g = adj.backward()
            res.append((J, fN.cpu(), g.cpu()))
    assert res[0][0] == res[1][0]
    assert torch.equal(res[0][1], res[1][1])
    assert torch.equal(res[0][2], res[1][2])


def _landau_eps_f0(torch, n, eps, k=0.5, vmax=6.0, dtype=None):
    """f0 = M(v) (1 + E(x, y) (cos kx + cos ky)), E = eps (m x m) upsampled to
    n x n by nearest neighbour, on x, y in [0, 2 pi / k), v in [-vmax, vmax)."""
    L = 2 * math.pi / k
    dev = eps.device
    x = torch.arange(n, dtype=torch.float64, device=dev) * (L / n)
    v = -vmax + torch.arange(n, dtype=torch.float64, device=dev) * (2 * vmax / n)
    rep = n // eps.shape[0]
    e = eps.repeat_interleave(rep, 0).repeat_interleave(rep, 1)  # (ny, nx)
    pert = 1 + e * (torch.cos(k * x)[None, :] + torch.cos(k * x)[:, None])
    m = torch.exp(-0.5 * v * v) / math.sqrt(2 * math.pi)
    f = m[:, None, None, None] * m[None, :, None, None] * pert[None, None, :, :]
    return f if dtype is None else f.to(dtype)


def test_energy_gradient_wrt_perturbation_field_fd_and_fp32(pkg, cuda):
    """The adjoint configuration: Landau 64^4, T = 20 (200 steps of 0.1), the
    gradient of the final electric energy with respect to a 32 x 32
    perturbation-amplitude field eps ~ U[0.02, 0.08] (seeded), checkpoints
    every 8 steps; FP64 against central differences (h = 1e-4) and FP32-f
    against FP64."""
    torch = cuda
    n, nsteps = 64, 200
    dom = pkg.landau_domain(n, dt=0.1, nbiter=nsteps, idcase=110)
    gen = torch.Generator().manual_seed(20261203)
    eps = (0.02 + 0.06 * torch.rand((32, 32), generator=gen, dtype=torch.float64)).cuda()
    grads = {}
    for dtype, tdt in (("f64", torch.float64), ("f32", torch.float32)):
        with pkg.Context(dom, dtype) as ctx, pkg.Adjoint(ctx, nsteps, 8) as adj:
            e = eps.clone().requires_grad_(True)
            J = pkg.vlp4d.energy_after_steps(_landau_eps_f0(torch, n, e, dtype=tdt), adj)
            J.backward()
            grads[dtype] = e.grad.detach().cpu().numpy()
            if dtype == "f64":
                rng = np.random.default_rng(7)
                h = 1e-4
                for idx in [tuple(rng.integers(0, 32, 2)) for _ in range(3)]:
                    def J_at(delta):
                        ep = eps.clone()
                        ep[idx] += delta
                        return adj.forward(_landau_eps_f0(torch, n, ep).contiguous())
                    fd = (J_at(h) - J_at(-h)) / (2 * h)
                    g = grads["f64"][idx]
                    assert abs(g - fd) <= 1e-5 * abs(fd) + 1e-12 * abs(J.item()), (idx, g, fd)
    g64, g32 = grads["f64"], grads["f32"]
    assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_graph_and_eager_reverse_sweeps_agree(pkg, cuda, dtype):
    """The forward and reverse sweeps run as captured CUDA graphs by default;
    VLP4D_ADJOINT_GRAPHS=0 runs them eagerly.  Same kernels, same order: the
    results are bit-identical, also on a second call through the cached graphs."""
    torch = cuda
    n, nsteps = (32, 16, 32, 24), 10
    dom = _dom(pkg, n, nbiter=nsteps)
    res = []
    for graphs in ("1", "0"):
        os.environ["VLP4D_ADJOINT_GRAPHS"] = graphs
        try:
            with pkg.Context(dom, dtype) as ctx, pkg.Adjoint(ctx, nsteps, 4) as adj:
                f0 = ctx.empty_f()
                ctx.init_case(f0, IC_LANDAU_SUM, 0.05, 0.5)
                for _ in range(2):
                    J = adj.forward(f0)
                    g = adj.backward()
                res.append((J, g.cpu()))
        finally:
            del os.environ["VLP4D_ADJOINT_GRAPHS"]
    assert res[0][0] == res[1][0]
    assert torch.equal(res[0][1], res[1][1])


@pytest.mark.parametrize("n", [(32, 16, 32, 24), (16, 8, 16, 8), (64, 64, 16, 16)])
def test_cluster_and_cufft_field_solves_give_the_same_reverse_step(pkg, cuda, n):
    """The reverse step through the cluster solves (forward D and D^T in one
    cluster launch each) and through the cuFFT path (VLP4D_FIELD=cufft)
    agree to FP64 rounding of the transforms."""
    torch = cuda
    dom = _dom(pkg, n)
    ora = Restatement(dom.nxmax, dom.min_phy, dom.max_phy, dom.dt, dom.idcase)
    f1 = ora.step(ora.init_case(IC_LANDAU_SUM, 0.05, 0.5))
    lam = np.random.default_rng(3).normal(size=ora.shape4)
    outs = []
    for mode in ("", "cufft"):
        os.environ["VLP4D_FIELD"] = mode
        try:
            with pkg.Context(dom, "f64") as ctx, pkg.Adjoint(ctx, 1, 1) as adj:
                out = ctx.empty_f()
                adj.step_adjoint(torch.from_numpy(f1).cuda(), torch.from_numpy(lam).cuda(), out)
                torch.cuda.synchronize()
                ctx.check()
                outs.append(out.cpu().numpy())
        finally:
            del os.environ["VLP4D_FIELD"]
    assert _rel(outs[0], outs[1]) < 1e-12
