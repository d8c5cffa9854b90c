"""CPU stand-in of a vy-slab context for the decomposition tests.

Implements the stage methods that distrib.SlabRun calls on a slab context
(the C ABI's vlp4d_ctx_create_slab contexts on the GPU) with the CPU oracle
(oracle/vlp4d_oracle.c), on torch CPU tensors so that gloo can exchange
them.  Test infrastructure only: the product path is the CUDA library.

The oracle works on whole periodic domains, so a slab's stages run on
sub-domains: the owned planes (vy in [vymin + ivy0*dvy, vymin + (ivy0 +
nloc)*dvy)) for x, y, vx and the moment, and owned planes plus halos for
the vy sweep, whose interior outputs then read exactly the global taps
(the sub-domain's periodic wrap only reaches the halo outputs, which are
discarded).  The sub-domains' dvy = width / n rounds differently from the
global one in the last bit, so results equal the one-domain oracle to
rounding, not bit for bit."""
from __future__ import annotations

import numpy as np
import torch

from oracle.oracle import Restatement


class CpuSlabContext:
    def __init__(self, n, minp, maxp, dt, idcase, ivy0, nloc, halo):
        self.n = tuple(int(v) for v in n)
        nx, ny, nvx, nvy = self.n
        self.ivy0, self.nvy_local, self.halo = ivy0, nloc, halo
        self.glob = Restatement(self.n, minp, maxp, dt, idcase)
        dvy = (maxp[3] - minp[3]) / nvy
        own_min, own_max = list(minp), list(maxp)
        own_min[3], own_max[3] = minp[3] + ivy0 * dvy, minp[3] + (ivy0 + nloc) * dvy
        self.own = Restatement((nx, ny, nvx, nloc), own_min, own_max, dt, idcase)
        ext_min, ext_max = list(minp), list(maxp)
        ext_min[3], ext_max[3] = minp[3] + (ivy0 - halo) * dvy, minp[3] + (ivy0 + nloc + halo) * dvy
        self.ext = Restatement((nx, ny, nvx, nloc + 2 * halo), ext_min, ext_max, dt, idcase)
        self.f_shape = (nloc + 2 * halo, nvx, ny, nx)
        self.rho = torch.zeros((ny, nx), dtype=torch.float64)
        self.ex = np.zeros((ny, nx))
        self.ey = np.zeros((ny, nx))
        self.nrj, self.mass = {}, {}

    def empty_f(self):
        return torch.full(self.f_shape, float("nan"), dtype=torch.float64)

    def owned(self, f):
        return f[self.halo:self.halo + self.nvy_local]

    def _own(self, f):
        return self.owned(f).numpy()

    def set_owned_from_global(self, f, f_glob):
        self.owned(f).copy_(torch.from_numpy(np.ascontiguousarray(f_glob[self.ivy0:self.ivy0 + self.nvy_local])))

    # -- stages (same names and meaning as the Context methods)
    def field_rho(self, f):
        self.rho.copy_(torch.from_numpy(self.own.field_rho(self._own(f))))

    def field_poisson(self):
        phi, self.ex, self.ey = self.glob.field_poisson(self.rho.numpy())
        self.rho.copy_(torch.from_numpy(phi))  # rho holds phi afterwards, as in the reference

    def diags_compute(self, it):
        self.nrj[it], self.mass[it] = self.glob.diags(self.rho.numpy(), self.ex, self.ey)

    def advect_xy(self, fn, fnp1, dt):
        out = self.own.advect_y(self.own.advect_x(self._own(fn), dt), dt)
        self.owned(fnp1).copy_(torch.from_numpy(out))

    def advect_xy_moment(self, fn, fnp1, dt):
        self.advect_xy(fn, fnp1, dt)
        self.field_rho(fnp1)

    def advect_xyxy(self, fn, fnp1, dt):
        tmp = self.empty_f()
        self.advect_xy(fn, tmp, dt)
        self.advect_xy_moment(tmp, fnp1, dt)

    def advect_vxvy(self, fn, fnp1, dt):
        a = self.ext.advect_vx(fn.numpy(), self.ex, dt)
        b = self.ext.advect_vy(a, self.ey, dt)
        self.owned(fnp1).copy_(torch.from_numpy(b[self.halo:self.halo + self.nvy_local]))
