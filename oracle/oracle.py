"""Test infrastructure: ctypes access to the two CPU checkers.

* ``Restatement`` wraps ``oracle/_build/liboracle_vlp4d.so`` (vlp4d_oracle.c),
  the plain-C restatement of the reference's algorithm.
* ``Reference`` wraps ``oracle/_ref/libvlp4d_ref.so``: the reference's own
  OpenMP vlp4d (miniapps/vlp4d/openmp) compiled from its sources by
  oracle/Makefile, driven through oracle/ref_driver.cpp.
* ``MpiRestatement`` wraps the restatement of the one-process vlp4d_mpi
  step (vlp4d_mpi_oracle.c, in the same library as ``Restatement``);
  ``MpiReference`` wraps ``oracle/_ref/libvlp4d_mpi_ref.so``, the
  reference's own OpenMP vlp4d_mpi (miniapps/vlp4d_mpi/openmp) driven
  through oracle/ref_mpi_driver.cpp.  Their 4D arrays are the reference's
  halo-extended views: numpy shape (nvy+6, nvx+6, ny+6, nx+6), index 3 is
  grid point 0.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module; the CUDA library never does.  Arrays are numpy float64 in the
reference's layout_left order, i.e. numpy arrays of shape (nvy, nvx, ny, nx)
in C order (``f[ivy, ivx, iy, ix]``), 2D fields of shape (ny, nx).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
RESTATEMENT_SO = HERE / "_build" / "liboracle_vlp4d.so"
REFERENCE_SO = HERE / "_ref" / "libvlp4d_ref.so"
REFERENCE_EXE = HERE / "_ref" / "vlp4d_ref"
MPI_REFERENCE_SO = HERE / "_ref" / "libvlp4d_mpi_ref.so"
HALO = 3

IC_CYL02, IC_CYL05, IC_SLD10, IC_TSI20, IC_LANDAU_SUM, IC_TWO_STREAM = 2, 5, 10, 20, 110, 120
IC_TSI20_MPI = 21

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build(reference: bool = True) -> None:
    """Compile the restatement (and the reference, when its tree is present)."""
    target = "all" if reference else "restatement"
    subprocess.run(["make", "-s", "-C", str(HERE), target], check=True)


class _Domain(C.Structure):
    _fields_ = [
        ("n", C.c_int * 4),
        ("minp", C.c_double * 4),
        ("maxp", C.c_double * 4),
        ("dx", C.c_double * 4),
        ("dt", C.c_double),
        ("idcase", C.c_int),
    ]


def _c_arr(t, vals):
    return (t * len(vals))(*vals)


class Restatement:
    """The plain-C restatement of miniapps/vlp4d/openmp (one domain)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not RESTATEMENT_SO.exists():
                build(reference=False)
            lib = C.CDLL(str(RESTATEMENT_SO))
            P = C.POINTER(_Domain)
            lib.orc_domain_init.argtypes = [P, C.c_int * 4, C.c_double * 4, C.c_double * 4, C.c_double, C.c_int]
            lib.orc_lag_basis5.argtypes = [C.c_double, _dp]
            for name in ("orc_advect_x", "orc_advect_y"):
                getattr(lib, name).argtypes = [P, _dp, _dp, C.c_double]
            for name in ("orc_advect_vx", "orc_advect_vy"):
                getattr(lib, name).argtypes = [P, _dp, _dp, _dp, C.c_double]
            lib.orc_field_rho.argtypes = [P, _dp, _dp]
            lib.orc_field_poisson.argtypes = [P, _dp, _dp, _dp]
            lib.orc_diags.argtypes = [P, _dp, _dp, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
            lib.orc_rfft2.argtypes = [C.c_int, C.c_int, _dp, _dp]
            lib.orc_irfft2.argtypes = [C.c_int, C.c_int, _dp, _dp]
            lib.orc_step.argtypes = [P, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
            lib.orc_diags_mpi.argtypes = [P, _dp, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
            lib.orc_l2norm.argtypes = [P, _dp]
            lib.orc_l2norm.restype = C.c_double
            lib.orc_run.argtypes = [P, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp]
            lib.orc_init_case.argtypes = [P, _dp, C.c_int, C.c_double, C.c_double, C.c_double]
            # FP64 discrete adjoint (vlp4d_adjoint.c).
            lib.orc_lag_basis5_deriv.argtypes = [C.c_double, _dp]
            for name in ("orc_advect_x_T", "orc_advect_y_T"):
                getattr(lib, name).argtypes = [P, _dp, _dp, C.c_double]
            for name in ("orc_advect_vx_T", "orc_advect_vy_T"):
                getattr(lib, name).argtypes = [P, _dp, _dp, _dp, C.c_double, _dp, _dp]
            lib.orc_field_poisson_T.argtypes = [P, _dp, _dp, _dp]
            lib.orc_energy_grad.argtypes = [P, _dp, C.POINTER(C.c_double), _dp]
            lib.orc_step_adjoint.argtypes = [P, _dp, _dp, _dp]
            lib.orc_adjoint_run.argtypes = [P, _dp, C.c_int, C.POINTER(C.c_double), _dp]
            # One-process vlp4d_mpi step (vlp4d_mpi_oracle.c).
            lib.orcm_size.argtypes = [P]
            lib.orcm_size.restype = C.c_size_t
            for name in ("orcm_halo_fill", "orcm_spline_xy", "orcm_spline_vxvy"):
                getattr(lib, name).argtypes = [P, _dp]
            lib.orcm_advect_2d.argtypes = [P, _dp, _dp, C.c_double]
            lib.orcm_advect_2d.restype = C.c_int
            lib.orcm_advect_4d.argtypes = [P, _dp, _dp, _dp, _dp]
            lib.orcm_advect_4d.restype = C.c_int
            lib.orcm_field_rho.argtypes = [P, _dp, _dp]
            lib.orcm_l2norm.argtypes = [P, _dp]
            lib.orcm_l2norm.restype = C.c_double
            lib.orcm_start.argtypes = [P, _dp, _dp, _dp, _dp, _dp]
            lib.orcm_step.argtypes = [P, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
            lib.orcm_step.restype = C.c_int
            lib.orcm_init_case.argtypes = [P, _dp, C.c_int]
            cls._lib = lib
        return cls._lib

    def __init__(self, n, minp, maxp, dt, idcase=10):
        self.L = self.lib()
        self.d = _Domain()
        self.L.orc_domain_init(C.byref(self.d), _c_arr(C.c_int, n), _c_arr(C.c_double, minp),
                               _c_arr(C.c_double, maxp), dt, idcase)
        self.n = tuple(int(v) for v in n)
        self.shape4 = (self.n[3], self.n[2], self.n[1], self.n[0])
        self.shape2 = (self.n[1], self.n[0])

    @property
    def dx(self):
        return tuple(self.d.dx)

    def empty4(self):
        return np.zeros(self.shape4, dtype=np.float64)

    def empty2(self):
        return np.zeros(self.shape2, dtype=np.float64)

    def init_case(self, ic, amp=0.05, k=0.5, u=2.4):
        f = self.empty4()
        self.L.orc_init_case(C.byref(self.d), f, ic, amp, k, u)
        return f

    def lag_basis(self, px):
        c = np.zeros(6)
        self.L.orc_lag_basis5(px, c)
        return c

    def advect_x(self, f, dt):
        out = self.empty4()
        self.L.orc_advect_x(C.byref(self.d), np.ascontiguousarray(f), out, dt)
        return out

    def advect_y(self, f, dt):
        out = self.empty4()
        self.L.orc_advect_y(C.byref(self.d), np.ascontiguousarray(f), out, dt)
        return out

    def advect_vx(self, f, ex, dt):
        out = self.empty4()
        self.L.orc_advect_vx(C.byref(self.d), np.ascontiguousarray(f), out, np.ascontiguousarray(ex), dt)
        return out

    def advect_vy(self, f, ey, dt):
        out = self.empty4()
        self.L.orc_advect_vy(C.byref(self.d), np.ascontiguousarray(f), out, np.ascontiguousarray(ey), dt)
        return out

    def field_rho(self, f):
        rho = self.empty2()
        self.L.orc_field_rho(C.byref(self.d), np.ascontiguousarray(f), rho)
        return rho

    def field_poisson(self, rho):
        """Returns (phi, ex, ey); the input is not modified."""
        phi = np.array(rho, dtype=np.float64, copy=True)
        ex, ey = self.empty2(), self.empty2()
        self.L.orc_field_poisson(C.byref(self.d), phi, ex, ey)
        return phi, ex, ey

    def diags(self, rho, ex, ey):
        nrj, mass = C.c_double(), C.c_double()
        self.L.orc_diags(C.byref(self.d), np.ascontiguousarray(rho), np.ascontiguousarray(ex),
                         np.ascontiguousarray(ey), C.byref(nrj), C.byref(mass))
        return nrj.value, mass.value

    def diags_mpi(self, ex, ey):
        """(nrjx, nrjy) of miniapps/vlp4d_mpi/thrust/Diags.cpp:63-64."""
        a, b = C.c_double(), C.c_double()
        self.L.orc_diags_mpi(C.byref(self.d), np.ascontiguousarray(ex), np.ascontiguousarray(ey), C.byref(a), C.byref(b))
        return a.value, b.value

    def l2norm(self, f):
        return self.L.orc_l2norm(C.byref(self.d), np.ascontiguousarray(f, dtype=np.float64))

    def rfft2(self, a):
        ny, nx = a.shape
        hat = np.zeros((ny, nx // 2 + 1, 2))
        self.L.orc_rfft2(nx, ny, np.ascontiguousarray(a, dtype=np.float64), hat)
        return hat[..., 0] + 1j * hat[..., 1]

    def irfft2(self, hat, nx):
        ny = hat.shape[0]
        buf = np.ascontiguousarray(np.stack([hat.real, hat.imag], axis=-1))
        out = np.zeros((ny, nx))
        self.L.orc_irfft2(nx, ny, buf, out)
        return out

    # ---- FP64 discrete adjoint (oracle/vlp4d_adjoint.c) ----

    def lag_basis_deriv(self, px):
        c = np.zeros(6)
        self.L.orc_lag_basis5_deriv(px, c)
        return c

    def advect_x_T(self, lam, dt):
        out = self.empty4()
        self.L.orc_advect_x_T(C.byref(self.d), np.ascontiguousarray(lam), out, dt)
        return out

    def advect_y_T(self, lam, dt):
        out = self.empty4()
        self.L.orc_advect_y_T(C.byref(self.d), np.ascontiguousarray(lam), out, dt)
        return out

    def advect_vx_T(self, lam, f_in, ex, dt):
        """Returns (A^T lam, dJ/dEx) for the vx stage evaluated at its input f_in."""
        out, g = self.empty4(), self.empty2()
        self.L.orc_advect_vx_T(C.byref(self.d), np.ascontiguousarray(lam), np.ascontiguousarray(f_in),
                               np.ascontiguousarray(ex), dt, out, g)
        return out, g

    def advect_vy_T(self, lam, f_in, ey, dt):
        out, g = self.empty4(), self.empty2()
        self.L.orc_advect_vy_T(C.byref(self.d), np.ascontiguousarray(lam), np.ascontiguousarray(f_in),
                               np.ascontiguousarray(ey), dt, out, g)
        return out, g

    def field_poisson_T(self, gex, gey):
        out = self.empty2()
        self.L.orc_field_poisson_T(C.byref(self.d), np.ascontiguousarray(gex), np.ascontiguousarray(gey), out)
        return out

    def energy_grad(self, f):
        """J = dx dy sum |E|^2 of the field solved from f, and dJ/df."""
        J = C.c_double()
        lam = self.empty4()
        self.L.orc_energy_grad(C.byref(self.d), np.ascontiguousarray(f), C.byref(J), lam)
        return J.value, lam

    def step_adjoint(self, f_state, lam_next):
        out = self.empty4()
        self.L.orc_step_adjoint(C.byref(self.d), np.ascontiguousarray(f_state), np.ascontiguousarray(lam_next), out)
        return out

    def adjoint_run(self, f0, nsteps):
        """J(f after nsteps steps) and dJ/df0."""
        J = C.c_double()
        grad = self.empty4()
        self.L.orc_adjoint_run(C.byref(self.d), np.ascontiguousarray(f0, dtype=np.float64), nsteps, C.byref(J), grad)
        return J.value, grad

    def step(self, f):
        """One Strang step of f (diagnostics discarded)."""
        fn = np.array(f, dtype=np.float64, copy=True)
        fnp1 = self.empty4()
        rho, ex, ey = self.empty2(), self.empty2(), self.empty2()
        nrj, mass = C.c_double(), C.c_double()
        self.L.orc_step(C.byref(self.d), fn, fnp1, rho, ex, ey, C.byref(nrj), C.byref(mass))
        return fn

    def energy(self, f):
        _, ex, ey = self.field_poisson(self.field_rho(f))
        return float((ex * ex + ey * ey).sum() * self.dx[0] * self.dx[1])

    def run(self, f0, nsteps):
        """Initial solve + nsteps Strang steps; returns (f, nrj[nsteps+1], mass[nsteps+1], ex, ey)."""
        fn = np.array(f0, dtype=np.float64, copy=True)
        fnp1 = self.empty4()
        rho, ex, ey = self.empty2(), self.empty2(), self.empty2()
        nrj = np.zeros(nsteps + 1)
        mass = np.zeros(nsteps + 1)
        self.L.orc_run(C.byref(self.d), fn, fnp1, rho, ex, ey, nsteps, nrj, mass)
        return fn, nrj, mass, ex, ey


class Reference:
    """The reference's own OpenMP vlp4d, compiled from its sources (oracle/_ref)."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return REFERENCE_SO.exists()

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = C.CDLL(str(REFERENCE_SO))
            lib.ref_create.restype = C.c_void_p
            lib.ref_create.argtypes = [C.c_int * 4, C.c_double * 4, C.c_double * 4, C.c_double, C.c_int, C.c_int]
            lib.ref_destroy.argtypes = [C.c_void_p]
            for name in ("ref_set_f", "ref_get_f", "ref_set_field", "ref_get_field"):
                getattr(lib, name).argtypes = [C.c_void_p, C.c_int, _dp]
            lib.ref_initcase.argtypes = [C.c_void_p, C.c_int]
            for name in ("ref_advect_x", "ref_advect_y", "ref_advect_vx", "ref_advect_vy"):
                getattr(lib, name).argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
            lib.ref_field_rho.argtypes = [C.c_void_p, C.c_int]
            lib.ref_field_poisson.argtypes = [C.c_void_p]
            lib.ref_diags_compute.argtypes = [C.c_void_p, C.c_int]
            lib.ref_diags_save.argtypes = [C.c_void_p, C.c_char_p]
            lib.ref_onetimestep.argtypes = [C.c_void_p, C.c_int]
            lib.ref_run.argtypes = [C.c_void_p, C.c_int]
            lib.ref_timer_seconds.restype = C.c_double
            lib.ref_timer_seconds.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
            lib.ref_reset_timers.argtypes = [C.c_void_p]
            lib.ref_rfft2.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp]
            lib.ref_irfft2.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp]
            cls._lib = lib
        return cls._lib

    TIMERS = ("total", "MainLoop", "advec1D_x", "advec1D_y", "advec1D_vx", "advec1D_vy",
              "field", "Fourier", "diag")

    def __init__(self, n, minp, maxp, dt, nbiter, idcase=10):
        self.L = self.lib()
        self.n = tuple(int(v) for v in n)
        self.shape4 = (self.n[3], self.n[2], self.n[1], self.n[0])
        self.shape2 = (self.n[1], self.n[0])
        self.nbiter = nbiter
        self.h = self.L.ref_create(_c_arr(C.c_int, n), _c_arr(C.c_double, minp), _c_arr(C.c_double, maxp),
                                   dt, nbiter, idcase)

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_f(self, which, f):
        self.L.ref_set_f(self.h, which, np.ascontiguousarray(f, dtype=np.float64))

    def get_f(self, which):
        out = np.zeros(self.shape4)
        self.L.ref_get_f(self.h, which, out)
        return out

    def set_field(self, which, a):
        self.L.ref_set_field(self.h, which, np.ascontiguousarray(a, dtype=np.float64))

    def get_field(self, which):
        out = np.zeros(self.shape2)
        self.L.ref_get_field(self.h, which, out)
        return out

    def initcase(self, which=0):
        self.L.ref_initcase(self.h, which)

    def advect_x(self, src, dst, dt):
        self.L.ref_advect_x(self.h, src, dst, dt)

    def advect_y(self, src, dst, dt):
        self.L.ref_advect_y(self.h, src, dst, dt)

    def advect_vx(self, src, dst, dt):
        self.L.ref_advect_vx(self.h, src, dst, dt)

    def advect_vy(self, src, dst, dt):
        self.L.ref_advect_vy(self.h, src, dst, dt)

    def field_rho(self, src=0):
        self.L.ref_field_rho(self.h, src)

    def field_poisson(self):
        self.L.ref_field_poisson(self.h)

    def diags_compute(self, it):
        self.L.ref_diags_compute(self.h, it)

    def diags(self):
        """nrj.out as written by Diags::save: rows (t, nrj, mass), nbiter+1 rows."""
        with tempfile.TemporaryDirectory() as d:
            rc = self.L.ref_diags_save(self.h, d.encode())
            if rc != 0:
                raise RuntimeError(f"ref_diags_save failed ({rc})")
            return np.loadtxt(os.path.join(d, "nrj.out"), ndmin=2)

    def onetimestep(self, it):
        self.L.ref_onetimestep(self.h, it)

    def run(self, nsteps):
        self.L.ref_run(self.h, nsteps)

    def timers(self):
        out = {}
        for i, name in enumerate(self.TIMERS):
            calls = C.c_int()
            s = self.L.ref_timer_seconds(self.h, i, C.byref(calls))
            out[name] = (s, calls.value)
        return out

    def reset_timers(self):
        self.L.ref_reset_timers(self.h)

    @classmethod
    def rfft2(cls, a3):
        """a3: (batch, ny, nx) float64 -> (batch, ny, nx//2+1) complex via Impl::FFT."""
        L = cls.lib()
        nb, ny, nx = a3.shape
        src = np.ascontiguousarray(a3, dtype=np.float64).copy()
        out = np.zeros((nb, ny, nx // 2 + 1, 2))
        L.ref_rfft2(nx, ny, nb, src, out)
        return out[..., 0] + 1j * out[..., 1]

    @classmethod
    def irfft2(cls, hat3, nx):
        L = cls.lib()
        nb, ny, _ = hat3.shape
        src = np.ascontiguousarray(np.stack([hat3.real, hat3.imag], axis=-1))
        out = np.zeros((nb, ny, nx))
        L.ref_irfft2(nx, ny, nb, src, out)
        return out


def interior(fh):
    """The grid points of a halo-extended array (a view)."""
    return fh[HALO:-HALO, HALO:-HALO, HALO:-HALO, HALO:-HALO]


class MpiRestatement(Restatement):
    """The plain-C restatement of the one-process vlp4d_mpi step."""

    def __init__(self, n, minp, maxp, dt, idcase=10):
        super().__init__(n, minp, maxp, dt, idcase)
        self.hshape4 = tuple(v + 2 * HALO for v in self.shape4)

    def empty_halo(self):
        return np.zeros(self.hshape4, dtype=np.float64)

    def init_halo(self, ic):
        fh = self.empty_halo()
        self.L.orcm_init_case(C.byref(self.d), fh, ic)
        return fh

    def halo_fill(self, fh):
        out = np.array(fh, dtype=np.float64, copy=True)
        self.L.orcm_halo_fill(C.byref(self.d), out)
        return out

    def spline_xy(self, fh):
        out = np.array(fh, dtype=np.float64, copy=True)
        self.L.orcm_spline_xy(C.byref(self.d), out)
        return out

    def spline_vxvy(self, fh):
        out = np.array(fh, dtype=np.float64, copy=True)
        self.L.orcm_spline_vxvy(C.byref(self.d), out)
        return out

    def advect_2d(self, coef, dt):
        """(values on the interior + coef's halo, out-of-range count)."""
        out = np.array(coef, dtype=np.float64, copy=True)
        tmp = self.empty_halo()
        err = self.L.orcm_advect_2d(C.byref(self.d), out, tmp, dt)
        return out, err

    def advect_4d(self, coef, ex, ey):
        out = np.array(coef, dtype=np.float64, copy=True)
        tmp = self.empty_halo()
        err = self.L.orcm_advect_4d(C.byref(self.d), np.ascontiguousarray(ex), np.ascontiguousarray(ey), out, tmp)
        return out, err

    def field_rho_halo(self, fh):
        rho = self.empty2()
        self.L.orcm_field_rho(C.byref(self.d), np.ascontiguousarray(fh), rho)
        return rho

    def l2norm_halo(self, fh):
        return float(self.L.orcm_l2norm(C.byref(self.d), np.ascontiguousarray(fh)))

    def start(self, fh):
        """Initial field and diagnostics: (phi, ex, ey, [nrj, nrjx, nrjy, mass, l2norm])."""
        rho, ex, ey = self.empty2(), self.empty2(), self.empty2()
        out = np.zeros(5)
        self.L.orcm_start(C.byref(self.d), np.ascontiguousarray(fh), rho, ex, ey, out)
        return rho, ex, ey, out

    def step_mpi(self, fh):
        """One step: (new state, ex, ey, half-step diags[4], end diags[5], out-of-range count)."""
        fn = np.array(fh, dtype=np.float64, copy=True)
        fnp1, tmp = self.empty_halo(), self.empty_halo()
        rho, ex, ey = self.empty2(), self.empty2(), self.empty2()
        half, out = np.zeros(4), np.zeros(5)
        err = self.L.orcm_step(C.byref(self.d), fn, fnp1, tmp, rho, ex, ey, half, out)
        return fn, ex, ey, half, out, err

    def run_mpi(self, fh, nsteps):
        """Initial solve + nsteps steps: (state, diags[nsteps+1, 5], ex, ey)."""
        f = np.array(fh, dtype=np.float64, copy=True)
        _, ex, ey, out = self.start(f)
        rows = [out]
        for _ in range(nsteps):
            f, ex, ey, _, out, err = self.step_mpi(f)
            if err:
                raise RuntimeError("time step too large for the interpolation range")
            rows.append(out)
        return f, np.array(rows), ex, ey


class MpiReference:
    """The reference's own OpenMP vlp4d_mpi as one process (oracle/_ref)."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return MPI_REFERENCE_SO.exists()

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = C.CDLL(str(MPI_REFERENCE_SO))
            lib.refm_create.restype = C.c_void_p
            lib.refm_create.argtypes = [C.c_int * 4, C.c_double * 4, C.c_double * 4, C.c_double, C.c_int, C.c_int]
            lib.refm_destroy.argtypes = [C.c_void_p]
            for name in ("refm_set_f", "refm_get_f", "refm_set_field", "refm_get_field"):
                getattr(lib, name).argtypes = [C.c_void_p, C.c_int, _dp]
            for name in ("refm_initcase", "refm_exchange_halo", "refm_spline_xy", "refm_spline_vxvy",
                         "refm_field", "refm_l2norm"):
                getattr(lib, name).argtypes = [C.c_void_p, C.c_int] + ([C.c_int] if name == "refm_l2norm" else [])
            lib.refm_advect_2d.argtypes = [C.c_void_p, C.c_int, C.c_double]
            lib.refm_advect_4d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
            lib.refm_diags.argtypes = [C.c_void_p, C.c_int]
            lib.refm_diags_save.argtypes = [C.c_void_p, C.c_char_p]
            lib.refm_onetimestep.argtypes = [C.c_void_p, C.c_int]
            lib.refm_run.argtypes = [C.c_void_p, C.c_int]
            lib.refm_timer_seconds.restype = C.c_double
            lib.refm_timer_seconds.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
            lib.refm_reset_timers.argtypes = [C.c_void_p]
            lib.refm_max_threads.restype = C.c_int
            cls._lib = lib
        return cls._lib

    TIMERS = ("total", "MainLoop", "pack", "comm", "unpack", "advec2D", "advec4D", "field", "all_reduce",
              "Fourier", "diag", "splinecoeff_xy", "splinecoeff_vxvy")

    def __init__(self, n, minp, maxp, dt, nbiter, idcase=10):
        self.L = self.lib()
        self.n = tuple(int(v) for v in n)
        self.hshape4 = (self.n[3] + 2 * HALO, self.n[2] + 2 * HALO, self.n[1] + 2 * HALO, self.n[0] + 2 * HALO)
        self.shape2 = (self.n[1], self.n[0])
        self.nbiter = nbiter
        self.h = self.L.refm_create(_c_arr(C.c_int, n), _c_arr(C.c_double, minp), _c_arr(C.c_double, maxp),
                                    dt, nbiter, idcase)

    def close(self):
        if self.h:
            self.L.refm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_f(self, which, fh):
        self.L.refm_set_f(self.h, which, np.ascontiguousarray(fh, dtype=np.float64))

    def get_f(self, which):
        out = np.zeros(self.hshape4)
        self.L.refm_get_f(self.h, which, out)
        return out

    def set_field(self, which, a):
        self.L.refm_set_field(self.h, which, np.ascontiguousarray(a, dtype=np.float64))

    def get_field(self, which):
        out = np.zeros(self.shape2)
        self.L.refm_get_field(self.h, which, out)
        return out

    def exchange_halo(self, which=0):
        self.L.refm_exchange_halo(self.h, which)

    def spline_xy(self, which=0):
        self.L.refm_spline_xy(self.h, which)

    def spline_vxvy(self, which=0):
        self.L.refm_spline_vxvy(self.h, which)

    def advect_2d(self, which, dt):
        self.L.refm_advect_2d(self.h, which, dt)

    def advect_4d(self, dst, src, dt):
        self.L.refm_advect_4d(self.h, dst, src, dt)

    def field(self, which=0):
        self.L.refm_field(self.h, which)

    def diags_compute(self, it):
        self.L.refm_diags(self.h, it)

    def l2norm(self, which, it):
        self.L.refm_l2norm(self.h, which, it)

    def diags(self):
        """(nrj.out rows (t, nrj, nrjx, nrjy, mass), l2norm.out rows (t, l2norm)), nbiter+1 rows each."""
        with tempfile.TemporaryDirectory() as d:
            rc = self.L.refm_diags_save(self.h, d.encode())
            if rc != 0:
                raise RuntimeError(f"refm_diags_save failed ({rc})")
            return (np.loadtxt(os.path.join(d, "nrj.out"), ndmin=2),
                    np.loadtxt(os.path.join(d, "l2norm.out"), ndmin=2))

    def onetimestep(self, it):
        self.L.refm_onetimestep(self.h, it)

    def run(self, nsteps):
        self.L.refm_run(self.h, nsteps)

    def timers(self):
        out = {}
        for i, name in enumerate(self.TIMERS):
            calls = C.c_int()
            s = self.L.refm_timer_seconds(self.h, i, C.byref(calls))
            out[name] = (s, calls.value)
        return out

    def reset_timers(self):
        self.L.refm_reset_timers(self.h)
