"""Test infrastructure: ctypes access to the two CPU checkers.

* ``Restatement`` wraps ``oracle/_build/liboracle_vlp4d.so`` (vlp4d_oracle.c),
  the plain-C restatement of the reference's algorithm.
* ``Reference`` wraps ``oracle/_ref/libvlp4d_ref.so``: the reference's own
  OpenMP vlp4d (miniapps/vlp4d/openmp) compiled from its sources by
  oracle/Makefile, driven through oracle/ref_driver.cpp.

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

IC_CYL02, IC_CYL05, IC_SLD10, IC_TSI20, IC_LANDAU_SUM, IC_TWO_STREAM = 2, 5, 10, 20, 110, 120

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
