"""ctypes binding of libvlp4d_b200 (include/vlp4d_b200.h) over torch CUDA tensors.

Tests and bench.py drive the CUDA library through this module; it adds no
computation of its own.  Device memory and streams come from PyTorch; every
call passes raw device pointers and a cudaStream_t through the C ABI.  If the
library is missing the import-time load raises: there is no CPU fallback.

Arrays use the reference's layout_left order, which for a C-ordered torch
tensor means shape (nvy, nvx, ny, nx) for f and (ny, nx) for 2D fields.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libvlp4d_b200.so"

OK, ERR_INVALID_ARG, ERR_CUDA, ERR_UNSUPPORTED, ERR_NO_DEVICE, ERR_IO, ERR_TIMEOUT, ERR_RANGE = 0, 1, 2, 3, 4, 5, 6, 7
F64, F32 = 0, 1
FIELD_RHO, FIELD_EX, FIELD_EY = 0, 1, 2
IC_CYL02, IC_CYL05, IC_SLD10, IC_TSI20, IC_LANDAU_SUM, IC_TWO_STREAM = 2, 5, 10, 20, 110, 120

# Every symbol include/vlp4d_b200.h declares.
EXPORTS = (
    "vlp4d_read_deck", "vlp4d_ctx_create", "vlp4d_ctx_destroy", "vlp4d_last_error", "vlp4d_ctx_dtype",
    "vlp4d_field_ptr", "vlp4d_init_case", "vlp4d_advect_x", "vlp4d_advect_y", "vlp4d_advect_vx",
    "vlp4d_advect_vy", "vlp4d_advect_xy", "vlp4d_advect_vxvy", "vlp4d_field_rho", "vlp4d_field_poisson",
    "vlp4d_diags_compute", "vlp4d_diags_read", "vlp4d_diags_save", "vlp4d_step", "vlp4d_run",
    "vlp4d_print_fxvx", "vlp4d_transpose", "vlp4d_check", "vlp4d_kernel_launches",
    "vlp4d_field_rho_noalloc", "vlp4d_steps", "vlp4d_advect_xyxy",
    "vlp4d_adjoint_create", "vlp4d_adjoint_destroy", "vlp4d_adjoint_forward", "vlp4d_adjoint_backward",
    "vlp4d_step_adjoint", "vlp4d_energy_grad",
    "vlp4d_ensemble_create", "vlp4d_ensemble_destroy", "vlp4d_ensemble_run", "vlp4d_ensemble_check",
    "vlp4d_ensemble_read", "vlp4d_ensemble_cells", "vlp4d_ensemble_set_tiles", "vlp4d_ensemble_get_tiles",
    "vlp4d_ensemble_autotune", "vlp4d_selftest_wait_timeout", "vlp4d_diags_l2norm", "vlp4d_diags_read_ext",
    "vlp4d_mpi_size", "vlp4d_mpi_init_case", "vlp4d_mpi_halo_fill", "vlp4d_mpi_spline_xy", "vlp4d_mpi_spline_vxvy", "vlp4d_mpi_advect_2d",
    "vlp4d_mpi_advect_4d", "vlp4d_mpi_field", "vlp4d_mpi_l2norm", "vlp4d_mpi_step",
    "vlp4d_ctx_create_slab", "vlp4d_f_size", "vlp4d_slab_info", "vlp4d_advect_xy_moment",
    "vlp4d_ensemble_set_idle_limit", "vlp4d_steps_joins_xy",
)
HALO = 3  # HALO_PTS of the vlp4d_mpi halo-extended arrays


class Vlp4dError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"vlp4d error {code}: {msg}")
        self.code = code


class CDomain(C.Structure):
    _fields_ = [
        ("nxmax", C.c_int32 * 4),
        ("min_phy", C.c_double * 4),
        ("max_phy", C.c_double * 4),
        ("dt", C.c_double),
        ("nbiter", C.c_int32),
        ("ifreq", C.c_int32),
        ("idcase", C.c_int32),
        ("fxvx", C.c_int32),
    ]


class CEnsMember(C.Structure):
    _fields_ = [
        ("n", C.c_int32 * 4),
        ("min_phy", C.c_double * 4),
        ("max_phy", C.c_double * 4),
        ("dt", C.c_double),
        ("amp", C.c_double),
        ("k", C.c_double),
    ]


_lib = None


def build() -> None:
    """Compile libvlp4d_b200.so in-tree (nvcc, sm_100a)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", str(HERE), "lib"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` (no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        vp, dp, i, d = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_double
        L.vlp4d_last_error.restype = C.c_char_p
        L.vlp4d_read_deck.argtypes = [C.c_char_p, C.POINTER(CDomain)]
        L.vlp4d_ctx_create.argtypes = [C.POINTER(CDomain), i, C.POINTER(vp)]
        L.vlp4d_ctx_destroy.argtypes = [vp]
        L.vlp4d_ctx_dtype.argtypes = [vp]
        L.vlp4d_field_ptr.argtypes = [vp, i, C.POINTER(vp)]
        L.vlp4d_init_case.argtypes = [vp, vp, i, d, d, d, vp]
        L.vlp4d_ctx_create_slab.argtypes = [C.POINTER(CDomain), i, i, i, i, C.POINTER(vp)]
        L.vlp4d_f_size.argtypes = [vp]
        L.vlp4d_steps_joins_xy.argtypes = [vp]
        L.vlp4d_slab_info.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
        for n in ("vlp4d_advect_x", "vlp4d_advect_y", "vlp4d_advect_vx", "vlp4d_advect_vy", "vlp4d_advect_xy",
                  "vlp4d_advect_vxvy", "vlp4d_advect_xyxy", "vlp4d_advect_xy_moment"):
            getattr(L, n).argtypes = [vp, vp, vp, d, vp]
        L.vlp4d_field_rho.argtypes = [vp, vp, vp]
        L.vlp4d_field_poisson.argtypes = [vp, vp]
        L.vlp4d_diags_compute.argtypes = [vp, i, vp]
        L.vlp4d_diags_read.argtypes = [vp, dp, dp, i]
        L.vlp4d_diags_save.argtypes = [vp, C.c_char_p]
        L.vlp4d_step.argtypes = [vp, vp, vp, i, vp]
        L.vlp4d_steps.argtypes = [vp, vp, vp, i, i, vp]
        L.vlp4d_run.argtypes = [vp, vp, vp, i, dp, dp, vp, vp, vp]
        L.vlp4d_print_fxvx.argtypes = [vp, vp, C.c_char_p]
        L.vlp4d_transpose.argtypes = [vp, vp, i, i, i, vp]
        L.vlp4d_check.argtypes = [vp]
        L.vlp4d_kernel_launches.argtypes = []
        L.vlp4d_field_rho_noalloc.argtypes = [vp, i, i, i, i, i, d, d, vp, vp]
        L.vlp4d_adjoint_create.argtypes = [vp, i, i, C.POINTER(vp)]
        L.vlp4d_adjoint_destroy.argtypes = [vp]
        L.vlp4d_adjoint_forward.argtypes = [vp, vp, vp, C.POINTER(d), vp]
        L.vlp4d_adjoint_backward.argtypes = [vp, vp, vp]
        L.vlp4d_step_adjoint.argtypes = [vp, vp, vp, vp, vp]
        L.vlp4d_energy_grad.argtypes = [vp, vp, C.POINTER(d), vp, vp]
        L.vlp4d_ensemble_create.argtypes = [C.POINTER(CEnsMember), i, i, C.POINTER(vp)]
        L.vlp4d_ensemble_destroy.argtypes = [vp]
        L.vlp4d_ensemble_run.argtypes = [vp, vp]
        L.vlp4d_ensemble_check.argtypes = [vp]
        L.vlp4d_ensemble_read.argtypes = [vp, i, vp, dp, vp]
        L.vlp4d_ensemble_cells.argtypes = [vp]
        L.vlp4d_ensemble_set_tiles.argtypes = [vp, i, i, i]
        L.vlp4d_ensemble_get_tiles.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
        L.vlp4d_ensemble_autotune.argtypes = [vp, i, C.c_char_p, vp]
        L.vlp4d_ensemble_set_idle_limit.argtypes = [vp, C.c_longlong]
        L.vlp4d_selftest_wait_timeout.argtypes = [vp, C.c_longlong, vp]
        L.vlp4d_diags_l2norm.argtypes = [vp, vp, i, vp]
        L.vlp4d_diags_read_ext.argtypes = [vp, dp, dp, dp, i]
        L.vlp4d_mpi_size.argtypes = [vp]
        for n in ("vlp4d_mpi_init_case", "vlp4d_mpi_halo_fill", "vlp4d_mpi_spline_xy", "vlp4d_mpi_spline_vxvy",
                  "vlp4d_mpi_field"):
            getattr(L, n).argtypes = [vp, vp, vp]
        L.vlp4d_mpi_advect_2d.argtypes = [vp, vp, vp, d, vp]
        L.vlp4d_mpi_advect_4d.argtypes = [vp, vp, vp, d, vp]
        L.vlp4d_mpi_l2norm.argtypes = [vp, vp, i, vp]
        L.vlp4d_mpi_step.argtypes = [vp, vp, vp, i, vp]
        for n in EXPORTS:
            if n not in ("vlp4d_last_error", "vlp4d_kernel_launches", "vlp4d_ensemble_cells", "vlp4d_mpi_size",
                         "vlp4d_f_size"):
                getattr(L, n).restype = C.c_int
        L.vlp4d_mpi_size.restype = C.c_size_t
        L.vlp4d_f_size.restype = C.c_size_t
        L.vlp4d_ensemble_cells.restype = C.c_longlong
        L.vlp4d_kernel_launches.restype = C.c_ulonglong
        _lib = L
    return _lib


def kernel_launches() -> int:
    """This library's own kernel launches so far in the process."""
    return int(lib().vlp4d_kernel_launches())


def _check(rc: int) -> None:
    if rc != OK:
        msg = lib().vlp4d_last_error()
        raise Vlp4dError(rc, msg.decode() if msg else "")


@dataclass
class Domain:
    """The reference's Domain (miniapps/vlp4d/thrust/config.hpp:8-20)."""

    nxmax: Sequence[int]
    min_phy: Sequence[float]
    max_phy: Sequence[float]
    dt: float
    nbiter: int = 1
    idcase: int = 10
    ifreq: int = 1
    fxvx: int = 0

    @property
    def dx(self):
        return tuple((self.max_phy[i] - self.min_phy[i]) / self.nxmax[i] for i in range(4))

    @property
    def shape4(self):
        nx, ny, nvx, nvy = self.nxmax
        return (nvy, nvx, ny, nx)

    @property
    def shape2(self):
        return (self.nxmax[1], self.nxmax[0])

    @property
    def cells(self) -> int:
        return int(math.prod(self.nxmax))

    def to_c(self) -> CDomain:
        c = CDomain()
        for k in range(4):
            c.nxmax[k] = int(self.nxmax[k])
            c.min_phy[k] = float(self.min_phy[k])
            c.max_phy[k] = float(self.max_phy[k])
        c.dt, c.nbiter, c.idcase, c.ifreq, c.fxvx = float(self.dt), int(self.nbiter), int(self.idcase), int(self.ifreq), int(self.fxvx)
        return c

    @classmethod
    def from_deck(cls, path: str) -> "Domain":
        c = CDomain()
        _check(lib().vlp4d_read_deck(str(path).encode(), C.byref(c)))
        return cls(list(c.nxmax), list(c.min_phy), list(c.max_phy), c.dt, c.nbiter, c.idcase, c.ifreq, c.fxvx)


def landau_domain(n, dt=0.125, nbiter=1, L=4 * math.pi, vmax=6.0, idcase=10) -> Domain:
    """Landau-damping geometry of the benchmark configurations: x, y in [0, L), v in [-vmax, vmax)."""
    if isinstance(n, int):
        n = (n, n, n, n)
    return Domain(list(n), [0.0, 0.0, -vmax, -vmax], [L, L, vmax, vmax], dt, nbiter, idcase)


class _DevArray:
    """Minimal __cuda_array_interface__ wrapper so torch can view a library-owned buffer."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def _stream_ptr(stream) -> Optional[int]:
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


class Context:
    """A vlp4d_ctx: the Efield + Diags state of one run on the current device.

    slab=(ivy0, nvy_local, halo) makes a vy-slab context of the run `dom`
    (vlp4d_ctx_create_slab): it owns the global vy planes
    [ivy0, ivy0 + nvy_local), and its f buffers (empty_f) hold `halo` more
    planes on each side, shape (nvy_local + 2*halo, nvx, ny, nx)."""

    def __init__(self, dom: Domain, dtype: str = "f64", slab=None):
        import torch

        self.dom = dom
        self.dtype_code = F64 if dtype in ("f64", "float64", torch.float64) else F32
        self.torch_dtype = torch.float64 if self.dtype_code == F64 else torch.float32
        self._c = dom.to_c()
        h = C.c_void_p()
        if slab is None:
            _check(lib().vlp4d_ctx_create(C.byref(self._c), self.dtype_code, C.byref(h)))
            self.ivy0, self.nvy_local, self.halo = 0, dom.nxmax[3], 0
        else:
            ivy0, nloc, halo = (int(v) for v in slab)
            _check(lib().vlp4d_ctx_create_slab(C.byref(self._c), self.dtype_code, ivy0, nloc, halo, C.byref(h)))
            self.ivy0, self.nvy_local, self.halo = ivy0, nloc, halo
        self.h = h
        self.is_slab = slab is not None
        nx, ny, nvx, _ = dom.nxmax
        self.f_shape = (self.nvy_local + 2 * self.halo, nvx, ny, nx)
        self.f_size = int(lib().vlp4d_f_size(self.h))
        # Whether vlp4d_steps joins consecutive x/y half steps on this context.
        self.joins_xy = bool(lib().vlp4d_steps_joins_xy(self.h))

    def owned(self, f):
        """View of the owned planes of an f buffer of this context."""
        return f[self.halo:self.halo + self.nvy_local]

    def close(self):
        if getattr(self, "h", None):
            lib().vlp4d_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- buffers
    def empty_f(self):
        import torch

        return torch.empty(self.f_shape, dtype=self.torch_dtype, device="cuda")

    def _f(self, t):
        if not (t.is_cuda and t.dtype == self.torch_dtype and t.is_contiguous() and t.numel() == self.f_size):
            raise ValueError(f"f must be a contiguous CUDA {self.torch_dtype} tensor of {self.f_size} elements")
        return C.c_void_p(t.data_ptr())

    def field(self, which: int):
        """Torch view (no copy) of the context-owned FP64 (ny, nx) field."""
        import torch

        p = C.c_void_p()
        _check(lib().vlp4d_field_ptr(self.h, which, C.byref(p)))
        return torch.as_tensor(_DevArray(p.value, self.dom.shape2, "<f8"), device="cuda")

    rho = property(lambda self: self.field(FIELD_RHO))
    ex = property(lambda self: self.field(FIELD_EX))
    ey = property(lambda self: self.field(FIELD_EY))

    # -- entry points (one per C function)
    def init_case(self, f, ic=IC_LANDAU_SUM, amp=0.05, k=0.5, u=2.4, stream=None):
        _check(lib().vlp4d_init_case(self.h, self._f(f), ic, amp, k, u, _stream_ptr(stream)))

    def advect_x(self, fn, fnp1, dt, stream=None):
        _check(lib().vlp4d_advect_x(self.h, self._f(fn), self._f(fnp1), dt, _stream_ptr(stream)))

    def advect_y(self, fn, fnp1, dt, stream=None):
        _check(lib().vlp4d_advect_y(self.h, self._f(fn), self._f(fnp1), dt, _stream_ptr(stream)))

    def advect_vx(self, fn, fnp1, dt, stream=None):
        _check(lib().vlp4d_advect_vx(self.h, self._f(fn), self._f(fnp1), dt, _stream_ptr(stream)))

    def advect_vy(self, fn, fnp1, dt, stream=None):
        _check(lib().vlp4d_advect_vy(self.h, self._f(fn), self._f(fnp1), dt, _stream_ptr(stream)))

    def advect_xy(self, fn, fnp1, dt, stream=None):
        _check(lib().vlp4d_advect_xy(self.h, self._f(fn), self._f(fnp1), dt, _stream_ptr(stream)))

    def advect_xyxy(self, fn, fnp1, dt, stream=None):
        """Two x/y shifts by dt in one pass, then the moment of fnp1 into rho."""
        _check(lib().vlp4d_advect_xyxy(self.h, self._f(fn), self._f(fnp1), dt, _stream_ptr(stream)))

    def advect_xy_moment(self, fn, fnp1, dt, stream=None):
        _check(lib().vlp4d_advect_xy_moment(self.h, self._f(fn), self._f(fnp1), dt, _stream_ptr(stream)))

    def advect_vxvy(self, fn, fnp1, dt, stream=None):
        _check(lib().vlp4d_advect_vxvy(self.h, self._f(fn), self._f(fnp1), dt, _stream_ptr(stream)))

    def field_rho(self, fn, stream=None):
        _check(lib().vlp4d_field_rho(self.h, self._f(fn), _stream_ptr(stream)))

    def field_poisson(self, stream=None):
        _check(lib().vlp4d_field_poisson(self.h, _stream_ptr(stream)))

    def diags_compute(self, it, stream=None):
        _check(lib().vlp4d_diags_compute(self.h, it, _stream_ptr(stream)))

    def diags_read(self, count=None):
        import numpy as np

        count = self.dom.nbiter + 1 if count is None else count
        nrj = (C.c_double * max(count, 1))()
        mass = (C.c_double * max(count, 1))()
        _check(lib().vlp4d_diags_read(self.h, nrj, mass, count))
        return np.array(nrj[:count]), np.array(mass[:count])

    def diags_l2norm(self, fn, it, stream=None):
        _check(lib().vlp4d_diags_l2norm(self.h, self._f(fn), it, _stream_ptr(stream)))

    def diags_read_ext(self, count=None):
        """(nrjx, nrjy, l2norm) histories, the vlp4d_mpi diagnostics."""
        import numpy as np

        count = self.dom.nbiter + 1 if count is None else count
        bufs = [(C.c_double * max(count, 1))() for _ in range(3)]
        _check(lib().vlp4d_diags_read_ext(self.h, bufs[0], bufs[1], bufs[2], count))
        return tuple(np.array(b[:count]) for b in bufs)

    def diags_save(self, path):
        _check(lib().vlp4d_diags_save(self.h, str(path).encode()))

    def step(self, f_state, f_next, it, stream=None):
        """One fused Strang step: reads f_state, writes the new state into f_next (f_state becomes scratch)."""
        _check(lib().vlp4d_step(self.h, self._f(f_state), self._f(f_next), it, _stream_ptr(stream)))

    def steps(self, f_state, f_next, iter0, nsteps, stream=None):
        """nsteps fused Strang steps (diagnostics iter0 ..): final state in f_next, f_state is scratch."""
        _check(lib().vlp4d_steps(self.h, self._f(f_state), self._f(f_next), iter0, nsteps, _stream_ptr(stream)))

    def run(self, f0_host, nsteps, fn, fnp1, f_out_host=None, stream=None):
        """vlp4d_run with host buffers (torch CPU tensors, ideally pinned). Returns (nrj, mass) numpy arrays."""
        import numpy as np

        if f0_host.is_cuda or f0_host.dtype != self.torch_dtype or not f0_host.is_contiguous():
            raise ValueError("f0_host must be a contiguous CPU tensor of the context dtype")
        nrj = (C.c_double * (nsteps + 1))()
        mass = (C.c_double * (nsteps + 1))()
        out_ptr = C.c_void_p(f_out_host.data_ptr()) if f_out_host is not None else None
        _check(lib().vlp4d_run(self.h, C.c_void_p(f0_host.data_ptr()), out_ptr, nsteps, nrj, mass, self._f(fn),
                               self._f(fnp1), _stream_ptr(stream)))
        return np.array(nrj[:]), np.array(mass[:])

    def check(self):
        """Synchronise and raise if a kernel reported a lost asynchronous copy."""
        _check(lib().vlp4d_check(self.h))

    def selftest_wait_timeout(self, limit_cycles: int, stream=None):
        """Launch a bounded wait that nothing completes (see the C header)."""
        _check(lib().vlp4d_selftest_wait_timeout(self.h, int(limit_cycles), _stream_ptr(stream)))

    def print_fxvx(self, fn, path):
        _check(lib().vlp4d_print_fxvx(self.h, self._f(fn), str(path).encode()))

    # -- vlp4d_mpi (one process): halo-extended FP64 arrays of shape
    #    (nvy+6, nvx+6, ny+6, nx+6); index 3 is grid point 0.
    @property
    def mpi_shape(self):
        nx, ny, nvx, nvy = self.dom.nxmax
        return (nvy + 2 * HALO, nvx + 2 * HALO, ny + 2 * HALO, nx + 2 * HALO)

    def mpi_empty(self):
        import torch

        return torch.zeros(self.mpi_shape, dtype=torch.float64, device="cuda")

    def _h(self, t):
        import torch

        n = int(lib().vlp4d_mpi_size(self.h))
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.numel() == n):
            raise ValueError(f"a vlp4d_mpi array must be a contiguous CUDA float64 tensor of {n} elements")
        return C.c_void_p(t.data_ptr())

    def mpi_init_case(self, fn, stream=None):
        """The domain's vlp4d_mpi initial condition (idcase 10, 20, 2, 5) on fn's grid points, halo zero."""
        _check(lib().vlp4d_mpi_init_case(self.h, self._h(fn), _stream_ptr(stream)))

    def mpi_halo_fill(self, fn, stream=None):
        _check(lib().vlp4d_mpi_halo_fill(self.h, self._h(fn), _stream_ptr(stream)))

    def mpi_spline_xy(self, fn, stream=None):
        _check(lib().vlp4d_mpi_spline_xy(self.h, self._h(fn), _stream_ptr(stream)))

    def mpi_spline_vxvy(self, fn, stream=None):
        _check(lib().vlp4d_mpi_spline_vxvy(self.h, self._h(fn), _stream_ptr(stream)))

    def mpi_advect_2d(self, fn, fn_tmp, dt, stream=None):
        _check(lib().vlp4d_mpi_advect_2d(self.h, self._h(fn), self._h(fn_tmp), dt, _stream_ptr(stream)))

    def mpi_advect_4d(self, fn, tmp_fn, dt, stream=None):
        _check(lib().vlp4d_mpi_advect_4d(self.h, self._h(fn), self._h(tmp_fn), dt, _stream_ptr(stream)))

    def mpi_field(self, fn, stream=None):
        _check(lib().vlp4d_mpi_field(self.h, self._h(fn), _stream_ptr(stream)))

    def mpi_l2norm(self, fn, it, stream=None):
        _check(lib().vlp4d_mpi_l2norm(self.h, self._h(fn), it, _stream_ptr(stream)))

    def mpi_step(self, fn, fnp1, it, stream=None):
        """One vlp4d_mpi step: state in fn's grid points -> fnp1's (fn is overwritten)."""
        _check(lib().vlp4d_mpi_step(self.h, self._h(fn), self._h(fnp1), it, _stream_ptr(stream)))

    def mpi_run(self, fn, fnp1, nsteps, stream=None):
        """Initial field and diagnostics, then nsteps steps (Vlp4d.cpp:30-49);
        returns the tensor that holds the final state (fn or fnp1)."""
        self.mpi_field(fn, stream)
        self.diags_compute(0, stream)
        self.mpi_l2norm(fn, 0, stream)
        a, b = fn, fnp1
        for it in range(1, nsteps + 1):
            self.mpi_step(a, b, it, stream)
            a, b = b, a
        return a


def field_rho_noalloc(f, rho, nxmax, dvx, dvy, stream=None):
    """vlp4d_field_rho_noalloc: the velocity moment of f into rho (FP64, (ny, nx))
    without a context and without allocating device memory."""
    import torch

    nx, ny, nvx, nvy = (int(v) for v in nxmax)
    # The C side sees only pointers: check here what it cannot.
    if not (f.is_cuda and f.is_contiguous() and f.dtype in (torch.float64, torch.float32)):
        raise ValueError("f must be a contiguous CUDA float64 or float32 tensor")
    if f.numel() != nx * ny * nvx * nvy:
        raise ValueError(f"f has {f.numel()} elements; nxmax {tuple(nxmax)} needs {nx * ny * nvx * nvy}")
    if not (rho.is_cuda and rho.is_contiguous() and rho.dtype == torch.float64 and rho.numel() == nx * ny):
        raise ValueError(f"rho must be a contiguous CUDA float64 tensor of nx*ny = {nx * ny} elements")
    if f.device != rho.device:
        raise ValueError("f and rho must be on the same device")
    dtype = F64 if f.dtype == torch.float64 else F32
    _check(lib().vlp4d_field_rho_noalloc(C.c_void_p(f.data_ptr()), dtype, nx, ny, nvx, nvy, float(dvx), float(dvy),
                                         C.c_void_p(rho.data_ptr()), _stream_ptr(stream)))


def transpose(a, out, stream=None):
    """Impl::Transpose::forward on a column-major (rows, cols) matrix held as a C-ordered (cols, rows) tensor."""
    cols, rows = a.shape
    _check(lib().vlp4d_transpose(C.c_void_p(a.data_ptr()), C.c_void_p(out.data_ptr()), rows, cols,
                                 a.element_size(), _stream_ptr(stream)))


class Adjoint:
    """Reverse mode of a Context (vlp4d_adjoint_*): checkpointed runs of
    `nsteps` steps with the objective J = dx dy sum |E(f_N)|^2; a checkpoint
    of f every `every` steps, or (every = 0) every step's stage input and
    field stored by the forward run, so that the reverse run recomputes
    nothing."""

    def __init__(self, ctx: Context, nsteps: int, every: int = 8):
        self.ctx = ctx
        self.nsteps = int(nsteps)
        self.h = C.c_void_p()
        _check(lib().vlp4d_adjoint_create(ctx.h, self.nsteps, int(every), C.byref(self.h)))

    def close(self):
        if self.h:
            lib().vlp4d_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    def forward(self, f0, f_out=None, stream=None) -> float:
        J = C.c_double()
        out = self.ctx._f(f_out) if f_out is not None else None
        _check(lib().vlp4d_adjoint_forward(self.h, self.ctx._f(f0), out, C.byref(J), _stream_ptr(stream)))
        return J.value

    def backward(self, grad=None, stream=None):
        if grad is None:
            grad = self.ctx.empty_f()
        _check(lib().vlp4d_adjoint_backward(self.h, self.ctx._f(grad), _stream_ptr(stream)))
        return grad

    def step_adjoint(self, f_state, lam_next, lam_out, stream=None):
        _check(lib().vlp4d_step_adjoint(self.h, self.ctx._f(f_state), self.ctx._f(lam_next), self.ctx._f(lam_out),
                                        _stream_ptr(stream)))

    def energy_grad(self, f, lam, stream=None) -> float:
        J = C.c_double()
        _check(lib().vlp4d_energy_grad(self.h, self.ctx._f(f), C.byref(J), self.ctx._f(lam), _stream_ptr(stream)))
        return J.value


def energy_after_steps(f0, adjoint: Adjoint):
    """torch.autograd binding for tests: J(f0) = electric energy after the
    adjoint's nsteps steps, differentiable in f0 through vlp4d_adjoint_backward."""
    import torch

    class _EnergyAfterSteps(torch.autograd.Function):
        @staticmethod
        def forward(ctx_, f):
            f = f.detach().contiguous()
            return torch.tensor(adjoint.forward(f), dtype=torch.float64, device=f.device)

        @staticmethod
        def backward(ctx_, gJ):
            g = adjoint.backward()
            return g * gJ.to(g.dtype)

    return _EnergyAfterSteps.apply(f0)


@dataclass
class EnsembleMember:
    """One member of a batched ensemble: grid, box, dt and the Landau initial
    condition f0 = M(vx) M(vy) (1 + amp (cos k x + cos k y))."""

    n: Sequence[int]
    min_phy: Sequence[float]
    max_phy: Sequence[float]
    dt: float
    amp: float
    k: float

    def domain(self, nbiter: int, idcase: int = 110) -> Domain:
        return Domain(list(self.n), list(self.min_phy), list(self.max_phy), self.dt, nbiter, idcase)


class Ensemble:
    """vlp4d_ensemble_*: members advanced together in one persistent launch."""

    def __init__(self, members: Sequence[EnsembleMember], nsteps: int):
        self.members = list(members)
        self.nsteps = int(nsteps)
        arr = (CEnsMember * len(self.members))()
        for i, m in enumerate(self.members):
            for k in range(4):
                arr[i].n[k] = int(m.n[k])
                arr[i].min_phy[k] = float(m.min_phy[k])
                arr[i].max_phy[k] = float(m.max_phy[k])
            arr[i].dt, arr[i].amp, arr[i].k = float(m.dt), float(m.amp), float(m.k)
        self.h = C.c_void_p()
        _check(lib().vlp4d_ensemble_create(arr, len(self.members), self.nsteps, C.byref(self.h)))

    def close(self):
        if self.h:
            lib().vlp4d_ensemble_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    @property
    def cells(self) -> int:
        return int(lib().vlp4d_ensemble_cells(self.h))

    def run(self, stream=None):
        _check(lib().vlp4d_ensemble_run(self.h, _stream_ptr(stream)))

    def check(self):
        _check(lib().vlp4d_ensemble_check(self.h))

    def read(self, i: int, stream=None):
        """(final f of member i as a float32 CUDA tensor (nvy, nvx, ny, nx), energy history)."""
        import numpy as np
        import torch

        m = self.members[i]
        f = torch.empty((m.n[3], m.n[2], m.n[1], m.n[0]), dtype=torch.float32, device="cuda")
        nrj = np.zeros(self.nsteps + 1)
        _check(lib().vlp4d_ensemble_read(self.h, int(i), C.c_void_p(f.data_ptr()),
                                         nrj.ctypes.data_as(C.POINTER(C.c_double)), _stream_ptr(stream)))
        return f, nrj

    def set_idle_limit(self, cycles: int):
        """Cycles a CTA may find no free tile before it flags a timeout (0: default)."""
        _check(lib().vlp4d_ensemble_set_idle_limit(self.h, int(cycles)))

    def set_tiles(self, threads: int, cols_per_tile: int, ctas_per_sm: int = 0):
        _check(lib().vlp4d_ensemble_set_tiles(self.h, threads, cols_per_tile, ctas_per_sm))

    def tiles(self):
        t, c, p = C.c_int(), C.c_int(), C.c_int()
        _check(lib().vlp4d_ensemble_get_tiles(self.h, C.byref(t), C.byref(c), C.byref(p)))
        return t.value, c.value, p.value

    def autotune(self, steps: int, csv_path: Optional[str] = None, stream=None):
        _check(lib().vlp4d_ensemble_autotune(self.h, int(steps), csv_path.encode() if csv_path else None,
                                             _stream_ptr(stream)))
        return self.tiles()


def landau_ensemble_members(nruns=256, sizes=(16, 24, 32, 48), seed=20261203, dt=0.1, vmax=6.0,
                            ks=(0.3, 0.5), amp_range=(0.01, 0.1)):
    """The batched-ensemble configuration: per member, N per dimension drawn
    independently from `sizes`, amp ~ U(amp_range), k from `ks`, box
    x, y in [0, 2 pi / k), v in [-vmax, vmax) (seeded)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nruns):
        n = [int(v) for v in rng.choice(sizes, size=4)]
        k = float(rng.choice(ks))
        amp = float(rng.uniform(*amp_range))
        L = 2 * math.pi / k
        out.append(EnsembleMember(n, [0.0, 0.0, -vmax, -vmax], [L, L, vmax, vmax], dt, amp, k))
    return out
