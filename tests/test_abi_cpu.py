"""CPU tests of the C ABI boundary: the library loads, exports every symbol
include/vlp4d_b200.h declares, parses the reference's decks, and rejects bad
arguments with status codes (no GPU needed, no compute launched)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess

import pytest

from conftest import ROOT


def _declared_symbols():
    text = (ROOT / "include" / "vlp4d_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vlp4d_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree(pkg):
    assert _declared_symbols() == sorted(pkg.vlp4d.EXPORTS)


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.lib()
    for name in _declared_symbols():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(pkg.vlp4d.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (vlp4d_[a-z0-9_]+)\b", out))
    assert set(_declared_symbols()) <= exported


def test_library_is_built_for_sm100a_only():
    """The build recipe compiles and links every CUDA source for sm_100a
    alone (one -gencode pair, no PTX for other targets)."""
    mk = (ROOT / "p3-miniapps_b200" / "Makefile").read_text()
    arch = re.search(r"^ARCH := (.*)$", mk, re.M).group(1).split()
    assert arch == ["-gencode", "arch=compute_100a,code=sm_100a"], arch
    assert "$(ARCH)" in re.search(r"^NVFLAGS := (.*)$", mk, re.M).group(1)
    assert "$(NVCC) $(ARCH) -shared" in mk
    assert "-arch" not in mk and "compute_90" not in mk


@pytest.mark.parametrize("deck,expect", [
    ("SLD10_large.dat", dict(nxmax=[128, 128, 128, 128], idcase=10, dt=0.125, nbiter=128)),
    ("TSI20.dat", dict(nxmax=[512, 4, 512, 4], idcase=20, dt=0.125, nbiter=512, fxvx=1)),
])
def test_read_deck(pkg, deck, expect):
    path = ROOT / "tests" / "golden" / "decks" / deck
    dom = pkg.Domain.from_deck(path)
    for k, v in expect.items():
        assert getattr(dom, k) == v, k
    assert dom.min_phy[2] == -9.0 and dom.max_phy[3] == 9.0


def test_read_deck_errors(pkg, tmp_path):
    with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
        pkg.Domain.from_deck(tmp_path / "missing.dat")
    assert e.value.code == pkg.vlp4d.ERR_IO
    bad = tmp_path / "bad.dat"
    bad.write_text("Number of points : 12\n")
    with pytest.raises(pkg.vlp4d.Vlp4dError) as e:
        pkg.Domain.from_deck(bad)
    assert e.value.code == pkg.vlp4d.ERR_IO


def test_invalid_arguments_rejected_before_any_device_work(pkg):
    L = pkg.lib()
    h = C.c_void_p()
    d = pkg.landau_domain(8).to_c()
    d.nxmax[1] = 0
    assert L.vlp4d_ctx_create(C.byref(d), 0, C.byref(h)) == pkg.vlp4d.ERR_INVALID_ARG
    d = pkg.landau_domain(8).to_c()
    assert L.vlp4d_ctx_create(C.byref(d), 7, C.byref(h)) == pkg.vlp4d.ERR_INVALID_ARG
    d.max_phy[0] = d.min_phy[0]
    assert L.vlp4d_ctx_create(C.byref(d), 0, C.byref(h)) == pkg.vlp4d.ERR_INVALID_ARG
    # NULL context / buffers.
    assert L.vlp4d_advect_x(None, None, None, 0.1, None) == pkg.vlp4d.ERR_INVALID_ARG
    assert L.vlp4d_step(None, None, None, 1, None) == pkg.vlp4d.ERR_INVALID_ARG
    assert L.vlp4d_transpose(None, None, 4, 4, 8, None) == pkg.vlp4d.ERR_INVALID_ARG
    assert b"NULL" in L.vlp4d_last_error()


def test_ctx_create_without_device_reports_no_device(pkg):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    L = pkg.lib()
    h = C.c_void_p()
    d = pkg.landau_domain(8).to_c()
    assert L.vlp4d_ctx_create(C.byref(d), 0, C.byref(h)) == pkg.vlp4d.ERR_NO_DEVICE
    assert not h.value


def test_host_line_stencil_matches_reference_per_cell(pkg):
    """The per-line stencil (lagrange.cuh), evaluated through the oracle's
    per-cell formula at every cell of a line, gives one offset and weights
    within 1e-13 of the line's: the basis for computing them once per line."""
    import numpy as np
    from oracle.oracle import Restatement

    R = Restatement((32, 32, 32, 32), (0, 0, -6, -6), (4 * np.pi, 4 * np.pi, 6, 6), 0.1)
    n, hmin, hmax = 32, 0.0, 4 * np.pi
    dh = (hmax - hmin) / n
    for disp in (0.0, 0.31, -0.77, 1e-17, 3.9, -11.2):
        pos = [((hmin + i * dh - disp - hmin) % (hmax - hmin)) / dh for i in range(n)]
        offs = {int(np.floor(p + 1e-9)) - i for i, p in enumerate(pos)}
        offs = {o % n for o in offs}
        assert len(offs) == 1, (disp, offs)
