"""CPU tests of the C-ABI library: it loads, exports every declared symbol,
its host-side FP64 scalar set-up equals the oracle's bit for bit, and it
fails loudly (no CPU fallback) when no GPU is present."""
import ctypes as C
import os
import re
import struct

import numpy as np
import pytest

from conftest import ROOT, has_gpu
import pyoracle as O
import pf3d
from pf3d import _abi, deck


def header_functions():
    src = open(os.path.join(ROOT, "include", "pf3d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_abi.LIB_PATH)
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    bound = {n for (n, _, _) in _abi.SIGNATURES}
    assert set(header_functions()) <= bound


def test_version():
    assert _abi.LIB.pf_version() == 1


@pytest.mark.parametrize("dx", [0.15e-6, 0.5e-6, 1.0e-6])
def test_w0_e0_equals_oracle(dx):
    p = deck.run6_params()
    g = deck.grid(8, 8, 8, dx)
    W0, E0, n = pf3d.w0_e0(g, p)
    W0o, E0o, no = O.w0_e0(p.Thin_Interface * dx, p.ajuste, p.Sigma)
    assert (struct.pack("d", W0), struct.pack("d", E0), n) == (struct.pack("d", W0o), struct.pack("d", E0o), no)


@pytest.mark.parametrize("TP", [922.0, 921.3, 917.0])
def test_auxiliar_equals_oracle(TP):
    p = deck.run6_params()
    g = deck.grid(8, 8, 8, 0.5e-6)
    W0, E0, _ = pf3d.w0_e0(g, p)
    Cs = ((p.Tm - TP) * float(np.float32(p.Ke))) / p.Me
    Cl = (p.Tm - TP) / p.Me
    assert pf3d.auxiliar_scalar(p, E0, W0, TP, Cs, Cl) == O.auxiliar(p, TP, Cs, Cl, E0, W0)


def test_rejects_small_grid():
    p = deck.run6_params()
    with pytest.raises(pf3d.PFError) as e:
        pf3d.Domain(deck.grid(4, 8, 8, 0.5e-6), p)
    assert e.value.code == _abi.PF_E_ARG


def test_math_log_argument_checks():
    # checked before any CUDA call, so this runs without a device
    x = np.ones(4)
    y = np.empty(4)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    assert _abi.LIB.pf_math_log(ptr(x), -1, ptr(y), ptr(y)) == _abi.PF_E_ARG
    assert _abi.LIB.pf_math_log(None, 4, ptr(y), ptr(y)) == _abi.PF_E_ARG
    assert _abi.LIB.pf_math_log(ptr(x), 1 << 29, ptr(y), ptr(y)) == _abi.PF_E_ARG
    assert _abi.LIB.pf_math_log(None, 0, None, None) == _abi.PF_OK


def test_ctx_bytes():
    g = deck.grid(512, 512, 1024, 0.5e-6)
    b64 = _abi.LIB.pf_ctx_bytes(C.byref(g), 64)
    b32 = _abi.LIB.pf_ctx_bytes(C.byref(g), 32)
    assert 7 * 512 * 512 * 1024 * 8 <= b64 < 7 * 512 * 512 * 1024 * 8 * 1.01
    assert abs(b64 / b32 - 2.0) < 0.01


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    p = deck.run6_params()
    with pytest.raises(pf3d.PFError) as e:
        pf3d.Domain(deck.grid(8, 8, 8, 0.5e-6), p)
    assert e.value.code == _abi.PF_E_NODEV


def test_read_entrada_reference_deck_format(tmp_path):
    # a deck in the reference's positional format (values of the run6 deck)
    lines = ["header", "", ""] + [
        "933.3 | Tm", "922 | T0", "0.891002000d+09 | dH", "1.055d-03 | E0", "673.2d+3 | w0", "1.9d-03 | M0",
        "6.59477338d-05 | Ds", "3.23646776d-05 | Dl", "2.926560e+06 | Cps", "2.626320e+06 | Cpl", "64 | Nx",
        "48 | Ny", "96 | Nz", "0.5d-06 | dy", "0.5d-06 | dx", "0.5d-06 | dz", "1.d-23 | small", "4.d0 | ANI",
        "1000000000 | itmax", "0.01d0 | AAA", "0.d0 | teta", "0.03d0 | DE", "1.5d-07 | DT", "3.0d-13 | Dsol",
        "3.0d-09 | Dliq", "0.14d0 | Ke", "640d0 | Me", "1.130d-05 | Vm", "8.31451D0 | R", "0.0196d0 | C0",
        "4.d0 | TI", "0.093d+0 | Sigma", "1 | Beta", "2.d0 | ajuste", "0.085d0 | stop", "7500 | write",
        "905.0d0 | TP", "3   0.d0 | tipo", "19.84d0  2 | taxa", "0  0 | h ruido"]
    f = tmp_path / "entrada.dat"
    f.write_text("\n".join(lines) + "\n")
    g, p, ex = deck.read_entrada(str(f))
    ref = deck.run6_params(AAA=0.01)
    assert (g.nx, g.ny, g.nz) == (64, 48, 96) and g.dx == 0.5e-6
    for name, _ in _abi.pf_params._fields_:
        assert getattr(p, name) == getattr(ref, name), name
    assert ex["tipo_inicial"] == 3
