"""GPU test of pf_diagnosticos_noalloc, the diagnostics entry point for
callers that cannot let the library allocate device memory (their device
memory belongs to another runtime, or a fixed budget forbids allocation).

It calls the entry point through the C-ABI on device fields the test owns
(torch tensors) and checks its output against pf_diagnosticos, the existing
entry point, within the tolerance of the other diagnostics tests (1e-12
relative), on two calls in a row with different domains.  The file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

import make_golden as MG
import pf3d
from pf3d import _abi, deck

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _state(nx, ny, nz, seed):
    p = deck.run6_params(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    g = deck.grid(nx, ny, nz, 0.5e-6)
    st = MG.small_state(nx, ny, nz, p)
    st["c"] = st["c"] + np.random.default_rng(seed).normal(0.0, 1e-4, st["c"].shape)
    return g, p, st


def _existing(g, p, st, precision):
    with pf3d.Domain(g, p, precision) as d:
        d.upload("phase_field_new", st["phi"])
        d.upload("conc_soluto_new", st["c"])
        out = d.diagnosticos()
        dv = d.derived()
    return out, dv


def _noalloc(g, st, precision, dv, pitch_pad=0):
    import torch
    dt = torch.float64 if precision == pf3d.PF_FP64 else torch.float32
    nz, ny, nx = st["phi"].shape
    pitch = nx + pitch_pad
    phi = torch.zeros((nz, ny, pitch), dtype=dt, device="cuda")
    c = torch.zeros((nz, ny, pitch), dtype=dt, device="cuda")
    phi[:, :, :nx] = torch.from_numpy(st["phi"]).to(dt)
    c[:, :, :nx] = torch.from_numpy(st["c"]).to(dt)
    torch.cuda.synchronize()
    out = (C.c_double * 5)()
    rc = _abi.LIB.pf_diagnosticos_noalloc(C.c_void_p(phi.data_ptr()), C.c_void_p(c.data_ptr()), nx, ny, nz, pitch,
                                          precision, g.dx, g.dy, g.dz, dv.E0, dv.W0, None, out)
    _abi.check(rc)
    return tuple(out)


@pytest.mark.parametrize("precision", [pf3d.PF_FP64, pf3d.PF_FP32])
def test_noalloc_matches_pf_diagnosticos_twice(gpu, precision):
    # first call: a deeper domain; second call: a shallower one, so partials
    # left behind by the first call must not leak into the second
    cases = [(_state(40, 33, 61, 1), 0), (_state(29, 24, 17, 2), 3)]
    for (g, p, st), pad in cases:
        want, dv = _existing(g, p, st, precision)
        got = _noalloc(g, st, precision, dv, pitch_pad=pad)
        for a, b in zip(got, want):
            assert abs(a - b) <= RTOL * abs(b), (got, want)


def test_noalloc_rejects_more_planes_than_its_scratch(gpu):
    out = (C.c_double * 5)()
    nz = _abi.PF_NOALLOC_MAX_PLANES + 1
    rc = _abi.LIB.pf_diagnosticos_noalloc(C.c_void_p(16), C.c_void_p(16), 8, 8, nz, 8, 64, 1e-6, 1e-6, 1e-6,
                                          1e-3, 1e5, None, out)
    assert rc == _abi.PF_E_ARG
    assert b"exceeds" in _abi.LIB.pf_last_error(None)
