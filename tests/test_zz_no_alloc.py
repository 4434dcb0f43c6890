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


def _exact(phi, c, dx, dy, dz, E0, W0):
    """diag_body.inc:8-22 with exactly rounded sums (math.fsum): L2, max,
    min, total solute, free energy (gradient term on interior cells only)."""
    import math
    nz, ny, nx = phi.shape
    g2 = np.zeros_like(phi)
    if nx > 2 and ny > 2 and nz > 2:
        gx = (phi[1:-1, 1:-1, 2:] - phi[1:-1, 1:-1, :-2]) * 0.5 / dx
        gy = (phi[1:-1, 2:, 1:-1] - phi[1:-1, :-2, 1:-1]) * 0.5 / dy
        gz = (phi[2:, 1:-1, 1:-1] - phi[:-2, 1:-1, 1:-1]) * 0.5 / dz
        g2[1:-1, 1:-1, 1:-1] = gx * gx + gy * gy + gz * gz
    w = W0 * phi * phi * (1.0 - phi) * (1.0 - phi)
    e = (0.5 * E0 * E0 * g2 + w) * dx * dy * dz
    return (math.sqrt(math.fsum((phi * phi).ravel())), float(phi.max()), float(phi.min()),
            math.fsum(c.ravel()), math.fsum(e.ravel()))


@pytest.mark.parametrize("shape", [(5, 4, 1), (5, 4, 2), (4, 4, _abi.PF_NOALLOC_MAX_PLANES)])
def test_noalloc_edge_shapes(gpu, shape):
    # one plane and two planes (no interior cell: the gradient term is zero
    # everywhere) and a thin domain whose rows fill the whole scratch, the
    # result row right after the last partial row; each called twice
    import torch
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 100 + nz)
    phi = rng.uniform(0.0, 1.0, (nz, ny, nx))
    c = 0.0196 * (1.0 - 0.86 * phi) + rng.normal(0.0, 1e-4, phi.shape)
    dx = dy = dz = 0.5e-6
    E0, W0 = 2.5e-4, 3.1e6
    want = _exact(phi, c, dx, dy, dz, E0, W0)
    tphi = torch.from_numpy(phi).cuda()
    tc = torch.from_numpy(c).cuda()
    torch.cuda.synchronize()
    for _ in range(2):
        out = (C.c_double * 5)()
        _abi.check(_abi.LIB.pf_diagnosticos_noalloc(C.c_void_p(tphi.data_ptr()), C.c_void_p(tc.data_ptr()), nx, ny,
                                                    nz, nx, pf3d.PF_FP64, dx, dy, dz, E0, W0, None, out))
        got = tuple(out)
        for a, b in zip(got, want):
            assert abs(a - b) <= RTOL * abs(b), (got, want)


def test_noalloc_rejects_more_planes_than_its_scratch(gpu):
    out = (C.c_double * 5)()
    nz = _abi.PF_NOALLOC_MAX_PLANES + 1
    rc = _abi.LIB.pf_diagnosticos_noalloc(C.c_void_p(16), C.c_void_p(16), 8, 8, nz, 8, 64, 1e-6, 1e-6, 1e-6,
                                          1e-3, 1e5, None, out)
    assert rc == _abi.PF_E_ARG
    assert b"exceeds" in _abi.LIB.pf_last_error(None)
