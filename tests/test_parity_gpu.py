"""GPU parity tests: the CUDA path through the C-ABI against the CPU oracle.

Plain form (FP64): every field within RTOL_FP64 = 1e-12 (normwise max
relative) of the oracle after N steps; everything that does not pass through
`log` is bit-identical in the per-subroutine kernels (the heat equation, the
noise stream).  The fused passes use the fast FP64 form and are held to the
same 1e-12 bar.
"""
import numpy as np
import pytest

import make_golden as MG
import pyoracle as O
import pf3d
from conftest import RTOL_FP64, max_rel
from pf3d import deck, init

pytestmark = pytest.mark.gpu

C1 = deck.WORKLOADS["c1_64x64x128_fp64"]


def small_case(nx, ny, nz, **over):
    p = deck.run6_params(T0=922.0, taxa_resfr=19.84, AAA=0.01, **over)
    g = deck.grid(nx, ny, nz, 0.5e-6)
    st = MG.small_state(nx, ny, nz, p)
    return g, p, st


def c1_case():
    return C1.grid(), C1.params(), init.workload_state(C1)


def compare(fd: dict, fo: dict, rtol=RTOL_FP64, exact=()):
    worst = {}
    for k in fo:
        if k in exact:
            assert np.array_equal(fd[k], fo[k]), f"{k} not bit-identical"
        r = max_rel(fd[k], fo[k])
        worst[k] = r
        assert r <= rtol, f"{k}: max rel {r:.3e} > {rtol:.1e}"
    return worst


def test_temperatura_bit_exact(gpu):
    g, p, st = small_case(33, 20, 24, D=2e-5)
    o = O.Oracle(g, p); o.load_state(st)
    st = dict(st, dpp=np.random.default_rng(1).normal(0, 1e-3, st["phi"].shape))
    o.set(6, st["dpp"])
    with pf3d.Domain(g, p) as d:
        d.load_state(st)
        d.temperatura(o.scalars()["TP"])
        o.temperatura()
        assert np.array_equal(d.download("TNEW"), o.get(5))


def test_phase_sweep_noise_bit_exact(gpu):
    """With M0 = 0 the sweep adds only the noise: DPP must equal the oracle bit for bit."""
    for rt in (0, 1, 2):
        g, p, st = small_case(40, 18, 22, ruido_tipo=rt, M0=0.0)
        o = O.Oracle(g, p); o.load_state(st)
        o.set_scalars(7, o.scalars()["TP"], 0.0, 0.0)
        with pf3d.Domain(g, p) as d:
            d.load_state(st)
            d.equacao_campo_fase(7, o.scalars()["TP"], 0.0)
            o.equacao_campo_fase()
            assert np.array_equal(d.download("DPP"), o.get(6)), f"ruido_tipo {rt}"
            assert np.array_equal(d.download("phase_field_new"), o.get(1))


@pytest.mark.parametrize("over", [{}, dict(h_quintico=1), dict(ruido_tipo=2)])
def test_per_subroutine_one_step(gpu, over):
    g, p, st = small_case(37, 29, 23, **over)
    o = O.Oracle(g, p); o.load_state(st)
    with pf3d.Domain(g, p) as d:
        d.load_state(st)
        d.step_reference_order(1)
        o.step(1)
        compare(d.fields(), o.fields(), exact=("T",))
        s = d.state()
        assert s.M0 == o.scalars()["M0"] and s.TP == o.scalars()["TP"] and s.it == 1


def test_solute_sets_old_like_reference(gpu):
    """concentracao_soluto leaves conc_soluto_old = the pre-decoration update."""
    g, p, st = small_case(20, 17, 19)
    o = O.Oracle(g, p); o.load_state(st)
    with pf3d.Domain(g, p) as d:
        d.load_state(st)
        d.concentracao_soluto()
        o.concentracao_soluto()
        assert max_rel(d.download("conc_soluto_new"), o.get(3)) <= RTOL_FP64
        assert max_rel(d.download("conc_soluto_old"), o.get(2)) <= RTOL_FP64


@pytest.mark.parametrize("shape,over", [
    ((64, 64, 128), {}),
    ((37, 29, 23), {}),
    ((5, 5, 5), {}),
    ((6, 9, 7), dict(n_varreduras=1)),
    ((33, 17, 40), dict(n_varreduras=3, h_quintico=1, ruido_tipo=1)),
    ((40, 40, 30), dict(D=2e-5, ruido_tipo=2)),
])
def test_fused_step_matches_oracle(gpu, shape, over):
    if shape == (64, 64, 128):
        g, p, st = c1_case()
    else:
        g, p, st = small_case(*shape, **over)
    o = O.Oracle(g, p); o.load_state(st)
    with pf3d.Domain(g, p) as d:
        d.load_state(st)
        for n in (1, 9):
            d.step(n)
            o.step(n)
            compare(d.fields(), o.fields())
        s = d.state()
        assert s.it == 10 and s.M0 == o.scalars()["M0"] and s.TP == o.scalars()["TP"]
        assert s.time == np.float32(o.scalars()["time"])


@pytest.mark.parametrize("tile_y,zchunk", [(4, 0), (8, 64), (16, 7), (8, 1)])
def test_fused_matches_per_subroutine(gpu, tile_y, zchunk):
    """The fused passes (fast FP64 form) against the per-subroutine kernels
    (reference form): tiling, z-chunking, node reuse and the closed-form
    decoration must not change anything beyond rounding."""
    g, p, st = small_case(70, 45, 50)
    with pf3d.Domain(g, p) as a, pf3d.Domain(g, p) as b:
        a.load_state(st); b.load_state(st)
        a.set_option(pf3d.PF_OPT_TILE_Y, tile_y)
        a.set_option(pf3d.PF_OPT_ZCHUNK, zchunk)
        b.set_option(pf3d.PF_OPT_FUSED, 0)
        a.step(3)
        b.step(3)
        compare(a.fields(), b.fields())


def exact_diagnostics(phi, c, dx, dy, dz, E0, w0):
    """diag_body.inc evaluated per cell in the reference's order, summed with
    math.fsum (exactly rounded) -- the reference's OpenMP reduction order is
    unspecified, so its rounding is not a target."""
    import math
    nz, ny, nx = phi.shape
    w_term = w0 * phi * phi * (1.0 - phi) * (1.0 - phi)
    grad2 = np.zeros_like(phi)
    gx = (phi[1:-1, 1:-1, 2:] - phi[1:-1, 1:-1, :-2]) * 0.5 / dx
    gy = (phi[1:-1, 2:, 1:-1] - phi[1:-1, :-2, 1:-1]) * 0.5 / dy
    gz = (phi[2:, 1:-1, 1:-1] - phi[:-2, 1:-1, 1:-1]) * 0.5 / dz
    grad2[1:-1, 1:-1, 1:-1] = gx ** 2 + gy ** 2 + gz ** 2
    fe = (0.5 * E0 * E0 * grad2 + w_term) * dx * dy * dz
    return (math.sqrt(math.fsum((phi * phi).ravel())), float(phi.max()), float(phi.min()),
            math.fsum(c.ravel()), math.fsum(fe.ravel()))


def test_diagnosticos_match_oracle(gpu):
    g, p, st = c1_case()
    o = O.Oracle(g, p); o.load_state(st)
    o.step(3)
    sc = o.scalars()
    fo = o.fields()
    ref = exact_diagnostics(fo["phi"], fo["c"], g.dx, g.dy, g.dz, sc["E0"], sc["W0"])
    naive = o.diagnosticos()        # serial sums (after the swap new == old)
    with pf3d.Domain(g, p) as d:
        d.load_state(st)
        out = d.step_diag(3)
    for a, b, c in zip(out, ref, naive):
        assert abs(a - b) <= 1e-12 * abs(b), (out, ref)
        assert abs(c - b) <= 1e-9 * abs(b)      # the naive serial sum, for scale


def test_diagnosticos_entry_point(gpu):
    """pf_diagnosticos reads phase_field_new / conc_soluto_new, as the reference."""
    g, p, st = small_case(30, 26, 34)
    with pf3d.Domain(g, p) as d:
        d.upload("phase_field_new", st["phi"])
        d.upload("conc_soluto_new", st["c"])
        out = d.diagnosticos()
        dv = d.derived()
    ref = exact_diagnostics(st["phi"], st["c"], g.dx, g.dy, g.dz, dv.E0, dv.W0)
    for a, b in zip(out, ref):
        assert abs(a - b) <= 1e-12 * abs(b), (out, ref)


@pytest.mark.slow
def test_config1_full_run(gpu):
    """Configuration 1: 64x64x128, FP64, 2000 steps, every field within 1e-12."""
    g, p, st = c1_case()
    o = O.Oracle(g, p); o.load_state(st)
    with pf3d.Domain(g, p) as d:
        d.load_state(st)
        d.step(C1.steps)
        o.step(C1.steps)
        w = compare(d.fields(), o.fields())
        print("config 1 after 2000 steps, max rel per field:", w)


def test_fp32_close_to_fp64(gpu):
    g, p, st = c1_case()
    with pf3d.Domain(g, p, pf3d.PF_FP64) as a, pf3d.Domain(g, p, pf3d.PF_FP32) as b:
        a.load_state(st); b.load_state(st)
        a.step(100); b.step(100)
        fa, fb = a.fields(), b.fields()
        for k in fb:
            assert np.isfinite(fb[k]).all(), f"FP32 {k} not finite"
        for k in ("phi", "c", "T", "dpp"):
            rel = np.linalg.norm(fb[k] - fa[k]) / np.linalg.norm(fa[k])
            print(k, "FP32 vs FP64 relative L2 after 100 steps:", rel)
            assert rel < (1e-2 if k == "dpp" else 1e-3), (k, rel)
        assert a.state().M0 == b.state().M0   # scalars stay FP64 in both


@pytest.mark.parametrize("prec", [pf3d.PF_FP64, pf3d.PF_FP32])
def test_flat_and_tiny_gradients_stay_finite(gpu, prec):
    """Flat liquid (phi = 0) and gradients near the underflow range of FP32."""
    nx = ny = nz = 24
    p = deck.run6_params(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    g = deck.grid(nx, ny, nz, 0.5e-6)
    rng = np.random.default_rng(0)
    for phi in (np.zeros((nz, ny, nx)), rng.uniform(0, 1e-16, (nz, ny, nx)), rng.uniform(0, 1e-30, (nz, ny, nx))):
        st = {"phi": phi, "c": p.C0 * np.ones_like(phi), "T": np.full_like(phi, 922.0)}
        o = O.Oracle(g, p); o.load_state(st); o.step(3)
        with pf3d.Domain(g, p, prec) as d:
            d.load_state(st)
            d.step(3)
            f = d.fields()
        fo = o.fields()
        for k in f:
            assert np.isfinite(f[k]).all(), k
            tol = RTOL_FP64 if prec == pf3d.PF_FP64 else 1e-6
            assert np.max(np.abs(f[k] - fo[k])) <= tol * max(1.0, np.max(np.abs(fo[k]))), k


def test_probe_and_stream(gpu):
    import torch
    g, p, st = small_case(30, 30, 30)
    with pf3d.Domain(g, p) as d:
        d.load_state(st)
        s = torch.cuda.Stream()
        d.set_stream(s.cuda_stream)
        d.step(2)
        d.sync()
        d.set_stream(None)
        phi = d.download("phase_field_old")
        assert d.probe("phase_field_old", 15, 10, 15) == phi[14, 9, 14]
