"""GPU test of the TMA-staged z-marching passes (PF_OPT_KERNEL = 1).

They keep the per-cell arithmetic of the element-wise cp.async passes
(PF_OPT_KERNEL = 0) and change how data moves (TMA plane loads on mbarriers,
4- or 3-plane node windows) and how the boundary is written (every cell runs
the same arithmetic and fans its value out to the cells copied from it).  So
every field after N steps must carry the bits of the cp.async passes: on
grids down to the 5-cell minimum, ragged tile edges, tiles that are all
boundary, z-chunks that split the domain anywhere, one, two and three
sweeps, every noise kind, quintic h, heat diffusion, one and two cells per
thread, every window mode (3- and 4-plane windows, the own column rolled in
registers), both precisions."""
import numpy as np
import pytest

import make_golden as MG
import pf3d
from pf3d import deck

pytestmark = pytest.mark.gpu


def run(g, p, st, prec, n, kernel, paired=1, nslot=0, zchunk=64):
    with pf3d.Domain(g, p, prec) as d:
        d.set_option(pf3d.PF_OPT_KERNEL, kernel)
        d.set_option(pf3d.PF_OPT_PAIRED, paired)
        d.set_option(pf3d.PF_OPT_NSLOT, nslot)
        d.set_option(pf3d.PF_OPT_ZCHUNK, zchunk)
        d.load_state(st)
        d.step(n)
        d.sync()
        return d.fields(), d.state()


def case(nx, ny, nz, **over):
    kw = dict(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    kw.update(over)
    p = deck.run6_params(**kw)
    return deck.grid(nx, ny, nz, 0.5e-6), p, MG.small_state(nx, ny, nz, p)


SHAPES = [
    ((5, 5, 5), {}),
    ((6, 7, 9), dict(n_varreduras=1)),
    ((33, 9, 12), {}),
    ((37, 41, 29), dict(h_quintico=1, ruido_tipo=1)),
    ((100, 60, 40), {}),
    ((70, 70, 30), dict(n_varreduras=1)),
    ((71, 52, 36), dict(n_varreduras=3, AAA=0.02)),
    ((67, 43, 33), dict(ruido_tipo=2)),
    ((69, 41, 31), dict(D=2e-5)),
]


@pytest.mark.parametrize("prec", [pf3d.PF_FP64, pf3d.PF_FP32])
@pytest.mark.parametrize("shape,over", SHAPES)
def test_march_equals_cpasync_passes(gpu, prec, shape, over):
    g, p, st = case(*shape, **over)
    want, sw = run(g, p, st, prec, 5, kernel=0, paired=0)
    for paired, nslot, zchunk in ((0, 3, 64), (2, 4, 64), (2, 3, 7), (0, 4, 4), (0, 5, 64), (2, 5, 5)):
        got, sg = run(g, p, st, prec, 5, kernel=1, paired=paired, nslot=nslot, zchunk=zchunk)
        for k in want:
            assert np.array_equal(got[k], want[k]), (k, paired, nslot, zchunk)
        assert (sg.it, sg.TP, sg.M0) == (sw.it, sw.TP, sw.M0)


def test_march_status_word_clean_after_steps(gpu):
    """No plane load timed out: the status word the bounded waits would set
    stays 0, so pf_sync reports success."""
    g, p, st = case(64, 48, 40)
    with pf3d.Domain(g, p, pf3d.PF_FP64) as d:
        d.load_state(st)
        d.step(20)
        d.sync()


@pytest.mark.parametrize("prec", [pf3d.PF_FP64, pf3d.PF_FP32])
@pytest.mark.parametrize("sweeps", [1, 2])
def test_march_batch_equals_cpasync_batch(gpu, prec, sweeps):
    """A batch of uneven small domains (tiles that are all boundary, ragged
    edges, mixed noise kinds) on the TMA passes, with one and two cells per
    thread and every window mode, against the same batch on the cp.async
    passes; a domain leaves mid-run at its target step."""
    cases = [case(40, 33, 50, n_varreduras=sweeps), case(21, 64, 17, T0=918.0, taxa_resfr=30.0, n_varreduras=sweeps),
             case(70, 12, 35, AAA=0.02, ruido_tipo=1, n_varreduras=sweeps),
             case(32, 32, 32, n_varreduras=sweeps, h_quintico=1)]
    targets = [0, 6, 0, 0]

    def run(kernel, paired, nslot):
        with pf3d.Batch(prec) as b:
            b.set_kernel(kernel, nslot)
            slots = []
            for (g, p, st), tgt in zip(cases, targets):
                s = b.add(g, p)
                b.load_state(s, st)
                b.set_target(s, tgt)
                slots.append(s)
            b.set_paired(paired)
            b.set_tile(8, 16)
            b.step(5)
            b.set_tile(8, 64)
            b.step(6)
            return [b.fields(s) for s in slots], [b.state(s).it for s in slots]

    want, wit = run(0, 0, 0)
    for paired, nslot in ((0, 3), (1, 4), (1, 3), (0, 5), (1, 5)):
        got, git = run(1, paired, nslot)
        assert git == wit
        for i, (a, b) in enumerate(zip(got, want)):
            for k in b:
                assert np.array_equal(a[k], b[k]), (i, k, paired, nslot)
