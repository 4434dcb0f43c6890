"""GPU test of the two-cells-per-thread fused passes: on 32 x 8 tiles the
paired kernels (packed f32x2 arithmetic in FP32, two FP64 chains per thread)
give every field the bits of the one-cell kernels, on grids with interior
and boundary tiles, ragged edges, one and two sweeps, both precisions; decks
they do not cover (smooth noise, heat diffusion) fall back to the one-cell
kernels with unchanged results."""
import numpy as np
import pytest

import make_golden as MG
import pf3d
from pf3d import deck

pytestmark = pytest.mark.gpu


def run(g, p, st, prec, paired, n):
    with pf3d.Domain(g, p, prec) as d:
        d.set_option(pf3d.PF_OPT_PAIRED, paired)   # 2: paired in both precisions
        d.load_state(st)
        d.step(n)
        return d.fields(), d.state()


@pytest.mark.parametrize("prec", [pf3d.PF_FP64, pf3d.PF_FP32])
@pytest.mark.parametrize("shape,over", [
    ((100, 60, 40), {}),
    ((77, 45, 70), dict(h_quintico=1, ruido_tipo=1)),
    ((70, 70, 30), dict(n_varreduras=1)),
    ((71, 52, 36), dict(n_varreduras=3, AAA=0.02)),
    ((67, 43, 33), dict(ruido_tipo=2)),          # one-cell fallback
    ((69, 41, 31), dict(D=2e-5)),                # one-cell fallback
])
def test_paired_equals_one_cell(gpu, prec, shape, over):
    nx, ny, nz = shape
    kw = dict(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    kw.update(over)
    p = deck.run6_params(**kw)
    g = deck.grid(nx, ny, nz, 0.5e-6)
    st = MG.small_state(nx, ny, nz, p)
    a, sa = run(g, p, st, prec, 2, 7)
    b, sb = run(g, p, st, prec, 0, 7)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert (sa.it, sa.TP, sa.M0) == (sb.it, sb.TP, sb.M0)
