"""GPU test against the reference's own recorded run: run6.

The reference's run log records the tip height (the highest point with
phi >= 0.5) of its 3-D run6 at 7.5, 15, 22.5, 30, 45 and 52.5 ms of real
time: 7, 14, 26, 43, 80 and 99 um (registro_runs.md:138-140;
docs/run6/README.md:58-59 gives 43 and 99 um at 30 and 52.5 ms).  That run
used the run6 deck (docs/run6/entrada_run6.dat: 340 x 340 x 700 cells,
dx = 0.15 um, T0 = 922 K cooled at 19.84 K/s, AAA = 0.03, cubic h(phi), the
positive cell noise, two phase sweeps a step, dt = dx^2/(7.5 D_liq) = 1 us,
entrada.f90:173) and the planar-front initial state (tipo_inicial 3:
phi = 1 and c = Ke C0 on the planes k <= 4, phi = 0 and c = C0 above,
T = T0; entrada.f90:226-262).  The reference's noise is a seedless hash of the cell
and the step (variaveis.f90:73-92), so the same deck and initial state give
the same run: the fused FP64 step of this library, stepped to the same
times, must give the recorded heights to the record's precision (whole
micrometres: |height - record| < 0.5 um).  This pins the product against
output of the reference itself, through 52 500 steps of the full physics.
About four minutes on a B200."""
import json

import numpy as np
import pytest

import pf3d
from pf3d import deck

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

NX, NY, NZ, DX = 340, 340, 700, 1.5e-7
RECORD_UM = [(7.5, 7.0), (15.0, 14.0), (22.5, 26.0), (30.0, 43.0), (45.0, 80.0), (52.5, 99.0)]


def planar_front_state(p):
    """tipo_inicial 3 of entrada.f90:226-262 (solid on the planes k <= 4)."""
    phi = np.zeros((NZ, NY, NX))
    phi[:4] = 1.0
    Ke = float(np.float32(p.Ke))   # Ke is REAL(4) in the reference
    c = np.where(phi >= 1.0, Ke * p.C0, p.C0)
    return {"phi": phi, "c": c, "T": np.full(phi.shape, p.T0)}


def test_run6_tip_heights_match_the_reference_record(gpu):
    p = deck.run6_params()
    g = deck.grid(NX, NY, NZ, DX)
    got = []
    with pf3d.Domain(g, p, pf3d.PF_FP64) as d:
        d.load_state(planar_front_state(p))
        dt = d.derived().DELTA_T
        assert abs(dt - 1e-6) < 1e-18            # dx^2 / (7.5 D_liq)
        it = 0
        for t_ms, _ in RECORD_UM:
            target = int(round(t_ms * 1e-3 / dt))
            d.step(target - it)
            it = target
            _, tip_cells, _ = d.track()
            got.append(tip_cells * DX * 1e6)
    print(json.dumps({"run6_tip_um": [round(h, 3) for h in got], "record_um": [r for _, r in RECORD_UM]}))
    for (t_ms, rec), h in zip(RECORD_UM, got):
        assert abs(h - rec) < 0.5, (t_ms, h, rec)
