"""GPU test of the Karma model against the reference's own recorded run.

The reference's run log records run3 of karma/karma3d.f90 (registro_runs.md:
99-107): the program's default namelist (karma/karma.nml: N = 200, lambda = 4,
eps4 = 0.02, dx = 0.8 W, dt = 0.008 tau0, a 1/8 seed of radius 8 W in the
corner, Fnoise = 0.01, Al-Cu at TP = 909.5 K), the tip printed every 5000
steps as karma3d.f90:300-302 prints it: ponta_eixo = tip_x dx and
ponta_diag = tip_d dx sqrt(3) (F7.1), tip_x and tip_d the largest i with
phi > 0 on the x axis and on the diagonal (karma3d.f90:294-297).  The noise
is a seedless hash of the cell and the step, so the run is reproducible: the
FP64 kernels, stepped the same way, must print every recorded value.  The
FP32 form must print the same axis tips and diagonal tips within one cell
(measured: equal up to step 40000, one cell short on the diagonal at
45000).  About a minute on a B200."""
import json
import math

import pytest

from pf3d import karma

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

# step: (ponta eixo, ponta diag) in W, as recorded
RECORD = {5000: ("26.4", "24.9"), 10000: ("38.4", "33.3"), 15000: ("53.6", "40.2"), 20000: ("70.4", "47.1"),
          25000: ("88.0", "52.7"), 30000: ("104.8", "58.2"), 35000: ("121.6", "65.1"), 40000: ("139.2", "72.1"),
          45000: ("155.2", "80.4")}


def run(prec):
    p = karma.karma_params(N=200, Fnoise=0.01)
    out = {}
    with karma.Karma(p, prec) as k:
        k.seed()
        it = 0
        for target in sorted(RECORD):
            k.step(target - it)
            it = target
            out[it] = k.tip()
    return p.dx, out


def test_karma_fp64_prints_the_recorded_tips(gpu):
    dx, tips = run(karma.FP64)
    printed = {it: (f"{tx * dx:.1f}", f"{td * dx * math.sqrt(3.0):.1f}") for it, (tx, td) in tips.items()}
    print(json.dumps({"karma_run3_fp64": printed}))
    assert printed == RECORD


def test_karma_fp32_tips_within_a_cell_of_the_record(gpu):
    dx, tips = run(karma.FP32)
    for it, (tx, td) in tips.items():
        ed = float(RECORD[it][1])
        assert f"{tx * dx:.1f}" == RECORD[it][0], (it, tx)
        assert abs(td - ed / (dx * math.sqrt(3.0))) <= 1.05, (it, td)
