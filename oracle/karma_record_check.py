"""Checks the Karma oracle against the reference's recorded run3.

TEST INFRASTRUCTURE: runs oracle/karma_oracle.c (through pyoracle) on the
host, never the product.  The reference's run log records run3 of
karma/karma3d.f90 (registro_runs.md:99-107: the default namelist of
karma/karma.nml, 200^3 cells, Fnoise = 0.01), its tip on the axis and on the
diagonal printed every 5000 steps to 45 000 as karma3d.f90:300-302 prints
them (ponta_eixo = tip_x dx, ponta_diag = tip_d dx sqrt(3), F7.1).  This
script steps the oracle from the program's seed (karma3d.f90:130-144) and
compares every printed pair with the record; it exits non-zero on a
mismatch.  About 100 minutes on 8 host threads (OMP_NUM_THREADS; measured:
5916 s, all nine pairs equal to the record), so it is a script, not part of
the test suite; tests/test_karma_record_gpu.py makes the
same check of the GPU kernels in about 30 s.

    OMP_NUM_THREADS=8 python oracle/karma_record_check.py
"""
import json
import math
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "phase-field-project-3d_b200"))

import pyoracle            # noqa: E402
from pf3d import karma     # noqa: E402  (host-side parameters and seed only)

# step: (ponta eixo, ponta diag) in W, as recorded
RECORD = {5000: ("26.4", "24.9"), 10000: ("38.4", "33.3"), 15000: ("53.6", "40.2"), 20000: ("70.4", "47.1"),
          25000: ("88.0", "52.7"), 30000: ("104.8", "58.2"), 35000: ("121.6", "65.1"), 40000: ("139.2", "72.1"),
          45000: ("155.2", "80.4")}


def main() -> int:
    p = karma.karma_params(N=200, Fnoise=0.01)
    o = pyoracle.KarmaOracle(p.nx, p.ny, p.nz, p.lambda_, p.eps4, p.dx, p.dt, p.Fnoise, p.k)
    o.set(*karma.seed_state(p))
    t0 = time.time()
    it = 0
    bad = 0
    for target in sorted(RECORD):
        o.step(target - it)
        it = target
        tx, td = o.tip()
        got = (f"{tx * p.dx:.1f}", f"{td * p.dx * math.sqrt(3.0):.1f}")
        ok = got == RECORD[it]
        bad += not ok
        print(json.dumps({"it": it, "printed": got, "record": RECORD[it], "ok": ok, "wall_s": round(time.time() - t0, 1)}),
              flush=True)
    return 1 if bad else 0


if __name__ == "__main__":
    sys.exit(main())
