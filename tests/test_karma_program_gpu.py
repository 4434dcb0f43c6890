"""GPU test of pf_karma3d, the Karma program of karma/karma3d.f90 on the
C-ABI: the tip lines equal the oracle's tip after the same steps, the Tecplot
file holds (1 + phi)/2 and the concentration of the oracle's fields to the
8 significant digits of ES15.7E3, and the tip-stop test ends the run."""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
import pyoracle as O  # noqa: E402
from pf3d import karma  # noqa: E402

pytestmark = pytest.mark.gpu
EXE = os.path.join(HERE, "..", "phase-field-project-3d_b200", "pf3d", "pf_karma3d")

NML = """&karma
  N = 24, lambda = 4.0, eps4 = 0.02
  dx = 0.8, dt = 0.008, R0 = 6.0
  Fnoise = 0.01     ! noise on
  nsteps = 30, nout = 10, tip_stop = 0.9
/
"""


def run(tmp_path, nml):
    (tmp_path / "karma.nml").write_text(nml)
    r = subprocess.run([EXE, "--dir", str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def test_program_tips_and_output_equal_oracle(gpu, tmp_path):
    out = run(tmp_path, NML)
    lines = [l for l in out.splitlines() if l.startswith("it=")]
    assert len(lines) == 3
    p = karma.karma_params(N=24, R0=6.0, Fnoise=0.01)
    o = O.KarmaOracle(24, 24, 24, p.lambda_, p.eps4, p.dx, p.dt, p.Fnoise, p.k)
    # the program seeds on the device: start the oracle from the device seed
    with karma.Karma(p) as g:
        g.seed()
        o.set(g.download(karma.PF_KARMA_PHI), g.download(karma.PF_KARMA_U))
    for line in lines:
        o.step(10)
        tx, td = o.tip()
        f = line.split()
        assert float(f[f.index("ponta_eixo=") + 1]) == pytest.approx(tx * p.dx, abs=0.051)
        assert float(f[f.index("ponta_diag=") + 1]) == pytest.approx(td * p.dx * np.sqrt(3.0), abs=0.051)
    data = np.loadtxt(tmp_path / "output" / "karma_0000030.dat", skiprows=4)
    assert data.shape == (24 ** 3, 6)
    phi, U, _ = o.get()
    d = karma.derived(p)
    conc = d.cl0 * 0.5 * (1.0 + p.k - (1.0 - p.k) * phi) * (1.0 + (1.0 - p.k) * U)
    np.testing.assert_allclose(data[:, 3], (0.5 * (1.0 + phi)).reshape(-1), rtol=6e-8, atol=1e-300)
    np.testing.assert_allclose(data[:, 5], conc.reshape(-1), rtol=6e-8)
    assert np.all(data[:, 4] == p.TP)


def test_program_stops_at_the_wall(gpu, tmp_path):
    out = run(tmp_path, NML.replace("tip_stop = 0.9", "tip_stop = 0.1").replace("nsteps = 30", "nsteps = 1000"))
    assert "ponta chegou perto da parede" in out
    assert len([l for l in out.splitlines() if l.startswith("it=")]) == 1
