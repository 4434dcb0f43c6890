"""GPU tests of pf_principal, the reference's main program (principal.f90)
in C++ on the C-ABI: deck reading, the entrada initial state, the step
order, the output cadence and the Tecplot POINT writer, against the oracle."""
import glob
import os
import subprocess

import numpy as np
import pytest

import pyoracle as O
from conftest import ROOT, RTOL_FP64, max_rel
from pf3d import deck

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "phase-field-project-3d_b200", "pf3d", "pf_principal")
NX, NY, NZ, STEPS, EVERY = 24, 20, 30, 10, 4


def write_deck(path, it_max=STEPS):
    vals = ["933.3", "922.0d0", "0.891002000d+09", "1.055d-03", "673.2d+3", "1.9d-03", "6.59477338d-05",
            "3.23646776d-05", "2.926560e+06", "2.626320e+06", str(NX), str(NY), str(NZ), "0.5d-06", "0.5d-06",
            "0.5d-06", "1.d-23", "4.d0", str(it_max), "0.01d0", "0.d0", "0.03d0", "1.5d-07", "3.0d-13", "3.0d-09",
            "0.14d0", "640d0", "1.130d-05", "8.31451D0", "0.0196d0", "4.d0", "0.093d+0", "1", "2.d0", "10.0d0",
            str(EVERY), "905.0d0", "3   0.d0", "19.84d0  2", "0  0"]
    with open(path, "w") as f:
        f.write("deck\n\n\n" + "\n".join(v + "   | comment" for v in vals) + "\n")


def oracle_after(n):
    g, p, _ = deck.read_entrada(str(DECK))
    o = O.Oracle(g, p)
    k = np.arange(1, NZ + 1)[:, None, None] * np.ones((NZ, NY, NX))
    solid = k <= 4
    ke = float(np.float32(p.Ke))
    o.load_state({"phi": np.where(solid, 1.0, 0.0), "c": np.where(solid, ke * p.C0, p.C0),
                  "T": np.full((NZ, NY, NX), p.T0)})
    o.step(n)
    return o


DECK = None


@pytest.fixture()
def rundir(tmp_path, gpu):
    global DECK
    DECK = tmp_path / "entrada.dat"
    write_deck(DECK)
    return tmp_path


def run(rundir, *args):
    r = subprocess.run([EXE, "--dir", str(rundir), *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def final_state(rundir):
    a = np.fromfile(rundir / "output" / "final_state.bin", dtype=np.float64)
    n = NX * NY * NZ
    return a[:n].reshape(NZ, NY, NX), a[n:].reshape(NZ, NY, NX)


def test_principal_matches_oracle(rundir):
    out = run(rundir)
    assert out.count("ESCREVENDO RESULTADOS") == 2               # it = 5 and 9
    files = sorted(glob.glob(str(rundir / "output" / "saida_*9_time_*.dat")))
    assert len(files) == 1
    rows = np.loadtxt(files[0], skiprows=4)
    assert rows.shape == (NX * NY * NZ, 6)
    o9 = oracle_after(9)
    phi9 = o9.get(1).ravel()
    assert np.allclose(rows[:, 3], phi9, rtol=1e-7, atol=1e-12)   # ES15.7E3 keeps 8 digits
    phi, c = final_state(rundir)
    o10 = oracle_after(10)
    assert max_rel(phi, o10.get(0)) <= RTOL_FP64 and max_rel(c, o10.get(2)) <= RTOL_FP64


def test_principal_fused_equals_per_subroutine(rundir):
    run(rundir, "--quiet")
    a = final_state(rundir)
    run(rundir, "--quiet", "--fused")
    b = final_state(rundir)
    assert max_rel(b[0], a[0]) <= RTOL_FP64 and max_rel(b[1], a[1]) <= RTOL_FP64
