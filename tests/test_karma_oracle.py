"""CPU tests of the Karma model's checker and host logic: the C oracle
(oracle/karma_oracle.c) and an independent numpy restatement
(tests/golden/np_karma.py), both written from karma/karma3d.f90, agree bit
for bit; the noise hash agrees; the namelist reader and the dimensional
scales follow karma3d.f90:80-124."""
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
sys.path.insert(0, os.path.join(HERE, "golden"))

import np_karma as NK  # noqa: E402
import pyoracle as O  # noqa: E402
from pf3d import karma  # noqa: E402


@pytest.mark.parametrize("nx,ny,nz,Fn", [(12, 10, 9, 0.01), (16, 16, 16, 0.0), (9, 14, 11, 0.05)])
def test_c_oracle_equals_numpy_restatement(nx, ny, nz, Fn):
    phi, U = NK.seed_state(nx, ny, nz, 0.8, 5.0, 0.55)
    o = O.KarmaOracle(nx, ny, nz, 4.0, 0.02, 0.8, 0.008, Fn, 0.14)
    o.set(phi, U)
    n = NK.Karma(nx, ny, nz, 4.0, 0.02, 0.8, 0.008, Fn, 0.14)
    n.set(phi, U)
    for _ in range(3):
        o.step(6)
        n.step(6)
        for a, b in zip(o.get(), n.get()):
            assert np.array_equal(a, b)
        assert o.tip() == n.tip()


def test_noise_hash_equals_numpy():
    r = NK.ruido_grid(5, 4, 3, 17)
    for k in range(3):
        for j in range(4):
            for i in range(5):
                assert O.karma_ruido(i + 1, j + 1, k + 1, 17) == r[k, j, i]
    assert all(-1.0 <= O.karma_ruido(i, 3, 5, 11) < 1.0 for i in range(1, 50))


NML = """! test deck in the karma.nml format
&karma
  N = 48,  lambda = 3.5     ! coupling
  eps4 = 0.015
  dx = 0.9, dt = 0.01
  Fnoise = 0.02
  nsteps = 1234
  nout = 100
  tip_stop = 0.8
  TP = 910.0
/
"""


def test_read_nml(tmp_path):
    f = tmp_path / "karma.nml"
    f.write_text(NML)
    p, run = karma.read_nml(str(f))
    assert (p.nx, p.ny, p.nz) == (48, 48, 48)
    assert (p.lambda_, p.eps4, p.dx, p.dt, p.Fnoise, p.TP) == (3.5, 0.015, 0.9, 0.01, 0.02, 910.0)
    assert (p.k, p.Tm, p.R0) == (0.14, 933.3, 8.0)   # program defaults
    assert run == {"nsteps": 1234, "nout": 100, "tip_stop": 0.8}


def test_derived_scales():
    p = karma.karma_params()
    d = karma.derived(p)
    a1, a2 = 0.8839, 0.6267
    cl0 = (p.Tm - p.TP) / p.mliq
    Om = (cl0 - p.C0) / ((1.0 - p.k) * cl0)
    Gam = p.sigma * p.Tm / p.dH
    d0 = Gam / (p.mliq * (1.0 - p.k) * cl0)
    W = p.lambda_ / a1 * d0
    tau0 = a2 * p.lambda_ * W * W / p.Dl
    assert (d.D, d.cl0, d.Omega, d.Gam, d.d0, d.W, d.tau0) == (a2 * p.lambda_, cl0, Om, Gam, d0, W, tau0)
    assert math.isclose(d.Omega, 0.55, rel_tol=1e-3)   # the classic case of Karma 2001


def test_karma_create_needs_a_device_or_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-device error path")
    with pytest.raises(Exception):
        karma.Karma(karma.karma_params(N=8))
