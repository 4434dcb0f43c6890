"""GPU parity of the Karma model (karma/karma3d.f90): the FP64 kernels give
the C oracle's bits after many steps (phi, U and dphi/dt, every cell) on
grids that are ragged against the 32 x 8 tiles and cross z-chunks, with and
without noise; the tip search equals the oracle's; the device seed equals
the host recipe to within the last bits of tanh; FP32 stays within a stated
error of FP64."""
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

pytestmark = pytest.mark.gpu


def pair(nx, ny, nz, Fn, precision=karma.FP64, R0=6.0):
    p = karma.karma_params(N=nx, nx=nx, ny=ny, nz=nz, Fnoise=Fn, R0=R0)
    phi, U = karma.seed_state(p)
    o = O.KarmaOracle(nx, ny, nz, p.lambda_, p.eps4, p.dx, p.dt, p.Fnoise, p.k)
    o.set(phi, U)
    g = karma.Karma(p, precision)
    g.upload(phi, U)
    return p, o, g


@pytest.mark.parametrize("nx,ny,nz,Fn", [(40, 33, 70, 0.01), (64, 64, 64, 0.0), (17, 9, 130, 0.05)])
def test_fp64_bit_identical_to_oracle(gpu, nx, ny, nz, Fn):
    p, o, g = pair(nx, ny, nz, Fn)
    with g:
        for n in (1, 19, 60):
            o.step(n)
            g.step(n)
            for name, a, b in zip(("phi", "U", "dphi"), g.fields(), o.get()):
                assert np.array_equal(a, b), (name, n, float(np.abs(a - b).max()))
            assert g.tip() == o.tip()
        assert g.it == 80


def test_noise_step_counter(gpu):
    """The noise of step n uses it = n; set_it moves the counter."""
    p, o, g = pair(20, 20, 20, 0.05)
    with g:
        g.it = 7
        o.set_it(7)
        o.step(3)
        g.step(3)
        assert g.it == 10
        for a, b in zip(g.fields(), o.get()):
            assert np.array_equal(a, b)


def test_device_seed_matches_host_recipe(gpu):
    p = karma.karma_params(N=30, nx=30, ny=22, nz=26, R0=7.0)
    phi, U = karma.seed_state(p)
    with karma.Karma(p) as g:
        g.seed()
        a, u, _ = g.fields()
    assert np.array_equal(u, U)
    assert np.max(np.abs(a - phi)) <= 4 * np.finfo(np.float64).eps


def test_fp32_error_against_fp64(gpu):
    """FP32 storage and arithmetic: after 300 steps the relative L2 error of
    phi and U against FP64 is below 1e-4 and the tip positions agree."""
    p, o, g64 = pair(48, 48, 48, 0.0)
    phi, U = karma.seed_state(p)
    with g64, karma.Karma(p, karma.FP32) as g32:
        g32.upload(phi, U)
        g64.step(300)
        g32.step(300)
        a64, u64, _ = g64.fields()
        a32, u32, _ = g32.fields()
        assert np.linalg.norm(a32 - a64) / np.linalg.norm(a64) < 1e-4
        assert np.linalg.norm(u32 - u64) / np.linalg.norm(u64) < 1e-4
        assert g32.tip() == g64.tip()
