"""Properties of the host initial-state recipe (pf3d.init), which the device
seed (pf_init_seeded) is held to bit for bit in the GPU tests."""
import numpy as np
import pytest

from pf3d import deck, init


@pytest.mark.parametrize("n", [1, 5, 16])
def test_bump_sites(n):
    s = init.bump_sites(40, 24, n, seed=7)
    assert s.shape == (n, 2)
    assert (s[:, 0] >= 1).all() and (s[:, 0] <= 40.5).all()
    assert (s[:, 1] >= 1).all() and (s[:, 1] <= 24.5).all()
    np.testing.assert_array_equal(s, init.bump_sites(40, 24, n, seed=7))     # seeded
    assert not np.array_equal(s, init.bump_sites(40, 24, n, seed=8))


def test_initial_state():
    p = deck.run6_params()
    nx, ny, nz = 24, 20, 48
    st = init.initial_state(nx, ny, nz, 4, 3, p)
    phi, c, T = st["phi"], st["c"], st["T"]
    assert phi.shape == c.shape == T.shape == (nz, ny, nx)
    assert phi.flags.c_contiguous
    assert phi.min() >= 0.0 and phi.max() <= 1.0
    assert (phi[:4] > 0.5).all()            # the slab k <= 4 (1-based) is solid
    assert (phi[-1] == 0.0).all()           # far above the interface tanh saturates exactly
    ke = float(np.float32(p.Ke))
    np.testing.assert_allclose(c, p.C0 * (1.0 - (1.0 - ke) * phi), rtol=0, atol=0)
    assert (T == p.T0).all()
    # bumps raise the interface above the flat slab somewhere
    flat = 0.5 * (1.0 - np.tanh(2.0 * (5.0 - init.SLAB_TOP) / float(p.Thin_Interface)))
    assert phi[4].max() > flat
