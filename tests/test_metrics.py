"""Known answers of the host solidification metrics (pf3d.metrics), which the
device tracking (pf_track) is held to bit for bit in the GPU tests."""
import numpy as np

from pf3d import metrics


def test_all_liquid():
    phi = np.zeros((8, 4, 4))
    assert metrics.solid_fraction(phi) == 0.0
    assert metrics.tip_position(phi) == 0.0


def test_solid_to_the_top():
    phi = np.ones((8, 4, 4))
    assert metrics.solid_fraction(phi) == 1.0
    assert metrics.tip_position(phi) == 8.0


def test_interpolated_tip_and_fraction():
    nz = 10
    phi = np.zeros((nz, 4, 4))
    phi[:3] = 1.0                       # planes k = 1..3 solid
    phi[3, 2, 1] = 0.75                 # one column reaches into plane 4
    phi[4, 2, 1] = 0.25
    # top solid plane 4 (1-based), crossing halfway to plane 5
    assert metrics.tip_position(phi) == 4.5
    assert metrics.solid_fraction(phi) == (3 * 16 + 1) / (nz * 16)


def test_l2_rel():
    b = np.array([3.0, 4.0])
    assert metrics.l2_rel(b, b) == 0.0
    assert metrics.l2_rel(np.array([3.0, 5.0]), b) == 0.2
    assert metrics.l2_rel(b, np.zeros(2)) == 5.0
