"""Solidification metrics of a phase field (arrays of shape (nz, ny, nx)).

solid_fraction : mean(phi >= 0.5)
tip_position   : largest height (cells, 1-based k) where any (i, j) column
                 has phi >= 0.5, linearly interpolated to the 0.5 crossing
                 above it (the "altura da ponta, phi >= 0,5" measure of the
                 reference's run log, docs/run6/README.md:54-62)
l2_rel         : |a - b|_2 / |b|_2
"""
from __future__ import annotations

import numpy as np


def solid_fraction(phi: np.ndarray) -> float:
    return float((phi >= 0.5).mean())


def tip_position(phi: np.ndarray) -> float:
    solid = (phi >= 0.5).any(axis=(1, 2))
    ks = np.nonzero(solid)[0]
    if len(ks) == 0:
        return 0.0
    k = int(ks[-1])                      # 0-based top solid plane
    if k + 1 >= phi.shape[0]:
        return float(k + 1)
    lo = phi[k].max()                    # >= 0.5
    hi = phi[k + 1].max()                # < 0.5
    frac = (lo - 0.5) / (lo - hi) if lo > hi else 0.0
    return float(k + 1 + frac)


def l2_rel(a: np.ndarray, b: np.ndarray) -> float:
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a))
