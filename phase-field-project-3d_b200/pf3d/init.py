"""Seeded synthetic initial states (host side, like the reference's entrada).

Fields are numpy arrays of shape (nz, ny, nx), C-contiguous float64, which
is the same memory order as the reference's Fortran arrays (i fastest).

Recipe (phase phi in [0, 1], 1 = solid, the reference's convention
phase_body.inc:198):
  * a bottom slab of 4 cells (k <= 4) carrying hemispherical bumps of radius
    3 cells at jittered lattice sites (numpy default_rng(seed));
  * phi = (1 - tanh(2 d / w)) / 2 with d the signed distance (in cells) to
    slab U bumps and w = Thin_Interface cells, the interface width
    Lambda = Thin_Interface*dx of entrada.f90:161;
  * c = C0 (1 - (1 - Ke) phi): Ke*C0 in the solid, C0 in the liquid;
  * T = T0 everywhere, DPP = 0 (entrada.f90:253-257).
"""
from __future__ import annotations

import math

import numpy as np

SLAB_TOP = 4.5      # cells k <= 4 (1-based) are solid
BUMP_R = 3.0


def bump_sites(nx: int, ny: int, n_bumps: int, seed: int) -> np.ndarray:
    """(n_bumps, 2) 1-based (i, j) centres on a jittered lattice."""
    rng = np.random.default_rng(seed)
    m = max(1, int(math.ceil(math.sqrt(n_bumps))))
    sx, sy = nx / m, ny / m
    ii, jj = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    base = np.stack([(ii.ravel() + 0.5) * sx, (jj.ravel() + 0.5) * sy], axis=1)
    jit = rng.uniform(-0.25, 0.25, size=base.shape) * np.array([sx, sy])
    sites = base + jit + 0.5          # to 1-based cell coordinates
    if n_bumps < m * m:
        pick = rng.choice(m * m, size=n_bumps, replace=False)
        sites = sites[np.sort(pick)]
    return sites


def phase_field(nx: int, ny: int, nz: int, n_bumps: int, seed: int, width_cells: float) -> np.ndarray:
    sites = bump_sites(nx, ny, n_bumps, seed)
    # beyond this many planes above the slab tanh saturates to exactly 1 in FP64
    kmax = min(nz, int(SLAB_TOP + BUMP_R + 20.0 * width_cells / 2.0) + 2)
    phi = np.zeros((nz, ny, nx), dtype=np.float64)
    k = np.arange(1, kmax + 1, dtype=np.float64)[:, None, None]
    j = np.arange(1, ny + 1, dtype=np.float64)[None, :, None]
    i = np.arange(1, nx + 1, dtype=np.float64)[None, None, :]
    d = np.broadcast_to(k - SLAB_TOP, (kmax, ny, nx)).copy()
    reach = BUMP_R + 10.0 * width_cells
    for (ci, cj) in sites:
        i0, i1 = max(1, int(ci - reach)), min(nx, int(ci + reach) + 1)
        j0, j1 = max(1, int(cj - reach)), min(ny, int(cj + reach) + 1)
        sub_i = i[:, :, i0 - 1:i1]
        sub_j = j[:, j0 - 1:j1, :]
        db = np.sqrt((sub_i - ci) ** 2 + (sub_j - cj) ** 2 + (k - SLAB_TOP) ** 2) - BUMP_R
        view = d[:, j0 - 1:j1, i0 - 1:i1]
        np.minimum(view, db, out=view)
    phi[:kmax] = 0.5 * (1.0 - np.tanh(2.0 * d / width_cells))
    return phi


def initial_state(nx: int, ny: int, nz: int, n_bumps: int, seed: int, params) -> dict:
    phi = phase_field(nx, ny, nz, n_bumps, seed, float(params.Thin_Interface))
    ke = float(np.float32(params.Ke))
    c = params.C0 * (1.0 - (1.0 - ke) * phi)
    T = np.full((nz, ny, nx), params.T0, dtype=np.float64)
    return {"phi": phi, "c": c, "T": T}


def workload_state(w) -> dict:
    return initial_state(w.nx, w.ny, w.nz, w.n_bumps, w.seed, w.params())
