"""Physics deck (the reference's entrada.dat) and the workload configurations.

`run6_params()` is the deck of the reference's documented run6
(entrada.dat:4-43, docs/run6/README.md:7-10): Al-4.5 wt% Cu, cubic h(phi),
positive cell noise, two phase sweeps per step, continuous cooling.
`read_entrada()` parses a deck file the way entrada.f90:17-89 reads it:
three header lines, then the first value of each line, positional.
"""
from __future__ import annotations

import ctypes as C
import re
from dataclasses import dataclass, field

from ._abi import pf_grid, pf_params, PF_BC_REFERENCE


def run6_params(**over) -> pf_params:
    p = pf_params()
    p.Tm = 933.3
    p.T0 = 922.0
    p.delta_H = 0.891002000e+09
    p.M0 = 1.9e-03
    p.Cp_s = 2.926560e+06
    p.D = 0.0            # module variable D is never assigned in the reference
    p.AAA = 0.03
    p.DELTA_EPSLON = 0.03
    p.D_sol = 3.0e-13
    p.D_liq = 3.0e-09
    p.Ke = 0.14
    p.Me = 640.0
    p.Vm = 1.130e-05
    p.R = 8.31451
    p.C0 = 0.0196
    p.Thin_Interface = 4.0
    p.Sigma = 0.093
    p.Beta = 1.0
    p.ajuste = 2.0
    p.TP = 905.0
    p.taxa_resfr = 19.84
    p.n_varreduras = 2
    p.h_quintico = 0
    p.ruido_tipo = 0
    p.bc = PF_BC_REFERENCE
    p.stoptime = 0.085
    p.WriteFileD_timeCounter = 7500
    for k, v in over.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def params_copy(p: pf_params, **over) -> pf_params:
    q = pf_params()
    C.pointer(q)[0] = p
    for k, v in over.items():
        setattr(q, k, v)
    return q


def grid(nx: int, ny: int, nz: int, dx: float, dy: float | None = None, dz: float | None = None) -> pf_grid:
    return pf_grid(nx, ny, nz, dx, dx if dy is None else dy, dx if dz is None else dz)


_NUM = re.compile(r"^\s*([-+0-9.eEdD]+)")


def read_entrada(path: str):
    """Parse an entrada.dat deck (positional, first value per line).

    Returns (pf_grid, pf_params, extras) where extras holds the values the
    hot path does not use (it_max, tipo_inicial, R_semente, ...).
    """
    with open(path, "r", encoding="latin-1") as f:
        lines = f.read().splitlines()[3:]

    def val(n, conv=float, default=None):
        if n >= len(lines):
            return default
        m = _NUM.match(lines[n])
        if not m:
            return default
        return conv(float(m.group(1).replace("d", "e").replace("D", "e")))

    def pair(n, c1, c2, default):
        if n >= len(lines):
            return default
        toks = lines[n].split()
        try:
            return (c1(float(toks[0].replace("d", "e").replace("D", "e"))),
                    c2(float(toks[1].replace("d", "e").replace("D", "e"))))
        except (IndexError, ValueError):
            return default

    p = pf_params()
    p.Tm, p.T0, p.delta_H = val(0), val(1), val(2)
    E0_deck, W0_deck = val(3), val(4)
    p.M0 = val(5)
    p.Cp_s = val(8)
    nx, ny, nz = val(10, int), val(11, int), val(12, int)
    dy, dx, dz = val(13), val(14), val(15)
    it_max = val(18, int)
    p.AAA = val(19)
    p.DELTA_EPSLON = val(21)
    p.D_sol, p.D_liq = val(23), val(24)
    p.Ke = val(25)
    p.Me, p.Vm, p.R, p.C0 = val(26), val(27), val(28), val(29)
    p.Thin_Interface = val(30)
    p.Sigma, p.Beta, p.ajuste = val(31), val(32), val(33)
    p.stoptime = val(34)
    p.WriteFileD_timeCounter = val(35, int)
    tp = val(36)
    p.TP = 919.0 if tp is None else tp
    tipo, r_sem = pair(37, int, float, (0, 0.0))
    taxa, nsw = pair(38, float, int, (0.0, 1))
    p.taxa_resfr = taxa
    p.n_varreduras = max(1, nsw)
    hq, rt = pair(39, int, int, (1, 2))
    p.h_quintico, p.ruido_tipo = hq, rt
    p.D = 0.0
    p.bc = PF_BC_REFERENCE
    g = pf_grid(nx, ny, nz, dx, dy, dz)
    extras = dict(it_max=it_max, tipo_inicial=tipo, R_semente=r_sem, E0_deck=E0_deck, W0_deck=W0_deck)
    return g, p, extras


@dataclass
class Workload:
    """One synthetic workload: grid, deck overrides, seeded initial state."""
    name: str
    nx: int
    ny: int
    nz: int
    dx: float
    steps: int
    seed: int
    n_bumps: int
    precision: int = 64
    overrides: dict = field(default_factory=dict)

    def grid(self) -> pf_grid:
        return grid(self.nx, self.ny, self.nz, self.dx)

    def params(self) -> pf_params:
        return run6_params(**self.overrides)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


# Configurations: Al-4.5wt%Cu, dx = 0.5 um, T0 = 922 K cooling at 19.84 K/s,
# noise amplitude 0.01, two sweeps per step (run6 deck otherwise).
_COMMON = dict(T0=922.0, taxa_resfr=19.84, AAA=0.01)
WORKLOADS = {
    "c1_64x64x128_fp64": Workload("c1_64x64x128_fp64", 64, 64, 128, 0.5e-6, 2000, 0, 9, 64, dict(_COMMON)),
    "c2_512x512x1024_fp64": Workload("c2_512x512x1024_fp64", 512, 512, 1024, 0.5e-6, 5000, 1, 64, 64, dict(_COMMON)),
    "c3_1024cube_fp32": Workload("c3_1024cube_fp32", 1024, 1024, 1024, 0.5e-6, 10000, 2, 256, 32, dict(_COMMON)),
    "c3_replica_256x256x512_fp64": Workload("c3_replica_256x256x512_fp64", 256, 256, 512, 0.5e-6, 10000, 2, 16, 64,
                                             dict(_COMMON)),
    # profiling cases: the same kernels on a state still larger than L2
    # (4 fields x 16.8M cells = 537 MB in FP64, 268 MB in FP32)
    "ncu_256x256x256_fp64": Workload("ncu_256x256x256_fp64", 256, 256, 256, 0.5e-6, 5, 1, 16, 64, dict(_COMMON)),
    "ncu_256x256x256_fp32": Workload("ncu_256x256x256_fp32", 256, 256, 256, 0.5e-6, 5, 1, 16, 32, dict(_COMMON)),
}
