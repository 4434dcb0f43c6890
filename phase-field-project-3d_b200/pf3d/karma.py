"""The reference's quantitative Karma model (karma/karma3d.f90) on the device.

`read_nml(path)` reads the `&karma` namelist of karma.nml (karma3d.f90:80-95)
into a `pf_karma_params` with the program's defaults for names the file does
not set; `Karma` is one domain resident on the GPU with the program's steps
(`seed`, `step`, `tip`) through the C-ABI of libpf3d.so; `seed_state` is the
program's initial state on the host (karma3d.f90:130-144).  Nothing here
computes the model on the CPU.
"""
from __future__ import annotations

import ctypes as C
import re

import numpy as np

from ._abi import (LIB, check, pf_karma_params, pf_karma_derived, PF_FP64, PF_FP32, PF_KARMA_PHI, PF_KARMA_U,
                   PF_KARMA_DPHI)

__all__ = ["Karma", "read_nml", "karma_params", "derived", "seed_state"]

# karma3d.f90:80-92 (program defaults)
DEFAULTS = dict(N=200, lambda_=4.0, eps4=0.02, dx=0.8, dt=0.008, R0=8.0, Fnoise=0.0, nsteps=100000, nout=2000,
                tip_stop=0.9, k=0.14, Tm=933.3, mliq=640.0, C0=0.0196, TP=909.5, sigma=0.093, dH=0.891002e9,
                Dl=3.0e-9)


def karma_params(**over) -> pf_karma_params:
    """Program defaults with overrides (N sets nx = ny = nz; `lambda_` is the
    namelist's `lambda`)."""
    v = dict(DEFAULTS)
    v.update(over)
    p = pf_karma_params()
    n = int(v["N"])
    p.nx = int(v.get("nx", n))
    p.ny = int(v.get("ny", n))
    p.nz = int(v.get("nz", n))
    for name in ("lambda_", "eps4", "dx", "dt", "R0", "Fnoise", "k", "Tm", "mliq", "C0", "TP", "sigma", "dH", "Dl"):
        setattr(p, name, float(v[name]))
    return p


def read_nml(path: str):
    """(pf_karma_params, run settings {nsteps, nout, tip_stop}) from a karma.nml
    file: `name = value` pairs inside `&karma ... /`, `!` comments, several
    pairs per line separated by commas."""
    text = open(path).read()
    m = re.search(r"&karma(.*?)^\s*/", text, flags=re.S | re.M | re.I)
    if not m:
        raise ValueError(f"{path}: no &karma namelist")
    vals = {}
    for line in m.group(1).splitlines():
        line = line.split("!", 1)[0]
        for item in line.split(","):
            if "=" not in item:
                continue
            key, val = (t.strip() for t in item.split("=", 1))
            if not key:
                continue
            key = "lambda_" if key.lower() == "lambda" else key
            vals[key] = float(val.replace("d", "e").replace("D", "e"))
    over = {k: v for k, v in vals.items() if k in DEFAULTS}
    run = {k: (int(over.get(k, DEFAULTS[k])) if k != "tip_stop" else float(over.get(k, DEFAULTS[k])))
           for k in ("nsteps", "nout", "tip_stop")}
    return karma_params(**over), run


def derived(p: pf_karma_params) -> pf_karma_derived:
    out = pf_karma_derived()
    check(LIB.pf_karma_derived_of(C.byref(p), C.byref(out)))
    return out


def seed_state(p: pf_karma_params):
    """karma3d.f90:130-144 on the host: phi = -tanh((r - R0)/sqrt 2) at the cell
    centres (i - 1/2) dx, U = -Omega; arrays of shape (nz, ny, nx)."""
    k, j, i = np.meshgrid(np.arange(1, p.nz + 1), np.arange(1, p.ny + 1), np.arange(1, p.nx + 1), indexing="ij")
    x, y, z = (i - 0.5) * p.dx, (j - 0.5) * p.dx, (k - 0.5) * p.dx
    r = np.sqrt(x * x + y * y + z * z)
    return -np.tanh((r - p.R0) / np.sqrt(2.0)), np.full(r.shape, -derived(p).Omega)


class Karma:
    """One Karma domain on the GPU."""

    def __init__(self, p: pf_karma_params, precision: int = PF_FP64):
        self.params = p
        self.precision = precision
        self.shape = (p.nz, p.ny, p.nx)
        self._h = C.c_void_p()
        check(LIB.pf_karma_create(C.byref(p), precision, C.byref(self._h)))

    def close(self):
        if self._h:
            LIB.pf_karma_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def derived(self) -> pf_karma_derived:
        return derived(self.params)

    @property
    def it(self) -> int:
        v = C.c_int()
        check(LIB.pf_karma_get_it(self._h, C.byref(v)))
        return v.value

    @it.setter
    def it(self, value: int):
        check(LIB.pf_karma_set_it(self._h, int(value)))

    def set_stream(self, stream: int):
        check(LIB.pf_karma_set_stream(self._h, C.c_void_p(stream)))

    def upload(self, phi: np.ndarray, U: np.ndarray):
        for f, a in ((PF_KARMA_PHI, phi), (PF_KARMA_U, U)):
            a = np.ascontiguousarray(a, dtype=np.float64)
            if a.size != self.params.nx * self.params.ny * self.params.nz:
                raise ValueError("array size does not match the grid")
            check(LIB.pf_karma_upload(self._h, f, a.ctypes.data_as(C.c_void_p)))

    def download(self, field: int = PF_KARMA_PHI) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        check(LIB.pf_karma_download(self._h, field, out.ctypes.data_as(C.c_void_p)))
        return out

    def fields(self):
        return self.download(PF_KARMA_PHI), self.download(PF_KARMA_U), self.download(PF_KARMA_DPHI)

    def seed(self):
        check(LIB.pf_karma_seed(self._h))

    def step(self, n: int = 1):
        check(LIB.pf_karma_step(self._h, int(n)))

    def sync(self):
        check(LIB.pf_karma_sync(self._h))

    def tip(self):
        a, b = C.c_int(), C.c_int()
        check(LIB.pf_karma_tip(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value


FP64, FP32 = PF_FP64, PF_FP32
DPHI = PF_KARMA_DPHI
