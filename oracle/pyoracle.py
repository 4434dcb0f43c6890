"""ctypes binding of the CPU oracle (oracle/build/libpf_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference arm of bench.py, never by the product package.
Builds the library with `make -C oracle` on first use if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libpf_oracle.so")


def build():
    subprocess.run(["make", "-C", HERE], check=True, stdout=subprocess.DEVNULL)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    return C.CDLL(LIB_PATH)


class _Params(C.Structure):
    """Same layout as pf_params of include/pf3d.h (the oracle reuses it)."""
    _fields_ = [
        ("Tm", C.c_double), ("T0", C.c_double), ("delta_H", C.c_double), ("M0", C.c_double),
        ("Cp_s", C.c_double), ("D", C.c_double), ("AAA", C.c_double), ("DELTA_EPSLON", C.c_double),
        ("D_sol", C.c_double), ("D_liq", C.c_double), ("Ke", C.c_float), ("Me", C.c_double),
        ("Vm", C.c_double), ("R", C.c_double), ("C0", C.c_double), ("Thin_Interface", C.c_double),
        ("Sigma", C.c_float), ("Beta", C.c_float), ("ajuste", C.c_float), ("TP", C.c_double),
        ("taxa_resfr", C.c_double), ("n_varreduras", C.c_int), ("h_quintico", C.c_int),
        ("ruido_tipo", C.c_int), ("bc", C.c_int), ("stoptime", C.c_double),
        ("WriteFileD_timeCounter", C.c_int),
    ]


LIB = _load()
_V = C.c_void_p
LIB.orc_pseudo_random.restype = C.c_double
LIB.orc_pseudo_random.argtypes = [C.c_int] * 5
LIB.orc_ruido_suave.restype = C.c_double
LIB.orc_ruido_suave.argtypes = [C.c_int] * 4
LIB.orc_w0_e0.restype = None
LIB.orc_w0_e0.argtypes = [C.c_double, C.c_float, C.c_float, C.POINTER(C.c_double), C.POINTER(C.c_double),
                          C.POINTER(C.c_long)]
LIB.orc_auxiliar.restype = C.c_double
LIB.orc_auxiliar.argtypes = [_V, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
LIB.orc_create.restype = _V
LIB.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _V]
for _n in ("orc_destroy", "orc_temperatura", "orc_equacao_campo_fase", "orc_copy_phase_new_to_old",
           "orc_concentracao_soluto", "orc_swap", "orc_step"):
    getattr(LIB, _n).restype = None
    getattr(LIB, _n).argtypes = [_V]
LIB.orc_set_field.argtypes = [_V, C.c_int, _V]
LIB.orc_get_field.argtypes = [_V, C.c_int, _V]
LIB.orc_diagnosticos.argtypes = [_V, C.POINTER(C.c_double)]
LIB.orc_run.argtypes = [_V, C.c_int]
LIB.orc_get_scalars.argtypes = [_V, C.POINTER(C.c_double)]
LIB.orc_set_scalars.argtypes = [_V, C.c_int, C.c_double, C.c_double, C.c_float]
LIB.orc_num_threads.restype = C.c_int


def as_params(p) -> _Params:
    q = _Params()
    C.memmove(C.byref(q), C.byref(p), C.sizeof(q))
    return q


def pseudo_random(i, j, k, it, salt) -> float:
    return LIB.orc_pseudo_random(i, j, k, it, salt)


def ruido_suave(i, j, k, it) -> float:
    return LIB.orc_ruido_suave(i, j, k, it)


def w0_e0(Lambda: float, ajuste: float, Sigma: float):
    W0, E0, n = C.c_double(), C.c_double(), C.c_long()
    LIB.orc_w0_e0(Lambda, ajuste, Sigma, C.byref(W0), C.byref(E0), C.byref(n))
    return W0.value, E0.value, n.value


def auxiliar(p, TP, Cs_eq, Cl_eq, E0, W0) -> float:
    q = as_params(p)
    return LIB.orc_auxiliar(C.byref(q), TP, Cs_eq, Cl_eq, E0, W0)


class Oracle:
    """The reference's module state + subroutines on the CPU."""

    def __init__(self, g, p):
        self._p = as_params(p)
        self.shape = (g.nz, g.ny, g.nx)
        self._h = LIB.orc_create(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, C.byref(self._p))
        if not self._h:
            raise ValueError("oracle: grid too small or out of memory")

    def close(self):
        if self._h:
            LIB.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set(self, field: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        LIB.orc_set_field(self._h, field, a.ctypes.data_as(_V))

    def get(self, field: int) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        LIB.orc_get_field(self._h, field, out.ctypes.data_as(_V))
        return out

    def load_state(self, st: dict):
        self.set(0, st["phi"])
        self.set(2, st["c"])
        self.set(4, st["T"])
        self.set(6, st.get("dpp", np.zeros(self.shape)))

    def scalars(self) -> dict:
        out = (C.c_double * 10)()
        LIB.orc_get_scalars(self._h, out)
        keys = ("dt", "AAA", "Lambda", "W0", "E0", "TP", "M0", "it", "time", "w0e0_iters")
        return dict(zip(keys, out))

    def set_scalars(self, it, TP, M0, time):
        LIB.orc_set_scalars(self._h, it, TP, M0, time)

    def temperatura(self):
        LIB.orc_temperatura(self._h)

    def equacao_campo_fase(self):
        LIB.orc_equacao_campo_fase(self._h)

    def copy_phase_new_to_old(self):
        LIB.orc_copy_phase_new_to_old(self._h)

    def concentracao_soluto(self):
        LIB.orc_concentracao_soluto(self._h)

    def swap(self):
        LIB.orc_swap(self._h)

    def diagnosticos(self):
        out = (C.c_double * 5)()
        LIB.orc_diagnosticos(self._h, out)
        return tuple(out)

    def step(self, n: int = 1):
        LIB.orc_run(self._h, int(n))

    def fields(self) -> dict:
        return {"phi": self.get(0), "c": self.get(2), "T": self.get(4), "dpp": self.get(6)}


def num_threads() -> int:
    return LIB.orc_num_threads()


# ---- the quantitative Karma model (karma/karma3d.f90) ----
LIB.orc_karma_ruido.restype = C.c_double
LIB.orc_karma_ruido.argtypes = [C.c_int] * 4
LIB.orc_karma_create.restype = _V
LIB.orc_karma_create.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_double] * 6
LIB.orc_karma_destroy.argtypes = [_V]
LIB.orc_karma_set.argtypes = [_V, _V, _V]
LIB.orc_karma_get.argtypes = [_V, _V, _V, _V]
LIB.orc_karma_step.argtypes = [_V, C.c_int]
LIB.orc_karma_set_it.argtypes = [_V, C.c_int]
LIB.orc_karma_tip.argtypes = [_V, C.POINTER(C.c_int), C.POINTER(C.c_int)]


def karma_ruido(i, j, k, it) -> float:
    return LIB.orc_karma_ruido(i, j, k, it)


class KarmaOracle:
    """karma3d.f90's time loop on the CPU (fields of shape (nz, ny, nx))."""

    def __init__(self, nx, ny, nz, lambda_, eps4, dx, dt, Fnoise, k):
        self.shape = (nz, ny, nx)
        self._h = LIB.orc_karma_create(nx, ny, nz, lambda_, eps4, dx, dt, Fnoise, k)

    def close(self):
        if self._h:
            LIB.orc_karma_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set(self, phi: np.ndarray, U: np.ndarray):
        a = np.ascontiguousarray(phi, dtype=np.float64)
        b = np.ascontiguousarray(U, dtype=np.float64)
        LIB.orc_karma_set(self._h, a.ctypes.data_as(_V), b.ctypes.data_as(_V))

    def get(self):
        phi, U, dphi = (np.empty(self.shape) for _ in range(3))
        LIB.orc_karma_get(self._h, phi.ctypes.data_as(_V), U.ctypes.data_as(_V), dphi.ctypes.data_as(_V))
        return phi, U, dphi

    def step(self, n: int = 1):
        LIB.orc_karma_step(self._h, n)

    def set_it(self, it: int):
        LIB.orc_karma_set_it(self._h, it)

    def tip(self):
        a, b = C.c_int(), C.c_int()
        LIB.orc_karma_tip(self._h, C.byref(a), C.byref(b))
        return a.value, b.value
