"""pf3d -- B200 implementation of the coupled explicit time step of the 3-D
Al-Cu phase-field model of ileaof/phase-field-project-3D.

`Domain` mirrors the reference's hot-path interface: one method per
subroutine the time loop of principal.f90 calls (temperatura,
equacao_campo_fase, concentracao_soluto, auxiliar, diagnosticos, the swap),
acting on the seven device-resident fields by their reference names, plus
`step()` (the fused form of the whole loop body).  Every call goes through
the C-ABI of libpf3d.so; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import (LIB, check, pf_grid, pf_params, pf_derived, pf_state, PFError,
                   PF_FP64, PF_FP32, PF_PHASE_OLD, PF_PHASE_NEW, PF_CONC_OLD, PF_CONC_NEW,
                   PF_TOLD, PF_TNEW, PF_DPP, PF_OPT_FUSED, PF_OPT_TILE_Y, PF_OPT_ZCHUNK,
                   PF_OPT_KTIMING, PF_OPT_PAIRED, PF_OPT_KERNEL, PF_OPT_NSLOT, PF_E_KERNEL, PF_E_NONFINITE, FIELD_NAMES)
from .deck import run6_params, params_copy, grid, read_entrada, WORKLOADS, Workload

__all__ = ["Domain", "PFError", "run6_params", "params_copy", "grid", "read_entrada", "WORKLOADS", "Workload",
           "w0_e0", "auxiliar_scalar", "math_log", "FIELDS", "PF_FP64", "PF_FP32"]

FIELDS = {n: q for q, n in enumerate(FIELD_NAMES)}
FIELDS.update({"phi_old": 0, "phi_new": 1, "c_old": 2, "c_new": 3, "T_old": 4, "T_new": 5, "dpp": 6})


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def w0_e0(g: pf_grid, p: pf_params):
    W0, E0, n = C.c_double(), C.c_double(), C.c_long()
    check(LIB.pf_w0_e0(C.byref(g), C.byref(p), C.byref(W0), C.byref(E0), C.byref(n)))
    return W0.value, E0.value, n.value


def auxiliar_scalar(p: pf_params, E0: float, W0: float, TP: float, Cs_eq: float, Cl_eq: float) -> float:
    M0 = C.c_double()
    check(LIB.pf_auxiliar_scalar(C.byref(p), E0, W0, TP, Cs_eq, Cl_eq, C.byref(M0)))
    return M0.value


def math_log(x) -> "tuple[np.ndarray, np.ndarray]":
    """The fused FP64 kernels' own logarithm and CUDA's log, both evaluated on
    the device for the values x (self-check of the fast form's arithmetic)."""
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    own = np.empty_like(x)
    lib = np.empty_like(x)
    check(LIB.pf_math_log(_dptr(x), x.size, _dptr(own), _dptr(lib)))
    return own, lib


class Domain:
    """One device-resident domain (a pf_ctx)."""

    def __init__(self, g: pf_grid, p: pf_params, precision: int = PF_FP64):
        self.grid = g
        self.params = p
        self.precision = precision
        h = C.c_void_p()
        check(LIB.pf_create(C.byref(g), C.byref(p), precision, C.byref(h)))
        self._h = h

    # ---- lifecycle ----
    def close(self):
        if self._h:
            LIB.pf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def shape(self):
        return (self.grid.nz, self.grid.ny, self.grid.nx)

    def _chk(self, rc):
        check(rc, self._h)

    def derived(self) -> pf_derived:
        d = pf_derived()
        self._chk(LIB.pf_get_derived(self._h, C.byref(d)))
        return d

    def state(self) -> pf_state:
        s = pf_state()
        self._chk(LIB.pf_get_state(self._h, C.byref(s)))
        return s

    def set_state(self, s: pf_state):
        self._chk(LIB.pf_set_state(self._h, C.byref(s)))

    def set_option(self, opt: int, value: int):
        self._chk(LIB.pf_set_option(self._h, opt, int(value)))

    def set_stream(self, stream_handle: int | None):
        self._chk(LIB.pf_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None))

    def sync(self):
        self._chk(LIB.pf_sync(self._h))

    # ---- data residency ----
    def upload(self, field, host: np.ndarray):
        q = FIELDS[field] if isinstance(field, str) else int(field)
        a = np.ascontiguousarray(host, dtype=np.float64)
        if a.size != self.grid.nx * self.grid.ny * self.grid.nz:
            raise ValueError("host array size does not match the grid")
        self._chk(LIB.pf_upload(self._h, q, _dptr(a)))

    def download(self, field, out: np.ndarray | None = None) -> np.ndarray:
        q = FIELDS[field] if isinstance(field, str) else int(field)
        if out is None:
            out = np.empty(self.shape, dtype=np.float64)
        self._chk(LIB.pf_download(self._h, q, _dptr(out)))
        return out

    def load_state(self, st: dict):
        """Upload an initial state {phi, c, T[, dpp]} into the *old* fields."""
        self.upload(PF_PHASE_OLD, st["phi"])
        self.upload(PF_CONC_OLD, st["c"])
        self.upload(PF_TOLD, st["T"])
        self.upload(PF_DPP, st.get("dpp", np.zeros(self.shape)))

    def probe(self, field, i: int, j: int, k: int) -> float:
        q = FIELDS[field] if isinstance(field, str) else int(field)
        v = C.c_double()
        self._chk(LIB.pf_probe(self._h, q, i, j, k, C.byref(v)))
        return v.value

    # ---- the reference's subroutines ----
    def temperatura(self, TP: float):
        self._chk(LIB.pf_temperatura(self._h, TP))

    def equacao_campo_fase(self, it: int, TP: float, M0: float):
        cs, cl = C.c_double(), C.c_double()
        self._chk(LIB.pf_equacao_campo_fase(self._h, it, TP, M0, C.byref(cs), C.byref(cl)))
        return cs.value, cl.value

    def copy_phase_new_to_old(self):
        self._chk(LIB.pf_copy_phase_new_to_old(self._h))

    def concentracao_soluto(self):
        self._chk(LIB.pf_concentracao_soluto(self._h))

    def auxiliar(self, TP: float, Cs_eq: float, Cl_eq: float) -> float:
        m = C.c_double()
        self._chk(LIB.pf_auxiliar(self._h, TP, Cs_eq, Cl_eq, C.byref(m)))
        return m.value

    def diagnosticos(self):
        out = (C.c_double * 5)()
        self._chk(LIB.pf_diagnosticos(self._h, out))
        return tuple(out)

    def swap(self):
        self._chk(LIB.pf_swap(self._h))

    # ---- time loop ----
    def step_reference_order(self, n: int = 1):
        """n iterations of principal.f90:93-226 issued as per-subroutine calls."""
        p = self.params
        d = self.derived()
        for _ in range(n):
            s = self.state()
            it = s.it + 1
            TP_prev = s.TP
            self.temperatura(TP_prev)
            TP = p.T0 - p.taxa_resfr * d.DELTA_T * it if p.taxa_resfr > 0.0 else TP_prev
            cs = cl = 0.0
            for sw in range(1, p.n_varreduras + 1):
                if sw > 1:
                    self.copy_phase_new_to_old()
                cs, cl = self.equacao_campo_fase(it, TP, s.M0)
            self.concentracao_soluto()
            M0 = self.auxiliar(TP, cs, cl)
            self.swap()
            ns = pf_state()
            ns.it, ns.TP, ns.M0, ns.Cs_eq, ns.Cl_eq = it, TP, M0, cs, cl
            ns.time = np.float32(np.float64(d.DELTA_T) + np.float64(s.time))
            self.set_state(ns)

    def step(self, n: int = 1):
        """n fused iterations of the time loop (pf_step)."""
        self._chk(LIB.pf_step(self._h, int(n)))

    def step_diag(self, n: int = 1):
        out = (C.c_double * 5)()
        self._chk(LIB.pf_step_diag(self._h, int(n), out))
        return tuple(out)

    # ---- tracking, checkpoints, moving frame ----
    def track(self):
        """(solid fraction, tip position in cells, solid cells) of the current
        phase field, evaluated on the device (pf_track)."""
        out = (C.c_double * 3)()
        self._chk(LIB.pf_track(self._h, out))
        return out[0], out[1], int(out[2])

    def checkpoint(self, path: str, wait: bool = False):
        """Binary checkpoint of the state; the file is written by a host
        thread while the domain keeps stepping (pf_checkpoint_save)."""
        self._chk(LIB.pf_checkpoint_save(self._h, os.fsencode(path)))
        if wait:
            self.checkpoint_wait()

    def checkpoint_wait(self):
        self._chk(LIB.pf_checkpoint_wait(self._h))

    def restore(self, path: str):
        self._chk(LIB.pf_checkpoint_load(self._h, os.fsencode(path)))

    def shift_frame(self, k_desl: int):
        """The reference's restart with a shift of k_desl planes, on the device."""
        self._chk(LIB.pf_shift_frame(self._h, int(k_desl)))

    def kernel_times(self, reset: bool = True):
        nf, nl = C.c_long(), C.c_long()
        mf, ml = C.c_double(), C.c_double()
        self._chk(LIB.pf_kernel_times(self._h, C.byref(nf), C.byref(mf), C.byref(nl), C.byref(ml), int(reset)))
        return nf.value, mf.value, nl.value, ml.value

    def fields(self) -> dict:
        """Current state after a step: the old fields + DPP (host copies)."""
        return {"phi": self.download(PF_PHASE_OLD), "c": self.download(PF_CONC_OLD),
                "T": self.download(PF_TOLD), "dpp": self.download(PF_DPP)}


def _sites_ptr(sites):
    a = np.ascontiguousarray(np.asarray(sites, dtype=np.float64).reshape(-1))
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def init_seeded(dom: "Domain", sites) -> None:
    """Device-side seeded initial state of a Domain (pf_init_seeded)."""
    a, ptr = _sites_ptr(sites)
    dom._chk(LIB.pf_init_seeded(dom.handle, len(a) // 2, ptr))


class Batch:
    """Many independent domains stepped together (pf_batch_*)."""

    def __init__(self, precision: int = PF_FP32, budget_bytes: int = 0, max_domains: int = 4096):
        h = C.c_void_p()
        check(LIB.pf_batch_create(precision, int(budget_bytes), int(max_domains), C.byref(h)))
        self._h = h
        self.precision = precision
        self._max = int(max_domains)
        self.grids = {}

    def close(self):
        if self._h:
            LIB.pf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, rc):
        check(rc, None)

    def set_stream(self, stream_handle):
        self._chk(LIB.pf_batch_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None))

    def add(self, g: pf_grid, p: pf_params) -> int:
        s = C.c_int()
        self._chk(LIB.pf_batch_add(self._h, C.byref(g), C.byref(p), C.byref(s)))
        self.grids[s.value] = g
        return s.value

    def remove(self, slot: int):
        self._chk(LIB.pf_batch_remove(self._h, slot))
        self.grids.pop(slot, None)

    def count(self) -> int:
        return LIB.pf_batch_count(self._h)

    def bytes_used(self) -> int:
        return LIB.pf_batch_bytes_used(self._h)

    def upload(self, slot: int, field, host: np.ndarray):
        q = FIELDS[field] if isinstance(field, str) else int(field)
        a = np.ascontiguousarray(host, dtype=np.float64)
        self._chk(LIB.pf_batch_upload(self._h, slot, q, _dptr(a)))

    def download(self, slot: int, field) -> np.ndarray:
        q = FIELDS[field] if isinstance(field, str) else int(field)
        g = self.grids[slot]
        out = np.empty((g.nz, g.ny, g.nx), dtype=np.float64)
        self._chk(LIB.pf_batch_download(self._h, slot, q, _dptr(out)))
        return out

    def load_state(self, slot: int, st: dict):
        self.upload(slot, PF_PHASE_OLD, st["phi"])
        self.upload(slot, PF_CONC_OLD, st["c"])
        self.upload(slot, PF_TOLD, st["T"])
        self.upload(slot, PF_DPP, st.get("dpp", np.zeros_like(st["phi"])))

    def init_seeded(self, slot: int, sites):
        a, ptr = _sites_ptr(sites)
        self._chk(LIB.pf_batch_init_seeded(self._h, slot, len(a) // 2, ptr))

    def set_target(self, slot: int, target_it: int):
        self._chk(LIB.pf_batch_set_target(self._h, slot, int(target_it)))

    def progress(self) -> np.ndarray:
        """Step count of every slot (-1 for a free slot), one library call."""
        it = np.empty(self._max, dtype=np.int32)
        self._chk(LIB.pf_batch_progress(self._h, it.ctypes.data_as(C.POINTER(C.c_int)), self._max))
        return it

    def state(self, slot: int) -> pf_state:
        st = pf_state()
        self._chk(LIB.pf_batch_get_state(self._h, slot, C.byref(st)))
        return st

    def step(self, n: int = 1) -> float:
        """Advance every active slot by up to n steps; returns device ms."""
        self._chk(LIB.pf_batch_step(self._h, int(n)))
        return LIB.pf_batch_last_ms(self._h)

    def step_async(self, n: int = 1):
        """Queue up to n steps on the batch's stream and return at once."""
        self._chk(LIB.pf_batch_step_async(self._h, int(n)))

    def wait(self) -> float:
        """Wait for the last step_async; returns its device ms."""
        self._chk(LIB.pf_batch_wait(self._h))
        return LIB.pf_batch_last_ms(self._h)

    def set_tile(self, tile_y: int, zchunk: int):
        self._chk(LIB.pf_batch_set_tile(self._h, tile_y, zchunk))

    def set_paired(self, paired: int):
        self._chk(LIB.pf_batch_set_paired(self._h, int(paired)))

    def set_kernel(self, kernel: int, nslot: int = 0):
        """1: the TMA-staged passes (default), 0: the cp.async passes."""
        self._chk(LIB.pf_batch_set_kernel(self._h, int(kernel), int(nslot)))

    def autotune(self, steps_per_candidate: int = 2):
        ty, zc, ms = C.c_int(), C.c_int(), C.c_double()
        self._chk(LIB.pf_batch_autotune(self._h, steps_per_candidate, C.byref(ty), C.byref(zc), C.byref(ms)))
        return ty.value, zc.value, ms.value

    def diagnosticos(self, slot: int):
        out = (C.c_double * 5)()
        self._chk(LIB.pf_batch_diagnosticos(self._h, slot, out))
        return tuple(out)

    def track(self, slot: int):
        out = (C.c_double * 3)()
        self._chk(LIB.pf_batch_track(self._h, slot, out))
        return out[0], out[1], int(out[2])

    def checkpoint(self, slot: int, path: str):
        self._chk(LIB.pf_batch_checkpoint_save(self._h, slot, os.fsencode(path)))

    def restore(self, slot: int, path: str):
        self._chk(LIB.pf_batch_checkpoint_load(self._h, slot, os.fsencode(path)))

    def fields(self, slot: int) -> dict:
        return {"phi": self.download(slot, PF_PHASE_OLD), "c": self.download(slot, PF_CONC_OLD),
                "T": self.download(slot, PF_TOLD), "dpp": self.download(slot, PF_DPP)}
