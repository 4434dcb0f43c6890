"""ctypes mirror of include/pf3d.h and the loader of the in-tree libpf3d.so.

The library is required: there is no Python or CPU fallback for any entry
point.  It is mapped on the first call through `LIB` (importing the package
for its host-side modules -- the deck and the initial-state recipe -- maps
nothing); if libpf3d.so is missing that first call raises ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpf3d.so")

PF_OK, PF_E_ARG, PF_E_CUDA, PF_E_NOMEM, PF_E_STATE, PF_E_NODEV, PF_E_KERNEL, PF_E_NONFINITE = (
    0, -1, -2, -3, -4, -5, -6, -7)
PF_PHASE_OLD, PF_PHASE_NEW, PF_CONC_OLD, PF_CONC_NEW, PF_TOLD, PF_TNEW, PF_DPP = range(7)
FIELD_NAMES = ("phase_field_old", "phase_field_new", "conc_soluto_old", "conc_soluto_new", "TOLD", "TNEW", "DPP")
PF_FP64, PF_FP32 = 64, 32
PF_BC_REFERENCE = 0
PF_OPT_FUSED, PF_OPT_TILE_Y, PF_OPT_ZCHUNK, PF_OPT_KTIMING, PF_OPT_PAIRED, PF_OPT_KERNEL, PF_OPT_NSLOT = 1, 2, 3, 4, 5, 6, 7
PF_NOALLOC_MAX_PLANES = 4096


class pf_grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class pf_params(C.Structure):
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


class pf_derived(C.Structure):
    _fields_ = [("DELTA_T", C.c_double), ("AAA", C.c_double), ("Lambda", C.c_double),
                ("W0", C.c_double), ("E0", C.c_double), ("w0e0_iterations", C.c_long)]


class pf_state(C.Structure):
    _fields_ = [("it", C.c_int), ("TP", C.c_double), ("M0", C.c_double),
                ("Cs_eq", C.c_double), ("Cl_eq", C.c_double), ("time", C.c_float)]


class pf_karma_params(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int)] + [
        (n, C.c_double) for n in ("lambda_", "eps4", "dx", "dt", "R0", "Fnoise", "k", "Tm", "mliq", "C0", "TP",
                                  "sigma", "dH", "Dl")]


class pf_karma_derived(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("D", "cl0", "Omega", "Gam", "d0", "W", "tau0")]


PF_KARMA_PHI, PF_KARMA_U, PF_KARMA_DPHI = 0, 1, 2

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)

# (name, restype, argtypes) for every function include/pf3d.h declares
SIGNATURES = [
    ("pf_version", C.c_int, []),
    ("pf_last_error", C.c_char_p, [_P]),
    ("pf_ctx_bytes", C.c_longlong, [C.POINTER(pf_grid), C.c_int]),
    ("pf_create", C.c_int, [C.POINTER(pf_grid), C.POINTER(pf_params), C.c_int, C.POINTER(_P)]),
    ("pf_destroy", C.c_int, [_P]),
    ("pf_get_derived", C.c_int, [_P, C.POINTER(pf_derived)]),
    ("pf_get_state", C.c_int, [_P, C.POINTER(pf_state)]),
    ("pf_set_state", C.c_int, [_P, C.POINTER(pf_state)]),
    ("pf_sync", C.c_int, [_P]),
    ("pf_set_stream", C.c_int, [_P, _P]),
    ("pf_set_option", C.c_int, [_P, C.c_int, C.c_int]),
    ("pf_get_option", C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    ("pf_kernel_times", C.c_int, [_P, C.POINTER(C.c_long), _D, C.POINTER(C.c_long), _D, C.c_int]),
    ("pf_upload", C.c_int, [_P, C.c_int, _P]),
    ("pf_download", C.c_int, [_P, C.c_int, _P]),
    ("pf_probe", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, _D]),
    ("pf_w0_e0", C.c_int, [C.POINTER(pf_grid), C.POINTER(pf_params), _D, _D, C.POINTER(C.c_long)]),
    ("pf_auxiliar_scalar", C.c_int, [C.POINTER(pf_params), C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double, _D]),
    ("pf_temperatura", C.c_int, [_P, C.c_double]),
    ("pf_equacao_campo_fase", C.c_int, [_P, C.c_int, C.c_double, C.c_double, _D, _D]),
    ("pf_copy_phase_new_to_old", C.c_int, [_P]),
    ("pf_concentracao_soluto", C.c_int, [_P]),
    ("pf_auxiliar", C.c_int, [_P, C.c_double, C.c_double, C.c_double, _D]),
    ("pf_diagnosticos", C.c_int, [_P, _D]),
    ("pf_swap", C.c_int, [_P]),
    ("pf_step", C.c_int, [_P, C.c_int]),
    ("pf_step_diag", C.c_int, [_P, C.c_int, _D]),
    ("pf_init_seeded", C.c_int, [_P, C.c_int, _D]),
    ("pf_track", C.c_int, [_P, _D]),
    ("pf_checkpoint_save", C.c_int, [_P, C.c_char_p]),
    ("pf_checkpoint_wait", C.c_int, [_P]),
    ("pf_checkpoint_load", C.c_int, [_P, C.c_char_p]),
    ("pf_shift_frame", C.c_int, [_P, C.c_int]),
    ("pf_batch_create", C.c_int, [C.c_int, C.c_longlong, C.c_int, C.POINTER(_P)]),
    ("pf_batch_destroy", C.c_int, [_P]),
    ("pf_batch_set_stream", C.c_int, [_P, _P]),
    ("pf_batch_bytes_used", C.c_longlong, [_P]),
    ("pf_batch_count", C.c_int, [_P]),
    ("pf_batch_add", C.c_int, [_P, C.POINTER(pf_grid), C.POINTER(pf_params), C.POINTER(C.c_int)]),
    ("pf_batch_remove", C.c_int, [_P, C.c_int]),
    ("pf_batch_upload", C.c_int, [_P, C.c_int, C.c_int, _P]),
    ("pf_batch_download", C.c_int, [_P, C.c_int, C.c_int, _P]),
    ("pf_batch_init_seeded", C.c_int, [_P, C.c_int, C.c_int, _D]),
    ("pf_batch_set_target", C.c_int, [_P, C.c_int, C.c_longlong]),
    ("pf_batch_get_state", C.c_int, [_P, C.c_int, C.POINTER(pf_state)]),
    ("pf_batch_progress", C.c_int, [_P, _I, C.c_int]),
    ("pf_batch_step", C.c_int, [_P, C.c_int]),
    ("pf_batch_step_async", C.c_int, [_P, C.c_int]),
    ("pf_batch_wait", C.c_int, [_P]),
    ("pf_batch_last_ms", C.c_double, [_P]),
    ("pf_batch_set_tile", C.c_int, [_P, C.c_int, C.c_int]),
    ("pf_batch_set_paired", C.c_int, [_P, C.c_int]),
    ("pf_batch_set_kernel", C.c_int, [_P, C.c_int, C.c_int]),
    ("pf_batch_autotune", C.c_int, [_P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _D]),
    ("pf_batch_diagnosticos", C.c_int, [_P, C.c_int, _D]),
    ("pf_batch_track", C.c_int, [_P, C.c_int, _D]),
    ("pf_batch_checkpoint_save", C.c_int, [_P, C.c_int, C.c_char_p]),
    ("pf_batch_checkpoint_load", C.c_int, [_P, C.c_int, C.c_char_p]),
    ("pf_karma_derived_of", C.c_int, [C.POINTER(pf_karma_params), C.POINTER(pf_karma_derived)]),
    ("pf_karma_create", C.c_int, [C.POINTER(pf_karma_params), C.c_int, C.POINTER(_P)]),
    ("pf_karma_destroy", C.c_int, [_P]),
    ("pf_karma_set_stream", C.c_int, [_P, _P]),
    ("pf_karma_get_it", C.c_int, [_P, _I]),
    ("pf_karma_set_it", C.c_int, [_P, C.c_int]),
    ("pf_karma_upload", C.c_int, [_P, C.c_int, _P]),
    ("pf_karma_download", C.c_int, [_P, C.c_int, _P]),
    ("pf_karma_seed", C.c_int, [_P]),
    ("pf_karma_step", C.c_int, [_P, C.c_int]),
    ("pf_karma_tip", C.c_int, [_P, _I, _I]),
    ("pf_karma_sync", C.c_int, [_P]),
    ("pf_diagnosticos_noalloc", C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                          C.c_double, C.c_double, C.c_double, C.c_double, _P, _D]),
    ("pf_math_log", C.c_int, [_P, C.c_longlong, _P, _P]),
]


def load_library(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"libpf3d.so not found at {path}; build it with "
            "`make -C phase-field-project-3d_b200/csrc` (or __graft_entry__.build())")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class _LazyLib:
    """Forwards attribute access to libpf3d.so, loading it on first use."""

    _lib = None

    def __getattr__(self, name):
        lib = _LazyLib._lib
        if lib is None:
            lib = _LazyLib._lib = load_library()
        return getattr(lib, name)

    @property
    def loaded(self) -> bool:
        return _LazyLib._lib is not None


LIB = _LazyLib()


class PFError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pf3d error {code}: {msg}")
        self.code = code


def check(rc: int, ctx=None) -> None:
    if rc != PF_OK:
        msg = LIB.pf_last_error(ctx)
        raise PFError(rc, msg.decode() if msg else "")
