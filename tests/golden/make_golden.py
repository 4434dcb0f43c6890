"""Generates the committed known-answer fixtures under tests/golden/.

Run from the repository root:  python tests/golden/make_golden.py

Every fixture is produced by the C oracle (oracle/) AND by the independent
numpy restatement (np_restatement.py) and written only if both agree bit for
bit.  The reference itself cannot be run here (no Fortran compiler), so these
fixtures pin the restatements against each other and against regressions,
not against the reference's own output.
"""
from __future__ import annotations

import json
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "phase-field-project-3d_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import np_restatement as NR  # noqa: E402
import pyoracle as O         # noqa: E402
from pf3d import deck, init  # noqa: E402


def hx(v: float) -> str:
    return struct.pack(">d", v).hex()


NOISE_INPUTS = [
    (1, 1, 1, 1, 1), (3, 3, 3, 1, 1), (32, 10, 64, 1, 1), (64, 64, 128, 2000, 1), (340, 340, 700, 52470, 1),
    (3, 3, 3, 1, 2), (17, 5, 9, 123, 2), (1, 1, 1, 0, 3), (0, 0, 0, 0, 0), (1024, 1024, 1024, 10000, 1),
    (512, 1, 1024, 5000, 1), (2, 999, 77, 65535, 3), (100000, 200000, 300000, 400000, 1),
]
SUAVE_INPUTS = [(3, 3, 3, 1), (7, 13, 5, 19), (7, 13, 5, 20), (64, 64, 128, 2000), (6, 12, 18, 40), (35, 3, 90, 77)]

SMALL_CASES = [
    ("base", (14, 12, 16), {}),
    ("quintic_zero_mean_one_sweep", (9, 7, 11), dict(h_quintico=1, ruido_tipo=1, n_varreduras=1)),
    ("smooth_noise_three_sweeps_heat_lap", (8, 10, 9), dict(ruido_tipo=2, n_varreduras=3, D=2e-5)),
    ("minimum_5cube", (5, 5, 5), {}),
]
SMALL_STEPS = 5


def small_state(nx, ny, nz, p):
    st = init.initial_state(nx, ny, nz, 4, 0, p)
    st["phi"] = np.roll(st["phi"], nz // 3, axis=0)
    st["c"] = p.C0 * (1.0 - (1.0 - float(np.float32(p.Ke))) * st["phi"])
    st["T"] = st["T"] + np.random.default_rng(5).normal(0.0, 0.1, st["T"].shape)
    return st


def main():
    # ---- noise KATs ----
    noise = []
    for (i, j, k, it, salt) in NOISE_INPUTS:
        a = O.pseudo_random(i, j, k, it, salt)
        b = NR.pseudo_random(i, j, k, it, salt)
        assert struct.pack("d", a) == struct.pack("d", b), (i, j, k, it, salt)
        noise.append(dict(i=i, j=j, k=k, it=it, salt=salt, hash63=hex(NR.pseudo_random_int(i, j, k, it, salt)),
                          ran64=hx(a), ran32=struct.pack(">f", np.float32(a)).hex()))
    suave = []
    for (i, j, k, it) in SUAVE_INPUTS:
        a = O.ruido_suave(i, j, k, it)
        b = NR.ruido_suave(i, j, k, it)
        assert struct.pack("d", a) == struct.pack("d", b), (i, j, k, it)
        suave.append(dict(i=i, j=j, k=k, it=it, r64=hx(a)))
    with open(os.path.join(HERE, "noise_kat.json"), "w") as f:
        json.dump({"pseudo_random": noise, "ruido_suave": suave}, f, indent=1)

    # ---- scalar KATs: W0/E0 scan, dt/AAA, M0 ----
    p = deck.run6_params()
    scal = []
    for dx in (0.15e-6, 0.25e-6, 0.5e-6, 1.0e-6):
        W0a, E0a, na = O.w0_e0(p.Thin_Interface * dx, p.ajuste, p.Sigma)
        W0b, E0b, nb = NR.w0_e0(p.Thin_Interface * dx, p.ajuste, p.Sigma)
        assert (W0a, E0a, na) == (W0b, E0b, nb), dx
        ms = []
        for TP in (922.0, 921.0, 919.5, 915.0):
            Cs = ((p.Tm - TP) * float(np.float32(p.Ke))) / p.Me
            Cl = (p.Tm - TP) / p.Me
            m1 = O.auxiliar(p, TP, Cs, Cl, E0a, W0a)
            m2 = NR.auxiliar(p, TP, Cs, Cl, E0a, W0a)
            assert m1 == m2, (dx, TP)
            ms.append(dict(TP=TP, Cs_eq=hx(Cs), Cl_eq=hx(Cl), M0=hx(m1)))
        scal.append(dict(dx=dx, W0=hx(W0a), E0=hx(E0a), iterations=na, M0=ms))
    with open(os.path.join(HERE, "scalars_kat.json"), "w") as f:
        json.dump({"deck": "run6", "cases": scal}, f, indent=1)

    # ---- small-grid runs ----
    out = {}
    for name, (nx, ny, nz), over in SMALL_CASES:
        pp = deck.run6_params(T0=922.0, taxa_resfr=19.84, AAA=0.01, **over)
        g = deck.grid(nx, ny, nz, 0.5e-6)
        st = small_state(nx, ny, nz, pp)
        o = O.Oracle(g, pp)
        o.load_state(st)
        r = NR.NpRef(g, pp)
        r.load_state(st)
        o.step(SMALL_STEPS)
        r.step(SMALL_STEPS)
        fo, fr = o.fields(), r.fields()
        for key in fo:
            assert np.array_equal(fo[key].view(np.uint64), fr[key].view(np.uint64)), (name, key)
        for key in ("phi", "c", "T"):
            out[f"{name}/in_{key}"] = st[key]
        for key in fo:
            out[f"{name}/out_{key}"] = fo[key]
        out[f"{name}/M0"] = np.array([o.scalars()["M0"]])
    np.savez_compressed(os.path.join(HERE, "small_runs.npz"), **out)
    print("fixtures written")


if __name__ == "__main__":
    main()
