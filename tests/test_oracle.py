"""CPU tests: the oracle against the committed known-answer fixtures and the
independent numpy restatement; closed-form boundary mapping."""
import json
import os
import struct

import numpy as np
import pytest

import np_restatement as NR
import pyoracle as O
from pf3d import deck

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def unhex(s):
    return struct.unpack(">d", bytes.fromhex(s))[0]


def test_noise_kat():
    kat = json.load(open(os.path.join(HERE, "noise_kat.json")))
    for e in kat["pseudo_random"]:
        v = O.pseudo_random(e["i"], e["j"], e["k"], e["it"], e["salt"])
        assert struct.pack(">d", v).hex() == e["ran64"]
        assert hex(NR.pseudo_random_int(e["i"], e["j"], e["k"], e["it"], e["salt"])) == e["hash63"]
        assert struct.pack(">f", np.float32(v)).hex() == e["ran32"]
        assert 0.0 <= v <= 1.0
    for e in kat["ruido_suave"]:
        v = O.ruido_suave(e["i"], e["j"], e["k"], e["it"])
        assert struct.pack(">d", v).hex() == e["r64"]


def test_hash_grid_matches_scalar():
    h = NR.hash_grid(7, 5, 3, 42, 1)
    for (k, j, i) in [(0, 0, 0), (2, 4, 6), (1, 3, 2)]:
        assert int(h[k, j, i]) == NR.pseudo_random_int(i + 1, j + 1, k + 1, 42, 1)


def test_scalar_kat():
    kat = json.load(open(os.path.join(HERE, "scalars_kat.json")))
    p = deck.run6_params()
    for case in kat["cases"]:
        W0, E0, n = O.w0_e0(p.Thin_Interface * case["dx"], p.ajuste, p.Sigma)
        assert struct.pack(">d", W0).hex() == case["W0"]
        assert struct.pack(">d", E0).hex() == case["E0"]
        assert n == case["iterations"]
        for m in case["M0"]:
            M0 = O.auxiliar(p, m["TP"], unhex(m["Cs_eq"]), unhex(m["Cl_eq"]), E0, W0)
            assert struct.pack(">d", M0).hex() == m["M0"]


@pytest.mark.parametrize("name", ["base", "quintic_zero_mean_one_sweep", "smooth_noise_three_sweeps_heat_lap",
                                  "minimum_5cube"])
def test_small_runs_fixture(name):
    import make_golden as MG
    z = np.load(os.path.join(HERE, "small_runs.npz"))
    (nx, ny, nz), over = [(s, o) for (n, s, o) in MG.SMALL_CASES if n == name][0]
    p = deck.run6_params(T0=922.0, taxa_resfr=19.84, AAA=0.01, **over)
    g = deck.grid(nx, ny, nz, 0.5e-6)
    o = O.Oracle(g, p)
    o.load_state({k: z[f"{name}/in_{k}"] for k in ("phi", "c", "T")})
    o.step(MG.SMALL_STEPS)
    f = o.fields()
    for key in f:
        assert np.array_equal(f[key].view(np.uint64), z[f"{name}/out_{key}"].view(np.uint64)), key
    assert o.scalars()["M0"] == z[f"{name}/M0"][0]


def test_oracle_matches_numpy_restatement_longer():
    import make_golden as MG
    p = deck.run6_params(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    g = deck.grid(12, 11, 13, 0.5e-6)
    st = MG.small_state(12, 11, 13, p)
    o = O.Oracle(g, p); o.load_state(st)
    r = NR.NpRef(g, p); r.load_state(st)
    o.step(20); r.step(20)
    fo, fr = o.fields(), r.fields()
    for key in fo:
        assert np.array_equal(fo[key].view(np.uint64), fr[key].view(np.uint64)), key


def _plane_copy_phase(a):
    """equacao_campo_fase.f90:151-167 applied literally to an index array."""
    a = a.copy()
    nz, ny, nx = a.shape
    a[:, 0, :] = a[:, 1, :]; a[:, 1, :] = a[:, 2, :]
    a[:, ny - 1, :] = a[:, ny - 2, :]; a[:, ny - 2, :] = a[:, ny - 3, :]
    a[:, :, 0] = a[:, :, 1]; a[:, :, 1] = a[:, :, 2]
    a[:, :, nx - 1] = a[:, :, nx - 2]; a[:, :, nx - 2] = a[:, :, nx - 3]
    a[0] = a[1]; a[1] = a[2]; a[nz - 1] = a[nz - 2]; a[nz - 2] = a[nz - 3]
    return a


def _fmap(x, n):
    if x == 0: return 1
    if x == 1: return 2
    if x == n - 1: return n - 2
    if x == n - 2: return n - 3
    return x


@pytest.mark.parametrize("shape", [(5, 5, 5), (6, 7, 5), (9, 8, 12), (5, 11, 6)])
def test_phase_decoration_closed_form(shape):
    nz, ny, nx = shape
    idx = np.arange(nz * ny * nx).reshape(shape)
    lit = _plane_copy_phase(idx)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                assert lit[z, y, x] == idx[_fmap(z, nz), _fmap(y, ny), _fmap(x, nx)]


@pytest.mark.parametrize("shape", [(5, 5, 5), (6, 7, 5), (9, 8, 12)])
def test_solute_decoration_closed_form(shape):
    nz, ny, nx = shape
    idx = np.arange(nz * ny * nx).reshape(shape)
    cn = idx.copy()
    co = idx
    cn[:, 0, :] = co[:, 1, :]; cn[:, ny - 1, :] = co[:, ny - 2, :]
    cn[:, :, 0] = co[:, :, 1]; cn[:, :, nx - 1] = co[:, :, nx - 2]
    cn[0] = co[1]; cn[nz - 1] = co[nz - 2]
    g = lambda v, n: 1 if v == 0 else (n - 2 if v == n - 1 else v)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                if z in (0, nz - 1):
                    src = (g(z, nz), y, x)
                elif x in (0, nx - 1):
                    src = (z, y, g(x, nx))
                elif y in (0, ny - 1):
                    src = (z, g(y, ny), x)
                else:
                    src = (z, y, x)
                assert cn[z, y, x] == idx[src]
