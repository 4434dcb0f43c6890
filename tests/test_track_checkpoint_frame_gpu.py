"""GPU tests of the rows around the hot path: on-device tracking (solid
fraction and tip position, equal bit for bit to the host metrics on the
downloaded field), binary checkpoints (a run continued from a checkpoint
gives the same bits as the run never stopped, for a domain and for a batch
slot that leaves and rejoins) and the moving frame (the reference's restart
with a shift of k_desl planes, entrada.f90:284-321, restated in numpy below
as the checker)."""
import numpy as np
import pytest

import make_golden as MG
import pf3d
from pf3d import deck, metrics

pytestmark = pytest.mark.gpu

PRECS = [pf3d.PF_FP64, pf3d.PF_FP32]


def case(nx, ny, nz, **over):
    kw = dict(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    kw.update(over)
    p = deck.run6_params(**kw)
    return deck.grid(nx, ny, nz, 0.5e-6), p, MG.small_state(nx, ny, nz, p)


def host_track(phi):
    return metrics.solid_fraction(phi), metrics.tip_position(phi), int((phi >= 0.5).sum())


@pytest.mark.parametrize("prec", PRECS)
def test_track_equals_host_metrics(gpu, prec):
    g, p, st = case(37, 29, 41)
    with pf3d.Domain(g, p, prec) as d:
        d.load_state(st)
        for n in (0, 7, 13):
            d.step(n)
            assert d.track() == host_track(d.download("phase_field_old")), n


@pytest.mark.parametrize("prec", PRECS)
def test_track_edge_cases(gpu, prec):
    g, p, st = case(16, 12, 10)
    shape = st["phi"].shape
    with pf3d.Domain(g, p, prec) as d:
        # all liquid: no tip
        d.upload("phase_field_old", np.zeros(shape))
        assert d.track() == (0.0, 0.0, 0)
        # solid up to the top plane: tip = nz
        d.upload("phase_field_old", np.ones(shape))
        assert d.track() == (1.0, 10.0, 16 * 12 * 10)
        # one solid cell below the top, interpolation against the plane above
        phi = np.zeros(shape)
        phi[6, 3, 5] = 0.75
        phi[7, 1, 1] = 0.25
        phi[8, 2, 2] = -0.5          # negative values order correctly
        d.upload("phase_field_old", phi)
        got = d.track()
        assert got == host_track(d.download("phase_field_old"))
        assert got[2] == 1 and abs(got[1] - (7.0 + 0.5)) < 1e-15


@pytest.mark.parametrize("prec", PRECS)
def test_batch_track_equals_alone(gpu, prec):
    cases = [case(30, 20, 26), case(20, 33, 18, T0=918.0)]
    with pf3d.Batch(prec) as b:
        slots = []
        for g, p, st in cases:
            s = b.add(g, p)
            b.load_state(s, st)
            slots.append(s)
        b.step(6)
        for (g, p, st), s in zip(cases, slots):
            with pf3d.Domain(g, p, prec) as d:
                d.load_state(st)
                d.step(6)
                assert b.track(s) == d.track() == host_track(d.download("phase_field_old"))


@pytest.mark.parametrize("prec", PRECS)
def test_checkpoint_continues_bit_identical(gpu, prec, tmp_path):
    g, p, st = case(33, 21, 27)
    path = str(tmp_path / "a.ckpt")
    with pf3d.Domain(g, p, prec) as a:
        a.load_state(st)
        a.step(5)
        a.checkpoint(path)   # asynchronous: the domain keeps stepping
        a.step(6)
        a.checkpoint_wait()
        want, wst = a.fields(), a.state()
    with pf3d.Domain(g, p, prec) as b:
        b.restore(path)
        assert b.state().it == 5
        b.step(6)
        got, gst = b.fields(), b.state()
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    assert (gst.it, gst.TP, gst.M0, gst.Cs_eq, gst.Cl_eq, gst.time) == \
           (wst.it, wst.TP, wst.M0, wst.Cs_eq, wst.Cl_eq, wst.time)


def test_checkpoint_rejects_other_grid_or_precision(gpu, tmp_path):
    """A checkpoint loads only into a domain of the same precision, cells,
    grid spacing and deck; anything else is an error, not a silent mix."""
    g, p, st = case(20, 16, 14)
    path = str(tmp_path / "b.ckpt")
    with pf3d.Domain(g, p, pf3d.PF_FP64) as a:
        a.load_state(st)
        a.checkpoint(path, wait=True)
    with pf3d.Domain(g, p, pf3d.PF_FP32) as d, pytest.raises(pf3d.PFError):
        d.restore(path)
    with pf3d.Domain(deck.grid(20, 16, 15, 0.5e-6), p, pf3d.PF_FP64) as d, pytest.raises(pf3d.PFError):
        d.restore(path)
    with pf3d.Domain(g, p, pf3d.PF_FP64) as d, pytest.raises(pf3d.PFError):
        d.restore(str(tmp_path / "missing.ckpt"))
    with pf3d.Domain(deck.grid(20, 16, 14, 0.25e-6), p, pf3d.PF_FP64) as d, pytest.raises(pf3d.PFError):
        d.restore(path)
    p2 = deck.params_copy(p, taxa_resfr=p.taxa_resfr * 2)
    with pf3d.Domain(g, p2, pf3d.PF_FP64) as d, pytest.raises(pf3d.PFError):
        d.restore(path)
    with pf3d.Domain(g, deck.params_copy(p, stoptime=1.0), pf3d.PF_FP64) as d:
        d.restore(path)   # driver-only values do not enter the deck check


@pytest.mark.parametrize("prec", PRECS)
def test_batch_preempt_and_resume(gpu, prec, tmp_path):
    """A request preempted (checkpoint, slot removed) and resumed later in
    another slot ends with the bits of the same request run alone."""
    cases = [case(28, 22, 24), case(24, 24, 20, AAA=0.02)]
    path = str(tmp_path / "slot.ckpt")
    with pf3d.Batch(prec) as b:
        s0 = b.add(*cases[0][:2])
        b.load_state(s0, cases[0][2])
        s1 = b.add(*cases[1][:2])
        b.load_state(s1, cases[1][2])
        b.step(4)
        b.checkpoint(s1, path)
        b.remove(s1)
        b.step(3)                       # the other request keeps going
        s2 = b.add(*cases[1][:2])       # resume
        b.restore(s2, path)
        assert b.state(s2).it == 4
        b.step(5)
        got0, got1 = b.fields(s0), b.fields(s2)
    for (g, p, st), n, got in ((cases[0], 12, got0), (cases[1], 9, got1)):
        with pf3d.Domain(g, p, prec) as d:
            d.load_state(st)
            d.step(n)
            want = d.fields()
        for k in want:
            assert np.array_equal(got[k], want[k]), (n, k)


def shift_restart_np(phi, c, k_desl, T0):
    """entrada.f90:284-321 (ler_restart) on arrays of shape (nz, ny, nx),
    after entrada's initial fill (entrada.f90:239-262)."""
    nz = phi.shape[0]
    phi_n = np.zeros_like(phi)
    c_n = np.empty_like(c)
    keep = nz - k_desl
    phi_n[:keep] = phi[k_desl:]
    c_n[:keep] = c[k_desl:]
    c_n[keep:] = c[nz - 1]
    return {"phase_field_old": phi_n, "conc_soluto_old": c_n, "conc_soluto_new": c_n,
            "phase_field_new": np.zeros_like(phi), "TOLD": np.full_like(phi, T0), "TNEW": np.full_like(phi, T0),
            "DPP": np.zeros_like(phi)}


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("k_desl", [0, 1, 7])
def test_shift_frame_equals_restart(gpu, prec, k_desl):
    g, p, st = case(26, 19, 23)
    with pf3d.Domain(g, p, prec) as d:
        d.load_state(st)
        d.step(4)
        phi, c = d.download("phase_field_old"), d.download("conc_soluto_old")
        t0 = float(np.float32(p.T0)) if prec == pf3d.PF_FP32 else p.T0
        want = shift_restart_np(phi, c, k_desl, t0)
        d.shift_frame(k_desl)
        for name, arr in want.items():
            assert np.array_equal(d.download(name), arr), name
        d.step(3)
        got = d.fields()
    # the shifted state steps like the same state uploaded into a new domain
    # that carries the same pf_state (the shift leaves the state alone)
    with pf3d.Domain(g, p, prec) as f:
        f.load_state(st)
        f.step(4)
        keep = f.state()
        f.load_state({"phi": want["phase_field_old"], "c": want["conc_soluto_old"], "T": want["TOLD"],
                      "dpp": want["DPP"]})
        f.set_state(keep)
        f.step(3)
        ref = f.fields()
    for k in ref:
        assert np.array_equal(got[k], ref[k]), k


def test_shift_frame_rejects_bad_shift(gpu):
    g, p, st = case(16, 12, 10)
    with pf3d.Domain(g, p) as d:
        for bad in (-1, 10, 11):
            with pytest.raises(pf3d.PFError):
                d.shift_frame(bad)
