"""GPU tests of the non-finite watchdog folded into the diagnostics reduction.

A blown-up run is made on the host: a NaN or an Inf is written into an
uploaded field (nothing faults, traps or hangs the GPU).  The diagnostics
then return PF_E_NONFINITE with max/min propagated as NaN (fmax/fmin would
have dropped the NaN and reported finite extremes), for a single domain,
for the fused step with diagnostics, and for a batch slot; the server
retires such a request as failed instead of returning its numbers.  The
phase update's clamp turns a NaN or infinite update into 1, so after a step
a blow-up may show only in DPP and T: the watchdog counts those fields too.
A NaN written into phi is therefore absorbed within a step or two (the cell
becomes solid, the heat equation's interior update does not read TOLD); a
NaN in c is not clamped and spreads, so the stepped cases poison c.  A
finite state still reports success with the same values as before."""
import math

import numpy as np
import pytest

import make_golden as MG
import pf3d
from pf3d import deck, serve

pytestmark = pytest.mark.gpu


def case(nx=24, ny=20, nz=18, **over):
    kw = dict(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    kw.update(over)
    p = deck.run6_params(**kw)
    return deck.grid(nx, ny, nz, 0.5e-6), p, MG.small_state(nx, ny, nz, p)


@pytest.mark.parametrize("prec", [pf3d.PF_FP64, pf3d.PF_FP32])
@pytest.mark.parametrize("bad", [float("nan"), float("inf")])
def test_diagnosticos_flag_a_nonfinite_cell(gpu, prec, bad):
    g, p, st = case()
    with pf3d.Domain(g, p, prec) as d:
        d.upload("phase_field_new", st["phi"])
        d.upload("conc_soluto_new", st["c"])
        clean = d.diagnosticos()
        assert all(math.isfinite(v) for v in clean)
        phi = st["phi"].copy()
        phi[5, 7, 9] = bad
        d.upload("phase_field_new", phi)
        with pytest.raises(pf3d.PFError) as e:
            d.diagnosticos()
        assert e.value.code == pf3d.PF_E_NONFINITE
        assert "1 cells" in str(e.value)
        c = st["c"].copy()
        c[0, 0, 0] = bad
        c[-1, -1, -1] = bad
        d.upload("phase_field_new", st["phi"])
        d.upload("conc_soluto_new", c)
        with pytest.raises(pf3d.PFError) as e:
            d.diagnosticos()
        assert e.value.code == pf3d.PF_E_NONFINITE and "2 cells" in str(e.value)


def test_max_min_propagate_nan(gpu):
    g, p, st = case()
    phi = st["phi"].copy()
    phi[3, 4, 5] = np.nan
    with pf3d.Domain(g, p, pf3d.PF_FP64) as d:
        d.upload("phase_field_new", phi)
        d.upload("conc_soluto_new", st["c"])
        out = (pf3d._abi.C.c_double * 5)()
        rc = pf3d.LIB.pf_diagnosticos(d.handle, out)
        assert rc == pf3d.PF_E_NONFINITE
        assert math.isnan(out[1]) and math.isnan(out[2]) and math.isnan(out[0])
        assert math.isfinite(out[3])   # the solute total does not read phi


def test_a_nan_in_phi_is_absorbed_by_the_clamp(gpu):
    """The reference's clamp dmax1(0, dmin1(1, .)) maps a NaN update to 1:
    a NaN written into phi leaves, after two steps, a finite state (the
    watchdog rightly reports nothing; the next sweep recomputes the cell)."""
    g, p, st = case()
    st = dict(st)
    st["phi"] = st["phi"].copy()
    st["phi"][9, 10, 11] = np.nan
    with pf3d.Domain(g, p, pf3d.PF_FP64) as d:
        d.load_state(st)
        out = d.step_diag(2)
        assert all(math.isfinite(v) for v in out)
        assert np.isfinite(d.download("phase_field_old")).all()


def test_step_diag_reports_a_blown_up_state(gpu):
    g, p, st = case()
    st = dict(st)
    st["c"] = st["c"].copy()
    st["c"][9, 10, 11] = np.nan
    with pf3d.Domain(g, p, pf3d.PF_FP64) as d:
        d.load_state(st)
        with pytest.raises(pf3d.PFError) as e:
            d.step_diag(2)
        assert e.value.code == pf3d.PF_E_NONFINITE
    g, p, st = case()
    with pf3d.Domain(g, p, pf3d.PF_FP64) as d:
        d.load_state(st)
        out = d.step_diag(2)
        assert all(math.isfinite(v) for v in out)


@pytest.mark.parametrize("prec", [pf3d.PF_FP64, pf3d.PF_FP32])
def test_batch_diagnosticos_flag_the_bad_slot_only(gpu, prec):
    (g1, p1, s1), (g2, p2, s2) = case(), case(30, 22, 20)
    s2 = dict(s2)
    s2["phi"] = s2["phi"].copy()
    s2["phi"][10, 11, 12] = np.inf
    with pf3d.Batch(prec) as b:
        a = b.add(g1, p1)
        b.load_state(a, s1)
        c = b.add(g2, p2)
        b.load_state(c, s2)
        assert all(math.isfinite(v) for v in b.diagnosticos(a))
        with pytest.raises(pf3d.PFError) as e:   # as uploaded
            b.diagnosticos(c)
        assert e.value.code == pf3d.PF_E_NONFINITE
        s2["phi"][10, 11, 12] = s1["phi"][0, 0, 0]
        s2["c"] = s2["c"].copy()
        s2["c"][10, 11, 12] = np.inf
        b.load_state(c, s2)
        b.step(2)                                  # a c that is not finite spreads
        out = b.diagnosticos(a)
        assert all(math.isfinite(v) for v in out)
        with pytest.raises(pf3d.PFError) as e:
            b.diagnosticos(c)
        assert e.value.code == pf3d.PF_E_NONFINITE


def test_server_retires_a_blown_up_request_as_failed(gpu):
    """A request whose state goes non-finite is retired with `failed` set
    and no numbers; the others complete normally."""
    jobs = serve.request_stream(seed=4, n=4, step_scale=0.002)
    for j in jobs:
        j.nx = j.ny = 32
        j.nz = 40
        j.steps = 24
        j.arrival = 0.0
    victim = jobs[1]

    def poison(srv, done, waiting):
        # after the first quantum, write a NaN into the victim's concentration
        prec = victim.precision
        if victim.slot >= 0 and victim.slot in srv.active[prec] and not getattr(poison, "done", False):
            b = srv.batches[prec]
            c = b.download(victim.slot, "conc_soluto_old")
            c[20, 16, 16] = np.nan
            b.upload(victim.slot, "conc_soluto_old", c)
            poison.done = True

    srv = serve.Server(budget_bytes=8e9, quantum=8)
    try:
        st = srv.run(jobs, on_quantum=poison)
    finally:
        srv.close()
    assert st["requests"] == 4 and st["failed"] == 1
    assert victim.failed and victim.result == ()
    for j in jobs:
        if j is not victim:
            assert not j.failed and all(math.isfinite(v) for v in j.result)
