"""GPU tests of the batched and served forms: every domain of a batch gives
the same bits as the same domain stepped alone with pf_step, whatever the
tile shape, the z-chunk and the other domains; admission respects the
device-memory budget; the continuous-batching server returns, for each
request, the result the request has when run alone."""
import numpy as np
import pytest

import make_golden as MG
import pf3d
from pf3d import deck, init, serve

pytestmark = pytest.mark.gpu


def case(nx, ny, nz, **over):
    kw = dict(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    kw.update(over)
    p = deck.run6_params(**kw)
    return deck.grid(nx, ny, nz, 0.5e-6), p, MG.small_state(nx, ny, nz, p)


def alone(g, p, st, prec, n):
    with pf3d.Domain(g, p, prec) as d:
        d.load_state(st)
        d.step(n)
        return d.fields(), d.state()


@pytest.mark.parametrize("prec", [pf3d.PF_FP64, pf3d.PF_FP32])
def test_batch_equals_alone(gpu, prec):
    cases = [case(40, 33, 50), case(21, 64, 17, T0=918.0, taxa_resfr=30.0), case(70, 12, 35, AAA=0.02)]
    targets = [0, 6, 0]
    with pf3d.Batch(prec) as b:
        slots = []
        for (g, p, st), tgt in zip(cases, targets):
            s = b.add(g, p)
            b.load_state(s, st)
            b.set_target(s, tgt)
            slots.append(s)
        b.step(5)
        b.set_tile(4, 16)
        b.step(6)          # the second domain stops at its target (6 steps)
        for (g, p, st), s, tgt in zip(cases, slots, targets):
            n = tgt if tgt else 11
            want, wst = alone(g, p, st, prec, n)
            got = b.fields(s)
            assert b.state(s).it == n and b.state(s).M0 == wst.M0 and b.state(s).TP == wst.TP
            for k in want:
                assert np.array_equal(got[k], want[k]), (s, k)


def test_async_batches_run_together(gpu):
    """Two batches (FP64 and FP32) queued with step_async run on their own
    streams at the same time; after wait() every domain has its alone bits,
    and steps spanning several graphs (more than 8) keep them too."""
    cases = [case(40, 30, 36), case(28, 44, 30, T0=919.0)]
    with pf3d.Batch(pf3d.PF_FP64) as b64, pf3d.Batch(pf3d.PF_FP32) as b32:
        slots = {}
        for b in (b64, b32):
            for i, (g, p, st) in enumerate(cases):
                s = b.add(g, p)
                b.load_state(s, st)
                slots[(id(b), i)] = s
        for n in (5, 19):
            b64.step_async(n)
            b32.step_async(n)
            assert b64.wait() > 0 and b32.wait() > 0
        for b, prec in ((b64, pf3d.PF_FP64), (b32, pf3d.PF_FP32)):
            for i, (g, p, st) in enumerate(cases):
                want, _ = alone(g, p, st, prec, 24)
                got = b.fields(slots[(id(b), i)])
                for k in want:
                    assert np.array_equal(got[k], want[k]), (prec, i, k)


def test_paired_batch_equals_alone(gpu):
    """FP32 batch with two cells per thread: every domain keeps its alone bits
    (domains big enough to have interior tiles, and small ragged ones)."""
    cases = [case(100, 70, 40), case(40, 33, 50), case(75, 90, 24, h_quintico=1)]
    with pf3d.Batch(pf3d.PF_FP32) as b:
        b.set_paired(1)
        slots = []
        for g, p, st in cases:
            s = b.add(g, p)
            b.load_state(s, st)
            slots.append(s)
        b.step(9)
        for (g, p, st), s in zip(cases, slots):
            want, _ = alone(g, p, st, pf3d.PF_FP32, 9)
            got = b.fields(s)
            for k in want:
                assert np.array_equal(got[k], want[k]), (s, k)


@pytest.mark.parametrize("prec", [pf3d.PF_FP64, pf3d.PF_FP32])
def test_batch_mixed_noise_kinds(gpu, prec):
    """A batch whose domains draw different noise (the smooth noise selects the
    kernels that carry it) still gives each domain its alone result, before and
    after the smooth-noise domain leaves."""
    cases = [case(36, 20, 30), case(24, 40, 26, ruido_tipo=2, AAA=0.02), case(30, 30, 24, ruido_tipo=1)]
    with pf3d.Batch(prec) as b:
        slots = []
        for g, p, st in cases:
            s = b.add(g, p)
            b.load_state(s, st)
            slots.append(s)
        b.step(4)
        g, p, st = cases[1]
        want, _ = alone(g, p, st, prec, 4)
        got = b.fields(slots[1])
        for k in want:
            assert np.array_equal(got[k], want[k]), ("smooth", k)
        b.remove(slots[1])
        b.step(5)
        for i in (0, 2):
            g, p, st = cases[i]
            want, _ = alone(g, p, st, prec, 9)
            got = b.fields(slots[i])
            for k in want:
                assert np.array_equal(got[k], want[k]), (i, k)


def test_batch_budget_and_membership(gpu):
    g, p, st = case(32, 32, 32)
    per = pf3d._abi.LIB.pf_ctx_bytes(pf3d._abi.C.byref(g), 32)
    with pf3d.Batch(pf3d.PF_FP32, budget_bytes=int(2.5 * per)) as b:
        s0 = b.add(g, p)
        s1 = b.add(g, p)
        with pytest.raises(pf3d.PFError) as e:
            b.add(g, p)
        assert e.value.code == pf3d._abi.PF_E_NOMEM
        b.remove(s0)
        s2 = b.add(g, p)        # the freed memory admits the next domain
        assert b.count() == 2 and s2 == s0
        b.load_state(s1, st)
        b.load_state(s2, st)
        b.step(3)
        assert np.array_equal(b.download(s1, "phase_field_old"), b.download(s2, "phase_field_old"))


@pytest.mark.parametrize("prec", [pf3d.PF_FP64, pf3d.PF_FP32])
def test_device_init_matches_host_recipe(gpu, prec):
    nx, ny, nz = 48, 40, 64
    p = deck.run6_params(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    g = deck.grid(nx, ny, nz, 0.5e-6)
    sites = init.bump_sites(nx, ny, 4, 7)
    st = init.initial_state(nx, ny, nz, 4, 7, p)
    with pf3d.Domain(g, p, prec) as d:
        pf3d.init_seeded(d, sites)
        tol = 1e-15 if prec == pf3d.PF_FP64 else 1e-7
        for key, field in (("phi", "phase_field_old"), ("c", "conc_soluto_old"), ("T", "TOLD")):
            got = d.download(field)
            assert np.max(np.abs(got - st[key])) <= tol * max(1.0, np.max(np.abs(st[key]))), key
        assert not d.download("DPP").any()


def test_autotune_keeps_results(gpu):
    cases = [case(64, 48, 80), case(33, 33, 40)]
    with pf3d.Batch(pf3d.PF_FP32) as b:
        slots = []
        for g, p, st in cases:
            s = b.add(g, p)
            b.load_state(s, st)
            slots.append(s)
        ty, zc, ms = b.autotune(1)
        assert ty in (4, 8, 16) and zc in (16, 32, 64, 128)
        n = b.state(slots[0]).it
        # the TMA passes (the default) run 32 x 8 tiles: 4 z-chunks x one or
        # two cells per thread, x (1 warm-up + 1 timed) real steps
        assert n == 16
        b.step(2)
        for (g, p, st), s in zip(cases, slots):
            want, _ = alone(g, p, st, pf3d.PF_FP32, n + 2)
            got = b.fields(s)
            for k in want:
                assert np.array_equal(got[k], want[k]), k


def test_server_alone_vs_mix(gpu):
    """Requests served together give, each, the result it has alone."""
    jobs = serve.request_stream(seed=11, n=6, rate_per_s=1000.0, step_scale=0.004)
    for j in jobs:
        j.nx = j.ny = min(j.nx, 48)
        j.nz = min(j.nz, 64)
    srv = serve.Server(budget_bytes=3e9, quantum=4)
    try:
        stats = srv.run(jobs)
    finally:
        srv.close()
    assert stats["requests"] == len(jobs)
    for j in jobs:
        with pf3d.Domain(j.grid(), j.params(), j.precision) as d:
            pf3d.init_seeded(d, j.sites())
            out = d.step_diag(j.steps)
            tr = d.track()
        assert np.array_equal(np.array(out), np.array(j.result)), j.jid
        assert tr == j.track, j.jid
