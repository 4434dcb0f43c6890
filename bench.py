#!/usr/bin/env python
"""Benchmark of the coupled explicit phase-field step on B200.

One bench "step" = one time step of the reference's loop (principal.f90:93-226:
temperatura, two phase sweeps, solute, M0, swap) over the whole domain.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

ours       value = GCell-updates/s of the fused FP64 step, device-resident
           (CUDA events, max over ranks); e2e = the same job through the C-ABI
           with the state uploaded from / downloaded to pinned host memory and
           a per-step probe read; roofline of the dominant kernel from CUDA
           events around each launch; cpu_baseline = the CPU oracle on the
           same full grid for a bounded number of steps (rank 0, N = 1).
reference  the reference's CPU path, i.e. the CPU oracle (C restatement of
           the Fortran OpenMP path; the Fortran cannot be compiled here) on the
           same full grid, all host threads, rank 0 only, K steps after W.
Multi-GPU: the path shards by domain (replicas only): every rank runs its own
domain, no data-path collective; value = all ranks' cell updates / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "phase-field-project-3d_b200"))

METRIC = "GCell-updates/s & %HBM peak, FP32 vs FP64 plain; p50/p99 batched-solve latency"
UNIT = "GCell-updates/s"
# algorithmic HBM bytes per cell and step of the fused step: phi, c, T, DPP
# each read once and written once (8 B FP64 / 4 B FP32)
STEP_BYTES_PER_CELL = {64: 64, 32: 32}
# the step's algorithmic bytes split between the two fused passes, each state
# byte counted in the pass that must move it:
#   first = temperatura + sweep 1: reads phi, c, T, DPP; writes T   (5 fields)
#   last  = sweep 2 + solute     : writes phi, DPP, c               (3 fields)
# The passes also move phi_mid, the noise hand-over and a second read of c
# (104 B/cell in FP64 by design); ncu's per-launch DRAM bytes are "traffic".
PASS_BYTES_PER_CELL = {"fused_first": {64: 40, 32: 20}, "fused_last": {64: 24, 32: 12}}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def step_hbm_frac_of(gbs: float, peak: float) -> float:
    return gbs / peak


def ncu_figures(kernel: str, precision: int) -> dict:
    """Per-cell figures of a fused pass from the committed ncu summary
    (profiles/ncu_passes.txt: `<pass> fp<NN> key=value ...`): DRAM bytes,
    executed thread instructions and FP64 flops per cell, issue-active and
    FP64-pipe fractions of the captured launch."""
    path = os.path.join(ROOT, "profiles", "ncu_passes.txt")
    out = {}
    try:
        for line in open(path):
            t = line.split()
            if len(t) >= 3 and not t[0].startswith("#") and t[0] == kernel and t[1] == f"fp{precision}":
                for kv in t[2:]:
                    k, v = kv.split("=")
                    out[k] = float(v)
    except Exception:
        pass
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.idx = gpu_index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if len(r) > 8]
        mx = max(float(r[2]) for r in rows if len(r) > 8)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) > 8:
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
        loaded = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows)}


def oracle_on_workload(w, st, warmup: int, steps: int = 0, seconds: float = 0.0):
    """Time the CPU oracle (the C restatement of the reference's CPU OpenMP
    path, all host threads) on the workload's full grid from the state `st`.
    Runs `steps` timed steps, or, with steps = 0, as many as fit `seconds`
    (at least 2).  Returns (GCell-updates/s, steps, seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    p = w.params()
    o = pyoracle.Oracle(w.grid(), p)
    try:
        o.load_state(st)
        o.step(warmup)
        n, t0 = 0, time.perf_counter()
        if steps > 0:
            o.step(steps)
            n = steps
        else:
            while n < 2 or time.perf_counter() - t0 < seconds:
                o.step(1)
                n += 1
        dt = time.perf_counter() - t0
    finally:
        o.close()
    return w.cells * n / dt / 1e9, n, dt, pyoracle.num_threads()


def workload_config(w, p, world: int) -> dict:
    es = 8 if w.precision == 64 else 4
    return {"workload": w.name, "grid": [w.nx, w.ny, w.nz], "cells": w.cells, "precision": f"fp{w.precision}",
            "sweeps_per_step": p.n_varreduras, "parallelism": f"replicas{world}",
            "l2": f"inputs larger than L2 (resident state of 4 fields x {es} B x {w.cells / 1e6:.0f}M cells)"}


def run_reference(args, rank: int, world: int):
    """The reference's CPU path on the same workload as our arm: the oracle on
    the full grid, all host threads.  Imports only the package's host-side
    modules (deck, initial-state recipe); libpf3d.so is never mapped."""
    if rank != 0:
        return 0
    from pf3d import deck, init
    w = deck.WORKLOADS[args.workload]
    p = w.params()
    st = init.initial_state(w.nx, w.ny, w.nz, w.n_bumps, w.seed, p)
    v, n, dt, threads = oracle_on_workload(w, st, args.warmup, steps=args.steps)
    del st
    sample = (f"the full {w.nx}x{w.ny}x{w.nz} workload (same deck and seeded initial state as the GPU arm), "
              f"{n} steps after {args.warmup} warm-up, {threads} threads")
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": n, "warmup": args.warmup, "ms_per_step": dt / n * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(w, p, world),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU OpenMP path as the C restatement in oracle/ (no Fortran compiler in the image)",
    }
    print(json.dumps(line))
    return 0


def bench_fp32(args, torch, pf3d, deck, init, stream, world):
    """1024^3 FP32 (configuration 3), state created on the device."""
    w = deck.WORKLOADS["c3_1024cube_fp32"]
    g, p = w.grid(), w.params()
    d = pf3d.Domain(g, p, pf3d.PF_FP32)
    d.set_stream(stream.cuda_stream)
    pf3d.init_seeded(d, init.bump_sites(w.nx, w.ny, w.n_bumps, w.seed))
    d.step(args.warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = max(4, args.steps // 2)
    e0.record(stream)
    d.step(n)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    peak, _ = measured_peaks()
    v = w.cells * world / (ms / 1e3) / 1e9
    d.close()
    return {"workload": w.name, "cells": w.cells, "steps": n, "ms_per_step": ms, "value": v, "unit": UNIT,
            "hbm_frac_step": v / world * STEP_BYTES_PER_CELL[32] / peak, "init": "device (pf_init_seeded)"}


def bench_batch(args, pf3d, serve, init, world=1, rank=0, barrier=None, max_over_ranks=None):
    """96 FP32 domains of uneven size (configuration 4), autotuned tiles.
    With N ranks the domains are routed longest-first (replicas.assign on
    their cells) and every rank runs its share as one batch; the same 96
    domains in total, so the scaling is strong, timed as the slowest rank."""
    from pf3d import replicas
    jobs_all = serve.batch_domains(seed=3)
    costs = [j.cells for j in jobs_all]
    jobs = [jobs_all[i] for i in replicas.my_share(costs, world, rank)]
    b = pf3d.Batch(pf3d.PF_FP32)
    for j in jobs:
        s = b.add(j.grid(), j.params())
        b.init_seeded(s, j.sites())
        j.slot = s
    t0 = time.perf_counter()
    ty, zc, _ = b.autotune(2)
    tune_s = time.perf_counter() - t0
    b.step(8)
    n = max(16, args.steps)
    if barrier:
        barrier()
    ms = b.step(n)
    if max_over_ranks:
        ms = max_over_ranks(ms)
    cells = sum(costs)
    b.close()
    out = {"workload": "c4_96_domains_fp32", "domains": len(jobs_all), "cells": cells, "steps": n,
           "ms_per_step": ms / n, "value": cells * n / (ms / 1e3) / 1e9, "unit": UNIT,
           "tile": [32, ty, zc], "autotune_s": tune_s, "launch": "persistent work-list kernels, CUDA graph of 8 steps"}
    if world > 1:
        out["scaling"] = "strong"
        out["routing"] = "longest-first on cells; rank 0 holds %d domains, %.1f M cells" % (
            len(jobs), sum(j.cells for j in jobs) / 1e6)
    return out


def bench_karma(args, torch, stream):
    """The reference's second model (karma/karma3d.f90) on 512^3, FP64 and
    FP32, seeded on the device, with a CPU-oracle sample for scale."""
    from pf3d import karma
    out = {"workload": "karma_512cube_Fnoise0.01", "unit": UNIT}
    for prec in (64, 32):
        p = karma.karma_params(N=512, Fnoise=0.01)
        with karma.Karma(p, prec) as k:
            k.set_stream(stream.cuda_stream)
            k.seed()
            k.step(args.warmup)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            n = max(10, args.steps // 2)
            e0.record(stream)
            k.step(n)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / n
            out[f"fp{prec}"] = {"ms_per_step": ms, "value": 512 ** 3 / (ms / 1e3) / 1e9, "steps": n,
                                "launches_per_step": 2}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    N = 96
    pk = karma.karma_params(N=N, Fnoise=0.01)
    o = pyoracle.KarmaOracle(N, N, N, pk.lambda_, pk.eps4, pk.dx, pk.dt, pk.Fnoise, pk.k)
    o.set(*karma.seed_state(pk))
    o.step(1)
    t0, n = time.perf_counter(), 0
    while n < 3 or time.perf_counter() - t0 < 3.0:
        o.step(1)
        n += 1
    dt = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": N ** 3 * n / dt / 1e9, "unit": UNIT, "cores": pyoracle.num_threads(),
                           "kind": "port", "sample": f"{N}^3, {n} steps (C restatement of karma3d.f90, OpenMP)"}
    return out


def bench_serve(args, serve):
    """The serving configuration (5): the seeded Poisson stream of 2000
    requests at 20/s under the 150 GB budget, every step count scaled by
    step_scale (1 = as configured)."""
    jobs = serve.request_stream(seed=4, n=args.serve_requests, step_scale=args.serve_step_scale)
    srv = serve.Server(budget_bytes=150e9, quantum=args.serve_quantum)
    try:
        st = srv.run(jobs)
    finally:
        srv.close()
    scale = "as configured" if args.serve_step_scale == 1.0 else f"every step count x {args.serve_step_scale}"
    st.update({"workload": "c5_poisson_20_per_s_seed4",
               "sample": f"{len(jobs)} requests of the seeded stream, {scale}",
               "fp64_share": sum(1 for j in jobs if j.precision == 64) / len(jobs), "quantum_steps": args.serve_quantum})
    return st


def bench_fp32_error(args):
    """FP32 against FP64 on the 256x256x512 replica (seed 2): worst relative
    errors of tip position, solid fraction, tip velocity and L2(phi, c)."""
    from pf3d import study
    r = study.run(256, 256, 512, steps=args.error_steps, every=max(1, args.error_steps // 4), seed=2, n_bumps=16)
    return {"workload": "c3_replica_256x256x512_seed2", "steps": r["steps"], "windows": len(r["windows"]),
            "worst_rel_error": r["worst"], "bound_tip_and_solid_fraction": 5e-3,
            "tip_cells": [r["windows"][0]["tip_64"], r["windows"][-1]["tip_64"]], "wall_s": r["wall_s"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c2_512x512x1024_fp64")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-karma", action="store_true")
    ap.add_argument("--no-error", action="store_true")
    ap.add_argument("--error-steps", type=int, default=2000)
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-step-scale", type=float, default=0.05)
    ap.add_argument("--serve-quantum", type=int, default=16)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist
    import pf3d
    from pf3d import deck, init

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    from pf3d import replicas
    barrier = replicas.barrier

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, device="cuda")

    w = deck.WORKLOADS[args.workload]
    g, p = w.grid(), w.params()
    prec = w.precision
    cells = w.cells
    st = init.initial_state(w.nx, w.ny, w.nz, w.n_bumps, w.seed + rank, p)
    # a dedicated (non-legacy) stream: the library runs on it and the events see it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    dom = pf3d.Domain(g, p, prec)
    dom.set_stream(stream.cuda_stream)
    dom.load_state(st)
    dom.step(args.warmup)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        dom.step(1)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    clk = clocks.stop()
    value = replicas.aggregate_rate(cells, args.steps, world, ms / 1e3)
    launches_per_step = 2 if p.n_varreduras >= 2 else 1
    launches_per_step += max(0, p.n_varreduras - 2)

    # ---- per-kernel timing (CUDA events around every fused launch, same stream) ----
    dom.set_option(pf3d.PF_OPT_KTIMING, 1)
    dom.kernel_times(reset=True)
    dom.step(args.steps)
    nf, mf, nl, ml = dom.kernel_times(reset=True)
    dom.set_option(pf3d.PF_OPT_KTIMING, 0)
    peak, peak_kind = measured_peaks()
    kname, n_k, ms_k = ("fused_first", nf, mf) if mf >= ml else ("fused_last", nl, ml)
    alg_bytes = PASS_BYTES_PER_CELL[kname][prec] * cells
    avg_s = ms_k / max(1, n_k) / 1e3
    achieved = alg_bytes / avg_s / 1e9
    fig = ncu_figures(kname, prec)
    tr = fig.get("dram_bytes_per_cell")
    step_gbs = value / world * STEP_BYTES_PER_CELL[prec]
    # the other two ceilings of the dominant pass, from this run's kernel time
    # and the per-cell counts of its ncu capture: the FP64 pipe (nominal peak
    # 148 SMs x 64 FP64 FMA a clock x 2 flops at the sampled SM clock) and
    # instruction issue (148 SMs x 4 schedulers x 1 warp instruction a clock)
    clk_hz = (clk["sm_mhz"] if clk and clk.get("sm_mhz") else 1965.0) * 1e6
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    ceilings = {"hbm": (tr * cells / avg_s / 1e9) / peak if tr else achieved / peak}
    fp64 = None
    if prec == 64 and "fp64_inst_per_cell" in fig:
        # FP64 pipe: lane-operations (DFMA, DMUL, DADD) per second against
        # 64 a clock per SM; flops count an FMA as two
        peak_ops = n_sm * 64 * clk_hz
        ops = fig["fp64_inst_per_cell"] * cells / avg_s
        other = ncu_figures("fused_first" if kname == "fused_last" else "fused_last", prec)
        step_ops = (fig["fp64_inst_per_cell"] + other.get("fp64_inst_per_cell", 0.0)) * cells * args.steps / (ms / 1e3)
        step_flops = fig.get("fp64_flops_per_cell", 0.0) + other.get("fp64_flops_per_cell", 0.0)
        fp64 = {"achieved_tflops": fig.get("fp64_flops_per_cell", 0.0) * cells / avg_s / 1e12,
                "peak_tflops": 2 * peak_ops / 1e12, "pipe_frac": ops / peak_ops,
                "inst_per_cell": fig["fp64_inst_per_cell"], "flops_per_cell": fig.get("fp64_flops_per_cell"),
                "step": {"inst_per_cell": fig["fp64_inst_per_cell"] + other.get("fp64_inst_per_cell", 0.0),
                         "flops_per_cell": step_flops, "pipe_frac": step_ops / peak_ops,
                         "achieved_tflops": step_flops * cells * args.steps / (ms / 1e3) / 1e12},
                "peak_source": f"nominal: {n_sm} SMs x 64 FP64 lane-operations a clock at the sampled "
                               f"{clk_hz / 1e6:.0f} MHz"}
        ceilings["fp64_pipe"] = ops / peak_ops
    if "inst_per_cell" in fig:
        ceilings["issue"] = fig["inst_per_cell"] / 32 * cells / avg_s / (n_sm * 4 * clk_hz)
    limiter = max(ceilings, key=ceilings.get)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (tr * cells if tr is not None else None), "kernel": kname,
                "kernel_ms": avg_s * 1e3, "peak_source": f"{peak_kind} hbm_gbs",
                "alg_bytes_per_cell": PASS_BYTES_PER_CELL[kname][prec], "traffic_bytes_per_cell": tr,
                "shares": {"fused_first": mf / max(1e-9, mf + ml), "fused_last": ml / max(1e-9, mf + ml)},
                "step": {"achieved": step_gbs, "frac": step_hbm_frac_of(step_gbs, peak),
                         "alg_bytes_per_cell": STEP_BYTES_PER_CELL[prec]},
                "fp64": fp64,
                "ceiling_fracs": ceilings,
                "limiter": limiter,
                "ncu_figures": fig}
    step_hbm_frac = step_gbs / peak

    # ---- the diagnostics reduction (a separate pass, run at output events):
    # its cost beside a step, from CUDA events around pf_diagnosticos ----
    dom.diagnosticos()
    torch.cuda.synchronize()
    dms = []
    for _ in range(3):
        d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        d0.record(stream)
        dom.diagnosticos()
        d1.record(stream)
        torch.cuda.synchronize()
        dms.append(d0.elapsed_time(d1))
    diag = {"ms": min(dms), "alg_bytes_per_cell": 4 * (8 if prec == 64 else 4),
            "frac_of_step": min(dms) / (ms / args.steps),
            "reads": "phi, c, T, DPP (sums, extremes, free energy, non-finite count)"}

    # ---- end to end through the C-ABI with pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        host = {k: torch.from_numpy(st[k]).pin_memory() for k in ("phi", "c", "T")}
        host["dpp"] = torch.zeros(st["phi"].shape, dtype=torch.float64).pin_memory()
        out = {k: torch.empty_like(v).pin_memory() for k, v in host.items()}
        fields_in = [("phase_field_old", "phi"), ("conc_soluto_old", "c"), ("TOLD", "T"), ("DPP", "dpp")]
        dom2 = pf3d.Domain(g, p, prec)
        dom2.set_stream(stream.cuda_stream)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for fname, key in fields_in:
            dom2.upload(fname, host[key].numpy())
        probe = 0.0
        for _ in range(args.steps):
            dom2.step(1)
            # the reference's per-sweep progress print reads 2 cells per sweep
            probe += dom2.probe("phase_field_old", w.nx // 2, 10, max(w.nz // 2, 1))
            probe += dom2.probe("phase_field_old", w.nx // 2, min(100, w.ny - 1), max(w.nz // 2, 1))
        for fname, key in fields_in:
            dom2.download(fname, out[key].numpy())
        torch.cuda.synchronize()
        t_e2e = max_over_ranks(time.perf_counter() - t0)
        barrier()
        dom2.close()
        state_bytes = 4 * cells * 8
        e2e = {"value": cells * args.steps * world / t_e2e / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": state_bytes / args.steps + 2 * 8,
               "job": "upload 4 state fields, K steps with a 2-cell probe read each, download 4 fields"}
        del host, out

    dom.close()

    extra = {}
    if not args.no_fp32:
        extra["fp32"] = bench_fp32(args, torch, pf3d, deck, init, stream, world)
        extra["fp32"]["speedup_vs_fp64"] = extra["fp32"]["value"] / value
    from pf3d import serve as serve_mod
    if not args.no_batch:   # every rank: the 96 domains are spread over the ranks
        extra["batched"] = bench_batch(args, pf3d, serve_mod, init, world, rank, barrier, max_over_ranks)
    if rank == 0 and world == 1:
        if not args.no_error:
            extra["fp32_error"] = bench_fp32_error(args)
        if not args.no_serve:
            extra["serving"] = bench_serve(args, serve_mod)
        if not args.no_karma:
            extra["karma"] = bench_karma(args, torch, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, n, dt, thr = oracle_on_workload(w, st, 1, seconds=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"the full {w.nx}x{w.ny}x{w.nz} workload, {n} steps after 1 warm-up in {dt:.1f} s "
                         f"(C restatement of the reference CPU OpenMP path)"}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == 64 else "f32", "data": "synthetic",
        "config": workload_config(w, p, world),
        "hbm_frac_step": step_hbm_frac,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches_per_step * args.steps,
        "diagnostics": diag,
        "clocks": clk,
    }
    line.update(extra)
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
