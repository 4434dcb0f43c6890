"""FP32-vs-FP64 error study (configuration 3's 256x256x512 replica, seed 2).

    python -m pf3d.study [--steps 10000] [--every 1000] [--grid 256x256x512]

Runs the same seeded domain in FP64 and FP32 side by side, and at every
window reports the solid fraction, the tip position and velocity of both and
the relative L2 difference of phi and c.  Prints one JSON object.
"""
from __future__ import annotations

import argparse
import json
import time

from . import Domain, PF_FP32, PF_FP64, init_seeded
from .deck import run6_params, grid
from .init import bump_sites
from .metrics import l2_rel, solid_fraction, tip_position


def run(nx=256, ny=256, nz=512, steps=10000, every=1000, seed=2, n_bumps=16):
    p = run6_params(T0=922.0, taxa_resfr=19.84, AAA=0.01)
    g = grid(nx, ny, nz, 0.5e-6)
    sites = bump_sites(nx, ny, n_bumps, seed)
    doms = {64: Domain(g, p, PF_FP64), 32: Domain(g, p, PF_FP32)}
    for d in doms.values():
        init_seeded(d, sites)
    dt = doms[64].derived().DELTA_T
    rows, prev = [], {}
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        n = min(every, steps - done)
        for d in doms.values():
            d.step(n)
        done += n
        f = {k: (d.download("phase_field_old"), d.download("conc_soluto_old")) for k, d in doms.items()}
        row = {"step": done, "time_s": done * dt}
        for k, (phi, _) in f.items():
            row[f"fs_{k}"] = solid_fraction(phi)
            row[f"tip_{k}"] = tip_position(phi)
            if k in prev:
                row[f"v_{k}"] = (row[f"tip_{k}"] - prev[k]) * g.dz / (n * dt)   # m/s
            prev[k] = row[f"tip_{k}"]
        row["l2_phi"] = l2_rel(f[32][0], f[64][0])
        row["l2_c"] = l2_rel(f[32][1], f[64][1])
        row["err_fs"] = abs(row["fs_32"] - row["fs_64"]) / max(row["fs_64"], 1e-30)
        row["err_tip"] = abs(row["tip_32"] - row["tip_64"]) / max(row["tip_64"], 1e-30)
        rows.append(row)
    for d in doms.values():
        d.close()
    worst = {k: max(r[k] for r in rows) for k in ("err_fs", "err_tip", "l2_phi", "l2_c")}
    vs = [abs(r["v_32"] - r["v_64"]) / max(abs(r["v_64"]), 1e-30) for r in rows if "v_64" in r and abs(r["v_64"]) > 0]
    worst["err_v"] = max(vs) if vs else 0.0
    return {"grid": [nx, ny, nz], "steps": steps, "every": every, "seed": seed, "bumps": n_bumps,
            "wall_s": time.perf_counter() - t0, "worst": worst, "windows": rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--grid", default="256x256x512")
    a = ap.parse_args()
    nx, ny, nz = (int(v) for v in a.grid.split("x"))
    print(json.dumps(run(nx, ny, nz, a.steps, a.every)))


if __name__ == "__main__":
    main()
