"""Accuracy of the mixed form against the plain FP64 form over a long run.

  python -m swehr_b200.error_study [--nx 8192 --ny 8192 --steps 5000 --every 1000]
                                   [--no-envelope] [--out report.json]

Runs the moving-storm domain (8192^2 cells, dx = 1 m, fractal topography with
Hurst 0.7 and 60 m relief, 10 classes 1 um..4 mm, lognormal Ks, a 200 mm/h
Gaussian storm of 1 km radius moving at 2 m/s) in the plain FP64 form, the
mixed form and -- unless --no-envelope -- the FP64 form on the inputs
rounded to FP32 (the envelope: what an FP32 representation of the inputs
alone changes).  All three advance in lockstep; at every checkpoint each
field's relative L-infinity difference to the FP64 run is recorded, with
the water and per-class sediment budget closure of the FP64 and mixed runs.
The three states stay resident on one GPU (about 90 GB at 8192^2); fields
are compared one at a time on the host.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

from . import workloads as W
from .accuracy import quantized_case, rel_linf
from .params import FP64, MIXED

FIELDS = ("h", "hu", "hv", "vinf", "totsed", "totm")
CLASS_FIELDS = ("sed", "U", "M")


def budget_closure(b, sclass: int) -> dict:
    water_scale = max(abs(b.water_now), abs(b.rain_in), 1e-300)
    sed = []
    for k in range(sclass):
        sc = max(abs(b.sed_now[k]), abs(b.detach[k]), 1e-300)
        sed.append(abs(b.sed_residual[k]) / sc)
    return {"water": abs(b.water_residual) / water_scale, "sediment_max": max(sed) if sed else 0.0}


def run(nx: int = 8192, ny: int = 8192, steps: int = 5000, every: int = 1000, envelope: bool = True,
        log=sys.stderr) -> dict:
    from .lib import Simulation
    t0 = time.time()
    case = W.storm_domain(nx=nx, ny=ny, dx=1.0, seed=4, steps=steps)
    print(f"inputs ready in {time.time() - t0:.1f} s", file=log, flush=True)
    sims = {"fp64": Simulation(case, precision=FP64, budget=True),
            "mixed": Simulation(case, precision=MIXED, budget=True)}
    if envelope:
        sims["fp64_on_fp32_inputs"] = Simulation(quantized_case(case), precision=FP64)
    rows = []
    done = 0
    try:
        while done < steps:
            n = min(every, steps - done)
            prog = {k: s.advance(max_steps=n) for k, s in sims.items()}
            done += n
            row = {"step": done, "t": {k: p.t for k, p in prog.items()}, "steps": {k: p.steps for k, p in prog.items()},
                   "device_ms": {k: p.device_ms for k, p in prog.items()}, "rel_linf": {}, "envelope": {}}
            names = [(f, 0) for f in FIELDS] + [(f, k) for f in CLASS_FIELDS for k in range(1, case.sclass + 1)]
            for f, k in names:
                ref = sims["fp64"].field(f, k)
                key = f if k == 0 else f"{f}{k}"
                row["rel_linf"][key] = rel_linf(sims["mixed"].field(f, k), ref)
                if envelope:
                    row["envelope"][key] = rel_linf(sims["fp64_on_fp32_inputs"].field(f, k), ref)
                del ref
            for f in CLASS_FIELDS:
                ks = [f"{f}{k}" for k in range(1, case.sclass + 1)]
                row["rel_linf"][f + "_max"] = max(row["rel_linf"][x] for x in ks)
                if envelope:
                    row["envelope"][f + "_max"] = max(row["envelope"][x] for x in ks)
            row["budget"] = {k: budget_closure(sims[k].budget(), case.sclass) for k in ("fp64", "mixed")}
            rows.append(row)
            print(json.dumps({"step": done, "h": row["rel_linf"]["h"], "totsed": row["rel_linf"]["totsed"],
                              "sed_max": row["rel_linf"]["sed_max"],
                              "env_h": row["envelope"].get("h"), "budget": row["budget"]}), file=log, flush=True)
    finally:
        for s in sims.values():
            s.close()
    return {"workload": f"moving storm {nx}x{ny}, dx=1 m, S={case.sclass}, {steps} steps", "checkpoints": rows,
            "wall_s": time.time() - t0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=8192)
    ap.add_argument("--ny", type=int, default=8192)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--no-envelope", action="store_true")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    rep = run(a.nx, a.ny, a.steps, a.every, not a.no_envelope)
    text = json.dumps(rep, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text)
    else:
        print(text)


if __name__ == "__main__":
    main()
