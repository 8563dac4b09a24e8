"""Generate the golden fixtures in tests/golden/ from the reference program.

The reference (SWEHR.c) ships no tests, golden vectors or known answers;
its only example is the 3x51 strip in input.txt/topoin.txt.  The fixtures
here are outputs of the reference itself, built from its source by
oracle/build_ref.py, on:

  shipped.npz       the shipped example's input files and the reference's
                    state after 2000 and 20000 steps (inflow on, default BCs;
                    the last row of M is NaN, a reference 0/0 at t=0)
  tiny_*.npz        small random hillslopes, every boundary type, inflow
                    on and off, per-cell Ks, to the end of their event
  hillslope.npz     the 200x50 hillslope, full 1200 s run, and the state at
                    600 s (mid-event, wet)
  failure_*.npz     cross-sloped grids with the deposit cohesion lowered
                    (two small ones and the 200x50 hillslope to 600 s):
                    slope failure fires (SWEHR.c:1292-1312, 1497-1503)
  solid_*.npz       interior solid cells (two small grids and the 200x50
                    hillslope with buildings and a wall, to 600 s): the
                    topography fill, reflecting faces and the source skip
                    (SWEHR.c:288-322, 1137-1146, 1205-1214, 1233)
  shipped_files.npz the reference's own output files for the shipped
                    example run as shipped (movies on): the ten result
                    grids, stage.txt, saveflow.txt, every 30th frame of the
                    five movie files, the console's per-frame lines and its
                    header (the host driver's parity target)

Each file holds the Case (params as JSON, topo, rain, ds, pfrac, ks) and the
reference's %.17g dump of every state field.

Run (needs the reference checkout; it is not read anywhere else):
    SWEHR_REFERENCE=<checkout> python tests/golden/make_golden.py   (or --reference DIR)
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from swehr_b200 import io as swio, workloads as W  # noqa: E402
from swehr_b200.params import REFERENCE_DEFAULTS  # noqa: E402
import harness  # noqa: E402

TINY = [
    dict(nx=12, ny=9, S=3, seed=5, bndry=(0, 1, 1, 1), inflow=0, rain_mmh=90.0, tend=60.0),
    dict(nx=15, ny=11, S=4, seed=6, bndry=(1, 0, 1, 1), inflow=1, rain_mmh=300.0, tend=120.0),
    dict(nx=15, ny=11, S=4, seed=7, bndry=(0, 0, 0, 0), inflow=0, rain_mmh=300.0, tend=120.0),
    dict(nx=9, ny=14, S=2, seed=8, bndry=(1, 1, 1, 1), inflow=1, rain_mmh=200.0, tend=90.0, per_cell_ks=False),
    dict(nx=20, ny=6, S=7, seed=9, bndry=(0, 1, 0, 1), inflow=0, rain_mmh=500.0, tend=150.0),
]

FAILURE = [
    dict(slope_y=0.5, cohesion=5.0, nx=20, ny=16, S=4, seed=31, bndry=(0, 1, 1, 1), rain_mmh=300.0, tend=120.0),
    dict(slope_y=0.7, cohesion=50.0, nx=17, ny=13, S=7, seed=32, bndry=(1, 1, 0, 0), rain_mmh=200.0, tend=150.0),
]

SOLID = [
    dict(bndry=(1, 1, 1, 1), inflow=1, S=3, seed=52),
    dict(bndry=(0, 0, 0, 0), rain_mmh=500.0, seed=53),
]

DUMP_KEYS = ("h", "hu", "hv", "z", "vinf", "totm", "dep", "totsed", "maxvel", "maxdepth", "U", "M", "sed",
             "stage", "saveflow")


def save(path, case, dumps: dict):
    arrs = {"params_json": np.array(json.dumps(case.params)), "topo": case.topo, "rain": case.rain,
            "ds": case.ds, "pfrac": case.pfrac, "name": np.array(case.name)}
    if case.ks is not None:
        arrs["ks"] = case.ks
    if getattr(case, "solid", None) is not None:
        arrs["solid"] = case.solid
    for tag, d in dumps.items():
        arrs[f"{tag}__steps"] = np.array(d["steps"])
        arrs[f"{tag}__t"] = np.array(d["t"])
        for k in DUMP_KEYS:
            arrs[f"{tag}__{k}"] = d[k]
    np.savez_compressed(path, **arrs)
    print("wrote", path, os.path.getsize(path), "bytes")


def shipped_case(reference):
    c = swio.read_inputs(reference)
    for k in ("bndry", "inflow", "roughness", "ks", "theta0", "thetas", "hf", "vinf0", "uc", "uc2"):
        c.params[k] = REFERENCE_DEFAULTS[k]
    c.params["bndry"] = list(c.params["bndry"])
    c.name = "shipped"
    return c


RESULT_FILES = ("topoout", "depth", "uh", "vh", "ch", "m", "c", "vel", "maxvel", "maxdepth")
MOVIE_FILES = ("topomovie", "depthmovie", "velocitymovie", "cmovie", "Mmovie")
FRAME_STRIDE = 30


def read_table(path):
    with open(path) as f:
        return np.array([[float(v) for v in line.split()] for line in f if line.strip()])


def shipped_files(reference):
    """Run the reference binary on the shipped input files exactly as shipped
    and parse everything it writes."""
    import shutil
    import subprocess
    import tempfile
    wd = tempfile.mkdtemp(prefix="swehr_files_")
    for fn in ("input.txt", "rain.txt", "particlesizein.txt", "particlepercentin.txt", "topoin.txt"):
        shutil.copy(os.path.join(reference, fn), wd)
    r = subprocess.run([harness.ref_binary(False)], cwd=wd, capture_output=True, text=True, timeout=3600)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    lines = r.stdout.splitlines()
    frames = [ln for ln in lines if ln.count("\t") == 3 and not ln.startswith(("Point", "SWEHR"))]
    header = [ln for ln in lines if ln.split(":")[0] in ("Grid Size (Spacing)", "Number of conserved variables",
                                                          "Number of particle size classes", "a0", "ad0", "F",
                                                          "J", "h0", "mtstar0", "b", "Basin Outlet Pixel",
                                                          "Basin Outlet Elevation (m)")
              or ln.startswith("Point ") or ln.startswith("H-R Parameters")]
    arrs = {"header": np.array("\n".join(header)),
            "frame_lines": np.array([[float(v) for v in ln.split()] for ln in frames])}
    ny = int(read_table(os.path.join(wd, "depth.txt")).shape[0])
    for n in RESULT_FILES:
        arrs[n] = read_table(os.path.join(wd, n + ".txt"))
    arrs["stage"] = read_table(os.path.join(wd, "stage.txt"))
    arrs["saveflow"] = read_table(os.path.join(wd, "saveflow.txt"))
    for n in MOVIE_FILES:
        m = read_table(os.path.join(wd, n + ".txt"))
        arrs[n + "_frames"] = np.array(m.shape[0] // ny)
        arrs[n] = m.reshape(-1, ny, m.shape[1])[::FRAME_STRIDE]
    arrs["frame_stride"] = np.array(FRAME_STRIDE)
    shutil.rmtree(wd, ignore_errors=True)
    path = os.path.join(HERE, "shipped_files.npz")
    np.savez_compressed(path, **arrs)
    print("wrote", path, os.path.getsize(path), "bytes")


def failure_fixtures():
    for n, kw in enumerate(FAILURE):
        c = W.failure_tiny(**kw)
        c.params["bndry"] = list(c.params["bndry"])
        d, _ = harness.run_reference(c)
        save(os.path.join(HERE, f"failure_{n}.npz"), c, {"end": d})
    c = W.failure_hillslope()
    c.params["bndry"] = list(c.params["bndry"])
    d, _ = harness.run_reference(c)
    save(os.path.join(HERE, "failure_hillslope.npz"), c, {"end": d})


def solid_fixtures():
    for n, kw in enumerate(SOLID):
        c = W.solid_tiny(**kw)
        c.params["bndry"] = list(c.params["bndry"])
        d, _ = harness.run_reference(c)
        save(os.path.join(HERE, f"solid_{n}.npz"), c, {"end": d})
    c = W.solid_hillslope()
    c.params["bndry"] = list(c.params["bndry"])
    d, _ = harness.run_reference(c)
    save(os.path.join(HERE, "solid_hillslope.npz"), c, {"end": d})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="reference checkout (default: $SWEHR_REFERENCE)")
    ap.add_argument("--only", default=None, help="shipped_files | failure | solid: only regenerate those fixtures")
    a = ap.parse_args()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import build_ref
    a.reference = build_ref.reference_dir(a.reference)
    if not build_ref.build(a.reference):
        raise SystemExit("reference not available")
    if a.only == "shipped_files":
        shipped_files(a.reference)
        return
    if a.only in (None, "failure"):
        failure_fixtures()
        if a.only == "failure":
            return
    if a.only in (None, "solid"):
        solid_fixtures()
        if a.only == "solid":
            return
    c = shipped_case(a.reference)
    d1, _ = harness.run_reference(c, max_steps=2000)
    d2, _ = harness.run_reference(c, max_steps=20000)
    save(os.path.join(HERE, "shipped.npz"), c, {"s2000": d1, "s20000": d2})
    for n, kw in enumerate(TINY):
        c = W.tiny_case(**kw)
        c.params["bndry"] = list(c.params["bndry"])
        d, _ = harness.run_reference(c)
        save(os.path.join(HERE, f"tiny_{n}.npz"), c, {"end": d})
    c = W.hillslope200x50()
    c.params["bndry"] = list(c.params["bndry"])
    c600 = W.hillslope200x50()
    c600.params["bndry"] = list(c600.params["bndry"])
    c600.params["tend"] = 600.0
    dmid, _ = harness.run_reference(c600)
    dend, _ = harness.run_reference(c)
    save(os.path.join(HERE, "hillslope.npz"), c, {"t600": dmid, "end": dend})
    shipped_files(a.reference)


if __name__ == "__main__":
    main()
