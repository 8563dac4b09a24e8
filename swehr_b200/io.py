"""The reference's file formats.

Inputs (read by SWEHR.c from the working directory, SWEHR.c:468-522, 218-227):
  input.txt               14 numbers: nx ny dx F manning0 tend a ad h0 mtstar0 rnum rint sclass J
  rain.txt                rnum rain rates [m/s]
  topoin.txt              nx*ny elevations, i-major
  particlesizein.txt      sclass diameters
  particlepercentin.txt   sclass fractions
Outputs (SWEHR.c:1705-1761): one row per j, nx values per row, "%10.10lf"
separated by tabs; stage.txt / saveflow.txt rows of "%lf".

Everything here is written with "%.17g" so a reader gets the exact doubles.
"""
from __future__ import annotations

import os

import numpy as np

from .params import INPUT_TXT_ORDER

OUTPUT_FILES = {
    "topoout.txt": "z", "depth.txt": "h", "uh.txt": "hu", "vh.txt": "hv", "ch.txt": "U1",
    "m.txt": "totm", "c.txt": "totsed", "vel.txt": "vel", "maxvel.txt": "maxvel",
    "maxdepth.txt": "maxdepth",
}


def _fmt(v) -> str:
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v))


def write_inputs(case, directory: str) -> None:
    """Write the five reference input files (and ks.txt when Ks varies per cell)."""
    os.makedirs(directory, exist_ok=True)
    p = case.params
    vals = [p[k] for k in INPUT_TXT_ORDER]
    with open(os.path.join(directory, "input.txt"), "w") as f:
        f.write("\t".join(_fmt(v) for v in vals) + "\n")
    with open(os.path.join(directory, "rain.txt"), "w") as f:
        f.write("\t".join(repr(float(v)) for v in case.rain) + "\n")
    with open(os.path.join(directory, "particlesizein.txt"), "w") as f:
        f.write("\n".join(repr(float(v)) for v in case.ds) + "\n")
    with open(os.path.join(directory, "particlepercentin.txt"), "w") as f:
        f.write("\n".join(repr(float(v)) for v in case.pfrac) + "\n")
    np.savetxt(os.path.join(directory, "topoin.txt"), case.topo.reshape(-1), fmt="%.17g")
    if case.ks is not None:
        np.savetxt(os.path.join(directory, "ks.txt"), case.ks.reshape(-1), fmt="%.17g")
    if getattr(case, "solid", None) is not None:
        np.savetxt(os.path.join(directory, "solid.txt"), case.solid.reshape(-1).astype(np.int64), fmt="%d")


def write_ref_cfg(case, directory: str, max_steps: int = -1, movies: int = 0) -> None:
    """Run-time switches understood by the patched reference (oracle/build_ref.py)."""
    p = case.params
    b = p.get("bndry", (1, 0, 1, 1))
    lines = [
        f"bndry1 {b[0]}", f"bndry2 {b[1]}", f"bndry3 {b[2]}", f"bndry4 {b[3]}",
        f"inflow {p.get('inflow', 1)}", f"maxsteps {max_steps}", f"movies {movies}",
        f"roughness {p.get('roughness', 0.1)!r}", f"ks {p.get('ks', 0.0)!r}",
        f"ksfile {1 if case.ks is not None else 0}",
        f"theta0 {p.get('theta0', 0.05)!r}", f"thetas {p.get('thetas', 0.4)!r}",
        f"hf {p.get('hf', 0.001)!r}", f"vinf0 {p.get('vinf0', 1e-4)!r}",
        f"uc {p.get('uc', 0.0)!r}", f"uc2 {p.get('uc2', 0.0)!r}",
        f"cohesion {p.get('cohesion', 400.0)!r}",
        f"solidfile {1 if getattr(case, 'solid', None) is not None else 0}",
    ]
    with open(os.path.join(directory, "swehr_ref.cfg"), "w") as f:
        f.write("\n".join(lines) + "\n")


def read_inputs(directory: str):
    """Parse the five reference input files from a directory into a Case."""
    from .workloads import Case
    with open(os.path.join(directory, "input.txt")) as f:
        vals = [float(v) for v in f.read().split()[:14]]
    p = dict(zip(INPUT_TXT_ORDER, vals))
    for k in ("nx", "ny", "rnum", "sclass"):
        p[k] = int(p[k])
    with open(os.path.join(directory, "rain.txt")) as f:
        rain = np.array([float(v) for v in f.read().split()[: p["rnum"]]])
    with open(os.path.join(directory, "particlesizein.txt")) as f:
        ds = np.array([float(v) for v in f.read().split()[: p["sclass"]]])
    with open(os.path.join(directory, "particlepercentin.txt")) as f:
        pf = np.array([float(v) for v in f.read().split()[: p["sclass"]]])
    with open(os.path.join(directory, "topoin.txt")) as f:
        topo = np.array([float(v) for v in f.read().split()[: p["nx"] * p["ny"]]]).reshape(p["nx"], p["ny"])
    return Case("files", p, topo, rain, ds, pf)


def read_ref_dump(path: str) -> dict:
    """Parse swehr_dump.txt written by the patched reference (%.17g)."""
    with open(path) as f:
        head = f.readline().split()
        nx, ny, S, steps = int(head[0]), int(head[1]), int(head[2]), int(head[3])
        t = float(head[4])
        data = np.array([float(v) for v in f.read().split()])
    N = nx * ny
    out = {"nx": nx, "ny": ny, "S": S, "steps": steps, "t": t}
    names = ["h", "hu", "hv", "z", "vinf", "totm", "dep", "totsed", "maxvel", "maxdepth"]
    pos = 0
    for n in names:
        out[n] = data[pos:pos + N].reshape(nx, ny)
        pos += N
    for group in ("U", "M", "sed"):
        out[group] = data[pos:pos + S * N].reshape(S, nx, ny)
        pos += S * N
    cnt = int(data[pos])
    pos += 1
    out["stage"] = data[pos:pos + cnt * 24].reshape(cnt, 24)
    pos += cnt * 24
    out["saveflow"] = data[pos:pos + cnt * 18].reshape(cnt, 18)
    return out


def write_outputs(fields: dict, directory: str, nx: int, ny: int) -> None:
    """Final output files in the reference's layout: row j, columns i, %10.10lf."""
    os.makedirs(directory, exist_ok=True)
    for fname, key in OUTPUT_FILES.items():
        a = fields[key]
        with open(os.path.join(directory, fname), "w") as f:
            for j in range(ny):
                f.write("\t".join("%10.10f" % a[i, j] for i in range(nx)) + "\n")
