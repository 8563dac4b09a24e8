"""Seeded synthetic SWEHR workloads.

No public dataset is involved: every domain is generated here from numpy's
default_rng(seed), so the CPU oracle, the reference program (through the
text files written by swehr_b200.io) and the GPU read identical bits.

  hillslope200x50()  200x50 planar hillslope, 10 % slope + 5 mm roughness,
                     60 mm/h for 600 s then dry, 7 classes (the CPU-runnable case)
  fractal_domain()   diamond-square catchment tilted toward i=1, uniform rain
                     from a seeded hyetograph, lognormal per-cell Ks
                     (4096x4096, dx=2, 2000 steps is the roofline workload)
  ensemble()         256 square catchments of side 64-1024 (log-uniform)
  storm_domain()     8192x8192 fractal domain with a moving Gaussian storm
  tiny_case()        small random grids for parity tests
  failure_tiny(), failure_hillslope()
                     cross-sloped grids with the deposit cohesion lowered,
                     so the slope-failure branch fires
  solid_tiny(), solid_hillslope()
                     grids with interior solid cells (blocks, a wall, a
                     cell in the first column whose mask the last column's
                     y-face test reads)
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

from .params import make_params, SwehrParams

MMH = 1.0 / 3.6e6          # 1 mm/h in m/s


@dataclasses.dataclass
class Case:
    name: str
    params: dict                      # keyword arguments for make_params
    topo: np.ndarray                  # (nx, ny) float64, i-major
    rain: np.ndarray                  # (rnum,) m/s
    ds: np.ndarray                    # (S,) m
    pfrac: np.ndarray                 # (S,)
    ks: Optional[np.ndarray] = None   # (nx, ny) m/s or None
    max_steps: int = -1               # -1: run to tend
    solid: Optional[np.ndarray] = None  # (nx, ny) int32 interior solid mask or None

    @property
    def nx(self):
        return int(self.params["nx"])

    @property
    def ny(self):
        return int(self.params["ny"])

    @property
    def sclass(self):
        return int(self.params["sclass"])

    def make_params(self) -> SwehrParams:
        return make_params(**self.params)

    def cells(self) -> int:
        return self.nx * self.ny


def seven_classes(seed: int = 0):
    """7 diameters log-spaced 2 um .. 2 mm and Dirichlet(alpha=2) fractions."""
    ds = 2e-6 * 1000.0 ** (np.arange(7) / 6.0)
    pf = np.random.default_rng(seed).dirichlet([2.0] * 7)
    return ds, pf


def common_soil(**over):
    """Hillslope soil / erosion parameters shared by the synthetic cases."""
    d = dict(F=0.01, manning0=0.03, a=200.0, ad=2000.0, h0=0.00099, mtstar0=3.0, J=30.0,
             roughness=0.03, ks=5 * MMH, hf=0.11, theta0=0.1, thetas=0.4, uc=0.2, uc2=0.2,
             bndry=(0, 1, 1, 1), inflow=0)
    d.update(over)
    return d


def hillslope200x50(nx: int = 200, ny: int = 50, seed: int = 0) -> Case:
    """200x50 cells, dx=1 m, z = 0.1 x + N(0, 5 mm), outflow at i=1 (x=0),
    walls elsewhere, dry bed, 60 mm/h for 600 s then 0 for 600 s."""
    rng = np.random.default_rng(seed)
    dx = 1.0
    x = (np.arange(1, nx + 1) - 1) * dx
    topo = 0.1 * x[:, None] + rng.normal(0.0, 0.005, size=(nx, ny))
    ds, pf = seven_classes(seed)
    rain = np.array([60 * MMH, 0.0])
    params = common_soil(nx=nx, ny=ny, dx=dx, tend=1200.0, rnum=2, rint=600.0, sclass=7)
    return Case("hillslope200x50", params, topo.astype(np.float64), rain, ds, pf)


def diamond_square(n: int, hurst: float, seed: int) -> np.ndarray:
    """(2^n+1)^2 fractal surface by the diamond-square algorithm (Fournier,
    Fussell & Carpenter 1982); amplitude shrinks by 2^-H per level."""
    size = 2 ** n + 1
    rng = np.random.default_rng(seed)
    z = np.zeros((size, size))
    z[0, 0], z[0, -1], z[-1, 0], z[-1, -1] = rng.normal(size=4)
    step = size - 1
    scale = 1.0
    while step > 1:
        half = step // 2
        c = (z[0:-1:step, 0:-1:step] + z[step::step, 0:-1:step]
             + z[0:-1:step, step::step] + z[step::step, step::step])
        z[half::step, half::step] = c * 0.25 + scale * rng.normal(size=c.shape)
        for r0, c0 in ((half, 0), (0, half)):
            rr = np.arange(r0, size, step)
            cc = np.arange(c0, size, step)
            acc = np.zeros((rr.size, cc.size))
            cnt = np.zeros((rr.size, cc.size))
            for dr, dc in ((-half, 0), (half, 0), (0, -half), (0, half)):
                r2 = rr + dr
                c2 = cc + dc
                vr = (r2 >= 0) & (r2 < size)
                vc = (c2 >= 0) & (c2 < size)
                sub = np.zeros((rr.size, cc.size))
                sub[np.ix_(vr, vc)] = z[np.ix_(r2[vr], c2[vc])]
                acc += sub
                cnt += np.outer(vr, vc)
            z[np.ix_(rr, cc)] = acc / cnt + scale * rng.normal(size=acc.shape)
        scale *= 2.0 ** (-hurst)
        step = half
    return z


def fractal_topo(nx: int, ny: int, dx: float, hurst: float, relief: float, tilt: float, seed: int):
    n = max(1, math.ceil(math.log2(max(nx, ny) - 1 if max(nx, ny) > 2 else 2)))
    z = diamond_square(n, hurst, seed)[:nx, :ny]
    z = (z - z.min()) / max(z.max() - z.min(), 1e-300) * relief
    x = (np.arange(1, nx + 1) - 1) * dx
    return z + tilt * x[:, None]


def fractal_domain(nx: int = 4096, ny: int = 4096, dx: float = 2.0, seed: int = 1,
                   steps: int = 2000, hurst: float = 0.8, relief: float = 40.0) -> Case:
    """Diamond-square (Hurst 0.8, 40 m relief) tilted 3 % toward i=1,
    30-entry hyetograph U(0,120) mm/h with rint = 60 s, Ks lognormal
    (median 5 mm/h, sigma_ln 0.5), 7 classes, outflow at i=1."""
    rng = np.random.default_rng(seed)
    topo = fractal_topo(nx, ny, dx, hurst, relief, 0.03, seed)
    rain = rng.uniform(0.0, 120.0, size=30) * MMH
    ks = (5 * MMH) * np.exp(0.5 * rng.standard_normal(size=(nx, ny)))
    ds, pf = seven_classes(0)
    params = common_soil(nx=nx, ny=ny, dx=dx, tend=1.0e9, rnum=30, rint=60.0, sclass=7)
    return Case(f"fractal{nx}x{ny}", params, topo, rain, ds, pf, ks=ks, max_steps=steps)


def ensemble(count: int = 256, seed: int = 2, side_min: int = 64, side_max: int = 1024, only=None):
    """Independent square catchments for batched runs: sides log-uniform,
    dx = 1 m, per-scenario fractal seeds, rain U(20,150) mm/h for U(300,1800) s,
    Manning n U(0.02, 0.08), 7 classes; each runs to the end of its event.
    only: indices whose topography is generated (the others are None in the
    returned list; their parameters are drawn all the same)."""
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(math.log(side_min), math.log(side_max), size=count)).astype(int)
    cases = []
    ds, pf = seven_classes(0)
    for s in range(count):
        side = int(sides[s])
        intensity = rng.uniform(20.0, 150.0) * MMH
        duration = float(rng.uniform(300.0, 1800.0))
        n = float(rng.uniform(0.02, 0.08))
        if only is not None and s not in only:
            cases.append(None)
            continue
        topo = fractal_topo(side, side, 1.0, 0.8, 40.0, 0.03, 1000 + s)
        params = common_soil(nx=side, ny=side, dx=1.0, tend=duration, rnum=1, rint=duration,
                             sclass=7, roughness=n, manning0=n)
        cases.append(Case(f"ensemble{s}", params, topo, np.array([intensity]), ds, pf))
    return cases


def storm_domain(nx: int = 8192, ny: int = 8192, dx: float = 1.0, seed: int = 4, steps: int = 5000) -> Case:
    """Fractal (Hurst 0.7, 60 m relief), 10 classes log-spaced 1 um..4 mm, Ks
    lognormal (median 10 mm/h, sigma_ln 0.8), moving Gaussian storm with a
    200 mm/h peak, 1 km radius, 2 m/s along +y."""
    rng = np.random.default_rng(seed)
    topo = fractal_topo(nx, ny, dx, 0.7, 60.0, 0.03, seed)
    ks = (10 * MMH) * np.exp(0.8 * rng.standard_normal(size=(nx, ny)))
    ds = 1e-6 * 4000.0 ** (np.arange(10) / 9.0)
    pf = rng.dirichlet([2.0] * 10)
    params = common_soil(nx=nx, ny=ny, dx=dx, tend=1.0e9, rnum=1, rint=1.0e9, sclass=10,
                         ks=10 * MMH, storm_peak=200 * MMH, storm_radius=1000.0,
                         storm_x0=nx * dx / 2, storm_y0=0.0, storm_vx=0.0, storm_vy=2.0)
    return Case(f"storm{nx}x{ny}", params, topo, np.array([0.0]), ds, pf, ks=ks, max_steps=steps)


def tiny_case(nx: int = 12, ny: int = 9, S: int = 3, seed: int = 5, bndry=(0, 1, 1, 1), inflow: int = 0,
              rain_mmh: float = 90.0, tend: float = 60.0, per_cell_ks: bool = True, **over) -> Case:
    """Small random hillslope for fast parity checks."""
    rng = np.random.default_rng(seed)
    dx = 0.5
    x = (np.arange(1, nx + 1) - 1) * dx
    topo = 0.08 * x[:, None] + rng.normal(0.0, 0.01, size=(nx, ny))
    ds = 2e-5 * 50.0 ** (np.arange(S) / max(S - 1, 1))
    pf = rng.dirichlet([2.0] * S)
    rain = np.array([rain_mmh * MMH, 0.5 * rain_mmh * MMH, 0.0])
    ks = (5 * MMH) * np.exp(0.5 * rng.standard_normal(size=(nx, ny))) if per_cell_ks else None
    params = common_soil(nx=nx, ny=ny, dx=dx, tend=tend, rnum=3, rint=tend / 3, sclass=S,
                         bndry=tuple(bndry), inflow=inflow)
    params.update(over)
    return Case(f"tiny{nx}x{ny}s{S}", params, topo, rain, ds, pf, ks=ks)


def failure_tiny(slope_y: float = 0.5, cohesion: float = 5.0, **kw) -> Case:
    """tiny_case tilted across the slope (z += slope_y * y) with the deposit
    cohesion lowered from the reference's 400 Pa: the slope-failure test
    (SWEHR.c:1292-1312) then fires in many cells and moves deposited mass
    back into suspension (SWEHR.c:1497-1503)."""
    c = tiny_case(**kw)
    y = (np.arange(1, c.ny + 1) - 1) * float(c.params["dx"])
    c.topo = c.topo + slope_y * y[None, :]
    c.params["cohesion"] = cohesion
    c.name = f"failure{c.nx}x{c.ny}s{c.sclass}"
    return c


def failure_hillslope(cross: float = 0.4, cohesion: float = 20.0, tend: float = 600.0) -> Case:
    """The 200x50 hillslope with a cross slope (z += cross * y), cohesion
    lowered to `cohesion` Pa, run to `tend`: slope failure in ~1.5 % of the
    cell-steps, deposits and resuspension over the whole event."""
    c = hillslope200x50()
    y = (np.arange(1, c.ny + 1) - 1) * float(c.params["dx"])
    c.topo = c.topo + cross * y[None, :]
    c.params["cohesion"] = cohesion
    c.params["tend"] = tend
    c.name = "failure_hillslope200x50"
    return c


def solid_tiny(nx: int = 20, ny: int = 16, S: int = 4, seed: int = 51, **kw) -> Case:
    """tiny_case with interior solid cells: a 4x4 block, a one-cell-wide wall
    with a gap, and the cell (3, 1) -- the reference's y-face test at j = ny
    reads SOLID[i][ny+1], which is SOLID[i+1][1] (SWEHR.c:1206,1211), so
    cell (2, ny) gets a reflecting top face from it."""
    c = tiny_case(nx=nx, ny=ny, S=S, seed=seed, **kw)
    m = np.zeros((nx, ny), dtype=np.int32)
    m[5:9, 4:8] = 1
    m[12, 2:ny - 3] = 1
    m[12, ny // 2] = 0
    m[2, 0] = 1
    c.solid = m
    c.name = f"solid{nx}x{ny}s{S}"
    return c


def solid_hillslope(tend: float = 600.0) -> Case:
    """The 200x50 hillslope with three rectangular buildings and a wall
    across part of the slope, run to `tend`."""
    c = hillslope200x50()
    m = np.zeros((c.nx, c.ny), dtype=np.int32)
    m[40:52, 10:18] = 1
    m[90:96, 30:44] = 1
    m[150:170, 5:9] = 1
    m[120, 0:35] = 1
    c.solid = m
    c.params["tend"] = tend
    c.name = "solid_hillslope200x50"
    return c
