"""FP64 GPU path vs the CPU oracle, through the C ABI (libswehr.so).

The plain FP64 form shares its elementary functions with the oracle's
project-math build and disables FP contraction, so every field must be
bit-identical (NaN positions included).  Against the reference itself
(golden fixtures from SWEHR.c with glibc libm) the only difference left is
libm's last-bit rounding; those tests assert the north-star bar of 1e-10
relative L-infinity where the reference's own floor allows it, and report
the measured value.
"""
import os

import numpy as np
import pytest

from harness import OracleRun, compare, load_golden, STATE_FIELDS, CLASS_FIELDS
from swehr_b200 import workloads as W

pytestmark = pytest.mark.gpu

ALL = STATE_FIELDS + CLASS_FIELDS + ("vel",)


def _sim(case, **kw):
    from swehr_b200.lib import Simulation
    return Simulation(case, **kw)


def _assert_bitexact(gpu: dict, orc: dict, names=ALL):
    res = compare(gpu, orc, names)
    bad = {k: v for k, v in res.items() if not v[2]}
    assert not bad, f"fields differ from the oracle: {bad}"


TINY = [
    dict(nx=12, ny=9, S=3, seed=5, bndry=(0, 1, 1, 1), inflow=0, rain_mmh=90.0, tend=60.0),
    dict(nx=15, ny=11, S=4, seed=6, bndry=(1, 0, 1, 1), inflow=1, rain_mmh=300.0, tend=120.0),
    dict(nx=15, ny=11, S=4, seed=7, bndry=(0, 0, 0, 0), inflow=0, rain_mmh=300.0, tend=120.0),
    dict(nx=9, ny=14, S=2, seed=8, bndry=(1, 1, 1, 1), inflow=1, rain_mmh=200.0, tend=90.0, per_cell_ks=False),
    dict(nx=20, ny=6, S=7, seed=9, bndry=(0, 1, 0, 1), inflow=0, rain_mmh=500.0, tend=150.0),
    dict(nx=33, ny=70, S=10, seed=10, bndry=(0, 1, 1, 0), inflow=0, rain_mmh=400.0, tend=100.0),
    dict(nx=2, ny=2, S=1, seed=11, bndry=(0, 0, 0, 0), inflow=0, rain_mmh=100.0, tend=30.0),
    dict(nx=40, ny=3, S=16, seed=12, bndry=(1, 1, 0, 1), inflow=1, rain_mmh=250.0, tend=80.0),
]


# cases whose inflow ghost (500 kg/m^3 per class) drives TOTSED past 0.2
# (debris forcing, SWEHR.c:1315-1316) and 0.4 (override, SWEHR.c:1392-1400)
DEBRIS = {1: ("dfmask", "debris"), 3: ("dfmask",), 7: ("dfmask", "debris")}


@pytest.mark.parametrize("kw", TINY, ids=[f"tiny{i}" for i in range(len(TINY))])
def test_tiny_bitexact(kw):
    c = W.tiny_case(**kw)
    o = OracleRun(c, "shim")
    o.advance()
    for branch in DEBRIS.get(TINY.index(kw), ()):
        assert o.counters()[branch] > 0, (branch, o.counters())
    with _sim(c) as g:
        pr = g.advance()
        assert pr.steps == o.steps
        assert pr.t == o.t
        _assert_bitexact(g.fields(), o.fields())
        st_g, sf_g = g.series()
        st_o, sf_o = o.series()
        assert st_g.shape == st_o.shape
        assert np.array_equal(st_g, st_o, equal_nan=True)
        assert np.array_equal(sf_g, sf_o, equal_nan=True)


def test_shipped_example_bitexact_and_reference():
    case, dumps = load_golden("shipped")
    o = OracleRun(case, "shim")
    with _sim(case) as g:
        for tag in ("s2000", "s20000"):
            n = dumps[tag]["steps"]
            g.advance(max_steps=n - g.advance(max_steps=0).steps)
            o.advance(max_steps=n - o.steps)
            gf = g.fields()
            _assert_bitexact(gf, o.fields())
            # reference: NaN positions identical (M's last row), values within the libm floor
            res = compare(gf, dumps[tag], ("h", "hu", "hv", "vinf", "U", "M", "z"))
            for name, (rel, same_nan, _) in res.items():
                assert same_nan, name
                assert rel < 1e-6, (tag, name, rel)


def test_hillslope_full_run_vs_reference():
    """200x50 hillslope, full 1200 s: bit-exact vs the oracle and within 1e-10
    of the reference on h, hu, hv, cumulative infiltration and per-class
    suspended / deposited mass."""
    case, dumps = load_golden("hillslope")
    o = OracleRun(case, "shim")
    with _sim(case, budget=True) as g:
        g.advance(t_stop=600.0)
        o.advance(t_stop=600.0)
        _assert_bitexact(g.fields(), o.fields())
        g.advance()
        o.advance()
        gf = g.fields()
        _assert_bitexact(gf, o.fields())
        res = compare(gf, dumps["end"], ("h", "hu", "hv", "vinf", "U", "M"))
        for name, (rel, same_nan, _) in res.items():
            assert same_nan and rel <= 1e-10, (name, rel)
        st_g, _ = g.series()
        assert st_g.shape[0] == dumps["end"]["stage"].shape[0]
        b = g.budget()
        scale = max(abs(b.water_now), abs(b.rain_in), 1e-300)
        assert abs(b.water_residual) <= 1e-9 * scale, (b.water_residual, scale)
        for k in range(case.sclass):
            sc = max(abs(b.sed_now[k]), abs(b.detach[k]), 1e-300)
            assert abs(b.sed_residual[k]) <= 1e-9 * sc, (k, b.sed_residual[k], sc)


def test_fractal_small_bitexact():
    c = W.fractal_domain(nx=96, ny=80, dx=2.0, steps=400)
    o = OracleRun(c, "shim")
    o.advance(max_steps=400)
    with _sim(c) as g:
        pr = g.advance(max_steps=400)
        assert pr.steps == 400
        _assert_bitexact(g.fields(), o.fields())


def test_storm_bitexact():
    c = W.storm_domain(nx=64, ny=48, dx=4.0, steps=300)
    c.params["storm_radius"] = 60.0
    c.params["storm_x0"] = 128.0
    c.params["storm_vy"] = 0.5
    c.params["storm_peak"] = 800 * W.MMH
    o = OracleRun(c, "shim")
    o.advance(max_steps=300)
    with _sim(c) as g:
        g.advance(max_steps=300)
        _assert_bitexact(g.fields(), o.fields())


def test_cfl_error_matches_oracle():
    c = W.tiny_case(nx=10, ny=10, S=2, seed=3, rain_mmh=500.0, tend=1000.0, cstable=40.0, maxstep=50.0)
    o = OracleRun(c, "shim")
    o.advance()
    assert o.status == 1
    with _sim(c) as g:
        pr = g.advance()
        assert pr.status == 1 and g.status == 1
        assert pr.steps == o.steps
        _assert_bitexact(g.fields(), o.fields())
        pr2 = g.advance()
        assert pr2.status == 1 and pr2.steps_this_call == 0


def test_pause_resume_does_not_change_trajectory():
    c = W.tiny_case(nx=16, ny=12, S=3, seed=21, rain_mmh=300.0, tend=60.0)
    with _sim(c) as a, _sim(c) as b:
        a.advance()
        for ts in (3.3, 10.0, 27.5, 41.0):
            b.advance(t_stop=ts)
        b.advance(max_steps=7)
        b.advance()
        _assert_bitexact(a.fields(), b.fields())


@pytest.mark.parametrize("name", ["failure_0", "failure_1", "failure_hillslope"])
def test_slope_failure_bitexact_and_reference(name):
    """Cross-sloped grids with the deposit cohesion lowered: slope failure
    (SWEHR.c:1292-1312) fires in many cells, 99 % of the deposit goes back
    into suspension and TOTM/DEP restart from zero (SWEHR.c:1497-1503).  The
    GPU takes the exact test wherever its no-failure bound cannot rule
    failure out, so it must match the oracle bit for bit; against the
    reference itself the libm floor applies (1e-10)."""
    case, dumps = load_golden(name)
    o = OracleRun(case, "shim")
    o.advance()
    assert o.counters()["fail"] > 0, o.counters()
    with _sim(case) as g:
        pr = g.advance()
        assert pr.steps == o.steps == dumps["end"]["steps"]
        gf = g.fields()
        _assert_bitexact(gf, o.fields())
        res = compare(gf, dumps["end"], ("h", "hu", "hv", "vinf", "U", "M"))
        for field, (rel, same_nan, _) in res.items():
            assert same_nan and rel <= 1e-10, (field, rel)


@pytest.mark.parametrize("name", ["solid_0", "solid_1", "solid_hillslope"])
def test_solid_cells_bitexact_and_reference(name):
    """Interior solid cells: the topography fill at creation, reflecting
    faces in both passes (including the j = ny face the reference tests
    against the next row's first cell), no sources and no water in solid
    cells -- bit for bit against the oracle, within the libm floor of the
    reference itself."""
    case, dumps = load_golden(name)
    o = OracleRun(case, "shim")
    o.advance()
    with _sim(case, budget=True) as g:
        pr = g.advance()
        assert pr.steps == o.steps == dumps["end"]["steps"]
        gf = g.fields()
        _assert_bitexact(gf, o.fields())
        res = compare(gf, dumps["end"], ("h", "hu", "hv", "vinf", "U", "M", "z"))
        for field, (rel, same_nan, _) in res.items():
            assert same_nan and rel <= 1e-10, (field, rel)
        b = g.budget()
        scale = max(abs(b.water_now), abs(b.rain_in), 1e-300)
        assert abs(b.water_residual) <= 1e-9 * scale, (b.water_residual, scale)


def test_solid_cells_mixed_and_pool():
    """The mixed form and the pool take the same solid-cell paths: the pooled
    FP64 run equals the single-domain run bit for bit, and the mixed form
    keeps solid cells dry."""
    from swehr_b200.lib import Pool
    case, _ = load_golden("solid_1")
    with _sim(case) as g:
        g.advance()
        alone = g.fields()
    with Pool(precision=0, max_classes=8, max_scenarios=4) as pool:
        sc = pool.submit(case)
        pool.run(-1)
        _assert_bitexact(sc.fields(), alone)
    with _sim(case, precision=1) as m:
        m.advance()
        f = m.fields()
        solid = case.solid.astype(bool)
        assert (f["h"][solid] == 0).all() and (f["U"][:, solid] == 0).all()
        assert np.isfinite(f["h"]).all()


def _mem_available_gb() -> float:
    """Host memory this process may still use: MemAvailable, capped by the
    container's cgroup limit (a container sees the whole host's meminfo)."""
    avail = 0.0
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                avail = int(line.split()[1]) / 2 ** 20
    except OSError:
        pass
    for path, used in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                       ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        try:
            lim = open(path).read().strip()
            if lim != "max":
                cur = int(open(used).read().strip()) if os.path.exists(used) else 0
                avail = min(avail, (int(lim) - cur) / 2 ** 30)
        except (OSError, ValueError):
            pass
    return avail


def test_roofline_domain_bitexact():
    """The 4096x4096 roofline domain (state planes of 134 MB, offsets past
    2^31 bytes) for 20 steps against the oracle (all host threads), field by
    field.  The oracle holds ~14 GB of host memory at this size; with less
    than 48 GB available to this process (cgroup limit included) the
    2048x2048 corner of the same domain runs instead, and with less than
    12 GB the 1024x1024 corner (said in the output)."""
    gb = _mem_available_gb()
    n = 4096 if gb >= 48 else (2048 if gb >= 12 else 1024)
    c = W.fractal_domain(nx=4096, ny=4096, dx=2.0, steps=20)
    if n != 4096:
        c = W.Case(c.name + "_corner", dict(c.params, nx=n, ny=n), c.topo[:n, :n].copy(), c.rain, c.ds, c.pfrac,
                   ks=c.ks[:n, :n].copy(), max_steps=20)
    print(f"roofline domain parity at {n}x{n}, 20 steps")
    o = OracleRun(c, "shim")
    o.advance(max_steps=20)
    with _sim(c) as g:
        pr = g.advance(max_steps=20)
        assert pr.steps == o.steps == 20 and pr.t == o.t
        for name in ("h", "hu", "hv", "z", "vinf", "totm", "dep", "totsed", "maxvel", "maxdepth", "vel"):
            a, b = g.field(name), o.field(name)
            assert np.array_equal(a, b, equal_nan=True), name
        for name in ("U", "M", "sed"):
            for k in range(1, c.sclass + 1):
                a, b = g.field(name, k), o.field(name, k)
                assert np.array_equal(a, b, equal_nan=True), (name, k)


# four of the smallest scenarios of the 256-scenario ensemble (sides 64-67),
# each run to the end of its event: 141 (427 s at 131 mm/h, 25 k steps, slope
# failure), 64 (1497 s at 43 mm/h, 42 k steps, failure and debris forcing),
# 97 (1704 s at 46 mm/h, 134 k steps, failure, debris forcing and the
# debris-flow override) and 187 (1053 s at 29 mm/h: all infiltrates, 4 k dry steps)
ENSEMBLE_TO_END = (141, 64, 97, 187)


def test_pool_ensemble_scenarios_to_event_end():
    """Config-2 scenarios stepped together in one pool until each event ends,
    against the oracle run alone: same step count and every field bit for
    bit.  These fractal catchments pond, erode, deposit and fail on their
    steep slopes well before their events end."""
    from swehr_b200.lib import Pool
    cases = W.ensemble(256, only=ENSEMBLE_TO_END)
    picked = [cases[k] for k in ENSEMBLE_TO_END]
    counts = []
    with Pool(precision=0, max_classes=8, max_scenarios=8) as pool:
        scs = [pool.submit(c) for c in picked]
        assert all(s is not None for s in scs)
        pool.run(-1)
        for k, (c, sc) in enumerate(zip(picked, scs)):
            pr = sc.progress()
            assert pr.done, k
            o = OracleRun(c, "shim")
            o.advance()
            assert o.steps == pr.steps and o.t == pr.t, (k, o.steps, pr.steps)
            _assert_bitexact(sc.fields(), o.fields())
            counts.append(o.counters())
    assert sum(c["fail"] > 0 for c in counts) >= 3 and sum(c["dfmask"] > 0 for c in counts) >= 2
    assert any(c["debris"] > 0 for c in counts)
