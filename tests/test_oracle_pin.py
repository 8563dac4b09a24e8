"""Pin the CPU oracle to the reference (CPU only).

The oracle's glibc build must reproduce the reference program bit-for-bit:
against the committed golden fixtures (outputs of SWEHR.c itself, see
tests/golden/make_golden.py), and -- when the reference program is built in
oracle/_ref -- against live runs on fresh random cases.  The project-math
build (the GPU's twin) is then within the libm floor of the glibc build.
"""
import numpy as np
import pytest

from harness import OracleRun, compare, load_golden, run_reference, have_reference_binary, STATE_FIELDS, CLASS_FIELDS
from swehr_b200 import workloads as W

FIELDS = STATE_FIELDS + CLASS_FIELDS


def _bitexact(a, b, names=FIELDS):
    res = compare(a, b, names)
    return {k: v for k, v in res.items() if not v[2]}


# the inflow cases carry the hard-wired 500 kg/m^3 ghost concentration of
# every class into the domain: TOTSED passes 0.2 (debris forcing, SWEHR.c:
# 1315-1316) and 0.4 (the debris-flow override, SWEHR.c:1392-1400)
DEBRIS_TINY = {1: ("dfmask", "debris"), 3: ("dfmask",)}


@pytest.mark.parametrize("n", range(5))
def test_glibc_oracle_matches_reference_tiny(n):
    case, dumps = load_golden(f"tiny_{n}")
    o = OracleRun(case, "glibc")
    o.advance()
    d = dumps["end"]
    assert o.steps == d["steps"] and o.t == d["t"]
    assert not _bitexact(o.fields(), d)
    for branch in DEBRIS_TINY.get(n, ()):
        assert o.counters()[branch] > 0, (n, branch, o.counters())
    st, sf = o.series()
    assert np.array_equal(st, d["stage"], equal_nan=True)
    # the reference clamps its sample points into the grid; compare the points that are inside
    assert st.shape[0] == d["saveflow"].shape[0]


@pytest.mark.parametrize("name", ["failure_0", "failure_1", "failure_hillslope"])
def test_glibc_oracle_matches_reference_slope_failure(name):
    """Cross-sloped grids with the deposit cohesion lowered: the slope
    failure test fires (SWEHR.c:1292-1312) and the class loop moves 99 % of
    the deposit into suspension and zeroes TOTM and DEP (SWEHR.c:1497-1503);
    the oracle still matches the reference bit for bit."""
    case, dumps = load_golden(name)
    o = OracleRun(case, "glibc")
    o.advance()
    d = dumps["end"]
    assert o.steps == d["steps"] and o.t == d["t"]
    assert not _bitexact(o.fields(), d)
    n = o.counters()
    assert n["fail"] > 0, n
    st, _ = o.series()
    assert np.array_equal(st, d["stage"], equal_nan=True)


@pytest.mark.parametrize("name", ["solid_0", "solid_1", "solid_hillslope"])
def test_glibc_oracle_matches_reference_solid_cells(name):
    """Interior solid cells (a SOLID mask the patched reference reads from
    solid.txt): the topography fill (SWEHR.c:288-322), reflecting faces
    (SWEHR.c:1137-1146, 1205-1214, including the y-face test's read of the
    next row's first cell at j = ny) and the source skip (SWEHR.c:1233)."""
    case, dumps = load_golden(name)
    assert case.solid is not None and case.solid.any()
    o = OracleRun(case, "glibc")
    o.advance()
    d = dumps["end"]
    assert o.steps == d["steps"] and o.t == d["t"]
    f = o.fields()
    assert not _bitexact(f, d)
    m = case.solid.astype(bool)
    assert (f["h"][m] == 0).all() and (f["U"][:, m] == 0).all()


def test_glibc_oracle_matches_reference_shipped_example():
    case, dumps = load_golden("shipped")
    o = OracleRun(case, "glibc")
    for tag in ("s2000", "s20000"):
        d = dumps[tag]
        o.advance(max_steps=d["steps"] - o.steps)
        f = o.fields()
        assert not _bitexact(f, d), tag
        # the reference's 0/0 in the inflow ghost at t=0 leaves NaN in the last row of M
        assert np.isnan(f["M"][0, :, -1]).all() and not np.isnan(f["M"][0, :, :-1]).any()


@pytest.mark.slow
def test_glibc_oracle_matches_reference_hillslope():
    case, dumps = load_golden("hillslope")
    half = W.Case(case.name, dict(case.params, tend=600.0), case.topo, case.rain, case.ds, case.pfrac)
    o = OracleRun(half, "glibc")     # the 600 s fixture ran with tend = 600 (last dt clamped to it)
    o.advance()
    mid = dumps["t600"]
    assert o.steps == mid["steps"]
    assert not _bitexact(o.fields(), mid)
    o = OracleRun(case, "glibc")
    o.advance()
    end = dumps["end"]
    assert o.steps == end["steps"] and o.t == end["t"]
    assert not _bitexact(o.fields(), end)
    st, _ = o.series()
    assert np.array_equal(st, end["stage"], equal_nan=True)


def test_shim_oracle_within_libm_floor_of_reference():
    """The project-math build differs from glibc only by last-bit rounding of
    the elementary functions: identical step counts, small field drift."""
    case, dumps = load_golden("tiny_1")
    o = OracleRun(case, "shim")
    o.advance()
    d = dumps["end"]
    assert o.steps == d["steps"]
    res = compare(o.fields(), d, ("h", "hu", "hv", "vinf", "U", "M"))
    for name, (rel, same_nan, _) in res.items():
        assert same_nan and rel < 1e-8, (name, rel)


@pytest.mark.skipif(not have_reference_binary(), reason="reference program not built (oracle/build_ref.py)")
@pytest.mark.parametrize("seed", [31, 32, 33])
def test_glibc_oracle_matches_live_reference(seed):
    rng = np.random.default_rng(seed)
    bndry = tuple(int(b) for b in rng.integers(0, 2, size=4))
    case = W.tiny_case(nx=int(rng.integers(3, 20)), ny=int(rng.integers(3, 20)), S=int(rng.integers(1, 8)),
                       seed=seed, bndry=bndry, inflow=int(rng.integers(0, 2)), rain_mmh=float(rng.uniform(50, 600)),
                       tend=60.0)
    d, _ = run_reference(case)
    o = OracleRun(case, "glibc")
    o.advance()
    assert o.steps == d["steps"]
    assert not _bitexact(o.fields(), d)
