"""Field reads of large planes, which go through the pinned two-buffer
download (planes of 32 MB and more), and the derived fields computed on the
device (|v|, SED_k): a plane written with swehr_write_field must read back
unchanged (FP64) or as its FP32 rounding (mixed form), and |v| and SED_k must
equal the same expressions evaluated by numpy on the read-back state."""
import numpy as np
import pytest

from swehr_b200 import workloads as W
from swehr_b200.params import FP64, MIXED

pytestmark = pytest.mark.gpu

# 2048^2 doubles and 2900^2 floats are both above the 32 MB staging threshold
SIDES = {FP64: (2048, 2080), MIXED: (2900, 2912)}


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_large_plane_roundtrip_and_derived(precision):
    from swehr_b200.lib import Simulation
    nx, ny = SIDES[precision]
    case = W.fractal_domain(nx=nx, ny=ny, dx=2.0, seed=3, steps=10)
    rng = np.random.default_rng(11)
    hfilm = 1e-5
    with Simulation(case, precision=precision) as s:
        s.advance(max_steps=2)
        h = rng.uniform(0.0, 0.05, (nx, ny))
        h[rng.random((nx, ny)) < 0.2] = 0.5 * hfilm        # dry cells
        hu = rng.normal(0.0, 0.01, (nx, ny))
        hv = rng.normal(0.0, 0.01, (nx, ny))
        u1 = rng.normal(0.0, 1e-4, (nx, ny))
        for name, a, k in (("h", h, 0), ("hu", hu, 0), ("hv", hv, 0), ("U", u1, 1)):
            s.write_field(name, a, k)
        got = {n: s.field(n) for n in ("h", "hu", "hv", "vel")}
        got["U"] = s.field("U", 1)
        got["sed"] = s.field("sed", 1)
    if precision == FP64:
        want = {"h": h, "hu": hu, "hv": hv, "U": u1}
    else:
        want = {n: a.astype(np.float32).astype(np.float64) for n, a in (("h", h), ("hu", hu), ("hv", hv), ("U", u1))}
    for n in ("h", "hu", "hv", "U"):
        assert np.array_equal(got[n], want[n]), n
    hh = got["h"]
    wet = hh > hfilm
    with np.errstate(divide="ignore", invalid="ignore"):
        v1 = np.where(wet, got["hu"] / hh, 0.0)
        v2 = np.where(wet, got["hv"] / hh, 0.0)
        vel = np.sqrt(v1 * v1 + v2 * v2)
        sed = np.where(wet, got["U"] / hh, 0.0)
    sed = np.where(wet & (sed < -1e-5), 0.0, sed)
    assert np.array_equal(got["vel"], vel)
    assert np.array_equal(got["sed"], sed)
    assert wet.any() and (~wet).any()
