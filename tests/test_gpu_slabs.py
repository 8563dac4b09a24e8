"""One domain split into row slabs on the GPU (swehr_slab_*, SlabDomain):
every slab updates only its own rows, reads two rows of each neighbour,
takes the largest wave speed over all slabs for the time step, and has its
halo rows refreshed after every step.  The slabs' own rows must equal the
whole domain run by swehr_create / swehr_advance bit for bit, in both forms
-- the same evidence the CPU test (test_slab_split.py) gives for the
oracle, now for the kernels (SWEHR.c:1135, 1243-1312, 1408)."""
import numpy as np
import pytest

from swehr_b200 import workloads as W
from swehr_b200.lib import Simulation, SlabDomain
from swehr_b200.params import FP64, MIXED

pytestmark = pytest.mark.gpu

NAMES = ("h", "hu", "hv", "z", "vinf", "totm", "dep", "totsed", "maxvel", "maxdepth", "U", "M")


def _compare(case, slabs, steps, precision):
    with Simulation(case, precision=precision) as whole:
        pw = whole.advance(max_steps=steps)
        ref = whole.fields(NAMES)
    with SlabDomain(case, slabs, precision) as split:
        split.step(steps)
        ps = split.progress()
        got = split.fields(NAMES)
    assert ps.steps == pw.steps == steps
    assert ps.t == pw.t and ps.dt == pw.dt
    bad = [n for n in NAMES if not np.array_equal(got[n], ref[n], equal_nan=True)]
    assert not bad, (case.name, slabs, bad)
    return ref


@pytest.mark.parametrize("slabs", [2, 3])
def test_slabs_match_whole_domain_with_failure_and_inflow(slabs):
    # slope failure, inflow at j = ny, per-cell Ks, walls on three sides: every
    # branch of the step crosses the slab seams
    case = W.failure_tiny(slope_y=0.5, cohesion=5.0, nx=26, ny=14, S=3, seed=71, bndry=(0, 1, 1, 1), inflow=1,
                          rain_mmh=300.0, tend=1.0e6)
    ref = _compare(case, slabs, 600, FP64)
    assert np.nanmax(ref["h"]) > 1e-3          # the run ponds: the seams carry flow


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_slabs_match_whole_fractal_domain(precision):
    case = W.fractal_domain(nx=64, ny=48, dx=2.0, seed=1, steps=400)
    _compare(case, 4, 400, precision)


def test_slabs_match_whole_domain_under_a_moving_storm():
    # the storm's rain depends on each cell's global row (the slab's row offset)
    case = W.storm_domain(nx=48, ny=40, dx=1.0, seed=4, steps=200)
    _compare(case, 3, 200, FP64)


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_two_row_slabs(precision):
    # the thinnest split: every slab owns two rows, so each halo is a whole
    # neighbour slab, and the first and last slabs hold the domain's boundary rows
    case = W.tiny_case(nx=8, ny=9, S=3, seed=5, bndry=(0, 1, 1, 1), inflow=1, rain_mmh=300.0, tend=60.0)
    _compare(case, 4, 150, precision)
