"""Writing the topography through swehr_write_field before stepping gives the
same run as creating the simulation with it: the lagged GZ the wave pass
reads (computed one step ahead by the update) is rebuilt from the written
topography."""
import copy

import numpy as np
import pytest

from harness import compare
from swehr_b200 import workloads as W
from swehr_b200.params import FP64, MIXED

pytestmark = pytest.mark.gpu

FIELDS = ("h", "hu", "hv", "z", "vinf", "totsed", "U", "M")


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_written_topography_equals_created(precision):
    from swehr_b200.lib import Simulation
    a = W.tiny_case(nx=40, ny=30, S=4, seed=41, bndry=(0, 1, 1, 1), inflow=0, rain_mmh=120.0, tend=60.0)
    other = copy.deepcopy(a)                               # same case on another topography
    other.topo = a.topo + np.random.default_rng(3).normal(0.0, 0.05, a.topo.shape)
    with Simulation(a, precision=precision) as sa:
        pa = sa.advance()
        fa = sa.fields(FIELDS)
    with Simulation(other, precision=precision) as sc:
        sc.write_field("z", a.topo)
        pc = sc.advance()
        fc = sc.fields(FIELDS)
    assert pa.steps == pc.steps
    bad = {k: v for k, v in compare(fa, fc, FIELDS).items() if not v[2]}
    assert not bad, bad
