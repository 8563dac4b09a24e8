"""Serving on the GPU: a Poisson stream of uneven requests through the
continuous-batching loop, with an HBM limit small enough that requests wait
for memory, then every result compared with the same request run alone.

Mixed form: alone = the request alone in a pool, and results must be
bit-identical (the per-cell arithmetic never depends on the batch).  Plain
FP64: alone = swehr_create / swehr_advance, also bit-identical."""
import numpy as np
import pytest

from harness import compare
from swehr_b200 import serving as SV
from swehr_b200.params import FP64, MIXED

pytestmark = pytest.mark.gpu

FIELDS = ("h", "hu", "hv", "totsed", "vinf", "U", "M")


def _stream():
    reqs = SV.poisson_stream(rate=25.0, duration=1.0, seed=21, side_min=16, side_max=96, step_len=(2.0, 6.0),
                             hyeto_steps=(1, 3))
    SV.prepare(reqs)
    return reqs


def _bitequal(a, b):
    res = compare(a, b, FIELDS)
    return {k: v for k, v in res.items() if not v[2]}


@pytest.mark.parametrize("precision", [MIXED, FP64], ids=["mixed", "fp64"])
def test_serving_results_same_alone_and_in_mix(precision):
    from swehr_b200.lib import Pool, Simulation
    reqs = _stream()
    assert len(reqs) >= 10
    srv = SV.Server(precision=precision, hbm_limit=48 * 2 ** 20, max_classes=16, chunk_steps=16,
                    result_fields=FIELDS)
    rep = srv.serve(reqs, time_limit=600.0)
    assert rep.completed == len(reqs), rep.summary()
    assert rep.max_resident > 1                     # requests overlapped on the GPU
    assert rep.peak_hbm_bytes <= rep.hbm_limit
    assert rep.p99_s >= rep.p50_s > 0
    byid = {r.rid: r for r in rep.results}
    for r in reqs:
        got = byid[r.rid]
        assert got.status == 0
        if precision == MIXED:
            with Pool(precision=MIXED, max_classes=16) as pool:
                sc = pool.submit(r.case)
                pool.run(-1)
                pr = sc.progress()
                ref = sc.fields(FIELDS)
        else:
            with Simulation(r.case, precision=FP64) as s:
                pr = s.advance()
                ref = s.fields(FIELDS)
        assert got.steps == pr.steps, (r.rid, got.steps, pr.steps)
        bad = _bitequal(got.fields, ref)
        assert not bad, (r.rid, bad)
