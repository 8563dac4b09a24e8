"""Error measures used to report the mixed form's accuracy (CPU only)."""
import numpy as np

from swehr_b200 import workloads as W
import pytest

from swehr_b200.accuracy import KEEP64, EmptyField, quantized_case, rel_linf


def test_rel_linf():
    b = np.array([[1.0, -4.0], [np.nan, 2.0]])
    a = b.copy()
    assert rel_linf(a, b) == 0.0
    a[0, 0] += 0.4
    assert abs(rel_linf(a, b) - 0.1) < 1e-15
    a[1, 1] = np.nan
    assert rel_linf(a, b) == float("inf")
    assert rel_linf(np.zeros(3), np.zeros(3)) == 0.0
    # an empty reference field cannot pass for an accuracy result
    with pytest.raises(EmptyField):
        rel_linf(np.zeros(3), np.zeros(3), require_nonzero=True)
    with pytest.raises(EmptyField):
        rel_linf(np.full(2, np.nan), np.full(2, np.nan), require_nonzero=True)
    assert rel_linf(np.array([1.0, 2.0]), np.array([1.0, 4.0]), require_nonzero=True) == 0.5


def test_quantized_case_rounds_only_fp32_inputs():
    c = W.tiny_case(nx=10, ny=8, S=3)
    q = quantized_case(c)
    assert np.array_equal(q.topo, c.topo)                      # z stays FP64
    for a, b in ((q.rain, c.rain), (q.ds, c.ds), (q.pfrac, c.pfrac), (q.ks, c.ks)):
        assert np.array_equal(a, b.astype(np.float32).astype(np.float64))
    for k, v in q.params.items():
        if isinstance(v, float):
            if k in KEEP64:
                assert v == c.params.get(k, v)
            else:
                assert v == float(np.float32(v))
