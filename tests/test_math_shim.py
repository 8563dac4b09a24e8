"""Accuracy of the project's elementary functions (swehr_math.h), called
through the oracle's project-math build, against 50-digit decimal values.

These are the bodies the FP64 kernels use; being (almost) correctly rounded
keeps the GPU within the libm floor of the reference's glibc results.
"""
import math
from decimal import Decimal, getcontext

import numpy as np
import pytest

from harness import OracleRun

getcontext().prec = 50


def _ulp_err(got: float, exact: Decimal) -> float:
    if not math.isfinite(got):
        return float("inf")
    e = float(exact)
    u = math.ulp(e) if e != 0 else 5e-324
    return float(abs(Decimal(got) - exact) / Decimal(u))


@pytest.fixture(scope="module")
def shim():
    return OracleRun.lib("shim")


@pytest.fixture(scope="module")
def glibc():
    return OracleRun.lib("glibc")


def test_exp(shim):
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-745, 709, 3000), rng.uniform(-60, 0, 3000), rng.uniform(-1e-3, 1e-3, 500)])
    worst = max(_ulp_err(shim.orc_m_exp(float(x)), Decimal(float(x)).exp()) for x in xs)
    assert worst < 0.53, worst
    assert shim.orc_m_exp(0.0) == 1.0
    assert shim.orc_m_exp(-800.0) == 0.0
    assert math.isinf(shim.orc_m_exp(710.0))
    assert math.isnan(shim.orc_m_exp(float("nan")))


@pytest.mark.parametrize("y", [3.333, 2.333, -0.33, 0.6, 4.0, 1.7, -2.5])
def test_pow(shim, y):
    rng = np.random.default_rng(int(abs(y) * 1000))
    xs = np.concatenate([10 ** rng.uniform(-6, 1, 2000), rng.uniform(0.5, 1.5, 500)])
    worst = 0.0
    for x in xs:
        exact = (Decimal(float(x)).ln() * Decimal(y)).exp()
        worst = max(worst, _ulp_err(shim.orc_m_pow(float(x), y), exact))
    assert worst < 0.52, (y, worst)


def test_pow_special_cases(shim):
    p = shim.orc_m_pow
    assert p(0.0, 3.333) == 0.0
    assert math.isinf(p(0.0, -0.33))
    assert p(-0.0, 0.5) == 0.0 and math.copysign(1, p(-0.0, 0.5)) > 0
    assert math.isnan(p(-2.0, 0.6))
    assert p(-2.0, 3.0) == -8.0
    assert p(5.0, 0.0) == 1.0 and p(1.0, float("nan")) == 1.0
    assert p(7.25, 1.0) == 7.25 and p(1.5, 2.0) == 2.25
    assert p(2.0, 0.5) == math.sqrt(2.0)
    assert math.isinf(p(float("inf"), 0.6)) and p(float("inf"), -0.6) == 0.0


def test_cos_sin_atan(shim):
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.uniform(0, 2, 2000), 10 ** rng.uniform(-8, 6, 1000)])
    wc = ws = 0.0
    for x in xs:
        d = Decimal(float(x))
        r = (1 + d * d).sqrt()
        wc = max(wc, _ulp_err(shim.orc_m_cosatan(float(x)), 1 / r))
        ws = max(ws, _ulp_err(shim.orc_m_sinatan(float(x)), d / r))
    assert wc < 0.52 and ws < 0.52, (wc, ws)
    assert shim.orc_m_cosatan(0.0) == 1.0 and shim.orc_m_sinatan(0.0) == 0.0


def test_agreement_with_glibc(shim, glibc):
    """Both are nearly correctly rounded, so they agree on almost every input."""
    rng = np.random.default_rng(4)
    xs = 10 ** rng.uniform(-5, 0, 4000)
    same_pow = np.mean([shim.orc_m_pow(float(x), 3.333) == glibc.orc_m_pow(float(x), 3.333) for x in xs])
    same_exp = np.mean([shim.orc_m_exp(-float(x) * 50) == glibc.orc_m_exp(-float(x) * 50) for x in xs])
    same_sqrt = np.mean([shim.orc_m_powh(float(x)) == glibc.orc_m_powh(float(x)) for x in xs])
    assert same_pow > 0.99 and same_exp > 0.98 and same_sqrt > 0.99, (same_pow, same_exp, same_sqrt)



def test_constant_divisor_by_remainder_correction_is_ieee_division():
    """The update kernel divides by the run's constant divisors (rho_s(1-phi),
    rho_s, J, 6 h0, 0.2, theta_s - theta_0) through their correctly rounded
    reciprocals and two remainder corrections; it must give the IEEE
    quotient bit for bit: millions of random dividends over the guarded
    range, for those constants and random ones, plus the edge cases."""
    import ctypes as C
    import math
    from harness import OracleRun
    L = OracleRun.lib("shim")
    L.orc_divk.restype = C.c_double
    L.orc_divk.argtypes = [C.c_double, C.c_double, C.c_double]
    L.orc_divk_check.restype = C.c_int64
    L.orc_divk_check.argtypes = [C.c_double, C.c_int64, C.c_uint64]
    consts = [2600 * (1 - 0.4), 2600.0, 30.0, 6 * 0.00099, 0.2, 0.4 - 0.1, 0.3]
    rng = np.random.default_rng(7)
    consts += [float(c) for c in np.exp2(rng.uniform(-100, 100, size=40)) * rng.uniform(1, 2, size=40)]
    # significands right below 2 (reciprocals right above a power of two): the hardest case
    consts += [math.ldexp(2 - 2 ** -52, e) for e in (-3, 0, 7)] + [math.ldexp(1 + 2 ** -52, e) for e in (-2, 5)]
    for k, c in enumerate(consts):
        assert L.orc_divk_check(c, 400000 if k < 7 else 100000, 1234 + k) == 0, c
    for a in (0.0, -0.0, 2 ** -1074, -(2 ** -1022), 2 ** -901, 1e300, -1e308, float("inf"), float("-inf"), float("nan")):
        for c in (1560.0, 0.2):
            got, want = L.orc_divk(a, c, 1.0 / c), a / c
            assert (math.isnan(got) and math.isnan(want)) or (got == want and math.copysign(1, got) == math.copysign(1, want)), (a, c)
