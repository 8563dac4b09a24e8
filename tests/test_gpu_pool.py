"""The scenario pool (swehr_pool_*): many scenarios of uneven sizes stepped
by shared persistent launches.

Every scenario's per-cell arithmetic in the pool is the single-domain
arithmetic, so its fields, stage rows and step count must be bit-identical
to the same case run alone -- alone through swehr_create/swehr_advance, alone
in a pool, and in a mix of other scenarios joining at different times.
Budgets in a pool are summed with atomics (order-dependent rounding of the
budget terms only) and must still close.
"""
import numpy as np
import pytest

from harness import OracleRun, compare, STATE_FIELDS, CLASS_FIELDS
from swehr_b200 import workloads as W
from swehr_b200.params import FP64, MIXED

pytestmark = pytest.mark.gpu

ALL = STATE_FIELDS + CLASS_FIELDS + ("vel",)

MIX = [
    dict(nx=12, ny=9, S=3, seed=5, bndry=(0, 1, 1, 1), inflow=0, rain_mmh=90.0, tend=60.0),
    dict(nx=15, ny=11, S=4, seed=6, bndry=(1, 0, 1, 1), inflow=1, rain_mmh=300.0, tend=120.0),
    dict(nx=40, ny=30, S=4, seed=41, bndry=(0, 1, 1, 1), inflow=0, rain_mmh=120.0, tend=90.0),
    dict(nx=33, ny=70, S=7, seed=42, bndry=(0, 1, 1, 0), inflow=0, rain_mmh=200.0, tend=70.0),
    dict(nx=2, ny=2, S=1, seed=11, bndry=(0, 0, 0, 0), inflow=0, rain_mmh=100.0, tend=30.0),
    dict(nx=97, ny=65, S=8, seed=43, bndry=(0, 0, 1, 1), inflow=0, rain_mmh=250.0, tend=45.0),
]


def _cases():
    return [W.tiny_case(**kw) for kw in MIX]


def _alone(case, precision):
    from swehr_b200.lib import Simulation
    with Simulation(case, precision=precision) as s:
        pr = s.advance()
        return pr.steps, s.fields(), s.series()


def _same(a, b, names=ALL):
    res = compare(a, b, names)
    return {k: v for k, v in res.items() if not v[2]}


def _pool_all(cases, precision, join_after=None, tune=False, max_classes=8):
    """Run cases to completion in one pool; case k joins after join_after[k]
    pool steps (0 = from the start)."""
    from swehr_b200.lib import Pool
    join_after = join_after or [0] * len(cases)
    out = {}
    with Pool(precision=precision, max_classes=max_classes, max_scenarios=64) as pool:
        pending = sorted(range(len(cases)), key=lambda k: join_after[k])
        live = {}
        step = 0
        while pending or live:
            if not live:
                step = max(step, join_after[pending[0]])
            while pending and join_after[pending[0]] <= step:
                k = pending.pop(0)
                live[k] = pool.submit(cases[k])
                assert live[k] is not None
            if tune and step == 0:
                st = pool.tune(4)
                assert st.tuned == 1 and st.grid_update > 0 and st.grid_wave > 0
                # the tuner ran real steps in both tile shapes and kept one
                assert (st.tile_i, st.tile_j) in ((8, 32), (16, 16))
                step += st.pool_steps
            else:
                nxt = min([join_after[k] for k in pending], default=step + 10 ** 9)
                st = pool.run(min(nxt - step, 10 ** 6) if pending else -1)
                step += st.pool_steps
            for k, sc in list(live.items()):
                pr = sc.progress()
                if pr.done:
                    out[k] = (pr.steps, sc.fields(), sc.series())
                    pool.release(sc)
                    del live[k]
    return [out[k] for k in range(len(cases))]


def _check_same(got, ref, label):
    for k, (g, r) in enumerate(zip(got, ref)):
        assert g[0] == r[0], (label, k, g[0], r[0])
        bad = _same(g[1], r[1])
        assert not bad, (label, k, bad)
        assert np.array_equal(g[2][0], r[2][0], equal_nan=True), (label, k, "stage rows")
        assert np.array_equal(g[2][1], r[2][1], equal_nan=True), (label, k, "point series")


def test_pool_fp64_matches_single_and_oracle():
    cases = _cases()
    alone = [_alone(c, FP64) for c in cases]
    got = _pool_all(cases, FP64)
    _check_same(got, alone, "pool vs alone")
    # and the oracle, for the two smallest
    for k in (0, 4):
        o = OracleRun(cases[k], "shim")
        o.advance()
        assert o.steps == got[k][0]
        bad = _same(got[k][1], o.fields())
        assert not bad, (k, bad)


def test_pool_fp64_join_mid_run_and_tuned():
    """Continuous batching: scenarios join while others are on the GPU; the
    tuner changes the launch shape; no result changes."""
    cases = _cases()
    alone = [_alone(c, FP64) for c in cases]
    got = _pool_all(cases, FP64, join_after=[0, 7, 0, 33, 50, 5], tune=True)
    _check_same(got, alone, "joined pool vs alone")


def test_pool_mixed_alone_vs_mix():
    cases = _cases()
    each = [_pool_all([c], MIXED)[0] for c in cases]
    mix = _pool_all(cases, MIXED, join_after=[0, 3, 9, 0, 20, 1])
    _check_same(mix, each, "mixed mix vs alone-in-pool")
    # and the pooled mixed form meets the mixed form's accuracy rule against
    # FP64: within 1e-4, or 10x the drift FP32-rounded inputs alone cause
    from swehr_b200.accuracy import quantized_case
    for k, (g, c) in enumerate(zip(mix, cases)):
        f64 = _alone(c, FP64)                  # all three end at t = tend (the last step is clamped);
        fq = _alone(quantized_case(c), FP64)   # their step counts may differ by one
        em, eq = compare(g[1], f64[1], ("h", "totsed", "sed")), compare(fq[1], f64[1], ("h", "totsed", "sed"))
        for name in ("h", "totsed", "sed"):
            env = eq[name][0]
            bound = 1e-4 if env < 1e-5 else max(1e-4, 10 * env)
            assert em[name][1] and em[name][0] <= bound, (k, name, em[name][0], env)


def test_pool_budget_closes():
    from swehr_b200.lib import Pool
    cases = _cases()[2:4]
    with Pool(precision=FP64, max_classes=8, budget=True) as pool:
        scs = [pool.submit(c, budget=True) for c in cases]
        pool.run(-1)
        for c, sc in zip(cases, scs):
            b = sc.budget()
            assert b.valid == 1
            scale = max(abs(b.water_now), abs(b.rain_in))
            assert abs(b.water_residual) <= 1e-9 * scale, (b.water_residual, scale)
            for k in range(c.sclass):
                s = max(abs(b.sed_now[k]), abs(b.detach[k]), 1e-300)
                assert abs(b.sed_residual[k]) <= 1e-9 * s, (k, b.sed_residual[k], s)


def test_pool_admission_by_footprint_and_slots():
    from swehr_b200.lib import Pool
    cases = _cases()
    big = cases[5]
    with Pool(precision=FP64, max_classes=8) as pool:
        pool.submit(big)
        held = pool.stats().hbm_used          # device bytes one such scenario holds
    assert held > 0
    # room for one large scenario only
    with Pool(precision=FP64, max_classes=8, hbm_limit=int(held * 1.5), max_scenarios=8) as pool:
        a = pool.submit(big)
        assert a is not None
        assert pool.submit(big) is None            # footprint: busy, nothing allocated
        st = pool.stats()
        assert st.resident == 1 and st.hbm_used <= st.hbm_limit
        pool.run(-1)
        assert a.progress().done
        pool.release(a)
        b = pool.submit(big)                        # memory freed: admitted, its block reused
        assert b is not None
        assert pool.stats().hbm_used == held
    with Pool(precision=FP64, max_classes=8, max_scenarios=2) as pool:
        assert pool.submit(cases[0]) is not None
        assert pool.submit(cases[1]) is not None
        assert pool.submit(cases[2]) is None        # slots: busy
    with Pool(precision=FP64, max_classes=4) as pool:
        from swehr_b200.lib import SwehrError
        with pytest.raises(SwehrError):
            pool.submit(cases[3])                   # 7 classes > max_classes 4


def test_pool_step_limit_and_cfl_error():
    from swehr_b200.lib import Pool
    c0 = W.tiny_case(nx=40, ny=30, S=4, seed=41, bndry=(0, 1, 1, 1), inflow=0, rain_mmh=120.0, tend=90.0)
    c1 = W.tiny_case(nx=15, ny=11, S=4, seed=6, bndry=(1, 0, 1, 1), inflow=1, rain_mmh=300.0, tend=1000.0,
                     cstable=40.0, maxstep=50.0)
    with Pool(precision=FP64, max_classes=8) as pool:
        a = pool.submit(c0, max_steps=25)
        b = pool.submit(c1)
        pool.run(-1)
        pa, pb = a.progress(), b.progress()
        assert pa.done and pa.steps == 25 and pa.status == 0
        assert pb.done and pb.status == 1
    from swehr_b200.lib import Simulation
    with Simulation(c1) as s:
        pr = s.advance()
        assert pr.steps == pb.steps and s.status == 1


def test_pool_exact_class_count_kernels():
    """A pool whose running scenarios all have 7 (or all 10) classes steps them
    with the batched kernel built for exactly that count; every scenario still
    equals its single-domain run bit for bit."""
    for S in (7, 10):
        cases = [W.tiny_case(nx=20 + 3 * k, ny=15 + k, S=S, seed=60 + k, bndry=(0, 1, 1, 1), inflow=k % 2,
                             rain_mmh=200.0, tend=40.0) for k in range(3)]
        alone = [_alone(c, FP64) for c in cases]
        got = _pool_all(cases, FP64, max_classes=16)
        _check_same(got, alone, f"exact {S} classes")
