"""Host logic of the serving loop (swehr_b200/serving.py) on the CPU: the
request stream, FIFO admission against an HBM limit, overlap of requests,
completion and the latency report, against a fake pool and a fake clock."""
import math

import numpy as np
import pytest

from swehr_b200 import serving as SV


def test_poisson_stream_shape():
    reqs = SV.poisson_stream(rate=50.0, duration=20.0, seed=3)
    n = len(reqs)
    assert abs(n - 1000) < 4 * math.sqrt(1000)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0) and arr[0] >= 0 and arr[-1] < 20.0
    sides = np.array([r.side for r in reqs])
    assert sides.min() >= 32 and sides.max() <= 2048
    # log-uniform: median side near sqrt(32 * 2048) = 256
    assert 180 < np.median(sides) < 360
    for r in reqs[:50]:
        p = r.params
        assert 5 <= r.sclass <= 10 and p["sclass"] == r.sclass
        assert 1 <= p["rnum"] <= 10 and 10.0 <= p["rint"] <= 60.0
        assert p["tend"] == pytest.approx(p["rnum"] * p["rint"])
        assert np.all((r.rain >= 0) & (r.rain <= 150.0 / 3.6e6))
    again = SV.poisson_stream(rate=50.0, duration=20.0, seed=3)
    assert [(r.arrival, r.side, r.seed) for r in again] == [(r.arrival, r.side, r.seed) for r in reqs]


def test_make_case_inputs():
    reqs = SV.poisson_stream(rate=10.0, duration=3.0, seed=7, side_max=96)
    for r in reqs:
        c = SV.make_case(r)
        assert c.topo.shape == (r.side, r.side) and np.all(np.isfinite(c.topo))
        assert c.ds.shape == (r.sclass,) and abs(c.pfrac.sum() - 1) < 1e-12
        assert c.rain.shape == (r.params["rnum"],)


def test_percentile_nearest_rank():
    xs = list(range(1, 101))
    assert SV.percentile(xs, 50) == 50
    assert SV.percentile(xs, 99) == 99
    assert SV.percentile([3.0], 99) == 3.0
    assert SV.percentile([], 50) is None


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-3)


class _Prog:
    def __init__(self, steps, done, t=0.0):
        self.steps, self.done, self.status, self.t = steps, done, 0, t


class _Stats:
    def __init__(self, **kw):
        self.__dict__.update(kw)


class FakeScenario:
    def __init__(self, pool, sid, case, need):
        self.pool, self.id, self.case, self.need, self.steps = pool, sid, case, need, 0

    def progress(self):
        # one pool step advances the fake event by one simulated second
        return _Prog(self.steps, self.steps >= self.need, float(min(self.steps, self.need)))

    def fields(self, names):
        return {n: np.full((self.case.nx, self.case.ny), float(self.id)) for n in names}


class FakePool:
    """Admits by footprint (cells x 100 bytes) under a limit; a scenario
    needs int(tend) pool steps; each pool step costs 1 ms plus 1 ms per 1e4
    resident cells on the fake clock."""

    def __init__(self, clock, limit):
        self.clock, self.limit, self.used = clock, limit, 0
        self.live, self.next = {}, 1
        self.order = []
        self.max_used = 0

    def submit(self, case):
        b = case.nx * case.ny * 100
        if b > self.limit:
            e = RuntimeError("never fits")
            e.status = 5
            raise e
        if self.used + b > self.limit:
            return None
        sc = FakeScenario(self, self.next, case, max(1, int(case.params["tend"])))
        self.next += 1
        self.used += b
        self.max_used = max(self.max_used, self.used)
        self.live[sc.id] = sc
        self.order.append(case.name)
        return sc

    def run(self, steps):
        cells = sum(s.case.nx * s.case.ny for s in self.live.values() if s.steps < s.need)
        cs = 0
        for s in self.live.values():
            k = min(steps, max(0, s.need - s.steps))
            s.steps += k
            cs += k * s.case.nx * s.case.ny
        self.clock.t += steps * 1e-3 * (1.0 + cells / 1e4)
        return _Stats(cell_steps=cs, pool_steps=steps, device_ms=0.0, resident=len(self.live), hbm_used=self.used,
                      hbm_limit=self.limit)

    def release(self, sc):
        self.used -= sc.case.nx * sc.case.ny * 100
        del self.live[sc.id]

    def close(self):
        pass


def _serve(reqs, limit, chunk=4):
    clk = FakeClock()
    box = {}

    def factory():
        box["pool"] = FakePool(clk, limit)
        return box["pool"]

    srv = SV.Server(pool_factory=factory, chunk_steps=chunk, clock=clk, sleep=clk.sleep)
    rep = srv.serve(reqs)
    return rep, box["pool"]


def test_server_admits_in_order_overlaps_and_reports():
    reqs = SV.poisson_stream(rate=20.0, duration=5.0, seed=11, side_min=16, side_max=128, step_len=(10, 30),
                             hyeto_steps=(1, 3))
    SV.prepare(reqs)
    limit = 128 * 128 * 100 * 3
    rep, pool = _serve(reqs, limit)
    assert rep.completed == len(reqs) and rep.incomplete == 0 and not rep.rejected
    # FIFO admission, HBM limit respected, several requests resident at once
    assert pool.order == [f"req{r.rid}" for r in sorted(reqs, key=lambda r: r.arrival)]
    assert pool.max_used <= limit
    assert rep.max_resident > 1
    for res in rep.results:
        assert res.finished >= res.admitted >= res.arrival
        assert res.steps == max(1, int(reqs[res.rid].params["tend"]))
        assert np.all(res.fields["h"] == res.fields["h"].flat[0])
    lat = sorted(r.latency for r in rep.results)
    assert rep.p50_s == SV.percentile(lat, 50) and rep.p99_s == SV.percentile(lat, 99)
    assert rep.p99_s >= rep.p50_s > 0
    assert rep.cell_steps == sum(r.cells * r.steps for r in rep.results)
    offered = sum(r.cells * r.params["tend"] for r in reqs)
    assert rep.offered_cell_s == pytest.approx(offered) and rep.served_cell_s == pytest.approx(offered)


def test_server_reports_served_fraction_when_cut_off():
    """A stream that is stopped early: finished requests count fully, resident
    ones up to the time they reached, queued ones not at all."""
    reqs = SV.poisson_stream(rate=20.0, duration=5.0, seed=11, side_min=16, side_max=128, step_len=(10, 30),
                             hyeto_steps=(1, 3))
    SV.prepare(reqs)
    clk = FakeClock()
    box = {}

    def factory():
        box["pool"] = FakePool(clk, 128 * 128 * 100 * 3)
        return box["pool"]

    rep = SV.Server(pool_factory=factory, chunk_steps=4, clock=clk, sleep=clk.sleep).serve(reqs, time_limit=2.0)
    assert rep.incomplete > 0
    s = rep.summary()
    assert 0 < s["served_over_offered"] < 1
    arrived = [r for r in reqs if r.arrival <= rep.wall_s]
    assert rep.offered_cell_s <= sum(r.cells * r.params["tend"] for r in arrived) + 1e-9


def test_topo_bank_crops_are_seeded():
    bank = SV.TopoBank(seed=5, side=64, fields=2)
    reqs = SV.poisson_stream(rate=20.0, duration=1.0, seed=13, side_min=8, side_max=64)
    a = [SV.make_case(r, bank).topo for r in reqs]
    b = [SV.make_case(r, bank).topo for r in reqs]
    for x, y, r in zip(a, b, reqs):
        assert x.shape == (r.side, r.side) and np.array_equal(x, y) and np.all(np.isfinite(x))


def test_server_rejects_what_can_never_fit_and_waits_for_memory():
    reqs = SV.poisson_stream(rate=20.0, duration=2.0, seed=12, side_min=16, side_max=256, hyeto_steps=(1, 2))
    SV.prepare(reqs)
    limit = 200 * 200 * 100
    rep, pool = _serve(reqs, limit)
    too_big = {r.rid for r in reqs if r.cells * 100 > limit}
    assert set(rep.rejected) == too_big and too_big
    assert rep.completed == len(reqs) - len(too_big)
    assert pool.max_used <= limit
