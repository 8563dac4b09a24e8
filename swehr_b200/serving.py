"""Serving: a request loop over a scenario pool (continuous batching).

Requests arrive over time, each a catchment with its own hyetograph, size
classes and soil.  The server admits them into one Pool in arrival order as
soon as the pool's HBM limit and slots allow (a request that does not fit
waits; nothing is preempted), steps every resident scenario together in
chunks of pool steps, and hands each result back -- the requested output
fields copied to the host -- once its rain event has ended (t >= tend), then
frees its device memory.  Requests that arrive while others are on the GPU
join the running batch at the next chunk boundary, so their work overlaps.

Time-to-result of a request = (result on the host) - (arrival); the report
gives its p50/p99 beside the aggregate cell-steps/s.  SWEHR.c serves one
catchment per process and has no counterpart.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import workloads as W
from .params import MIXED

INVALID = 5   # swehr_status SWEHR_INVALID


@dataclass
class Request:
    rid: int
    arrival: float                 # seconds after the stream starts
    kind: str                      # "hillslope" or "fractal"
    side: int
    sclass: int
    seed: int
    params: dict = field(default_factory=dict)
    rain: Optional[np.ndarray] = None
    case: Optional[W.Case] = None  # materialised inputs (see prepare)

    @property
    def cells(self) -> int:
        return self.side * self.side


def poisson_stream(rate: float = 50.0, duration: float = 60.0, seed: int = 3, side_min: int = 32,
                   side_max: int = 2048, dx: float = 1.0, classes=(5, 10), step_len=(10.0, 60.0),
                   hyeto_steps=(1, 10), max_mmh: float = 150.0) -> List[Request]:
    """Poisson arrivals at `rate` per second for `duration` seconds; each
    request a hillslope or fractal square catchment with side log-uniform in
    [side_min, side_max], sclass uniform in `classes` (inclusive) with
    Dirichlet fractions, and its own hyetograph of `hyeto_steps` steps, each
    `step_len` seconds long at U(0, max_mmh) mm/h; the event (tend) is the
    hyetograph's length."""
    rng = np.random.default_rng(seed)
    reqs = []
    t = 0.0
    rid = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        side = int(round(math.exp(rng.uniform(math.log(side_min), math.log(side_max)))))
        side = max(2, side)
        kind = "hillslope" if rng.uniform() < 0.5 else "fractal"
        S = int(rng.integers(classes[0], classes[1] + 1))
        nsteps = int(rng.integers(hyeto_steps[0], hyeto_steps[1] + 1))
        rint = float(rng.uniform(step_len[0], step_len[1]))
        rain = rng.uniform(0.0, max_mmh, size=nsteps) * W.MMH
        n = float(rng.uniform(0.02, 0.08))
        params = W.common_soil(nx=side, ny=side, dx=dx, tend=rint * nsteps, rnum=nsteps, rint=rint, sclass=S,
                               roughness=n, manning0=n)
        reqs.append(Request(rid, t, kind, side, S, int(rng.integers(0, 2 ** 31)), params, rain))
        rid += 1
    return reqs


class TopoBank:
    """A few large seeded diamond-square fields (Hurst 0.8) from which fractal
    requests crop their topography at a seeded offset: O(cells) per request
    instead of a diamond-square per request, for streams too fast to generate
    inputs one by one."""

    def __init__(self, seed: int = 3, side: int = 2048, fields: int = 4):
        self.side = side
        n = max(1, math.ceil(math.log2(side - 1 if side > 2 else 2)))
        self.fields = [W.diamond_square(n, 0.8, seed * 1000 + k)[:side, :side] for k in range(fields)]

    def crop(self, side: int, rng) -> np.ndarray:
        f = self.fields[int(rng.integers(0, len(self.fields)))]
        i0 = int(rng.integers(0, self.side - side + 1))
        j0 = int(rng.integers(0, self.side - side + 1))
        return f[i0:i0 + side, j0:j0 + side]


def make_case(r: Request, bank: Optional[TopoBank] = None) -> W.Case:
    """The request's inputs: topography, size classes (diameters log-spaced
    2 um..2 mm, Dirichlet(2) fractions) and Ks, from its own seed.  Fractal
    relief grows with the catchment (1 m + 40 m x side/2048) on a 3 % tilt;
    with a bank the fractal field is a crop of one of its fields."""
    rng = np.random.default_rng(r.seed)
    side, dx = r.side, float(r.params["dx"])
    if r.kind == "hillslope":
        slope = rng.uniform(0.05, 0.15)
        x = (np.arange(1, side + 1) - 1) * dx
        topo = slope * x[:, None] + rng.normal(0.0, 0.005, size=(side, side))
    elif bank is not None and side <= bank.side:
        z = bank.crop(side, rng)
        relief = 40.0 * side / 2048.0 + 1.0
        z = (z - z.min()) / max(z.max() - z.min(), 1e-300) * relief
        topo = z + 0.03 * ((np.arange(1, side + 1) - 1) * dx)[:, None]
    else:
        topo = W.fractal_topo(side, side, dx, 0.8, 40.0 * side / 2048.0 + 1.0, 0.03, r.seed % (2 ** 31))
    S = r.sclass
    ds = 2e-6 * 1000.0 ** (np.arange(S) / max(S - 1, 1))
    pf = rng.dirichlet([2.0] * S)
    return W.Case(f"req{r.rid}", dict(r.params), topo, np.asarray(r.rain, dtype=np.float64), ds, pf)


def prepare(reqs: Sequence[Request], bank: Optional[TopoBank] = None) -> None:
    """Materialise every request's inputs on the host (the client side; done
    before the stream starts so that input generation is not timed)."""
    for r in reqs:
        if r.case is None:
            r.case = make_case(r, bank)


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    status: int
    cells: int
    fields: Dict[str, np.ndarray]

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class Report:
    submitted: int
    completed: int
    incomplete: int
    rejected: List[int]
    wall_s: float
    device_ms: float
    cell_steps: int
    pool_steps: int
    p50_s: Optional[float]
    p99_s: Optional[float]
    mean_s: Optional[float]
    max_resident: int
    peak_hbm_bytes: int
    hbm_limit: int
    results: List[Result]
    offered_cell_s: float = 0.0     # sum over arrived requests of cells x event length (simulated s)
    served_cell_s: float = 0.0      # sum of cells x simulated time reached by the end
    host_s: Dict[str, float] = field(default_factory=dict)   # wall time per loop phase

    @property
    def cell_steps_per_s(self) -> float:
        return self.cell_steps / self.wall_s if self.wall_s > 0 else 0.0

    def split(self) -> dict:
        """Per-request time-to-result split into queueing (arrival ->
        admission: waiting for HBM or a slot) and residency (admission ->
        result on the host: the request's steps, shared with everything
        resident), p50 / p99 / max over the completed requests."""
        q = [x.admitted - x.arrival for x in self.results]
        d = [x.finished - x.admitted for x in self.results]
        out = {}
        for name, xs in (("queue_s", q), ("resident_s", d)):
            out[name] = {"p50": percentile(xs, 50), "p99": percentile(xs, 99), "max": max(xs) if xs else None}
        # the slowest 1 %: how much of their time was queueing
        lat = sorted(self.results, key=lambda x: x.latency)
        tail = lat[int(0.99 * len(lat)):] if lat else []
        out["p99_tail"] = {"n": len(tail),
                           "queue_share": (sum(x.admitted - x.arrival for x in tail) / sum(x.latency for x in tail))
                           if tail and sum(x.latency for x in tail) > 0 else None,
                           "mean_cells": (sum(x.cells for x in tail) / len(tail)) if tail else None,
                           "mean_steps": (sum(x.steps for x in tail) / len(tail)) if tail else None}
        return out

    def summary(self) -> dict:
        return {"submitted": self.submitted, "completed": self.completed, "incomplete": self.incomplete,
                "latency_split": self.split(),
                "rejected": len(self.rejected),
                "wall_s": self.wall_s, "device_ms": self.device_ms, "cell_steps": self.cell_steps,
                "pool_steps": self.pool_steps, "cell_steps_per_s": self.cell_steps_per_s,
                "p50_s": self.p50_s, "p99_s": self.p99_s, "mean_s": self.mean_s,
                "max_resident": self.max_resident, "peak_hbm_bytes": self.peak_hbm_bytes,
                "hbm_limit": self.hbm_limit, "host_s": self.host_s,
                "offered_cell_seconds": self.offered_cell_s, "served_cell_seconds": self.served_cell_s,
                "served_over_offered": (self.served_cell_s / self.offered_cell_s) if self.offered_cell_s else None}


def percentile(xs: Sequence[float], q: float) -> Optional[float]:
    """Nearest-rank percentile (q in 0..100)."""
    if not xs:
        return None
    s = sorted(xs)
    k = max(1, int(math.ceil(q / 100.0 * len(s))))
    return float(s[k - 1])


class Server:
    """Continuous-batching request loop over one Pool.

    pool_factory: callable returning a Pool-like object (tests pass a fake);
    chunk_steps: pool steps between admission / completion checks;
    result_fields: fields copied to the host for every finished request."""

    def __init__(self, precision: int = MIXED, hbm_limit: int = 150 * 10 ** 9, max_classes: int = 16,
                 max_scenarios: int = 4096, chunk_steps: int = 32, result_fields=("h", "totsed"),
                 pool_factory: Optional[Callable] = None, clock: Callable[[], float] = time.perf_counter,
                 sleep: Callable[[float], None] = time.sleep):
        if pool_factory is None:
            from .lib import Pool

            def pool_factory():
                return Pool(precision=precision, max_classes=max_classes, hbm_limit=hbm_limit,
                            max_scenarios=max_scenarios)
        self.pool_factory = pool_factory
        self.chunk_steps = chunk_steps
        self.result_fields = tuple(result_fields)
        self.clock = clock
        self.sleep = sleep

    def serve(self, reqs: Sequence[Request], time_limit: Optional[float] = None,
              on_result: Optional[Callable[[Result], None]] = None) -> Report:
        reqs = sorted(reqs, key=lambda r: r.arrival)
        pool = self.pool_factory()
        try:
            return self._loop(pool, reqs, time_limit, on_result)
        finally:
            pool.close()

    def _loop(self, pool, reqs, time_limit, on_result) -> Report:
        t0 = self.clock()
        nxt = 0
        reqs_by_id = {r.rid: r for r in reqs}
        queue: List[Request] = []
        live = {}            # rid -> (request, scenario, admitted time)
        results: List[Result] = []
        rejected: List[int] = []
        cell_steps = pool_steps = 0
        device_ms = 0.0
        max_res = peak_hbm = 0
        hbm_limit = 0
        host = {"submit_s": 0.0, "run_s": 0.0, "poll_s": 0.0, "read_s": 0.0, "release_s": 0.0}
        clk = self.clock
        while nxt < len(reqs) or queue or live:
            now = self.clock() - t0
            if time_limit is not None and now >= time_limit:
                break
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                queue.append(reqs[nxt])
                nxt += 1
            # admission in arrival order while the pool has room
            while queue:
                r = queue[0]
                case = r.case if r.case is not None else make_case(r)
                ts = clk()
                try:
                    sc = pool.submit(case)
                    host["submit_s"] += clk() - ts
                except Exception as e:  # noqa: BLE001 -- a request the pool can never hold
                    if getattr(e, "status", None) != INVALID:
                        raise
                    queue.pop(0)
                    rejected.append(r.rid)
                    continue
                if sc is None:
                    break
                queue.pop(0)
                live[r.rid] = (r, sc, self.clock() - t0)
            if not live:
                if nxt < len(reqs):
                    self.sleep(max(0.0, min(reqs[nxt].arrival - (self.clock() - t0), 0.05)))
                    continue
                break
            ts = clk()
            st = pool.run(self.chunk_steps)
            host["run_s"] += clk() - ts
            cell_steps += int(st.cell_steps)
            pool_steps += int(st.pool_steps)
            device_ms += float(st.device_ms)
            max_res = max(max_res, int(st.resident))
            peak_hbm = max(peak_hbm, int(st.hbm_used))
            hbm_limit = int(st.hbm_limit)
            ts = clk()
            done = []
            for rid in list(live):
                pr = live[rid][1].progress()
                if pr.done:
                    done.append((rid, pr))
            host["poll_s"] += clk() - ts
            for rid, pr in done:
                r, sc, adm = live[rid]
                ts = clk()
                out = sc.fields(self.result_fields)
                fin = clk() - t0
                host["read_s"] += clk() - ts
                res = Result(rid, r.arrival, adm, fin, int(pr.steps), int(pr.status), r.cells, out)
                ts = clk()
                pool.release(sc)
                host["release_s"] += clk() - ts
                del live[rid]
                results.append(res)
                if on_result is not None:
                    on_result(res)
        wall = self.clock() - t0
        # offered vs served simulated work: finished requests count fully,
        # resident ones up to the time they reached, queued ones not at all
        offered = sum(r.cells * float(r.params["tend"]) for r in reqs[:nxt])
        served = sum(x.cells * float(reqs_by_id[x.rid].params["tend"]) for x in results)
        for rid, (r, sc, adm) in live.items():
            served += r.cells * float(sc.progress().t)
        lat = [x.latency for x in results]
        return Report(submitted=len(reqs), completed=len(results),
                      incomplete=len(reqs) - len(results) - len(rejected), rejected=rejected,
                      wall_s=wall, device_ms=device_ms, cell_steps=cell_steps, pool_steps=pool_steps,
                      p50_s=percentile(lat, 50), p99_s=percentile(lat, 99),
                      mean_s=(sum(lat) / len(lat)) if lat else None, max_resident=max_res,
                      peak_hbm_bytes=peak_hbm, hbm_limit=hbm_limit, results=results, host_s=host,
                      offered_cell_s=offered, served_cell_s=served)
