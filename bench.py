"""Benchmark of the SWEHR time step on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {swehr,reference}]

Workload (N=1): the roofline domain -- 4096 x 4096 cells, dx = 2 m,
diamond-square topography (Hurst 0.8, 40 m relief, seed 1) tilted 3 % toward
i=1, uniform rain from a seeded 30-entry hyetograph, lognormal per-cell Ks,
7 sediment classes -- run in the plain FP64 form.  A "step" is one SWEHR time
step over the whole domain.  W untimed steps, then exactly K timed steps
(the run continues the same trajectory); the 4096^2 state (6.7 GB) is far
larger than L2, so no flush is needed between steps.

N > 1 (torchrun): every rank advances its own replica of the domain (weak
scaling, no data-path collective -- independent domains do not exchange
anything); rank 0 prints the whole-job cell-steps/s from the max over ranks
of the device-timed region.  The batched-ensemble leg splits its scenarios
over the ranks by cell count (strong scaling of a fixed ensemble, again
without exchange); the CPU baseline and the serving leg run at N = 1 only.

--impl reference: the reference program (SWEHR.c built by oracle/build_ref.py
with its own OpenMP pragmas on) on a crop of the same domain, all host
threads, timed by its own loop timer; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def algo_bytes_f64(S: int) -> int:
    """Algorithmic bytes per cell-step of the plain FP64 form: every prognostic
    field (h hu hv z VINF MAXDEPTH MAXVEL, U_k, M_k) read and written once,
    plus the per-cell Ks read."""
    return 16 * (7 + 2 * S) + 8


def algo_bytes_mixed(S: int) -> int:
    """Algorithmic bytes per cell-step of the mixed form: FP32 h, hu, hv,
    MAXDEPTH, MAXVEL, U_k; FP64 z, VINF, M_k; FP32 Ks."""
    return 2 * (4 * (5 + S) + 8 * (2 + S)) + 4


def profiled(summary: str, key: str = "traffic_bytes_per_cell_step"):
    """A per-cell figure of a kernel from its committed ncu summary: DRAM
    bytes per cell-step (dram__bytes_read.sum + dram__bytes_write.sum of one
    captured launch on a 1024^2 case, divided by its cells; per-cell traffic
    is size independent once the state is far larger than L2), or FP64
    operations per cell-step (2 x DFMA + DMUL + DADD thread instructions)."""
    path = os.path.join(ROOT, "profiles", summary)
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def profiled_traffic(summary: str):
    return profiled(summary)


def fp64_peak():
    """The FP64 pipe's ceiling on this GPU in TFLOP/s, measured now by
    swehr_probe_fp64_peak (independent FMA chains at full occupancy)."""
    import ctypes
    try:
        lib = ctypes.CDLL(os.path.join(ROOT, "swehr_b200", "libswehr_probe.so"))
        v = ctypes.c_double()
        if lib.swehr_probe_fp64_peak(ctypes.byref(v)) == 0 and v.value > 0:
            return v.value
    except OSError:
        pass
    return None


def hbm_peak():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clock samples (every 20 ms) kept only where their timestamps
    fall inside the timed windows: the sampler starts before the simulation
    is created, so it is producing samples when the short timed regions run."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        self.idx = gpu_index
        self.proc = None
        self.windows = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def window(self, t0: float, t1: float):
        """a timed region, host wall-clock seconds (time.time()) around it"""
        self.windows.append((t0, t1))

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        import datetime
        rows = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) < 10:
                    continue
                try:
                    ts = datetime.datetime.strptime(p[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    rows.append((ts, float(p[2]), float(p[3]),
                                 {n for n, v in zip(names, p[6:10]) if v.lower() in ("active", "1", "yes")}))
                except ValueError:
                    continue
        except FileNotFoundError:
            pass
        try:
            os.unlink(self.path)
        except OSError:
            pass
        inside = [r for r in rows if any(a <= r[0] <= b for a, b in self.windows)]
        sel = inside
        if not sel and rows and self.windows:
            # no sample landed inside (windows of ~0.1 s): the samples nearest to them
            d = lambda r: min(min(abs(r[0] - a), abs(r[0] - b)) for a, b in self.windows)
            sel = sorted(rows, key=d)[:3]
        sm = [r[1] for r in sel]
        reasons = set().union(*[r[3] for r in sel]) if sel else set()
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(r[2] for r in sel) if sel else None,
                "reasons": sorted(reasons), "samples": len(sel), "samples_inside_windows": len(inside),
                "windows_s": [round(b - a, 3) for a, b in self.windows]}


def bench_workload(args):
    from swehr_b200 import workloads as W
    return W.fractal_domain(nx=args.nx, ny=args.ny, dx=2.0, seed=1, steps=args.warmup + args.steps)


def run_cpu_reference(case, crop: int, steps: int, threads: int):
    """The reference program (OpenMP build) on a crop x crop corner of the
    case for `steps` steps; returns (cell-steps/s, elapsed, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import harness
    from swehr_b200.workloads import Case
    p = dict(case.params)
    p["nx"], p["ny"] = crop, crop
    sub = Case(case.name + f"_crop{crop}", p, case.topo[:crop, :crop].copy(), case.rain, case.ds, case.pfrac,
               ks=None if case.ks is None else case.ks[:crop, :crop].copy())
    if not os.path.exists(harness.ref_binary(True)):
        raise FileNotFoundError("oracle/_ref/swehr_ref_omp not built")
    _, out = harness.run_reference(sub, max_steps=steps, omp=True, threads=threads, dump=False, timeout=900)
    for line in out.splitlines():
        if line.startswith("SWEHR_REF"):
            f = line.split()
            n, el, th = int(f[2]), float(f[4]), int(f[6])
            return crop * crop * n / el, el, th, n
    raise RuntimeError("reference printed no timing line")


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_arm(args, rank: int):
    if rank != 0:
        return
    case = bench_workload(args)
    threads = host_threads()
    # one timed "step" = one reference time step on a crop sized so K steps take ~1-2 minutes
    budget_cell_steps = 1.5e8
    crop = int(max(64, min(1024, (budget_cell_steps / max(args.steps, 1)) ** 0.5)))
    try:
        value, el, th, n = run_cpu_reference(case, crop, args.steps, threads)
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference program not runnable: {e}"}))
        return
    line = {
        "impl": "reference", "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": args.gpus,
        "steps": n, "warmup": 0, "ms_per_step": el * 1e3 / max(n, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"fractal {args.nx}x{args.ny} dx=2 S=7, plain FP64; reference run on a "
                               f"{crop}x{crop} crop of the same domain", "threads": th},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": th, "kind": "reference",
                         "sample": f"SWEHR.c (OpenMP pragmas on) on a {crop}x{crop} crop, {n} steps"},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def ensemble_leg(args, ranks):
    """The batched ensemble: scenarios with sides log-uniform in 64..1024
    cells (dx = 1 m, per-scenario fractal seeds, rain U(20,150) mm/h, Manning
    n U(0.02,0.08), 7 classes) resident in one pool and stepped by shared
    persistent launches, in the mixed and in the plain FP64 form; each form's
    launch shape picked by the pool's tuner first.  With N ranks the
    scenarios are split over the GPUs by cell count (no exchange: strong
    scaling of a fixed ensemble); throughput is all ranks' cell-steps over
    the slowest rank's device time.  Every scenario is capped at the same
    step count, so after the timed steps both pools hold the same steps of
    every scenario and a subset is compared field by field (mixed vs FP64,
    beside FP64 on FP32-rounded inputs: the envelope)."""
    from swehr_b200.accuracy import rel_linf, quantized_case
    from swehr_b200 import workloads as W
    from swehr_b200.lib import Pool, Simulation
    from swehr_b200.params import FP64, MIXED
    from swehr_b200.ranks import shard
    all_cases = W.ensemble(args.ens_count)
    mine = shard([c.cells() for c in all_cases], ranks.world)[ranks.rank]
    cases = [all_cases[k] for k in mine]
    cells = sum(c.cells() for c in all_cases)
    # pool steps every scenario runs: the tuner's (up to 2 shapes x 8 grids x
    # 3 rounds x 4 steps), the warm-up and the timed ones, so that every
    # scenario is still running through the whole timed window
    cap = 256 + args.ens_warmup + args.ens_steps
    every = max(1, len(all_cases) // 8)
    subset = [i for i, k in enumerate(mine) if k % every == 0 and k // every < 8]
    names = ("h", "totsed", "sed")
    out, keep = {}, {}
    for label, prec in (("fp64", FP64), ("mixed", MIXED)):
        with Pool(precision=prec, max_classes=8, max_scenarios=len(cases) + 1) as pool:
            t0 = time.perf_counter()
            scs = [pool.submit(c, max_steps=cap) for c in cases]
            if any(s is None for s in scs):
                raise RuntimeError("ensemble does not fit the pool")
            upload_s = time.perf_counter() - t0
            tu = pool.tune(4)
            pool.run(args.ens_warmup)
            ranks.barrier()
            st = pool.run(args.ens_steps)
            ranks.barrier()
            dev_ms = ranks.max(st.device_ms)
            cs = ranks.sum(st.cell_steps)
            pool.run(-1)
            keep[label] = [scs[k].fields(names) for k in subset]
            out[label] = {"value": cs / (dev_ms / 1e3), "unit": "cell-steps/s", "pool_steps": int(st.pool_steps),
                          "tuner_steps": int(tu.pool_steps), "scenario_steps_timed": cs / max(cells, 1),
                          "device_ms": dev_ms, "ms_per_pool_step": dev_ms / max(st.pool_steps, 1),
                          "grid_wave": int(tu.grid_wave), "grid_update": int(tu.grid_update),
                          "tile": f"{int(tu.tile_i)}x{int(tu.tile_j)}",
                          "upload_s": upload_s, "hbm_bytes_rank0": int(st.hbm_used)}
    # envelope: FP64 on the subset's inputs rounded to FP32
    env = []
    if subset:
        with Pool(precision=FP64, max_classes=8, max_scenarios=len(subset) + 1) as pool:
            scs = [pool.submit(quantized_case(cases[k]), max_steps=cap) for k in subset]
            pool.run(-1)
            env = [s.fields(names) for s in scs]
    # every compared field must carry something: an empty (all-zero) FP64
    # field would make any error look perfect
    # field: an all-zero FP64 field (a scenario that has not ponded yet
    # carries no sediment) is skipped and counted, never scored as a match
    from swehr_b200.accuracy import EmptyField
    err = {n: 0.0 for n in names}
    envm = {n: 0.0 for n in names}
    compared = {n: 0 for n in names}
    wet = []
    for a, b, q in zip(keep["mixed"], keep["fp64"], env):
        wet.append(float((b["h"] > 1e-4).mean()))
        for n in names:
            try:
                e = rel_linf(a[n], b[n], require_nonzero=True)
                v = rel_linf(q[n], b[n], require_nonzero=True)
            except EmptyField:
                continue
            err[n], envm[n] = max(err[n], e), max(envm[n], v)
            compared[n] += 1
    err = {n: ranks.max(v) for n, v in err.items()}
    envm = {n: ranks.max(v) for n, v in envm.items()}
    compared = {n: int(ranks.sum(v)) for n, v in compared.items()}
    # the same scenarios one at a time through the single-domain path
    step = max(1, len(all_cases) // 32)

    def solo_rate(prec):
        t_dev, cs = 0.0, 0
        for k in mine:
            if k % step:
                continue
            with Simulation(all_cases[k], precision=prec) as sim:
                sim.advance(max_steps=3)
                pr = sim.advance(max_steps=args.ens_solo_steps)
                t_dev += pr.device_ms
                cs += all_cases[k].cells() * pr.steps_this_call
        tot = ranks.sum(t_dev)
        return ranks.sum(cs) / (tot / 1e3) if tot > 0 else None

    solo = solo_rate(FP64)
    solo_mixed = solo_rate(MIXED)
    return {"workload": f"{len(all_cases)} scenarios, sides log-uniform 64..1024 (seed 2), {cells} cells, 7 classes",
            "scenarios": len(all_cases), "cells": cells, "steps_per_scenario": cap,
            "placement": f"split over {ranks.world} GPU(s) by cells, no exchange"
                         + (" (strong scaling)" if ranks.world > 1 else ""),
            "batched_mixed": out["mixed"], "batched_fp64": out["fp64"],
            "solo_fp64": {"value": solo, "unit": "cell-steps/s per GPU",
                          "sample": f"every {step}th scenario alone, {args.ens_solo_steps} steps each"},
            "solo_mixed": {"value": solo_mixed, "unit": "cell-steps/s per GPU",
                           "sample": f"every {step}th scenario alone, {args.ens_solo_steps} steps each"},
            "mixed_over_batched_fp64": out["mixed"]["value"] / out["fp64"]["value"],
            "mixed_over_solo_fp64": (out["mixed"]["value"] / ranks.world / solo) if solo else None,
            "error_vs_fp64": {"scenarios": [int(k) for k in range(0, len(all_cases), every)][:8],
                              "at_step": cap, "rel_linf": err, "fp32_input_envelope": envm,
                              "wet_fraction": wet, "scenarios_compared": compared,
                              "valid": all(v > 0 for v in compared.values())}}


def serving_leg(args):
    """A Poisson request stream through the continuous-batching server: the
    full stream by default (50/s for 60 s, sides to 2048, up to 10
    hyetograph steps, 150 GB admission limit), which offers more work than
    one GPU serves and is reported by its served fraction, served for 60 s
    more after the last arrival; --serve-small scales it to what one B200
    keeps up with."""
    from swehr_b200 import serving as SV
    from swehr_b200.params import MIXED
    if args.serve_small:
        args.serve_side_max, args.serve_hyeto_max = 512, 3
        args.serve_duration, args.serve_drain = 10.0, 50.0
    reqs = SV.poisson_stream(rate=args.serve_rate, duration=args.serve_duration, seed=3, side_min=32,
                             side_max=args.serve_side_max, hyeto_steps=(1, args.serve_hyeto_max))
    SV.prepare(reqs, SV.TopoBank(3, 2048, 4) if args.serve_side_max > 512 else None)
    srv = SV.Server(precision=MIXED, hbm_limit=150 * 10 ** 9, max_classes=16, chunk_steps=16)
    rep = srv.serve(reqs, time_limit=args.serve_duration + args.serve_drain)
    d = rep.summary()
    d.update({"workload": f"Poisson {args.serve_rate}/s for {args.serve_duration} s (seed 3), hillslope or "
                          f"fractal squares, side log-uniform 32..{args.serve_side_max}, 5-10 classes, "
                          f"1-{args.serve_hyeto_max} hyetograph steps of 10-60 s at 0-150 mm/h, dx=1 m, "
                          "mixed form, 150 GB HBM admission limit",
              "latency": "arrival -> result fields (h, totsed) on the host"})
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="swehr", choices=["swehr", "reference"])
    ap.add_argument("--nx", type=int, default=4096)
    ap.add_argument("--ny", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--ens-count", type=int, default=256)
    ap.add_argument("--ens-warmup", type=int, default=800,
                    help="untimed pool steps before the timed ones (the scenarios pond and erode by then)")
    ap.add_argument("--ens-steps", type=int, default=200)
    ap.add_argument("--ens-solo-steps", type=int, default=50)
    ap.add_argument("--serve-rate", type=float, default=50.0)
    ap.add_argument("--serve-duration", type=float, default=60.0)
    ap.add_argument("--serve-drain", type=float, default=60.0)
    ap.add_argument("--serve-side-max", type=int, default=2048)
    ap.add_argument("--serve-hyeto-max", type=int, default=10)
    ap.add_argument("--serve-small", action="store_true",
                    help="a scaled stream one B200 keeps up with (sides to 512, 1-3 hyetograph steps, 10 s)")
    ap.add_argument("--steady-at", type=int, default=1000,
                    help="step at which the second (wet, steady) timed window starts; 0 to skip it")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = vis.split(",") if vis else [str(i) for i in range(64)]
        os.environ["CUDA_VISIBLE_DEVICES"] = devs[local]

    if args.impl == "reference":
        reference_arm(args, rank)
        return

    if world > 1:
        import torch
        torch.cuda.set_device(0)
    from swehr_b200.ranks import Ranks
    ranks = Ranks("nccl", timeout_s=600.0)
    barrier, max_over_ranks = ranks.barrier, ranks.max

    from swehr_b200.lib import Simulation
    from swehr_b200.params import FP64, MIXED
    case = bench_workload(args)
    S = case.sclass
    cells = case.cells()

    def window(prw, B, prof):
        """throughput and update-kernel roofline of a timed window (prof: the
        committed ncu summary of the same kernel in the same flow state)"""
        ms = max_over_ranks(prw.device_ms)
        n = max(int(prw.steps_this_call), 1)
        upd = prw.kernel_ms / n
        ach = B * cells / (upd / 1e3) / 1e9 if upd > 0 else None
        first = int(prw.steps) - n
        tb, ff = profiled(prof), profiled(prof, "fp64_flop_per_cell_step")
        return {"steps": f"{first}..{int(prw.steps)}", "value": world * cells * n / (ms / 1e3),
                "unit": "cell-steps/s", "ms_per_step": ms / n, "update_ms_avg": upd, "achieved_gbs": ach,
                "frac": (ach / hbm_peak()[0]) if ach else None, "traffic": tb * cells if tb else None,
                "fp64_tflops": ff * cells / (upd / 1e3) / 1e12 if (ff and upd > 0) else None,
                "profile": "profiles/" + prof}

    def timed_run(precision, clocks=None):
        """W warm-up steps, K timed steps; then, untimed, on to the steady
        window (the domain wets up over the first ~1000 steps: dry at step 25,
        58 % wet at 600, wet everywhere by 1000) and K more timed steps there."""
        if clocks:
            clocks.start()
        sim = Simulation(case, precision=precision)
        sim.advance(max_steps=args.warmup)
        barrier()
        sim.set_timing(True)
        t0 = time.time()
        pr = sim.advance(max_steps=args.steps)
        if clocks:
            clocks.window(t0, time.time())
        sim.set_timing(False)
        barrier()
        steady = None
        if args.steady_at > args.warmup + args.steps:
            sim.advance(max_steps=args.steady_at - (args.warmup + args.steps))
            barrier()
            sim.set_timing(True)
            t0 = time.time()
            steady = sim.advance(max_steps=args.steps)
            if clocks:
                clocks.window(t0, time.time())
            sim.set_timing(False)
            barrier()
        clk = clocks.stop() if clocks else None
        sim.close()
        return pr, clk, steady

    clocks = ClockSampler(local)
    pr, clk, st64 = timed_run(FP64, clocks)
    elapsed_ms = max_over_ranks(pr.device_ms)
    kernel_ms = pr.kernel_ms
    steps_done = pr.steps_this_call
    value = world * cells * steps_done / (elapsed_ms / 1e3)

    mixed = None
    if not args.no_mixed:
        prm, _, stm = timed_run(MIXED)
        em = max_over_ranks(prm.device_ms)
        vm = world * cells * prm.steps_this_call / (em / 1e3)
        um = prm.kernel_ms / max(prm.steps_this_call, 1)
        Bm = algo_bytes_mixed(S)
        tm = profiled_traffic("k_update_tile_f32_dry_fractal1024.md")
        mixed = {"value": vm, "unit": "cell-steps/s", "ms_per_step": em / max(prm.steps_this_call, 1),
                 "steps": int(prm.steps_this_call), "gpu_launches": int(prm.kernel_launches),
                 "over_fp64": vm / value,
                 "roofline": {"bound": "hbm", "achieved": Bm * cells / (um / 1e3) / 1e9 if um > 0 else None,
                              "peak": hbm_peak()[0], "unit": "GB/s",
                              "frac": (Bm * cells / (um / 1e3) / 1e9 / hbm_peak()[0]) if um > 0 else None,
                              "traffic": tm * cells if tm else None,
                              "algo_bytes_per_cell_step": Bm, "update_ms_avg": um},
                 "dtype": "f32 bulk; f64 z, infiltration, deposited mass, budgets",
                 "error_bar": "<=1e-4 relative L-inf on depth and concentration vs FP64 (tests/test_gpu_mixed.py)"}
        if stm is not None:
            mixed["steady"] = window(stm, algo_bytes_mixed(S), "k_update_tile_f32_wet_fractal1024.md")

    # end-to-end through the C ABI from host buffers: create (H2D of every
    # input) + the same steps + D2H of the fields SWEHR.c writes at the end
    # of its run (depth, uh, vh, topoout, ch = U_1, m, c, vel, maxvel,
    # maxdepth: SWEHR.c:1718-1747), wall-clock
    e2e = None
    if not args.no_e2e:
        barrier()
        t0 = time.perf_counter()
        s2 = Simulation(case)
        ta = time.perf_counter()
        s2.advance(max_steps=args.warmup + args.steps)
        tb = time.perf_counter()
        out = s2.fields(("h", "hu", "hv", "z", "totm", "totsed", "vel", "maxvel", "maxdepth"))
        out["U1"] = s2.field("U", 1)
        t1 = time.perf_counter()
        s2.close()
        h2d = case.topo.nbytes + (case.ks.nbytes if case.ks is not None else 0) + case.rain.nbytes
        d2h = sum(v.nbytes for v in out.values())
        e2e_val = world * cells * (args.warmup + args.steps) / max_over_ranks(t1 - t0)
        n_e2e = args.warmup + args.steps
        e2e = {"value": e2e_val, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d / n_e2e,
               "d2h_bytes_per_step": d2h / n_e2e,
               "scope": "swehr_create + swehr_advance + swehr_read_field of the ten result grids SWEHR.c writes "
                        "(depth uh vh topoout ch m c vel maxvel maxdepth), host buffers",
               "phases_s": {"create": ta - t0, "advance": tb - ta, "read": t1 - tb}}

    steady = window(st64, algo_bytes_f64(S), "k_update_tile_f64_wet_fractal1024.md") if st64 is not None else None
    if steady is not None and mixed is not None and mixed.get("steady"):
        mixed["steady"]["over_fp64"] = mixed["steady"]["value"] / steady["value"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, el, th, n = run_cpu_reference(case, 1024, 150, host_threads())
            cpu = {"value": v, "unit": "cell-steps/s", "cores": th, "kind": "reference",
                   "sample": f"SWEHR.c with its OpenMP pragmas on, 1024x1024 corner of the same domain, "
                             f"first {n} steps, {el:.1f} s"}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "cell-steps/s", "cores": host_threads(), "kind": "reference",
                   "sample": f"unavailable: {e}"}

    ensemble = serving = None
    if not args.no_ensemble:
        if world == 1:
            try:
                ensemble = ensemble_leg(args, ranks)
            except Exception as e:  # noqa: BLE001
                ensemble = {"error": repr(e)}
        else:
            ensemble = ensemble_leg(args, ranks)   # every rank takes the same collective steps
    if rank == 0 and world == 1 and not args.no_serving:
        try:
            serving = serving_leg(args)
        except Exception as e:  # noqa: BLE001
            serving = {"error": repr(e)}

    if rank == 0:
        peak, peak_kind = hbm_peak()
        B = algo_bytes_f64(S)
        upd_ms = kernel_ms / max(steps_done, 1)
        achieved = B * cells / (upd_ms / 1e3) / 1e9 if upd_ms > 0 else None
        tb = profiled_traffic("k_update_tile_f64_dry_fractal1024.md")
        fpk = fp64_peak()
        ff = profiled("k_update_tile_f64_dry_fractal1024.md", "fp64_flop_per_cell_step")
        fach = ff * cells / (upd_ms / 1e3) / 1e12 if (ff and upd_ms > 0) else None
        fp64 = {"peak_tflops": fpk, "peak_kind": "measured now (FMA chains, swehr_b200/csrc/swehr_probe.cu)",
                "flop_per_cell_step": ff, "achieved_tflops": fach,
                "frac": (fach / fpk) if (fach and fpk) else None,
                "flop_source": "ncu thread-instruction counters of the same kernel and window "
                               "(profiles/k_update_tile_f64_dry_fractal1024.md)"}
        traffic = tb * cells if tb else None
        line = {
            "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": steps_done, "warmup": args.warmup, "ms_per_step": elapsed_ms / max(steps_done, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded diamond-square topography, hyetograph and lognormal Ks; no dataset)",
            "config": {"workload": f"fractal {args.nx}x{args.ny} dx=2 S=7 plain FP64 (roofline domain), "
                                   f"steps {args.warmup}..{args.warmup + steps_done}",
                       "cells": cells, "sclass": S, "l2": "inputs larger than L2 (state 6.7 GB), no flush",
                       "parallelism": f"replicas x{world}", "impl": "swehr_b200 FP64, 2 kernels/step, CUDA graphs off "
                                                                  "(per-launch event timing)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "peak_kind": peak_kind, "kernel": "k_update (FP64)",
                         "algo_bytes_per_cell_step": B, "update_ms_avg": upd_ms, "fp64": fp64,
                         "limiter": "issue and dependency latency: neither HBM nor the FP64 pipe is saturated "
                                    "(ncu: DRAM, FP64 pipe and issue-active fractions and stall reasons in "
                                    "profiles/k_update_tile_f64_*_fractal1024.md)"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "steady_state": steady,
            "mixed_form": mixed,
            "batched_ensemble": ensemble,
            "serving": serving,
            "clocks": clk,
            "gpu_launches": int(pr.kernel_launches),
            "impl": "swehr",
        }
        print(json.dumps(line))
    ranks.close()


if __name__ == "__main__":
    main()
