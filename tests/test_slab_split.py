"""The row-slab decomposition of one domain (swehr_b200.slabs) run on the
CPU: gloo ranks each step the oracle on their slab plus a two-row halo,
refresh the halos from their neighbours before every step and take the
largest wave speed over all ranks' faces for the time step.  Their owned
rows must equal the whole-domain oracle bit for bit -- the evidence that
HALO = 2 rows and one scalar max per step are what a multi-GPU split of a
single domain needs (SWEHR.c:1135, 1243-1312, 1408)."""
import ctypes as C
import datetime
import os
import socket

import numpy as np
import pytest

from swehr_b200 import workloads as W
from swehr_b200.slabs import HALO, exchanges, plan

STEPS = 600


def _case():
    # cross-sloped, low cohesion (slope failure), inflow at j = ny (debris),
    # per-cell Ks, walls on three sides: every branch crosses the slab seams
    c = W.failure_tiny(slope_y=0.5, cohesion=5.0, nx=26, ny=14, S=3, seed=71, bndry=(0, 1, 1, 1), inflow=1,
                       rain_mmh=300.0, tend=1.0e6)
    return c


def _sub(case, span):
    a, b = span
    p = dict(case.params, nx=b - a + 1)
    return W.Case(case.name + f"_rows{a}_{b}", p, case.topo[a - 1:b].copy(), case.rain, case.ds, case.pfrac,
                  ks=None if case.ks is None else case.ks[a - 1:b].copy())


def test_plan_covers_rows_once():
    for nx, world in ((26, 2), (26, 3), (4096, 8), (9, 4)):
        slabs = plan(nx, world)
        own = [r for s in slabs for r in range(s.own[0], s.own[1] + 1)]
        assert own == list(range(1, nx + 1))
        for s in slabs:
            assert s.span[0] == max(1, s.own[0] - HALO) and s.span[1] == min(nx, s.own[1] + HALO)
        for src, rows, dst, _ in exchanges(slabs):
            assert slabs[src].own[0] <= rows[0] <= rows[1] <= slabs[src].own[1]
            assert slabs[dst].span[0] <= rows[0] <= rows[1] <= slabs[dst].span[1]
            assert rows[1] - rows[0] + 1 == HALO
    with pytest.raises(ValueError):
        plan(5, 3)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, outdir):
    import torch
    import torch.distributed as dist
    from harness import OracleRun
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    case = _case()
    slabs = plan(case.nx, world)
    me = slabs[rank]
    o = OracleRun(_sub(case, me.span), "shim")
    L = o.L
    L.orc_set_own.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.orc_step_prepare.restype = C.c_double
    L.orc_step_prepare.argtypes = [C.c_void_p]
    L.orc_step_commit.restype = C.c_int
    L.orc_step_commit.argtypes = [C.c_void_p, C.c_double]
    L.orc_rows.restype = C.c_int
    L.orc_rows.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]
    lo, hi = me.local_own
    L.orc_set_own(o.ctx, lo, hi)
    per_row = (12 + 3 * case.sclass) * case.ny
    for _ in range(STEPS):
        for src, rows, dst, _ in exchanges(slabs):
            n = rows[1] - rows[0] + 1
            a, b = rows[0] - me.span[0] + 1, rows[1] - me.span[0] + 1
            if rank == src:
                buf = np.empty(n * per_row)
                assert L.orc_rows(o.ctx, a, b, buf.ctypes.data, 0) == 0
                dist.send(torch.from_numpy(buf), dst)
            elif rank == dst:
                buf = np.empty(n * per_row)
                dist.recv(torch.from_numpy(buf), src)
                assert L.orc_rows(o.ctx, a, b, buf.ctypes.data, 1) == 0
        t = torch.tensor([L.orc_step_prepare(o.ctx)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        L.orc_step_commit(o.ctx, float(t.item()))
    f = o.fields()
    out = {k: (v[:, lo - 1:hi] if v.ndim == 3 else v[lo - 1:hi]) for k, v in f.items()}
    out["t"] = np.array(o.t)
    out["steps"] = np.array(o.steps)
    np.savez(os.path.join(outdir, f"slab{rank}.npz"), **out)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_split_matches_whole_domain(tmp_path, world):
    import torch.multiprocessing as mp
    from harness import OracleRun
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    case = _case()
    whole = OracleRun(case, "shim")
    whole.advance(max_steps=STEPS)
    ref = whole.fields()
    assert whole.counters()["fail"] > 0
    parts = [np.load(os.path.join(tmp_path, f"slab{r}.npz")) for r in range(world)]
    for part in parts:
        assert int(part["steps"]) == STEPS and float(part["t"]) == whole.t
    for name, arr in ref.items():
        got = np.concatenate([p[name] for p in parts], axis=-2 if arr.ndim == 3 else 0)
        assert got.shape == arr.shape, name
        assert np.array_equal(got, arr, equal_nan=True), name
