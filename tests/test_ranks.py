"""Multi-process host logic on the CPU (gloo, world size 2): the rank
helpers bench.py uses around its timed regions, and the deterministic
placement of independent scenarios over GPUs."""
import json
import os
import socket

import pytest

from swehr_b200.ranks import shard


def test_shard_balances_and_covers():
    w = [float(s * s) for s in (1024, 64, 512, 900, 100, 300, 700, 64, 1000, 256)]
    for world in (1, 2, 3, 4, 8):
        parts = shard(w, world)
        assert len(parts) == world
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(w)))
        loads = [sum(w[k] for k in p) for p in parts]
        # greedy largest-first: no rank exceeds the mean by more than the largest item
        assert max(loads) <= sum(w) / world + max(w)
        assert all(p == sorted(p) for p in parts)
    assert shard(w, 2) == shard(list(w), 2)       # deterministic
    assert shard([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard(w, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, outdir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from swehr_b200.ranks import Ranks, shard as shard_
    r = Ranks("gloo", timeout_s=60.0)
    r.barrier()
    # a rank's device time and work, combined the way bench.py reports them
    ms = [12.5, 20.0][rank]
    work = [3e9, 1e9][rank]
    res = {"rank": r.rank, "world": r.world, "max_ms": r.max(ms), "sum_work": r.sum(work),
           "mine": shard_([5.0, 1.0, 4.0, 2.0, 3.0], r.world)[r.rank]}
    r.barrier()
    r.close()
    with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_ranks_gloo_world2(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    got = [json.load(open(os.path.join(tmp_path, f"rank{k}.json"))) for k in range(2)]
    for k, g in enumerate(got):
        assert g["rank"] == k and g["world"] == 2
        assert g["max_ms"] == 20.0 and g["sum_work"] == 4e9
    # together the two shards cover every item once, split by weight 8 : 7
    assert sorted(got[0]["mine"] + got[1]["mine"]) == [0, 1, 2, 3, 4]
    assert all(g["mine"] == sorted(g["mine"]) for g in got)
    loads = [sum([5.0, 1.0, 4.0, 2.0, 3.0][i] for i in g["mine"]) for g in got]
    assert sorted(loads) == [7.0, 8.0]
