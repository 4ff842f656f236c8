"""The multi-rank path on CPU: two `gloo` ranks (one process per GPU in a real
run) exercising what `bench.py --gpus N` and the sharding helper do across
ranks — independent seeded replicas, the max over ranks of a time, and a
deterministic, balanced split of independent transforms that every rank
computes alike without communication.  No GPU is used.
"""
import json
import os
import socket

import pytest

from ducc_b200 import shard


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WEIGHTS = [1e3 * (1 + (i * 37) % 17) * (4 if i % 5 == 0 else 1) for i in range(64)]


def _worker(rank, world, port, outdir):
    import datetime

    import torch
    import torch.distributed as td

    td.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                          world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        t = bench.max_over_ranks(1.5 + rank, torch.device("cpu"), True)
        coord, vals, grid = bench.make_inputs(1234 + rank, 1000, 16)
        mine = shard.local_units(WEIGHTS, rank, world)
        gathered = [None] * world
        td.all_gather_object(gathered, {"units": mine, "c0": float(coord[0, 0])})
        td.barrier()
    finally:
        td.destroy_process_group()
    with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
        json.dump({"max": t, "gathered": gathered}, f)


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(world)]
    for r in res:
        assert r["max"] == 2.5                       # the slower rank's time
        g = r["gathered"]
        assert g[0]["c0"] != g[1]["c0"]              # independent seeded replicas
        units = sorted(g[0]["units"] + g[1]["units"])
        assert units == list(range(len(WEIGHTS)))    # disjoint cover of all units
        assert g == res[0]["gathered"]               # every rank saw the same split


def test_assign_balances_and_is_deterministic():
    for world in (1, 2, 3, 8):
        parts = shard.assign(WEIGHTS, world)
        assert sorted(sum(parts, [])) == list(range(len(WEIGHTS)))
        loads = [sum(WEIGHTS[i] for i in p) for p in parts]
        # longest-processing-time bound: no rank exceeds the mean by more than
        # the largest unit
        assert max(loads) <= sum(WEIGHTS) / world + max(WEIGHTS)
        assert parts == shard.assign(WEIGHTS, world)
        assert all(shard.local_units(WEIGHTS, r, world) == parts[r] for r in range(world))
    with pytest.raises(ValueError):
        shard.assign([1.0, -1.0], 2)
    with pytest.raises(ValueError):
        shard.local_units([1.0], 2, 2)
