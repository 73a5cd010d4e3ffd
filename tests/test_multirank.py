"""Multi-process host logic of bench.py on CPU ranks (gloo, world size 2).

Pairs are independent, so N GPUs split one pair list of N x 4096 pairs by
LPT on the pairs' computed cells: every rank computes the same partition and
runs its shard, no collective touches the data, and the reported time is the
max over ranks.  These tests run that host logic with gloo.
"""

import json
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    w, r, local = bench.dist_init(torch, backend="gloo")
    assert (w, r, local) == (world, rank, rank)
    ln, idx, shards = bench.shard_of(w, r, 64)
    bench.barrier(torch, w)
    t_max = bench.max_over_ranks(torch, w, 10.0 + r)
    # every rank takes the same collective steps: a second reduction agrees
    t_max2 = bench.max_over_ranks(torch, w, -float(r))
    # the reference arm is rank 0's alone: other ranks return at once
    rc_ref = bench.run_reference(type("A", (), {"steps": 1, "warmup": 0})()) if r != 0 else 0
    with open(os.path.join(outdir, f"rank{r}.json"), "w") as f:
        json.dump({"lengths": ln.tolist(), "index": idx.tolist(), "shards": [x.tolist() for x in shards],
                   "t_max": t_max, "t_max2": t_max2, "rc_ref": rc_ref}, f)
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_shards(tmp_path):
    sys.path.insert(0, ROOT)
    import bench

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert all(x["t_max"] == 11.0 for x in res)      # max over ranks
    assert all(x["t_max2"] == 0.0 for x in res)
    assert all(x["rc_ref"] == 0 for x in res)
    # both ranks computed the same partition of the 128-pair job, and each ran its own shard
    assert res[0]["shards"] == res[1]["shards"]
    i0, i1 = (np.array(x["index"]) for x in res)
    assert len(np.intersect1d(i0, i1)) == 0 and len(i0) + len(i1) == 128
    job = bench.workload_lengths(3, 128)
    for x, i in zip(res, (i0, i1)):
        assert np.array_equal(np.array(x["lengths"]), job[i])


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        assert bench.dist_init(torch, backend="gloo") == (1, 0, 0)
        assert bench.max_over_ranks(torch, 1, 3.5) == 3.5
    finally:
        os.environ.update(env)
