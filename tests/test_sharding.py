"""One pair list across GPUs (ragged.ShardedPlan): the LPT partition, the
shard packing and the value gather, on CPU.

The partition runs on the host, so it is checked here on the bench's own
batch.  The gather is a collective; a world-size-2 gloo group runs it with
per-pair values from the oracle standing in for each rank's kernel results
(the kernels themselves need a GPU: tests/test_gpu_sharding.py)."""

import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.mark.parametrize("parts", [2, 4, 8])
def test_lpt_balances_the_bench_batch(parts):
    import bench
    from orihime_b200 import ragged

    ln = bench.workload_lengths(3)
    shards = ragged.lpt_partition(ln, parts)
    allidx = np.sort(np.concatenate(shards))
    assert np.array_equal(allidx, np.arange(len(ln)))          # every pair exactly once
    cost = ragged.pair_cost(ln)
    loads = np.array([cost[s].sum() for s in shards], dtype=np.float64)
    assert loads.max() <= 1.05 * loads.mean(), loads
    again = ragged.lpt_partition(ln, parts)                       # deterministic
    assert all(np.array_equal(a, b) for a, b in zip(shards, again))


def test_pair_cost_counts_band_work():
    from orihime_b200 import ragged

    c = ragged.pair_cost([[100, 1], [100, 128], [100, 129], [0, 50]])
    assert c[0] == c[1] == 131 * 128      # one band of 128 columns, 100 + 31 steps
    assert c[2] == 2 * 131 * 128          # a second, mostly dead band
    assert c[3] == 0


def test_shard_scores_round_trip():
    from orihime_b200 import ragged

    g = torch.Generator().manual_seed(0)
    mats = [torch.randn(int(a), int(b), generator=g) for a, b in [(3, 5), (1, 1), (7, 4), (0, 3), (6, 9)]]
    flat, off, ln = ragged.pack(mats)
    idx = np.array([4, 0, 3])
    sub, soff, sln = ragged.shard_scores(flat, off, ln, idx)
    assert np.array_equal(sln, ln[idx])
    for k, m in enumerate(ragged.unpack(sub, soff, sln)):
        assert torch.equal(m, mats[int(idx[k])])


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from oracle import oracle as O
    from orihime_b200 import ragged

    dist.init_process_group("gloo")
    rng = np.random.default_rng(5)
    ln = rng.integers(1, 40, size=(23, 2))
    shards = ragged.lpt_partition(ln, world)
    g = torch.Generator().manual_seed(1)
    mats = [torch.randn(int(a), int(b), generator=g) for a, b in ln]
    # this rank's pairs only (the kernel's results, stood in for by the oracle)
    mine = [float(O.affine(mats[b].numpy()[None], None, -2.0, -0.5, 0.5)["value"][0]) for b in shards[rank]]
    vals = ragged.all_gather_values(torch.tensor(mine, dtype=torch.float32), shards, len(ln))
    np.save(os.path.join(outdir, f"rank{rank}.npy"), vals.numpy())
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_gather_matches_single_rank(tmp_path):
    from oracle import oracle as O

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    rng = np.random.default_rng(5)
    ln = rng.integers(1, 40, size=(23, 2))
    g = torch.Generator().manual_seed(1)
    mats = [torch.randn(int(a), int(b), generator=g) for a, b in ln]
    want = np.array([O.affine(m.numpy()[None], None, -2.0, -0.5, 0.5)["value"][0] for m in mats],
                    dtype=np.float32)
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.array_equal(got, want)
