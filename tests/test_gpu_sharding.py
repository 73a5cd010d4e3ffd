"""ragged.ShardedPlan on the GPU: a packed batch split by LPT into shards,
each run as its own plan, gives the single plan's results bit for bit (pairs
are independent; the band decomposition of a pair does not depend on the
other pairs).  Two shards on one device stand in for two GPUs: the shards
never wait on each other."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")


@pytest.mark.parametrize("family", ["affine", "linear"])
def test_two_shards_equal_single_plan(family):
    from orihime_b200 import ragged

    rng = np.random.default_rng(7)
    ln = np.exp(rng.uniform(np.log(8), np.log(700), size=(40, 2))).round().astype(np.int64)
    ln[3] = (0, 12)
    g = torch.Generator().manual_seed(3)
    mats = [torch.randn(int(a), int(b), generator=g) * 1.5 for a, b in ln]
    flat, off, lens = ragged.pack(mats)
    params = dict(gap_open=-2.0, gap_ext=-0.5, temp=0.5) if family == "affine" else dict(gap=-1.0, temp=0.5)
    single = ragged.Plan(lens, off, family=family, device="cuda").run(flat.cuda(), **params)
    sp = ragged.ShardedPlan(lens, off, family=family, devices=["cuda:0", "cuda:0"])
    outs = sp.run(sp.scatter(flat.cuda()), **params)
    torch.cuda.synchronize()
    assert torch.equal(sp.gather_values(outs), single.value)
    for gidx, r in outs.items():
        idx = sp.shards[gidx]
        sub_off, sub_ln = ragged.layout(lens[idx])
        for k, b in enumerate(idx.tolist()):
            want = ragged.unpack(single.map, off, lens)[b]
            got = ragged.unpack(r.map, sub_off, sub_ln)[k]
            assert torch.equal(got, want), b
            assert torch.equal(r.grad_temp[k], single.grad_temp[b])
