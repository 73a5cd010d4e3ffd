"""ragged.MixedPlan on the GPU: columns per lane chosen per pair from the
bucket table, one plan per choice on the batch's own packed buffers.  Each
pair's results equal, bit for bit, a single plan at that pair's choice; the
oracle bounds hold; CUDA-graph replay works."""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")


def _batch(seed=3, B=60):
    rng = np.random.default_rng(seed)
    ln = np.exp(rng.uniform(np.log(8), np.log(1500), size=(B, 2))).round().astype(np.int64)
    ln[0] = (0, 40)
    g = torch.Generator().manual_seed(seed)
    mats = [torch.randn(int(a), int(b), generator=g) * 1.5 for a, b in ln]
    return mats


@pytest.mark.parametrize("family", ["affine", "linear"])
def test_mixed_plan_equals_single_plans_per_pair(family):
    from orihime_b200 import ragged

    mats = _batch()
    flat, off, lens = ragged.pack(mats)
    flat = flat.cuda()
    params = dict(gap_open=-2.0, gap_ext=-0.5, temp=0.5) if family == "affine" else dict(gap=-1.0, temp=0.5)
    mp = ragged.MixedPlan(lens, off, family=family, device="cuda")
    assert len(set(mp.cols.tolist())) >= 2      # the batch spans several buckets
    out = mp.run(flat, **params)
    vals = mp.values(flat, **params)
    torch.cuda.synchronize()
    assert mp.status() == 0
    assert torch.equal(vals, out.value)
    maps = ragged.unpack(out.map, off, lens)
    single = {R: ragged.Plan(lens, off, family=family, device="cuda", cols_per_lane=R).run(flat, **params)
              for R in sorted(set(mp.cols.tolist()))}
    torch.cuda.synchronize()
    for b in range(len(mats)):
        r = single[int(mp.cols[b])]
        assert torch.equal(out.value[b], r.value[b])
        assert torch.equal(out.grad_temp[b], r.grad_temp[b])
        assert torch.equal(maps[b], ragged.unpack(r.map, off, lens)[b])
    # oracle on the pairs of each choice
    for R in single:
        b = int(np.nonzero(mp.cols == R)[0][-1])
        s = mats[b][None].numpy()
        if family == "affine":
            r32, r64 = O.affine(s, None, -2.0, -0.5, 0.5), O.affine(s, None, -2.0, -0.5, 0.5, dtype=np.float64)
        else:
            r32, r64 = O.linear(s, None, -1.0, 0.5), O.linear(s, None, -1.0, 0.5, dtype=np.float64)
        assert abs(float(out.value[b]) - r32["value"][0]) <= 1e-5 * abs(r32["value"][0])
        err = np.abs(maps[b].cpu().numpy() - r64["map"][0]).max()
        assert err <= max(1e-5, np.abs(r32["map"][0] - r64["map"][0]).max())


def test_mixed_plan_graph_replay():
    from orihime_b200 import ragged

    mats = _batch(5, 40)
    flat, off, lens = ragged.pack(mats)
    flat = flat.cuda()
    mp = ragged.MixedPlan(lens, off, family="affine", device="cuda")
    g, gout = mp.graph(flat, gap_open=-2.0, gap_ext=-0.5, temp=0.5)
    flat.mul_(0.7)
    g.replay()
    torch.cuda.synchronize()
    want = mp.run(flat, gap_open=-2.0, gap_ext=-0.5, temp=0.5)
    torch.cuda.synchronize()
    assert torch.equal(gout.value, want.value) and torch.equal(gout.map, want.map)


def test_eight_columns_per_lane_matches_oracle():
    from orihime_b200 import ragged

    mats = _batch(7, 12)
    flat, off, lens = ragged.pack(mats)
    plan = ragged.Plan(lens, off, family="affine", device="cuda", cols_per_lane=8)
    out = plan.run(flat.cuda(), gap_open=-2.0, gap_ext=-0.5, temp=0.5)
    torch.cuda.synchronize()
    maps = ragged.unpack(out.map.cpu(), off, lens)
    for b, m in enumerate(mats):
        if m.numel() == 0:
            continue
        s = m[None].numpy()
        r32, r64 = O.affine(s, None, -2.0, -0.5, 0.5), O.affine(s, None, -2.0, -0.5, 0.5, dtype=np.float64)
        assert abs(float(out.value[b]) - r32["value"][0]) <= 1e-5 * abs(r32["value"][0])
        assert np.abs(maps[b].numpy() - r64["map"][0]).max() <= max(1e-5, np.abs(r32["map"][0] - r64["map"][0]).max())
