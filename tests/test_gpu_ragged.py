"""Packed ragged batches on the GPU: per-pair parity with the oracle, bitwise
agreement with the padded drop-in, zeroed pitch padding, CUDA-graph replay."""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")


def _emb(N, M, seed, d=64):
    g = torch.Generator().manual_seed(seed)
    e = torch.randn(N, d, generator=g)
    f = torch.randn(M, d, generator=g)
    return (3 * e @ f.T / d ** 0.5).float()


def _lengths(B, seed, lo=1, hi=400):
    rng = np.random.default_rng(seed)
    ln = np.exp(rng.uniform(np.log(lo), np.log(hi), size=(B, 2))).round().astype(np.int64)
    ln[0] = (0, 17)
    ln[1] = (9, 0)
    return ln


def _lib_cols(fam_code, L2, params):
    from orihime_b200 import _lib

    return _lib.load().swb_cols_per_lane(fam_code, int(L2), params.get("gap_open", params.get("gap", 0.0)),
                                         params.get("gap_ext", 0.0), params["temp"])


@pytest.mark.parametrize("family", ["affine", "linear"])
@pytest.mark.parametrize("cols", [2, 4, 8])
def test_ragged_matches_oracle_and_padded(family, cols):
    from orihime_b200 import ragged

    ln = _lengths(24, 1)
    mats = [_emb(int(a), int(b), 100 + i) for i, (a, b) in enumerate(ln)]
    flat, off, lens = ragged.pack(mats)
    plan = ragged.Plan(lens, off, family=family, device="cuda", cols_per_lane=cols)
    params = dict(gap_open=-2.0, gap_ext=-0.5, temp=0.5) if family == "affine" else dict(gap=-1.0, temp=0.5)
    out = plan.run(flat.cuda(), **params)
    assert plan.status() == 0
    maps = ragged.unpack(out.map.cpu(), off, lens)
    full = out.map.cpu()
    for b, (L1, L2) in enumerate(lens.tolist()):
        p = ragged.pitch_of(L2)
        if L1 * p:
            pad = full[int(off[b]):int(off[b]) + L1 * p].view(L1, p)[:, L2:]
            assert not pad.any(), "pitch padding must be written as 0"
        if L1 * L2 == 0:
            assert float(out.value[b]) == 0.0
            continue
        s = mats[b][None]
        if family == "affine":
            v, m = torch.ops.orihime.sw_affine_forward(s.cuda(), -2.0, -0.5, 0.5, None)
            r32 = O.affine(s.numpy(), None, -2.0, -0.5, 0.5)
            r64 = O.affine(s.numpy(), None, -2.0, -0.5, 0.5, dtype=np.float64)
        else:
            v, m = torch.ops.orihime.sw_forward(s.cuda(), -1.0, 0.5, None)
            r32 = O.linear(s.numpy(), None, -1.0, 0.5)
            r64 = O.linear(s.numpy(), None, -1.0, 0.5, dtype=np.float64)
        fam_code = 3 if family == "affine" else 1
        pad_cols = _lib_cols(fam_code, L2, params)
        if cols == pad_cols:  # same per-pair schedule as the padded drop-in: identical bits
            assert torch.equal(v.cpu()[0], out.value.cpu()[b])
            assert torch.equal(m.cpu()[0], maps[b])
        rel = abs(float(out.value[b]) - r32["value"][0]) / abs(r32["value"][0])
        assert rel <= 1e-5
        err = np.abs(maps[b].numpy() - r64["map"][0]).max()
        ref_err = np.abs(r32["map"][0] - r64["map"][0]).max()
        assert err <= max(1e-5, ref_err), (b, err, ref_err)


def test_ragged_cuda_graph_replay():
    from orihime_b200 import ragged

    ln = _lengths(40, 2, 32, 600)
    mats = [_emb(int(a), int(b), 200 + i) for i, (a, b) in enumerate(ln)]
    flat, off, lens = ragged.pack(mats)
    plan = ragged.Plan(lens, off, family="affine", device="cuda")
    static = flat.cuda()
    ref = plan.run(static.clone(), gap_open=-2.0, gap_ext=-0.5, temp=0.5)
    ref_v, ref_m = ref.value.clone(), ref.map.clone()
    g, out = plan.graph(static, gap_open=-2.0, gap_ext=-0.5, temp=0.5)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out.value, ref_v) and torch.equal(out.map, ref_m)
    # new scores through the same graph
    static.mul_(0.5)
    g.replay()
    direct = plan.run(static.clone(), gap_open=-2.0, gap_ext=-0.5, temp=0.5)
    torch.cuda.synchronize()
    assert torch.equal(out.value, direct.value) and torch.equal(out.map, direct.map)
    assert not torch.equal(out.value, ref_v)


def test_streamed_plan_from_pinned_host_matches_plan():
    """Copy/compute-overlapped run from pinned host memory: same bits as one Plan."""
    from orihime_b200 import ragged

    ln = _lengths(37, 3, 16, 500)
    mats = [_emb(int(a), int(b), 300 + i) for i, (a, b) in enumerate(ln)]
    flat, off, lens = ragged.pack(mats)
    host = flat.pin_memory()
    params = dict(gap_open=-2.0, gap_ext=-0.5, temp=0.5)
    ref = ragged.Plan(lens, off, family="affine", device="cuda").run(flat.cuda(), **params)
    sp = ragged.StreamedPlan(lens, off, family="affine", device="cuda", parts=5)
    assert len(sp.groups) == 5 and sp.groups[0][0] == 0 and sp.groups[-1][1] == len(lens)
    for _ in range(2):  # the second call reuses the device buffers
        out = sp.run(host, **params)
        torch.cuda.synchronize()
        assert sp.status() == 0
        assert torch.equal(out.value, ref.value) and torch.equal(out.map, ref.map)
        assert torch.equal(out.grad_open, ref.grad_open) and torch.equal(out.grad_temp, ref.grad_temp)


@pytest.mark.parametrize("family", ["affine", "linear"])
@pytest.mark.parametrize("cols", [2, 4])
def test_ragged_values_only_equal_full_run(family, cols):
    """Plan.values (forward wavefront only) gives the full run's values bit
    for bit, including empty pairs."""
    from orihime_b200 import ragged

    ln = _lengths(40, 7)
    mats = [_emb(int(a), int(b), 300 + i) for i, (a, b) in enumerate(ln)]
    flat, off, lens = ragged.pack(mats)
    plan = ragged.Plan(lens, off, family=family, device="cuda", cols_per_lane=cols)
    params = dict(gap_open=-2.0, gap_ext=-0.5, temp=0.5) if family == "affine" else dict(gap=-1.0, temp=0.5)
    fd = flat.cuda()
    full = plan.run(fd, **params).value.clone()
    vals = plan.values(fd, **params)
    again = plan.values(fd, **params)
    assert plan.status() == 0
    assert torch.equal(vals, full) and torch.equal(again, full)
