"""vmap, autocast and torch.compile through the registrations of the namespaced ops,
on the GPU (reference: orihime/_ops.py:178-406, orihime/_compile.py:323-452)."""

import pytest
import torch

from orihime_b200 import _ops

pytestmark = pytest.mark.gpu

o = torch.ops.orihime
AFF = (-2.0, -0.5, 0.5)
LIN = (-1.0, 0.5)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    if len(_ops.DEFINED_HERE) != len(_ops.SCHEMAS):
        pytest.skip("the reference extension defined the schemas; its package registers these")


def _scores(*shape, seed=0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(*shape, generator=g) * 1.5).cuda()


def test_vmap_forward_and_hvp_match_per_element_calls():
    s = _scores(3, 2, 37, 50)
    v = _scores(3, 2, 37, 50, seed=1)
    val, mp = torch.func.vmap(lambda a: o.sw_affine_forward(a, *AFF, None))(s)
    for k in range(3):
        v1, m1 = o.sw_affine_forward(s[k].contiguous(), *AFF, None)
        assert torch.equal(val[k], v1) and torch.equal(mp[k], m1)
    h = torch.func.vmap(lambda a, b: o.sw_marginals_hvp(a, b, *LIN, None))(s, v)
    for k in range(3):
        assert torch.allclose(h[k], o.sw_marginals_hvp(s[k].contiguous(), v[k].contiguous(), *LIN, None),
                              rtol=1e-5, atol=1e-7)


def test_vmap_mapped_lengths_and_unmapped_scores():
    s = _scores(2, 40, 33)
    ln = torch.tensor([[[40, 33], [12, 20]], [[5, 30], [40, 7]]], dtype=torch.int32).cuda()
    val, mp = torch.func.vmap(lambda n: o.sw_forward(s, *LIN, n), in_dims=0)(ln)
    for k in range(2):
        v1, m1 = o.sw_forward(s, *LIN, ln[k].contiguous())
        assert torch.equal(val[k], v1) and torch.equal(mp[k], m1)


def test_vmap_marginals_backward_sums_per_element():
    s = _scores(2, 3, 30, 26)
    g = _scores(2, 3, 30, 26, seed=3)
    out = torch.func.vmap(lambda a, b: o.sw_affine_marginals_backward(a, b, *AFF, None))(s, g)
    assert out[0].shape == (2, 3, 30, 26) and all(t.shape == (2, 1) for t in out[1:])
    for k in range(2):
        ref = o.sw_affine_marginals_backward(s[k].contiguous(), g[k].contiguous(), *AFF, None)
        assert torch.allclose(out[0][k], ref[0], rtol=1e-5, atol=1e-7)
        for a, b in zip(out[1:], ref[1:]):
            assert torch.allclose(a[k], b, rtol=1e-5, atol=1e-6)


def test_autocast_runs_in_float32():
    s = _scores(2, 64, 48).half()
    with torch.autocast("cuda", dtype=torch.float16):
        v, m = o.sw_affine_forward(s, *AFF, None)
    assert v.dtype == torch.float32 and m.dtype == torch.float32
    v32, m32 = o.sw_affine_forward(s.float(), *AFF, None)
    assert torch.equal(v, v32) and torch.equal(m, m32)


def test_torch_compile_fullgraph_matches_eager():
    s = _scores(2, 50, 60)

    def loss(a):
        v, m = o.sw_affine_forward(a, *AFF, None)
        return v.sum() + (m * a).sum()

    got = torch.compile(loss, fullgraph=True)(s)
    assert torch.allclose(got, loss(s), rtol=1e-6, atol=1e-5)


def test_vmap_global_alignment_ops_match_per_element_calls():
    s = _scores(2, 3, 29, 41)
    v = _scores(2, 3, 29, 41, seed=2)
    val, mp = torch.func.vmap(lambda a: o.nw_forward(a, *LIN, None))(s)
    h = torch.func.vmap(lambda a, b: o.nw_marginals_hvp(a, b, *LIN, None))(s, v)
    for k in range(2):
        v1, m1 = o.nw_forward(s[k].contiguous(), *LIN, None)
        assert torch.equal(val[k], v1) and torch.equal(mp[k], m1)
        assert torch.allclose(h[k], o.nw_marginals_hvp(s[k].contiguous(), v[k].contiguous(), *LIN, None),
                              rtol=1e-5, atol=1e-7)
