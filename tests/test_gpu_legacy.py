"""The 18 legacy soft_sw* / soft_nw* ops (src/sw*/registry.cpp,
src/nw/registry.cpp, src/sw*/torch_cuda.cpp:803-830, :917-946,
src/nw/torch_cuda.cpp:795-821) run the namespaced op bodies under their old
names: the same results bit for bit, param_type selecting the parameter,
autograd through the tensor-parameter forward."""

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
    if len(_ops.LEGACY_DEFINED_HERE) != len(_ops.LEGACY_SCHEMAS):
        pytest.skip("the reference extension defined the legacy schemas; they stay its own")


def _scores(*shape, seed=0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(*shape, generator=g) * 1.5).cuda()


def _eq(a, b):
    if isinstance(a, (list, tuple)):
        return len(a) == len(b) and all(_eq(x, y) for x, y in zip(a, b))
    return torch.equal(a, b)


def test_legacy_ops_equal_namespaced_ops():
    s = _scores(3, 40, 57)
    v = _scores(3, 40, 57, seed=1)
    ln = torch.tensor([[40, 57], [13, 9], [40, 30]], dtype=torch.int32).cuda()
    for lengths in (None, ln):
        assert _eq(o.soft_sw_affine_float(s, *AFF, lengths), o.sw_affine_forward(s, *AFF, lengths))
        assert _eq(o.soft_sw_float(s, *LIN, lengths), o.sw_forward(s, *LIN, lengths))
        vg = o.soft_sw_affine_with_grads(s, *AFF, lengths)
        assert _eq(vg[:2], o.sw_affine_forward(s, *AFF, lengths))
        assert _eq(vg[2:], o.sw_affine_value_grad_params(s, *AFF, lengths))
        lg = o.soft_sw_with_grads(s, *LIN, lengths)
        assert _eq(lg[:2], o.sw_forward(s, *LIN, lengths))
        assert _eq(lg[2:], o.sw_value_grad_params(s, *LIN, lengths))
        assert _eq(o.soft_sw_affine_hvp(s, v, *AFF, lengths), o.sw_affine_marginals_hvp(s, v, *AFF, lengths))
        assert _eq(o.soft_sw_hvp(s, v, *LIN, lengths), o.sw_marginals_hvp(s, v, *LIN, lengths))
        for k, name in enumerate(("gap_open", "gap_ext", "temp")):
            assert _eq(o.soft_sw_affine_param_jacobian(s, k, *AFF, lengths),
                       getattr(o, f"sw_affine_marginals_grad_{name}")(s, *AFF, lengths))
        for k, name in enumerate(("gap", "temp")):
            assert _eq(o.soft_sw_param_jacobian(s, k, *LIN, lengths),
                       getattr(o, f"sw_marginals_grad_{name}")(s, *LIN, lengths))
        assert _eq(o.soft_sw_affine_backward_full(s, v, *AFF, lengths),
                   o.sw_affine_marginals_backward(s, v, *AFF, lengths))
        assert _eq(o.soft_sw_backward_full(s, v, *LIN, lengths), o.sw_marginals_backward(s, v, *LIN, lengths))
    with pytest.raises(RuntimeError, match="param_type must be 0, 1, or 2"):
        o.soft_sw_affine_param_jacobian(s, 3, *AFF, None)
    with pytest.raises(RuntimeError, match="param_type must be 0 or 1"):
        o.soft_nw_param_jacobian(s, 2, *LIN, None)


def test_legacy_nw_ops_equal_namespaced_ops():
    s = _scores(3, 40, 57)
    v = _scores(3, 40, 57, seed=1)
    ln = torch.tensor([[40, 57], [13, 9], [0, 30]], dtype=torch.int32).cuda()
    for lengths in (None, ln):
        assert _eq(o.soft_nw_float(s, *LIN, lengths), o.nw_forward(s, *LIN, lengths))
        lg = o.soft_nw_with_grads(s, *LIN, lengths)
        assert _eq(lg[:2], o.nw_forward(s, *LIN, lengths))
        assert _eq(lg[2:], o.nw_value_grad_params(s, *LIN, lengths))
        assert _eq(o.soft_nw_hvp(s, v, *LIN, lengths), o.nw_marginals_hvp(s, v, *LIN, lengths))
        for k, name in enumerate(("gap", "temp")):
            assert _eq(o.soft_nw_param_jacobian(s, k, *LIN, lengths),
                       getattr(o, f"nw_marginals_grad_{name}")(s, *LIN, lengths))
        assert _eq(o.soft_nw_backward_full(s, v, *LIN, lengths), o.nw_marginals_backward(s, v, *LIN, lengths))
    full = torch.tensor([[40, 57]] * 3, dtype=torch.int32).cuda()
    assert _eq(o.soft_nw(s, torch.tensor(-1.0).cuda(), torch.tensor(0.5).cuda(), full),
               o.nw_forward(s, *LIN, full))


def test_legacy_tensor_parameter_forward_is_differentiable():
    s = _scores(2, 30, 33).requires_grad_(True)
    ln = torch.tensor([[30, 33], [20, 11]], dtype=torch.int32).cuda()
    go, ge, T = (torch.tensor(x, device="cuda", requires_grad=True) for x in AFF)
    v, m = o.soft_sw_affine(s, go, ge, T, ln)
    (v.sum() + (m * m).sum()).backward()
    s2 = s.detach().clone().requires_grad_(True)
    go2, ge2, T2 = (torch.tensor(x, device="cuda", requires_grad=True) for x in AFF)
    v2, m2 = o.sw_affine_forward_t(s2, go2, ge2, T2, ln)
    (v2.sum() + (m2 * m2).sum()).backward()
    assert torch.equal(s.grad, s2.grad)
    for a, b in ((go, go2), (ge, ge2), (T, T2)):
        assert torch.equal(a.grad, b.grad)
