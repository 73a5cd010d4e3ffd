"""Public functions under CUDA autocast, as the reference's
tests/test_autocast.py checks them: low-precision inputs compute in FP32, the
map and value back-propagate after the context exits, and every gradient is
the FP32 gradient rounded once to the input's dtype."""

import pytest
import torch

import orihime_b200 as ohm

pytestmark = pytest.mark.gpu

CASES = {
    "sw": dict(gap_score=-0.7, temperature=0.9),
    "sw_affine": dict(gap_open_score=-1.0, gap_extend_score=-0.3, temperature=0.9),
    "nw": dict(gap_score=-0.7, temperature=0.9),
    "nw_affine": dict(gap_open_score=-1.0, gap_extend_score=-0.3, temperature=0.9),
    "sv_linear": dict(gap_score=-0.7, temperature=0.9),
    "sv_affine": dict(gap_open_score=-1.0, gap_extend_score=-0.3, temperature=0.9),
}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")


def _x(name):
    g = torch.Generator().manual_seed(4200 + list(CASES).index(name))
    return (0.5 * torch.randn(2, 12, 17, generator=g)).cuda()


@pytest.mark.parametrize("name", list(CASES))
def test_map_backward_after_autocast_exit(name):
    x = _x(name).half().requires_grad_()
    with torch.autocast("cuda", dtype=torch.float16):
        m = getattr(ohm, name)(x, **CASES[name])
    assert m.dtype == torch.float32 and torch.isfinite(m).all()
    m.square().sum().backward()
    assert x.grad is not None and x.grad.dtype == torch.float16 and torch.isfinite(x.grad).all()
    ref = x.detach().float().requires_grad_()
    getattr(ohm, name)(ref, **CASES[name]).square().sum().backward()
    assert torch.equal(x.grad, ref.grad.half())


@pytest.mark.parametrize("dtype", (torch.float16, torch.bfloat16), ids=("fp16", "bf16"))
@pytest.mark.parametrize("name", list(CASES))
def test_value_backward_after_autocast_exit(name, dtype):
    fn = getattr(ohm, f"{name}_value")
    base = _x(name).to(dtype)
    pnames = list(CASES[name])
    pv = [torch.tensor(v, device="cuda").to(dtype) for v in CASES[name].values()]
    ex = base.float().requires_grad_()
    ep = [p.float().requires_grad_() for p in pv]
    want = fn(ex, **dict(zip(pnames, ep)))
    want.sum().backward()
    ax = base.clone().requires_grad_()
    ap = [p.clone().requires_grad_() for p in pv]
    with torch.autocast("cuda", dtype=dtype):
        got = fn(ax, **dict(zip(pnames, ap)))
    assert got.dtype == torch.float32
    torch.testing.assert_close(got, want, rtol=1e-5, atol=1e-5)
    got.sum().backward()
    assert ax.grad.dtype == dtype and torch.equal(ax.grad, ex.grad.to(dtype))
    for a, e in zip(ap, ep):
        assert a.grad.dtype == dtype and torch.equal(a.grad, e.grad.to(dtype))


@pytest.mark.parametrize("name", list(CASES))
def test_bf16_value_vjp_pullback_after_autocast_exit(name):
    fn = getattr(ohm, f"{name}_value")
    x = _x(name).bfloat16()
    with torch.autocast("cuda", dtype=torch.bfloat16):
        out, pull = torch.func.vjp(lambda a: fn(a, **CASES[name]), x)
    (g,) = pull(torch.ones_like(out))
    ref = x.float().requires_grad_()
    fn(ref, **CASES[name]).sum().backward()
    assert g.dtype == torch.bfloat16 and torch.equal(g, ref.grad.bfloat16())
