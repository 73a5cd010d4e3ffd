"""Checks of the raw tier (orihime_b200.raw), shared by the CPU run
(oracle-backed kernels) and the GPU run of tests/test_raw_tier.py."""

from __future__ import annotations

import torch

import orihime_b200 as ohm

PARAMS = {
    "sw": dict(gap_score=-0.7, temperature=0.9),
    "sw_affine": dict(gap_open_score=-1.0, gap_extend_score=-0.3, temperature=0.9),
    "nw": dict(gap_score=-0.7, temperature=0.9),
    "nw_affine": dict(gap_open_score=-1.0, gap_extend_score=-0.3, temperature=0.9),
    "sv_linear": dict(gap_score=-0.7, temperature=0.9),
    "sv_affine": dict(gap_open_score=-1.0, gap_extend_score=-0.3, temperature=0.9),
}
PUBLIC_OP = {"sv_linear": "sv"}


def check_values(family, device):
    """vjp_one / vjp equal the named backward's parameter fields (float
    parameter: shape [1]; tensor parameter: its own shape), and the kernel
    bindings equal the ops they bind."""
    raw = getattr(ohm.raw, family)
    op = getattr(ohm.ops, PUBLIC_OP.get(family, family))
    g = torch.Generator().manual_seed(77)
    x = (0.5 * torch.randn(2, 5, 6, generator=g)).to(device)
    cot = torch.randn(2, 5, 6, generator=g).to(device)
    kw = PARAMS[family]
    ref = op.backward(x, grad_map=cot, **kw)
    for f in raw.vjp_fields:
        one = raw.vjp_one(x, wrt=f, cotangent=cot, **kw)
        assert one.shape == (1,), (f, one.shape)
        torch.testing.assert_close(one.reshape(()), ref[f].reshape(()), rtol=1e-6, atol=1e-6)
    d = raw.vjp(x, wrt=raw.vjp_fields, cotangent=cot, **kw)
    assert list(d) == list(raw.vjp_fields)
    tkw = {k: torch.tensor([v], device=device, dtype=torch.float32) for k, v in kw.items()}
    for f in raw.vjp_fields:
        t = raw.vjp_one(x, wrt=f, cotangent=cot, **tkw)
        assert t.shape == (1,) and t.dtype == torch.float32
        torch.testing.assert_close(t, d[f], rtol=1e-6, atol=1e-6)
    fam_ops = torch.ops.orihime
    vals = list(kw.values())
    v1, m1 = raw.forward(x, *vals)
    v2, m2 = getattr(fam_ops, f"{family}_forward")(x, *vals, None)
    assert torch.equal(v1, v2) and torch.equal(m1, m2)
    ln = torch.tensor([[5, 6], [3, 4]], dtype=torch.int32, device=device)
    v3, m3 = raw.forward(x, *vals, ln)                      # lengths positionally, as in the reference
    v4, m4 = raw.forward(x, *vals, lengths=ln)
    assert torch.equal(v3, v4) and torch.equal(m3, m4) and not m3[1, 3:].any()
    h1 = raw.marginals_hvp(x, cot, *vals)
    h2 = getattr(fam_ops, f"{family}_marginals_hvp")(x, cot, *vals, None)
    assert torch.equal(h1, h2)


def check_errors(family, device):
    """The raw contract's errors, raised before any kernel runs."""
    raw = getattr(ohm.raw, family)
    x = torch.zeros(1, 3, 4, device=device)
    cot = torch.zeros(1, 3, 4, device=device)
    kw = PARAMS[family]
    cases = [
        (dict(wrt=1, cotangent=cot), TypeError, "wrt must be a string"),
        (dict(wrt="nope", cotangent=cot), ValueError, "invalid wrt field 'nope'"),
        (dict(wrt=raw.vjp_fields[0], cotangent=cot[:, :2]), ValueError, "cotangent must have same shape as map"),
        (dict(wrt=raw.vjp_fields[0], cotangent=cot.double()), TypeError, "cotangent must have dtype torch.float32"),
        (dict(wrt=raw.vjp_fields[0], cotangent=torch.zeros(1, 4, 3, device=device).transpose(1, 2)),
         ValueError, "cotangent must be contiguous"),
        (dict(wrt=raw.vjp_fields[0], cotangent=[0.0]), TypeError, "cotangent must be a tensor"),
    ]
    for args, exc, msg in cases:
        try:
            raw.vjp_one(x, **args, **kw)
        except exc as e:
            assert msg in str(e), (msg, str(e))
        else:
            raise AssertionError(f"{family}: {msg} must raise {exc.__name__}")
    for wrt, exc, msg in ((list(raw.vjp_fields), TypeError, "wrt must be a tuple"),
                          ((raw.vjp_fields[0],) * 2, ValueError, "must not contain duplicates")):
        try:
            raw.vjp(x, wrt=wrt, cotangent=cot, **kw)
        except exc as e:
            assert msg in str(e), (msg, str(e))
        else:
            raise AssertionError(f"{family}: {msg} must raise")
    vals = list(kw.values())
    for fn, name in ((raw.marginals_hvp, "tangent"), (raw.marginals_backward, "cotangent")):
        try:
            fn(x, cot.double(), *vals)
        except RuntimeError as e:
            assert f"{name} must have dtype torch.float32" in str(e), str(e)
        else:
            raise AssertionError(f"{family}: a float64 {name} must raise RuntimeError")
