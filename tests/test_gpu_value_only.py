"""Value-only ops (orihime_b200::sw_value / sw_affine_value, C ABI
swb_sw_value / swb_sw_affine_value): the forward wavefront alone, folded to S
per pair.  No reference counterpart; the values must equal the full forward's
bit for bit, and Operator.value uses them whenever no gradient can flow."""

import pytest
import torch

pytestmark = pytest.mark.gpu

AFF = (-2.0, -0.5, 0.5)
LIN = (-1.0, 0.5)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    import orihime_b200  # noqa: F401


def _scores(*shape, seed=0, scale=1.5):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(*shape, generator=g) * scale).cuda()


@pytest.mark.parametrize("fam", ["aff", "lin"])
@pytest.mark.parametrize("shape", [(5, 1, 1), (4, 70, 300), (3, 300, 70), (6, 129, 257)])
def test_value_only_equals_full_forward_bitwise(fam, shape):
    s = _scores(*shape)
    B, L1, L2 = shape
    ln = torch.tensor([[L1, L2], [0, L2], [L1 // 2, max(L2 // 3, 1)], [L1, 0], [1, 1], [L1, L2]][:B],
                      dtype=torch.int32).cuda()
    for lengths in (None, ln):
        if fam == "aff":
            want = torch.ops.orihime.sw_affine_forward(s, *AFF, lengths)[0]
            got = torch.ops.orihime_b200.sw_affine_value(s, *AFF, lengths)
        else:
            want = torch.ops.orihime.sw_forward(s, *LIN, lengths)[0]
            got = torch.ops.orihime_b200.sw_value(s, *LIN, lengths)
        assert torch.equal(got, want)


def test_operator_value_without_grad_matches_grad_path_and_is_faster():
    import orihime_b200 as ohm

    s = _scores(16, 512, 512, scale=3.0)
    kw = dict(gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.5)
    with torch.no_grad():
        v0 = ohm.sw_affine_value(s, **kw)
    v1 = ohm.sw_affine_value(s.clone().requires_grad_(True), **kw)
    assert torch.equal(v0, v1.detach())

    def tm(fn, n=5):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    t_val = tm(lambda: torch.ops.orihime_b200.sw_affine_value(s, *AFF, None))
    t_full = tm(lambda: torch.ops.orihime.sw_affine_forward(s, *AFF, None))
    print(f"  16 x 512^2: value only {t_val:.3f} ms, value + map {t_full:.3f} ms")
    assert t_val < t_full


def test_value_ops_under_vmap_and_compile():
    s = _scores(3, 2, 40, 50)
    got = torch.func.vmap(lambda a: torch.ops.orihime_b200.sw_affine_value(a, *AFF, None))(s)
    for k in range(3):
        assert torch.equal(got[k], torch.ops.orihime_b200.sw_affine_value(s[k].contiguous(), *AFF, None))
    f = torch.compile(lambda a: torch.ops.orihime_b200.sw_value(a, *LIN, None).sum(), fullgraph=True)
    assert torch.allclose(f(s[0]), torch.ops.orihime_b200.sw_value(s[0], *LIN, None).sum())


@pytest.mark.parametrize("fam", ["sw_affine", "sw", "nw", "nw_affine", "sv_affine", "sv_linear"])
def test_value_with_tensor_params_runs_one_native_call(fam, monkeypatch):
    """value(...).backward() with learnable gaps and temperature: the value,
    the map and dS/dparameters come from ONE forward pass (one forward +
    adjoint call, or, for the local families, the checkpointed forward and
    its adjoint in the backward), equal bit for bit to the op's value and
    value_grad_params."""
    import orihime_b200 as ohm
    from orihime_b200 import _ops

    s = _scores(3, 40, 57, seed=4).requires_grad_(True)
    affine = fam in ("sw_affine", "nw_affine", "sv_affine")
    names = ("gap_open", "gap_ext", "temp") if affine else ("gap", "temp")
    vals = (-2.0, -0.5, 0.5) if affine else (-1.0, 0.5)
    params = [torch.tensor(v, device="cuda", requires_grad=True) for v in vals]
    calls = []   # native forward passes: one-call forward + adjoint, or the checkpointed forward
    real_a, real_l, real_c = _ops.run_affine, _ops.run_linear, _ops.run_checkpoint
    monkeypatch.setattr(_ops, "run_affine", lambda *a, **k: calls.append(1) or real_a(*a, **k))
    monkeypatch.setattr(_ops, "run_linear", lambda *a, **k: calls.append(1) or real_l(*a, **k))
    monkeypatch.setattr(_ops, "run_checkpoint", lambda *a, **k: calls.append(1) or real_c(*a, **k))
    op = getattr(ohm, {"sw_affine": "sw_affine_value", "sw": "sw_value", "nw": "nw_value",
                       "nw_affine": "nw_affine_value", "sv_affine": "sv_affine_value",
                       "sv_linear": "sv_value"}[fam])
    kw = {"gap_open": "gap_open_score", "gap_ext": "gap_extend_score", "gap": "gap_score",
          "temp": "temperature"}
    v = op(s, **{kw[n]: p for n, p in zip(names, params)})
    v.sum().backward()
    torch.cuda.synchronize()
    assert len(calls) == 1, f"{len(calls)} native forward+adjoint calls"
    monkeypatch.undo()
    sd = s.detach()
    full = getattr(torch.ops.orihime_b200, f"{fam}_forward_with_grads")(sd, *vals, None)
    assert torch.equal(v.detach(), full[0])
    assert torch.equal(s.grad, full[1])
    for p, g in zip(params, full[2:]):
        assert torch.equal(p.grad.reshape(()), g.sum())
