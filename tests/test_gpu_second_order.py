"""Second-order ops on the GPU: HVP of the map, parameter Jacobians, the map's
full VJP (marginals_backward), and autograd through the map and the entropy.

Truth is the fp64 oracle; "ref32" is the oracle's float restatement of the
reference algorithm.  Bar: our error against fp64 may not exceed the
reference's own fp32 error, with an absolute floor of 1e-4 times the largest
entry of the exact result (these are derivatives of probabilities, scaled by
1/T, so their magnitude varies by case).
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

AFF = (-2.0, -0.5)
LIN = (-1.0,)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    import orihime_b200  # noqa: F401


def _scores(B, L1, L2, seed, scale=1.5):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(B, L1, L2, generator=g) * scale).float()


def _check(name, got, r32, r64, rel_floor=1e-4):
    got, r32, r64 = (np.asarray(x, np.float64) for x in (got, r32, r64))
    scale = max(float(np.abs(r64).max()), 1e-12)
    e64 = float(np.abs(got - r64).max())
    eref = float(np.abs(r32 - r64).max())
    bound = max(rel_floor * scale, eref)
    print(f"  {name:14s} ours-fp64 {e64:.2e}  ref32-fp64 {eref:.2e}  bound {bound:.2e}  scale {scale:.2e}")
    assert e64 <= bound, f"{name}: {e64:.3e} > {bound:.3e}"


CASES = [
    # (B, L1, L2, lengths or None, T, seed)
    (2, 24, 31, None, 0.7, 1),
    (3, 40, 33, [[40, 33], [17, 29], [1, 5]], 1.0, 2),
    (2, 64, 48, None, 0.3, 3),
    (1, 130, 70, None, 0.5, 4),
]


def _ln(lengths):
    return None if lengths is None else torch.tensor(lengths, dtype=torch.int32)


@pytest.mark.parametrize("B,L1,L2,lengths,T,seed", CASES)
@pytest.mark.parametrize("fam", ["affine", "linear"])
def test_hvp_matches_oracle(fam, B, L1, L2, lengths, T, seed):
    s = _scores(B, L1, L2, seed)
    v = _scores(B, L1, L2, seed + 100, scale=1.0)
    ln = _ln(lengths)
    lnd = None if ln is None else ln.cuda()
    sn, vn, lnn = s.numpy(), v.numpy(), (None if ln is None else ln.numpy())
    if fam == "affine":
        got = torch.ops.orihime.sw_affine_marginals_hvp(s.cuda(), v.cuda(), *AFF, T, lnd).cpu().numpy()
        r32 = O.affine_hvp(sn, vn, lnn, *AFF, T)
        r64 = O.affine_hvp(sn, vn, lnn, *AFF, T, dtype=np.float64)
    else:
        got = torch.ops.orihime.sw_marginals_hvp(s.cuda(), v.cuda(), *LIN, T, lnd).cpu().numpy()
        r32 = O.linear_hvp(sn, vn, lnn, *LIN, T)
        r64 = O.linear_hvp(sn, vn, lnn, *LIN, T, dtype=np.float64)
    _check("hvp", got, r32, r64)
    if lengths is not None:  # exactly zero outside lengths
        for b, (l1, l2) in enumerate(lengths):
            assert not got[b, l1:, :].any() and not got[b, :, l2:].any()


@pytest.mark.parametrize("B,L1,L2,lengths,T,seed", CASES)
@pytest.mark.parametrize("fam,param", [("affine", 0), ("affine", 1), ("affine", 2),
                                       ("linear", 0), ("linear", 1)])
def test_param_jacobian_matches_oracle(fam, param, B, L1, L2, lengths, T, seed):
    s = _scores(B, L1, L2, seed)
    ln = _ln(lengths)
    lnd = None if ln is None else ln.cuda()
    sn, lnn = s.numpy(), (None if ln is None else ln.numpy())
    ops = torch.ops.orihime
    if fam == "affine":
        fn = [ops.sw_affine_marginals_grad_gap_open, ops.sw_affine_marginals_grad_gap_ext,
              ops.sw_affine_marginals_grad_temp][param]
        got = fn(s.cuda(), *AFF, T, lnd).cpu().numpy()
        r32 = O.affine_param_grad(sn, lnn, *AFF, T, param)
        r64 = O.affine_param_grad(sn, lnn, *AFF, T, param, dtype=np.float64)
    else:
        fn = [ops.sw_marginals_grad_gap, ops.sw_marginals_grad_temp][param]
        got = fn(s.cuda(), *LIN, T, lnd).cpu().numpy()
        r32 = O.linear_param_grad(sn, lnn, *LIN, T, param)
        r64 = O.linear_param_grad(sn, lnn, *LIN, T, param, dtype=np.float64)
    _check(f"dP/dtheta{param}", got, r32, r64)


@pytest.mark.parametrize("fam", ["affine", "linear"])
def test_marginals_backward_matches_oracle_contractions(fam):
    B, L1, L2, T = 3, 37, 45, 0.6
    s = _scores(B, L1, L2, 11)
    gm = _scores(B, L1, L2, 12, scale=1.0)
    ln = torch.tensor([[37, 45], [20, 45], [37, 9]], dtype=torch.int32)
    sn, gn, lnn = s.numpy(), gm.numpy(), ln.numpy()
    if fam == "affine":
        out = torch.ops.orihime.sw_affine_marginals_backward(s.cuda(), gm.cuda(), *AFF, T, ln.cuda())
        h64 = O.affine_hvp(sn, gn, lnn, *AFF, T, dtype=np.float64)
        h32 = O.affine_hvp(sn, gn, lnn, *AFF, T)
        tots = [(gn * O.affine_param_grad(sn, lnn, *AFF, T, p, dtype=np.float64)).sum() for p in range(3)]
    else:
        out = torch.ops.orihime.sw_marginals_backward(s.cuda(), gm.cuda(), *LIN, T, ln.cuda())
        h64 = O.linear_hvp(sn, gn, lnn, *LIN, T, dtype=np.float64)
        h32 = O.linear_hvp(sn, gn, lnn, *LIN, T)
        tots = [(gn * O.linear_param_grad(sn, lnn, *LIN, T, p, dtype=np.float64)).sum() for p in range(2)]
    _check("grad_scores", out[0].cpu().numpy(), h32, h64)
    assert len(out) == 1 + len(tots)
    for k, want in enumerate(tots):
        got = float(out[1 + k].cpu())
        assert out[1 + k].shape == (1,)
        print(f"  param {k}: got {got:.6e} want {want:.6e}")
        assert abs(got - want) <= 2e-4 * max(1.0, abs(want)), (k, got, want)


def test_autograd_through_map_and_entropy():
    import orihime_b200 as ohm

    B, L1, L2, T = 2, 30, 26, 0.8
    s = _scores(B, L1, L2, 21).cuda().requires_grad_(True)
    go = torch.tensor(-2.0, device="cuda", requires_grad=True)
    gm = _scores(B, L1, L2, 22, scale=1.0).cuda()
    m = ohm.sw_affine(s, gap_open_score=go, gap_extend_score=-0.5, temperature=T)
    (m * gm).sum().backward()
    want = torch.ops.orihime.sw_affine_marginals_hvp(s.detach(), gm, -2.0, -0.5, T, None)
    assert torch.allclose(s.grad, want, rtol=0, atol=1e-6)
    field = torch.ops.orihime.sw_affine_marginals_grad_gap_open(s.detach(), -2.0, -0.5, T, None)
    assert torch.allclose(go.grad, (gm * field).sum(), rtol=1e-5, atol=1e-6)
    # entropy backward = dP/dT field (the Hessian's mixed block)
    s2 = s.detach().clone().requires_grad_(True)
    ent = ohm.sw_affine_entropy(s2, gap_open_score=-2.0, gap_extend_score=-0.5, temperature=T)
    ent.sum().backward()
    field_t = torch.ops.orihime.sw_affine_marginals_grad_temp(s2.detach(), -2.0, -0.5, T, None)
    assert torch.allclose(s2.grad, field_t, rtol=0, atol=1e-6)
    # cross-check against the fp64 oracle
    r64 = O.affine_param_grad(s.detach().cpu().numpy(), None, -2.0, -0.5, T, 2, dtype=np.float64)
    r32 = O.affine_param_grad(s.detach().cpu().numpy(), None, -2.0, -0.5, T, 2)
    _check("entropy grad", s2.grad.cpu().numpy(), r32, r64)


def test_hvp_symmetry_and_linearity():
    """u . H v == v . H u, and H (a u + b v) == a H u + b H v."""
    B, L1, L2, T = 2, 50, 41, 0.5
    s = _scores(B, L1, L2, 31).cuda()
    u = _scores(B, L1, L2, 32, 1.0).cuda()
    v = _scores(B, L1, L2, 33, 1.0).cuda()
    H = lambda x: torch.ops.orihime.sw_affine_marginals_hvp(s, x, *AFF, T, None)
    Hu, Hv = H(u), H(v)
    a = float((u * Hv).double().sum())
    b = float((v * Hu).double().sum())
    assert abs(a - b) <= 1e-4 * max(1.0, abs(a)), (a, b)
    lin = H(2.0 * u - 0.5 * v)
    assert torch.allclose(lin, 2.0 * Hu - 0.5 * Hv, rtol=0, atol=2e-5 * float(Hu.abs().max()))


@pytest.mark.parametrize("fam", ["affine", "linear"])
def test_forward_ops_are_differentiable(fam):
    """The namespaced forward ops carry their own autograd (as the reference's
    AutogradCUDA registration does): value cotangent x map + HVP of the map
    cotangent, plus parameter gradients for the tensor-parameter variant."""
    ops = torch.ops.orihime
    B, L1, L2, T = 2, 33, 27, 0.6
    s = _scores(B, L1, L2, 41).cuda().requires_grad_(True)
    a = torch.randn(B, device="cuda")
    g = _scores(B, L1, L2, 42, 1.0).cuda()
    if fam == "affine":
        v, m = ops.sw_affine_forward(s, *AFF, T, None)
        ((v * a).sum() + (m * g).sum()).backward()
        want = a.view(-1, 1, 1) * m.detach() + ops.sw_affine_marginals_hvp(s.detach(), g, *AFF, T, None)
    else:
        v, m = ops.sw_forward(s, *LIN, T, None)
        ((v * a).sum() + (m * g).sum()).backward()
        want = a.view(-1, 1, 1) * m.detach() + ops.sw_marginals_hvp(s.detach(), g, *LIN, T, None)
    assert torch.allclose(s.grad, want, rtol=1e-5, atol=1e-6)
    # tensor-parameter variant: parameter gradients
    s2 = s.detach().clone().requires_grad_(True)
    vals = AFF + (T,) if fam == "affine" else LIN + (T,)
    ps = [torch.tensor(x, device="cuda", requires_grad=True) for x in vals]
    ln = torch.tensor([[L1, L2]] * B, dtype=torch.int32, device="cuda")
    fwd_t = ops.sw_affine_forward_t if fam == "affine" else ops.sw_forward_t
    v2, m2 = fwd_t(s2, *ps, ln)
    ((v2 * a).sum() + (m2 * g).sum()).backward()
    vg = (ops.sw_affine_value_grad_params if fam == "affine" else ops.sw_value_grad_params)(
        s.detach(), *vals, ln)
    mb = (ops.sw_affine_marginals_backward if fam == "affine" else ops.sw_marginals_backward)(
        s.detach(), g, *vals, ln)
    assert torch.allclose(s2.grad, s.grad, rtol=1e-5, atol=1e-6)
    for k, p in enumerate(ps):
        want_p = float((a * vg[k]).sum() + mb[1 + k].sum())
        assert abs(float(p.grad) - want_p) <= 1e-4 * max(1.0, abs(want_p)), (k, float(p.grad), want_p)


def test_pair_groups_match_single_call(monkeypatch):
    """A batch whose field table exceeds the memory budget runs in pair
    groups; pairs are independent, so each group's outputs equal the
    single-call outputs bit for bit (both use 2 columns per lane here)."""
    from orihime_b200 import _ops

    s = _scores(5, 40, 70, 11).cuda()
    v = _scores(5, 40, 70, 12, scale=1.0).cuda()
    ln = torch.tensor([[40, 70], [17, 33], [0, 5], [40, 1], [23, 70]], dtype=torch.int32).cuda()
    want, want_gt = _ops.run_hvp("sw_affine", s, v, ln, (*AFF, 0.6), want_grads=True)
    want_p = _ops.run_param_jacobian("sw", s, ln, (*LIN, 0.6), 1)
    monkeypatch.setattr(_ops, "AUX_BUDGET_MAX", 1)
    assert _ops._aux_plan("sw_affine", 5, 40, 70, s.device, (*AFF, 0.6))[0] == 1
    got, got_gt = _ops.run_hvp("sw_affine", s, v, ln, (*AFF, 0.6), want_grads=True)
    got_p = _ops.run_param_jacobian("sw", s, ln, (*LIN, 0.6), 1)
    assert torch.equal(got, want) and torch.equal(got_gt, want_gt) and torch.equal(got_p, want_p)
    assert float(want[2].abs().max()) == 0.0 and float(want_gt[2].abs().max()) == 0.0


@pytest.mark.parametrize("fam", ["affine", "linear"])
def test_long_pair_quiet_chunks(fam):
    """A long pair where most backward chunks carry negligible flow (they push
    zeros instead of recomputing, dropping values below ~1e-15): the HVP and
    dP/dT stay within the fp64 bounds, and two runs agree bit for bit."""
    from orihime_b200 import _ops

    s = _scores(1, 900, 700, 21, scale=3.0).cuda()
    v = _scores(1, 900, 700, 22, scale=1.0).cuda()
    sn, vn = s.cpu().numpy(), v.cpu().numpy()
    T = 0.5
    if fam == "affine":
        got = _ops.run_hvp("sw_affine", s, v, None, (*AFF, T))[0]
        again = _ops.run_hvp("sw_affine", s, v, None, (*AFF, T))[0]
        _check("hvp", got.cpu().numpy(), O.affine_hvp(sn, vn, None, *AFF, T),
               O.affine_hvp(sn, vn, None, *AFF, T, dtype=np.float64))
        pt = _ops.run_param_jacobian("sw_affine", s, None, (*AFF, T), 2)
        _check("dP/dT", pt.cpu().numpy(), O.affine_param_grad(sn, None, *AFF, T, 2),
               O.affine_param_grad(sn, None, *AFF, T, 2, dtype=np.float64))
    else:
        got = _ops.run_hvp("sw", s, v, None, (*LIN, T))[0]
        again = _ops.run_hvp("sw", s, v, None, (*LIN, T))[0]
        _check("hvp", got.cpu().numpy(), O.linear_hvp(sn, vn, None, *LIN, T),
               O.linear_hvp(sn, vn, None, *LIN, T, dtype=np.float64))
        pt = _ops.run_param_jacobian("sw", s, None, (*LIN, T), 1)
        _check("dP/dT", pt.cpu().numpy(), O.linear_param_grad(sn, None, *LIN, T, 1),
               O.linear_param_grad(sn, None, *LIN, T, 1, dtype=np.float64))
    assert torch.equal(got, again)


@pytest.mark.parametrize("fam", ["affine", "linear"])
def test_workspace_for_parameters(fam):
    """The parameter-aware workspace size is exactly what the call launches:
    an HVP and a parameter Jacobian with that many bytes give the outputs of
    a call with the any-parameters size bit for bit, and one byte less is
    refused before anything runs (SWB_ERR_WORKSPACE, output untouched)."""
    import ctypes

    from orihime_b200 import _lib

    lib = _lib.load()
    s = _scores(3, 40, 70, 31).cuda()
    v = _scores(3, 40, 70, 32, scale=1.0).cuda()
    B, L1, L2 = s.shape
    f = ctypes.c_float
    if fam == "affine":
        ps, pfx = (f(AFF[0]), f(AFF[1]), f(0.6)), "swb_sw_affine"
    else:
        ps, pfx = (f(LIN[0]), f(0.6)), "swb_sw"
    n_for = int(getattr(lib, f"{pfx}_aux_workspace_bytes_for")(B, L1, L2, *ps))
    n_any = int(getattr(lib, f"{pfx}_aux_workspace_bytes")(B, L1, L2))
    assert 0 < n_for < n_any
    st = torch.cuda.current_stream().cuda_stream
    hvp, jac = getattr(lib, f"{pfx}_hvp"), getattr(lib, f"{pfx}_param_jacobian")
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    outs = {}
    for n in (n_any, n_for):
        ws = torch.empty(n, dtype=torch.uint8, device="cuda")
        o1, o2 = torch.empty_like(s), torch.empty_like(s)
        assert hvp(P(s), P(v), None, B, L1, L2, *ps, P(o1), None, P(ws), ctypes.c_size_t(n), ctypes.c_void_p(st)) == 0
        assert jac(P(s), None, B, L1, L2, *ps, 0, P(o2), P(ws), ctypes.c_size_t(n), ctypes.c_void_p(st)) == 0
        torch.cuda.synchronize()
        outs[n] = (o1, o2)
    assert torch.equal(outs[n_for][0], outs[n_any][0]) and torch.equal(outs[n_for][1], outs[n_any][1])
    ws = torch.empty(n_for, dtype=torch.uint8, device="cuda")
    o = torch.full_like(s, 7.0)
    rc = hvp(P(s), P(v), None, B, L1, L2, *ps, P(o), None, P(ws), ctypes.c_size_t(n_for - 1), ctypes.c_void_p(st))
    torch.cuda.synchronize()
    assert rc == -2 and bool((o == 7.0).all())
