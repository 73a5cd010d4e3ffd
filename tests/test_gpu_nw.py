"""Global alignment (soft Needleman-Wunsch, linear gap): the CUDA path vs the oracle.

The oracle's float restatement reproduces the reference CPU kernels
(src/nw/kernels_cpu.cpp) bit for bit ("ref32"); its double instantiation is
the truth ("fp64").  Bars: value error <= 1e-5 * max(|S|, 1) against ref32
(relative for |S| >= 1; a global alignment's S can sit near 0 by
cancellation, where relative error is ill-conditioned); map, dS/dgap and
dS/dT within max(floor, |ref32 - fp64|) of fp64 (map floor 1e-5 absolute,
gradient floor 1e-4 relative).
Cases follow the reference's own test grid and edge cases
(tests/test_soft_nw.py:114-130, :569-620, :729-835).
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

VAL_RTOL = 1e-5
MAP_ATOL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    import orihime_b200  # noqa: F401  registers the ops


def _gen(shape, seed, scale=1.0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(*shape, generator=g) * scale).float()


def _emb_scores(B, N, M, d, seed, scale=3.0):
    g = torch.Generator().manual_seed(seed)
    e = torch.randn(B, N, d, generator=g)
    f = torch.randn(B, M, d, generator=g)
    return (scale * torch.bmm(e, f.transpose(1, 2)) / d ** 0.5).float()


def _check(name, got, r32, r64, floor, rel=False):
    got = np.asarray(got, np.float64)
    if rel:
        scale = np.maximum(np.abs(np.asarray(r64, np.float64)), 1.0)
        e64 = float(np.max(np.abs(got - r64) / scale)) if got.size else 0.0
        eref = float(np.max(np.abs(np.asarray(r32, np.float64) - r64) / scale)) if got.size else 0.0
    else:
        e64 = float(np.abs(got - r64).max()) if got.size else 0.0
        eref = float(np.abs(np.asarray(r32, np.float64) - r64).max()) if got.size else 0.0
    bound = max(floor, eref)
    print(f"  {name:10s} ours-fp64 {e64:.2e}  ref32-fp64 {eref:.2e}  bound {bound:.2e}")
    assert e64 <= bound, f"{name}: error vs fp64 {e64:.3e} > {bound:.3e} (ref32 {eref:.3e})"


def _cmp(s, ln, gap, T, options=None):
    from orihime_b200 import _ops
    dev = torch.device("cuda")
    sd = s.to(dev).contiguous()
    lnd = None if ln is None else ln.to(dev)
    if options is None:
        v, m = torch.ops.orihime.nw_forward(sd, gap, T, lnd)
        gg = torch.ops.orihime.nw_value_grad_params(sd, gap, T, lnd)
    else:
        lr = _ops.resolve_lengths(lnd, *sd.shape, sd.device)
        v, m, g0, g1 = _ops.run_linear(sd, lr, gap, T, options, family="nw")
        gg = (g0, g1)
    torch.cuda.synchronize()
    sn, lnn = s.numpy(), (None if ln is None else ln.numpy())
    r32 = O.nw(sn, lnn, gap, T)
    r64 = O.nw(sn, lnn, gap, T, dtype=np.float64)
    v, m = v.cpu().numpy(), m.cpu().numpy()
    # value bar: 1e-5 of max(|S|, 1), relative for |S| >= 1 and absolute below,
    # where S comes from cancellation and relative error is ill-conditioned
    rel = np.abs(v - r32["value"]) / np.maximum(np.abs(r32["value"]), 1.0)
    print(f"  value err / max(|S|, 1) vs ref32 {rel.max() if rel.size else 0:.2e}")
    assert (rel.max() if rel.size else 0) <= VAL_RTOL
    _check("value", v, r32["value"], r64["value"], VAL_RTOL, rel=True)
    _check("map", m, r32["map"], r64["map"], MAP_ATOL)
    for got, key in zip(gg, ("grad_gap", "grad_temp")):
        g = got.cpu().numpy()
        floor = 1e-4 * (1.0 + np.abs(r64[key]).max()) if g.size else 1e-4
        _check(key, g, r32[key], r64[key], floor)
    if ln is not None:
        for b, (l1, l2) in enumerate(lnn.tolist()):
            assert not m[b, l1:, :].any() and not m[b, :, l2:].any()
    return v, m


@pytest.mark.parametrize("B", [1, 4])
@pytest.mark.parametrize("shape", [(8, 10), (16, 16), (5, 20)])
@pytest.mark.parametrize("gap", [-1.0, -0.5, -2.0])
@pytest.mark.parametrize("T", [0.1, 1.0, 2.0])
def test_nw_reference_grid(B, shape, gap, T):
    _cmp(_gen((B, *shape), 42), None, gap, T)


@pytest.mark.parametrize("shape", [(1, 1), (1, 3), (3, 1), (1, 300), (300, 1)])
def test_nw_vectors(shape):
    _cmp(_gen((2, *shape), 3), None, -1.0, 1.0)


@pytest.mark.parametrize("gap,T", [(0.0, 1.0), (0.5, 1.0), (-1.0, 0.01), (-1.0, 10.0)])
def test_nw_edge_parameters(gap, T):
    _, m = _cmp(_gen((2, 6, 8), 42), None, gap, T)
    assert m.min() >= -1e-6 and m.max() <= 1 + 1e-5


def test_nw_variable_lengths_with_empty_sides():
    s = _gen((8, 10, 12), 42)
    ln = torch.tensor([[8, 10], [10, 12], [6, 8], [9, 11], [0, 5], [7, 0], [0, 0], [1, 12]],
                      dtype=torch.int32)
    v, m = _cmp(s, ln, -1.0, 1.0)
    # an empty side leaves the boundary cell (L1 + L2) * gap as the value
    assert v[4] == np.float32(5 * -1.0) and v[5] == np.float32(7 * -1.0) and v[6] == 0.0


def test_nw_boundary_heavy_gap_gradient():
    """dS/dgap includes the beta mass that leaves through the row-0 / column-0
    boundary (tests/test_soft_nw.py:378-408)."""
    s = _gen((3, 5, 7), 7)
    s[:, 0, :] -= 2.5
    s[:, :, 0] -= 2.5
    _cmp(s, None, -1.0, 1.0)


@pytest.mark.parametrize("shape", [(300, 700), (129, 257), (40, 1000)])
def test_nw_multiband(shape):
    _cmp(_gen((3, *shape), 5, 1.5), None, -1.0, 1.0)


def test_nw_long_pairs_ragged():
    s = _emb_scores(3, 700, 1100, 64, 9)
    ln = torch.tensor([[700, 1100], [513, 1031], [650, 97]], dtype=torch.int32)
    _cmp(s, ln, -2.0, 0.5)


@pytest.mark.parametrize("cols", [2, 4])
def test_nw_cols_per_lane(cols):
    from orihime_b200 import _lib
    opt = _lib.Options(cols_per_lane=cols)
    _cmp(_gen((3, 90, 333), 8, 1.5), torch.tensor([[90, 333], [77, 300], [5, 200]], dtype=torch.int32),
         -0.7, 0.8, options=opt)


def test_nw_value_only_bitwise_and_deterministic():
    s = _emb_scores(4, 300, 500, 32, 11).cuda()
    ln = torch.tensor([[300, 500], [200, 450], [0, 10], [299, 1]], dtype=torch.int32, device="cuda")
    v1, m1 = torch.ops.orihime.nw_forward(s, -1.0, 0.7, ln)
    v2, m2 = torch.ops.orihime.nw_forward(s, -1.0, 0.7, ln)
    g1 = torch.ops.orihime.nw_value_grad_params(s, -1.0, 0.7, ln)
    g2 = torch.ops.orihime.nw_value_grad_params(s, -1.0, 0.7, ln)
    vo = torch.ops.orihime_b200.nw_value(s, -1.0, 0.7, ln)
    assert torch.equal(v1, v2) and torch.equal(m1, m2)
    assert all(torch.equal(a, b) for a, b in zip(g1, g2))
    assert torch.equal(vo, v1)


def test_nw_map_is_a_posterior_over_aligned_cells():
    """Sum of the map = expected number of aligned cells: (L1 + L2 - dS/dgap) / 2
    (every path has L1 + L2 - 2 * #aligned gap steps, boundaries included)."""
    s = _gen((2, 64, 90), 13, 1.5).cuda()
    v, m = torch.ops.orihime.nw_forward(s, -0.8, 0.9, None)
    gg, _ = torch.ops.orihime.nw_value_grad_params(s, -0.8, 0.9, None)
    lhs = m.double().sum((1, 2))
    rhs = (64 + 90 - gg.double()) / 2
    assert torch.allclose(lhs, rhs, rtol=1e-5, atol=1e-4), (lhs, rhs)


def test_nw_public_api_vs_golden(golden):
    import orihime_b200 as ob
    for case in ("sq", "rect", "ragged", "unit", "row"):
        s = torch.from_numpy(golden[f"{case}/scores"]).cuda()
        ln = (torch.from_numpy(golden[f"{case}/lengths"]).to(torch.int32).cuda()
              if f"{case}/lengths" in golden.files else None)
        g = lambda k: golden[f"{case}/nw/{k}"]  # noqa: E731
        kw = dict(gap_score=-1.0, temperature=0.7, lengths=ln)
        np.testing.assert_allclose(ob.nw_value(s, **kw).cpu().numpy(), g("value"), rtol=1e-5, atol=1e-5)
        x = s.clone().requires_grad_(True)
        v = ob.nw_value(x, **kw)
        (dx,) = torch.autograd.grad(-v.mean(), x)
        np.testing.assert_allclose(dx.cpu().numpy(), g("dvalue"), atol=1e-5)
        with torch.no_grad():
            np.testing.assert_allclose(ob.nw(s, **kw).cpu().numpy(), g("map"), atol=1e-5)
            np.testing.assert_allclose(ob.nw_entropy(s, **kw).cpu().numpy(), g("entropy"), atol=2e-5)
    s = torch.from_numpy(golden["mask/scores"]).cuda()
    mask = torch.from_numpy(golden["mask/mask"]).bool().cuda()
    gp = torch.tensor(-1.0, device="cuda", requires_grad=True)
    tp = torch.tensor(0.8, device="cuda", requires_grad=True)
    x = s.clone().requires_grad_(True)
    v = ob.nw_value(x, gap_score=gp, temperature=tp, mask=mask)
    dx, dg, dt = torch.autograd.grad(v.sum(), (x, gp, tp))
    np.testing.assert_allclose(v.detach().cpu().numpy(), golden["mask/nw/value"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(dx.cpu().numpy(), golden["mask/nw/dx"], atol=1e-5)
    np.testing.assert_allclose(dg.item(), golden["mask/nw/dgap"], atol=1e-4)
    np.testing.assert_allclose(dt.item(), golden["mask/nw/dtemp"], atol=1e-4)


# ---- second-order ops: HVP, parameter Jacobians, map VJP --------------------

def _check2(name, got, r32, r64, rel_floor=1e-4):
    """Bar of the second-order ops: error vs fp64 within the reference's own
    fp32 error, floor 1e-4 of the largest exact entry."""
    got, r32, r64 = (np.asarray(x, np.float64) for x in (got, r32, r64))
    scale = max(float(np.abs(r64).max()), 1e-12)
    e64 = float(np.abs(got - r64).max())
    eref = float(np.abs(r32 - r64).max())
    bound = max(rel_floor * scale, eref)
    print(f"  {name:14s} ours-fp64 {e64:.2e}  ref32-fp64 {eref:.2e}  bound {bound:.2e}  scale {scale:.2e}")
    assert e64 <= bound, f"{name}: {e64:.3e} > {bound:.3e}"


SECOND = [
    # (B, L1, L2, lengths or None, gap, T, seed)
    (2, 24, 31, None, -1.0, 0.7, 1),
    (4, 10, 12, [[8, 10], [10, 12], [0, 5], [7, 0]], -1.0, 1.0, 2),
    (2, 64, 48, None, -0.5, 0.3, 3),
    (1, 130, 300, None, -2.0, 0.5, 4),
    (3, 5, 7, None, -1.0, 1.0, 7),     # boundary-heavy (below)
]


def _second_inputs(B, L1, L2, seed):
    s = _gen((B, L1, L2), seed, 1.5)
    if seed == 7:   # push mass onto the row-0 / column-0 boundary
        s[:, 0, :] -= 2.5
        s[:, :, 0] -= 2.5
    return s, _gen((B, L1, L2), seed + 100)


@pytest.mark.parametrize("B,L1,L2,lengths,gap,T,seed", SECOND)
def test_nw_hvp_matches_oracle(B, L1, L2, lengths, gap, T, seed):
    s, v = _second_inputs(B, L1, L2, seed)
    ln = None if lengths is None else torch.tensor(lengths, dtype=torch.int32)
    lnd = None if ln is None else ln.cuda()
    lnn = None if ln is None else ln.numpy()
    got = torch.ops.orihime.nw_marginals_hvp(s.cuda(), v.cuda(), gap, T, lnd).cpu().numpy()
    _check2("hvp", got, O.nw_hvp(s.numpy(), v.numpy(), lnn, gap, T),
            O.nw_hvp(s.numpy(), v.numpy(), lnn, gap, T, dtype=np.float64))
    if lengths is not None:
        for b, (l1, l2) in enumerate(lengths):
            assert not got[b, l1:, :].any() and not got[b, :, l2:].any()


@pytest.mark.parametrize("B,L1,L2,lengths,gap,T,seed", SECOND)
@pytest.mark.parametrize("param", [0, 1])
def test_nw_param_jacobian_matches_oracle(param, B, L1, L2, lengths, gap, T, seed):
    s, _ = _second_inputs(B, L1, L2, seed)
    ln = None if lengths is None else torch.tensor(lengths, dtype=torch.int32)
    lnd = None if ln is None else ln.cuda()
    lnn = None if ln is None else ln.numpy()
    fn = (torch.ops.orihime.nw_marginals_grad_gap, torch.ops.orihime.nw_marginals_grad_temp)[param]
    got = fn(s.cuda(), gap, T, lnd).cpu().numpy()
    _check2(f"dP/dtheta{param}", got, O.nw_param_grad(s.numpy(), lnn, gap, T, param),
            O.nw_param_grad(s.numpy(), lnn, gap, T, param, dtype=np.float64))


def test_nw_marginals_backward_matches_oracle_contractions():
    B, L1, L2, gap, T = 3, 37, 145, -0.8, 0.6
    s, gm = _second_inputs(B, L1, L2, 11)
    ln = torch.tensor([[37, 145], [20, 45], [37, 9]], dtype=torch.int32)
    sn, gn, lnn = s.numpy(), gm.numpy(), ln.numpy()
    out = torch.ops.orihime.nw_marginals_backward(s.cuda(), gm.cuda(), gap, T, ln.cuda())
    _check2("grad_scores", out[0].cpu().numpy(), O.nw_hvp(sn, gn, lnn, gap, T),
            O.nw_hvp(sn, gn, lnn, gap, T, dtype=np.float64))
    for k in range(2):
        r64 = (gn.astype(np.float64) * O.nw_param_grad(sn, lnn, gap, T, k, dtype=np.float64)).sum()
        r32 = (gn.astype(np.float64) * O.nw_param_grad(sn, lnn, gap, T, k)).sum()
        got = float(out[1 + k].item())
        bound = max(abs(r32 - r64), 1e-4 * (1 + abs(r64)))
        print(f"  param {k}: ours {got:.6f} fp64 {r64:.6f} ref32 {r32:.6f}")
        assert abs(got - r64) <= bound


def test_nw_second_order_deterministic_and_grouped():
    s, v = _second_inputs(5, 70, 200, 21)
    s, v = s.cuda(), v.cuda()
    a = torch.ops.orihime.nw_marginals_hvp(s, v, -1.0, 0.8, None)
    b = torch.ops.orihime.nw_marginals_hvp(s, v, -1.0, 0.8, None)
    assert torch.equal(a, b)
    for k in range(5):   # pairs are independent: one call per pair gives the same bits
        assert torch.equal(torch.ops.orihime.nw_marginals_hvp(s[k:k + 1].contiguous(), v[k:k + 1].contiguous(),
                                                              -1.0, 0.8, None), a[k:k + 1])


def test_nw_public_api_second_order_vs_golden(golden):
    import orihime_b200 as ob
    for case in ("sq", "rect", "ragged", "unit", "row"):
        s = torch.from_numpy(golden[f"{case}/scores"]).cuda()
        cot = torch.from_numpy(golden[f"{case}/cot"]).cuda()
        ln = (torch.from_numpy(golden[f"{case}/lengths"]).to(torch.int32).cuda()
              if f"{case}/lengths" in golden.files else None)
        g = lambda k: golden[f"{case}/nw/{k}"]  # noqa: E731
        kw = dict(gap_score=-1.0, temperature=0.7, lengths=ln)
        x = s.clone().requires_grad_(True)
        (dm,) = torch.autograd.grad((ob.nw(x, **kw) * cot).sum(), x)
        np.testing.assert_allclose(dm.cpu().numpy(), g("dmap"), atol=1e-5)
        x = s.clone().requires_grad_(True)
        (de,) = torch.autograd.grad(ob.nw_entropy(x, **kw).sum(), x)
        np.testing.assert_allclose(de.cpu().numpy(), g("dentropy"), atol=1e-5)
        args = (s, -1.0, 0.7, ln)
        np.testing.assert_allclose(torch.ops.orihime.nw_marginals_grad_gap(*args).cpu().numpy(),
                                   g("sens_gap_score"), atol=1e-5)
        np.testing.assert_allclose(torch.ops.orihime.nw_marginals_grad_temp(*args).cpu().numpy(),
                                   g("sens_temperature"), atol=1e-5)
        bw = torch.ops.orihime.nw_marginals_backward(s, cot, -1.0, 0.7, ln)
        np.testing.assert_allclose(bw[0].cpu().numpy(), g("bw_pair_scores"), atol=1e-5)
        np.testing.assert_allclose(bw[1].item(), g("bw_gap_score"), atol=1e-4)
        np.testing.assert_allclose(bw[2].item(), g("bw_temperature"), atol=1e-4)


def test_nw_tensor_parameter_forward_backward():
    """orihime::nw_forward_t through AutogradCUDA: value and map cotangents reach
    the scores and both tensor parameters (value x grads + map VJP)."""
    s = _gen((2, 30, 41), 31, 1.5).cuda().requires_grad_(True)
    ln = torch.tensor([[30, 41], [22, 17]], dtype=torch.int32).cuda()
    gp = torch.tensor(-0.9, device="cuda", requires_grad=True)
    tp = torch.tensor(0.7, device="cuda", requires_grad=True)
    v, m = torch.ops.orihime.nw_forward_t(s, gp, tp, ln)
    cot = _gen((2, 30, 41), 32).cuda()
    (v.sum() + (m * cot).sum()).backward()
    sd = s.detach()
    gg, gT = torch.ops.orihime.nw_value_grad_params(sd, -0.9, 0.7, ln)
    mb = torch.ops.orihime.nw_marginals_backward(sd, cot, -0.9, 0.7, ln)
    vm = torch.ops.orihime.nw_forward(sd, -0.9, 0.7, ln)[1]
    assert torch.allclose(s.grad, vm + mb[0], rtol=1e-5, atol=1e-6)
    assert torch.allclose(gp.grad, gg.sum() + mb[1][0], rtol=1e-5, atol=1e-5)
    assert torch.allclose(tp.grad, gT.sum() + mb[2][0], rtol=1e-5, atol=1e-5)


def test_nw_ragged_plan_equals_padded_bitwise():
    """The packed ragged path (family "global") computes each pair exactly as
    the padded op with lengths does."""
    from orihime_b200 import ragged
    rng = np.random.default_rng(17)
    lens = np.stack([rng.integers(0, 300, 40), rng.integers(0, 520, 40)], 1)
    lens[3] = [0, 50]
    lens[5] = [70, 0]
    lens[7] = [1, 1]
    mats = [_gen((int(a), int(b)), 100 + k, 1.5) for k, (a, b) in enumerate(lens)]
    flat, off, l32 = ragged.pack([m.cuda() for m in mats])
    plan = ragged.Plan(l32, off, family="global", device="cuda")
    out = plan.run(flat.cuda(), gap=-0.9, temp=0.6)
    vals = plan.values(flat.cuda(), gap=-0.9, temp=0.6)
    L1m, L2m = int(lens[:, 0].max()), int(lens[:, 1].max())
    pad = torch.zeros(len(mats), L1m, L2m)
    for k, m in enumerate(mats):
        pad[k, :m.shape[0], :m.shape[1]] = m
    ln = torch.tensor(lens, dtype=torch.int32).cuda()
    v, m = torch.ops.orihime.nw_forward(pad.cuda(), -0.9, 0.6, ln)
    gg, gT = torch.ops.orihime.nw_value_grad_params(pad.cuda(), -0.9, 0.6, ln)
    assert torch.equal(out.value, v) and torch.equal(vals, v)
    assert torch.equal(out.grad_open, gg) and torch.equal(out.grad_temp, gT)
    for k, mk in enumerate(ragged.unpack(out.map, off, l32)):
        a, b = int(lens[k, 0]), int(lens[k, 1])
        assert torch.equal(mk, m[k, :a, :b]), k
