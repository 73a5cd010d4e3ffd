"""Global alignment with affine gaps (soft Needleman-Wunsch affine): the CUDA
path vs the oracle.

The oracle's float restatement reproduces the reference CPU kernels
(src/nw_affine/kernels_cpu.cpp) bit for bit ("ref32"); its double
instantiation is the truth ("fp64").  Bars: value error <= 1e-5 * max(|S|, 1)
against ref32 (a global alignment's S can sit near 0 by cancellation, where
relative error is ill-conditioned: the scaled-domain temperature alone,
log2(e)/T rounded to float, moves such an S by ~1e-6 absolute; the
reference's own test bar is rtol 1e-4 with atol 1e-5); map and gradients
within max(floor, |ref32 - fp64|) of fp64 (map floor 1e-5 absolute, gradient
floor 1e-4 relative).  Cases follow the reference's own grid and edge cases
(tests/test_soft_nw_affine.py:125-145, :248, :745, :1003-1100).
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


def _cmp(s, ln, go, ge, T, options=None):
    from orihime_b200 import _ops
    dev = torch.device("cuda")
    sd = s.to(dev).contiguous()
    lnd = None if ln is None else ln.to(dev)
    if options is None:
        v, m = torch.ops.orihime.nw_affine_forward(sd, go, ge, T, lnd)
        vg = torch.ops.orihime.nw_affine_value_grad_params(sd, go, ge, T, lnd)
        assert torch.equal(vg[0], v)
        gg = vg[1:]
    else:
        lr = _ops.resolve_lengths(lnd, *sd.shape, sd.device)
        v, m, g0, g1, g2 = _ops.run_affine(sd, lr, go, ge, T, options, family="nw_affine")
        gg = (g0, g1, g2)
    torch.cuda.synchronize()
    sn, lnn = s.numpy(), (None if ln is None else ln.numpy())
    r32 = O.nw_affine(sn, lnn, go, ge, T)
    r64 = O.nw_affine(sn, lnn, go, ge, T, dtype=np.float64)
    v, m = v.cpu().numpy(), m.cpu().numpy()
    # value bar: 1e-5 of max(|S|, 1), relative for |S| >= 1 and absolute below,
    # where S comes from cancellation and relative error is ill-conditioned
    rel = np.abs(v - r32["value"]) / np.maximum(np.abs(r32["value"]), 1.0)
    print(f"  value err / max(|S|, 1) vs ref32 {rel.max() if rel.size else 0:.2e}")
    assert (rel.max() if rel.size else 0) <= VAL_RTOL
    _check("value", v, r32["value"], r64["value"], VAL_RTOL, rel=True)
    _check("map", m, r32["map"], r64["map"], MAP_ATOL)
    for got, key in zip(gg, ("grad_open", "grad_ext", "grad_temp")):
        g = got.cpu().numpy()
        floor = 1e-4 * (1.0 + np.abs(r64[key]).max()) if g.size else 1e-4
        _check(key, g, r32[key], r64[key], floor)
    if ln is not None:
        for b, (l1, l2) in enumerate(lnn.tolist()):
            assert not m[b, l1:, :].any() and not m[b, :, l2:].any()
    return v, m


@pytest.mark.parametrize("B", [1, 4])
@pytest.mark.parametrize("shape", [(8, 10), (16, 16), (5, 20)])
@pytest.mark.parametrize("gaps", [(-2.0, -0.5), (-1.0, -0.3), (-3.0, -1.0)])
@pytest.mark.parametrize("T", [0.1, 1.0, 2.0])
def test_nw_affine_reference_grid(B, shape, gaps, T):
    _cmp(_gen((B, *shape), 42), None, *gaps, T)


@pytest.mark.parametrize("shape", [(1, 1), (1, 3), (3, 1), (1, 300), (300, 1)])
def test_nw_affine_vectors(shape):
    _cmp(_gen((2, *shape), 3), None, -2.0, -0.5, 1.0)


@pytest.mark.parametrize("go,ge,T", [(-1.0, -1.0, 1.0), (-2.0, 0.0, 1.0), (-2.0, -0.5, 0.01),
                                     (-2.0, -0.5, 10.0), (0.5, 0.2, 1.0)])
def test_nw_affine_edge_parameters(go, ge, T):
    _, m = _cmp(_gen((2, 6, 8), 42), None, go, ge, T)
    assert m.min() >= -1e-6 and m.max() <= 1 + 1e-5


def test_nw_affine_variable_lengths_with_empty_sides():
    s = _gen((8, 10, 12), 42)
    ln = torch.tensor([[8, 10], [10, 12], [6, 8], [9, 11], [0, 5], [7, 0], [0, 0], [1, 12]],
                      dtype=torch.int32)
    v, _ = _cmp(s, ln, -2.0, -0.5, 1.0)
    # an empty side leaves the boundary state go + (n - 1) ge; the origin is 0
    assert v[4] == np.float32(-2.0 + 4 * -0.5) and v[5] == np.float32(-2.0 + 6 * -0.5) and v[6] == 0.0


def test_nw_affine_boundary_heavy_gap_gradients():
    """dS/dgap_open and dS/dgap_ext include the leading-gap boundary states
    (tests/test_soft_nw_affine.py:248-298, :481-529)."""
    s = _gen((3, 5, 7), 7)
    s[:, 0, :] -= 2.5
    s[:, :, 0] -= 2.5
    _cmp(s, None, -1.0, -0.3, 1.0)


@pytest.mark.parametrize("shape", [(300, 700), (129, 257), (40, 1000)])
def test_nw_affine_multiband(shape):
    _cmp(_gen((3, *shape), 5, 1.5), None, -2.0, -0.5, 1.0)


def test_nw_affine_long_pairs_ragged():
    s = _emb_scores(3, 700, 1100, 64, 9)
    ln = torch.tensor([[700, 1100], [513, 1031], [650, 97]], dtype=torch.int32)
    _cmp(s, ln, -2.0, -0.5, 0.5)


@pytest.mark.parametrize("cols", [2, 4])
def test_nw_affine_cols_per_lane(cols):
    from orihime_b200 import _lib
    opt = _lib.Options(cols_per_lane=cols)
    _cmp(_gen((3, 90, 333), 8, 1.5), torch.tensor([[90, 333], [77, 300], [5, 200]], dtype=torch.int32),
         -2.0, -0.5, 0.8, options=opt)


def test_nw_affine_value_only_bitwise_and_deterministic():
    s = _emb_scores(4, 300, 500, 32, 11).cuda()
    ln = torch.tensor([[300, 500], [200, 450], [0, 10], [299, 1]], dtype=torch.int32, device="cuda")
    v1, m1 = torch.ops.orihime.nw_affine_forward(s, -2.0, -0.5, 0.7, ln)
    v2, m2 = torch.ops.orihime.nw_affine_forward(s, -2.0, -0.5, 0.7, ln)
    g1 = torch.ops.orihime.nw_affine_value_grad_params(s, -2.0, -0.5, 0.7, ln)
    g2 = torch.ops.orihime.nw_affine_value_grad_params(s, -2.0, -0.5, 0.7, ln)
    vo = torch.ops.orihime_b200.nw_affine_value(s, -2.0, -0.5, 0.7, ln)
    assert torch.equal(v1, v2) and torch.equal(m1, m2)
    assert all(torch.equal(a, b) for a, b in zip(g1, g2))
    assert torch.equal(vo, v1)


def test_nw_affine_ragged_plan_equals_padded_bitwise():
    from orihime_b200 import ragged
    rng = np.random.default_rng(19)
    lens = np.stack([rng.integers(0, 300, 40), rng.integers(0, 520, 40)], 1)
    lens[3] = [0, 50]
    lens[5] = [70, 0]
    lens[7] = [1, 1]
    mats = [_gen((int(a), int(b)), 200 + k, 1.5) for k, (a, b) in enumerate(lens)]
    flat, off, l32 = ragged.pack([m.cuda() for m in mats])
    plan = ragged.Plan(l32, off, family="global_affine", device="cuda")
    out = plan.run(flat.cuda(), gap_open=-2.0, gap_ext=-0.5, temp=0.6)
    vals = plan.values(flat.cuda(), gap_open=-2.0, gap_ext=-0.5, temp=0.6)
    L1m, L2m = int(lens[:, 0].max()), int(lens[:, 1].max())
    pad = torch.zeros(len(mats), L1m, L2m)
    for k, m in enumerate(mats):
        pad[k, :m.shape[0], :m.shape[1]] = m
    ln = torch.tensor(lens, dtype=torch.int32).cuda()
    v, m = torch.ops.orihime.nw_affine_forward(pad.cuda(), -2.0, -0.5, 0.6, ln)
    _, go, ge, gT = torch.ops.orihime.nw_affine_value_grad_params(pad.cuda(), -2.0, -0.5, 0.6, ln)
    assert torch.equal(out.value, v) and torch.equal(vals, v)
    assert torch.equal(out.grad_open, go) and torch.equal(out.grad_ext, ge)
    assert torch.equal(out.grad_temp, gT)
    for k, mk in enumerate(ragged.unpack(out.map, off, l32)):
        a, b = int(lens[k, 0]), int(lens[k, 1])
        assert torch.equal(mk, m[k, :a, :b]), k


def test_nw_affine_public_value_and_map():
    import orihime_b200 as ob
    s = _gen((3, 20, 27), 23, 1.5).cuda()
    ln = torch.tensor([[20, 27], [11, 19], [20, 3]], dtype=torch.int32).cuda()
    kw = dict(gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.7, lengths=ln)
    o = O.nw_affine(s.cpu().numpy(), ln.cpu().numpy(), -2.0, -0.5, 0.7)
    np.testing.assert_allclose(ob.nw_affine_value(s, **kw).cpu().numpy(), o["value"], rtol=1e-5)
    with torch.no_grad():
        np.testing.assert_allclose(ob.nw_affine(s, **kw).cpu().numpy(), o["map"], atol=1e-5)
        np.testing.assert_allclose(ob.nw_affine_entropy(s, **kw).cpu().numpy(), o["grad_temp"],
                                   atol=1e-4)
    x = s.clone().requires_grad_(True)
    (dx,) = torch.autograd.grad(ob.nw_affine_value(x, **kw).sum(), x)
    np.testing.assert_allclose(dx.cpu().numpy(), o["map"], atol=1e-5)


# ---- second-order ops: HVP, parameter Jacobians, map VJP --------------------

def _check2(name, got, r32, r64, rel_floor=1e-4):
    """Second-order bar: error vs fp64 within the reference's own fp32 error,
    floor 1e-4 of the largest exact entry."""
    got, r32, r64 = (np.asarray(x, np.float64) for x in (got, r32, r64))
    scale = max(float(np.abs(r64).max()), 1e-12)
    e64 = float(np.abs(got - r64).max())
    eref = float(np.abs(r32 - r64).max())
    bound = max(rel_floor * scale, eref)
    print(f"  {name:14s} ours-fp64 {e64:.2e}  ref32-fp64 {eref:.2e}  bound {bound:.2e}  scale {scale:.2e}")
    assert e64 <= bound, f"{name}: {e64:.3e} > {bound:.3e}"


SECOND = [
    # (B, L1, L2, lengths or None, go, ge, T, seed)
    (2, 24, 31, None, -2.0, -0.5, 0.7, 1),
    (4, 10, 12, [[8, 10], [10, 12], [0, 5], [7, 0]], -1.0, -0.3, 1.0, 2),
    (2, 64, 48, None, -2.0, -0.5, 0.3, 3),
    (1, 130, 300, None, -3.0, -1.0, 0.5, 4),
    (3, 5, 7, None, -1.0, -0.3, 1.0, 7),     # boundary-heavy
]


def _second_inputs(B, L1, L2, seed):
    s = _gen((B, L1, L2), seed, 1.5)
    if seed == 7:
        s[:, 0, :] -= 2.5
        s[:, :, 0] -= 2.5
    return s, _gen((B, L1, L2), seed + 100)


@pytest.mark.parametrize("B,L1,L2,lengths,go,ge,T,seed", SECOND)
def test_nw_affine_hvp_matches_oracle(B, L1, L2, lengths, go, ge, T, seed):
    s, v = _second_inputs(B, L1, L2, seed)
    ln = None if lengths is None else torch.tensor(lengths, dtype=torch.int32)
    lnd = None if ln is None else ln.cuda()
    lnn = None if ln is None else ln.numpy()
    got = torch.ops.orihime.nw_affine_marginals_hvp(s.cuda(), v.cuda(), go, ge, T, lnd).cpu().numpy()
    _check2("hvp", got, O.nw_affine_hvp(s.numpy(), v.numpy(), lnn, go, ge, T),
            O.nw_affine_hvp(s.numpy(), v.numpy(), lnn, go, ge, T, dtype=np.float64))
    if lengths is not None:
        for b, (l1, l2) in enumerate(lengths):
            assert not got[b, l1:, :].any() and not got[b, :, l2:].any()


@pytest.mark.parametrize("B,L1,L2,lengths,go,ge,T,seed", SECOND)
@pytest.mark.parametrize("param", [0, 1, 2])
def test_nw_affine_param_jacobian_matches_oracle(param, B, L1, L2, lengths, go, ge, T, seed):
    s, _ = _second_inputs(B, L1, L2, seed)
    ln = None if lengths is None else torch.tensor(lengths, dtype=torch.int32)
    lnd = None if ln is None else ln.cuda()
    lnn = None if ln is None else ln.numpy()
    ops = torch.ops.orihime
    fn = (ops.nw_affine_marginals_grad_gap_open, ops.nw_affine_marginals_grad_gap_ext,
          ops.nw_affine_marginals_grad_temp)[param]
    got = fn(s.cuda(), go, ge, T, lnd).cpu().numpy()
    _check2(f"dP/dtheta{param}", got, O.nw_affine_param_grad(s.numpy(), lnn, go, ge, T, param),
            O.nw_affine_param_grad(s.numpy(), lnn, go, ge, T, param, dtype=np.float64))


def test_nw_affine_marginals_backward_matches_oracle_contractions():
    B, L1, L2, go, ge, T = 3, 37, 145, -2.0, -0.5, 0.6
    s, gm = _second_inputs(B, L1, L2, 11)
    ln = torch.tensor([[37, 145], [20, 45], [37, 9]], dtype=torch.int32)
    sn, gn, lnn = s.numpy(), gm.numpy(), ln.numpy()
    out = torch.ops.orihime.nw_affine_marginals_backward(s.cuda(), gm.cuda(), go, ge, T, ln.cuda())
    _check2("grad_scores", out[0].cpu().numpy(), O.nw_affine_hvp(sn, gn, lnn, go, ge, T),
            O.nw_affine_hvp(sn, gn, lnn, go, ge, T, dtype=np.float64))
    for k in range(3):
        r64 = (gn.astype(np.float64) * O.nw_affine_param_grad(sn, lnn, go, ge, T, k, dtype=np.float64)).sum()
        r32 = (gn.astype(np.float64) * O.nw_affine_param_grad(sn, lnn, go, ge, T, k)).sum()
        got = float(out[1 + k].item())
        bound = max(abs(r32 - r64), 1e-4 * (1 + abs(r64)))
        print(f"  param {k}: ours {got:.6f} fp64 {r64:.6f} ref32 {r32:.6f}")
        assert abs(got - r64) <= bound


def test_nw_affine_public_autograd_and_legacy():
    import orihime_b200 as ob
    s = _gen((2, 30, 41), 31, 1.5).cuda()
    cot = _gen((2, 30, 41), 32).cuda()
    ln = torch.tensor([[30, 41], [22, 17]], dtype=torch.int32).cuda()
    kw = dict(gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.7, lengths=ln)
    x = s.clone().requires_grad_(True)
    (dm,) = torch.autograd.grad((ob.nw_affine(x, **kw) * cot).sum(), x)
    ref = torch.ops.orihime.nw_affine_marginals_hvp(s, cot, -2.0, -0.5, 0.7, ln)
    assert torch.allclose(dm, ref, rtol=1e-6, atol=1e-7)
    x = s.clone().requires_grad_(True)
    (de,) = torch.autograd.grad(ob.nw_affine_entropy(x, **kw).sum(), x)
    assert torch.allclose(de, torch.ops.orihime.nw_affine_marginals_grad_temp(s, -2.0, -0.5, 0.7, ln),
                          rtol=1e-6, atol=1e-7)
    # tensor parameters through the AutogradCUDA forward
    go = torch.tensor(-2.0, device="cuda", requires_grad=True)
    ge = torch.tensor(-0.5, device="cuda", requires_grad=True)
    tp = torch.tensor(0.7, device="cuda", requires_grad=True)
    x = s.clone().requires_grad_(True)
    v, m = torch.ops.orihime.nw_affine_forward_t(x, go, ge, tp, ln)
    (v.sum() + (m * cot).sum()).backward()
    _, g0, g1, gT = torch.ops.orihime.nw_affine_value_grad_params(s, -2.0, -0.5, 0.7, ln)
    mb = torch.ops.orihime.nw_affine_marginals_backward(s, cot, -2.0, -0.5, 0.7, ln)
    assert torch.allclose(go.grad, g0.sum() + mb[1][0], rtol=1e-5, atol=1e-5)
    assert torch.allclose(ge.grad, g1.sum() + mb[2][0], rtol=1e-5, atol=1e-5)
    assert torch.allclose(tp.grad, gT.sum() + mb[3][0], rtol=1e-5, atol=1e-5)
    from orihime_b200 import _ops
    if len(_ops.LEGACY_DEFINED_HERE) == len(_ops.LEGACY_SCHEMAS):
        o = torch.ops.orihime
        assert all(torch.equal(a, b) for a, b in zip(o.soft_nw_affine_float(s, -2.0, -0.5, 0.7, ln),
                                                      o.nw_affine_forward(s, -2.0, -0.5, 0.7, ln)))
        for k, name in enumerate(("gap_open", "gap_ext", "temp")):
            assert torch.equal(o.soft_nw_affine_param_jacobian(s, k, -2.0, -0.5, 0.7, ln),
                               getattr(o, f"nw_affine_marginals_grad_{name}")(s, -2.0, -0.5, 0.7, ln))
        with pytest.raises(RuntimeError, match="param_type must be 0, 1, or 2"):
            o.soft_nw_affine_param_jacobian(s, 3, -2.0, -0.5, 0.7, ln)


def test_nw_affine_public_api_vs_golden(golden):
    """ohm.nw_affine / nw_affine_value / nw_affine_entropy and the map VJP,
    against fixtures recorded from the reference's public API."""
    import orihime_b200 as ob
    for case in ("sq", "rect", "ragged", "unit", "row"):
        s = torch.from_numpy(golden[f"{case}/scores"]).cuda()
        cot = torch.from_numpy(golden[f"{case}/cot"]).cuda()
        ln = (torch.from_numpy(golden[f"{case}/lengths"]).to(torch.int32).cuda()
              if f"{case}/lengths" in golden.files else None)
        g = lambda k: golden[f"{case}/nwa/{k}"]  # noqa: E731
        kw = dict(gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.7, lengths=ln)
        np.testing.assert_allclose(ob.nw_affine_value(s, **kw).cpu().numpy(), g("value"), rtol=1e-5,
                                   atol=1e-5)
        x = s.clone().requires_grad_(True)
        (dx,) = torch.autograd.grad(-ob.nw_affine_value(x, **kw).mean(), x)
        np.testing.assert_allclose(dx.cpu().numpy(), g("dvalue"), atol=1e-5)
        x = s.clone().requires_grad_(True)
        (dm,) = torch.autograd.grad((ob.nw_affine(x, **kw) * cot).sum(), x)
        np.testing.assert_allclose(dm.cpu().numpy(), g("dmap"), atol=1e-5)
        x = s.clone().requires_grad_(True)
        h = ob.nw_affine_entropy(x, **kw)
        np.testing.assert_allclose(h.detach().cpu().numpy(), g("entropy"), atol=2e-5)
        (de,) = torch.autograd.grad(h.sum(), x)
        np.testing.assert_allclose(de.cpu().numpy(), g("dentropy"), atol=1e-5)
        bw = torch.ops.orihime.nw_affine_marginals_backward(s, cot, -2.0, -0.5, 0.7, ln)
        np.testing.assert_allclose(bw[0].cpu().numpy(), g("bw_pair_scores"), atol=1e-5)
        for k, name in enumerate(("gap_open_score", "gap_extend_score", "temperature")):
            np.testing.assert_allclose(bw[1 + k].item(), g(f"bw_{name}"), atol=1e-4)
