"""Saigo-Vert local alignment (linear and affine gaps): the CUDA path vs the oracle.

The oracle's float restatement reproduces the reference CPU kernels
(src/sv_affine/kernels_cpu.cpp, src/sv_linear/kernels_cpu.cpp) bit for bit
("ref32"); its double instantiation is the truth ("fp64").  The linear model
runs the affine kernels with gap_open = gap_ext = gap.  Bars: value error <=
1e-5 * max(|S|, 1) against ref32 (S = LSE(0, M cells) can sit near 0); map
and gradients within max(floor, |ref32 - fp64|) of fp64 (map floor 1e-5
absolute, gradient floor 1e-4 relative); second-order outputs within the
reference's own fp32 error, floor 1e-4 of the largest exact entry.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

VAL_RTOL = 1e-5
MAP_ATOL = 1e-5
GAPS = {True: (-1.0,), False: (-2.0, -0.5)}


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


def _oargs(lin, gaps):
    return (gaps[0], gaps[0]) if lin else gaps


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


def _cmp(lin, s, ln, gaps, T):
    o = torch.ops.orihime
    sd = s.cuda().contiguous()
    lnd = None if ln is None else ln.cuda()
    if lin:
        v, m = o.sv_linear_forward(sd, *gaps, T, lnd)
        gg = o.sv_linear_value_grad_params(sd, *gaps, T, lnd)
        keys = ("grad_open", "grad_temp")
    else:
        v, m = o.sv_affine_forward(sd, *gaps, T, lnd)
        gg = o.sv_affine_value_grad_params(sd, *gaps, T, lnd)
        keys = ("grad_open", "grad_ext", "grad_temp")
    torch.cuda.synchronize()
    sn, lnn = s.numpy(), (None if ln is None else ln.numpy())
    r32 = O.sv(sn, lnn, *_oargs(lin, gaps), T, linear=lin)
    r64 = O.sv(sn, lnn, *_oargs(lin, gaps), T, linear=lin, dtype=np.float64)
    v, m = v.cpu().numpy(), m.cpu().numpy()
    rel = np.abs(v - r32["value"]) / np.maximum(np.abs(r32["value"]), 1.0)
    print(f"  value err / max(|S|, 1) vs ref32 {rel.max() if rel.size else 0:.2e}")
    assert (rel.max() if rel.size else 0) <= VAL_RTOL
    _check("value", v, r32["value"], r64["value"], VAL_RTOL, rel=True)
    _check("map", m, r32["map"], r64["map"], MAP_ATOL)
    for got, key in zip(gg, keys):
        g = got.cpu().numpy()
        floor = 1e-4 * (1.0 + np.abs(r64[key]).max()) if g.size else 1e-4
        _check(key, g, r32[key], r64[key], floor)
    if ln is not None:
        for b, (l1, l2) in enumerate(lnn.tolist()):
            assert not m[b, l1:, :].any() and not m[b, :, l2:].any()
    return v, m


@pytest.mark.parametrize("lin", [False, True])
@pytest.mark.parametrize("B", [1, 4])
@pytest.mark.parametrize("shape", [(8, 10), (16, 16), (5, 20)])
@pytest.mark.parametrize("T", [0.1, 1.0, 2.0])
def test_sv_reference_grid(lin, B, shape, T):
    _cmp(lin, _gen((B, *shape), 42, 1.5), None, GAPS[lin], T)


@pytest.mark.parametrize("lin", [False, True])
def test_sv_lengths_multiband_and_edges(lin):
    s = _gen((6, 40, 300), 5, 1.5)
    ln = torch.tensor([[40, 300], [0, 7], [9, 0], [1, 1], [33, 129], [40, 5]], dtype=torch.int32)
    v, _ = _cmp(lin, s, ln, GAPS[lin], 0.8)
    assert v[1] == 0.0 and v[2] == 0.0   # an empty side leaves the empty alignment: S = 0
    _cmp(lin, _emb_scores(2, 513, 700, 64, 9), torch.tensor([[513, 700], [300, 651]],
                                                             dtype=torch.int32), GAPS[lin], 0.5)


def test_sv_value_only_ragged_plan_and_determinism():
    from orihime_b200 import ragged
    s = _emb_scores(4, 300, 500, 32, 11).cuda()
    ln = torch.tensor([[300, 500], [200, 450], [0, 10], [299, 1]], dtype=torch.int32, device="cuda")
    v1, m1 = torch.ops.orihime.sv_affine_forward(s, -2.0, -0.5, 0.7, ln)
    v2, m2 = torch.ops.orihime.sv_affine_forward(s, -2.0, -0.5, 0.7, ln)
    assert torch.equal(v1, v2) and torch.equal(m1, m2)
    assert torch.equal(torch.ops.orihime_b200.sv_affine_value(s, -2.0, -0.5, 0.7, ln), v1)
    assert torch.equal(torch.ops.orihime_b200.sv_linear_value(s, -1.0, 0.7, ln),
                       torch.ops.orihime.sv_linear_forward(s, -1.0, 0.7, ln)[0])
    rng = np.random.default_rng(23)
    lens = np.stack([rng.integers(0, 300, 30), rng.integers(0, 520, 30)], 1)
    lens[3] = [0, 50]
    mats = [_gen((int(a), int(b)), 300 + k, 1.5) for k, (a, b) in enumerate(lens)]
    flat, off, l32 = ragged.pack([m.cuda() for m in mats])
    plan = ragged.Plan(l32, off, family="saigo_vert", device="cuda")
    out = plan.run(flat.cuda(), gap_open=-2.0, gap_ext=-0.5, temp=0.6)
    vals = plan.values(flat.cuda(), gap_open=-2.0, gap_ext=-0.5, temp=0.6)
    pad = torch.zeros(len(mats), int(lens[:, 0].max()), int(lens[:, 1].max()))
    for k, m in enumerate(mats):
        pad[k, :m.shape[0], :m.shape[1]] = m
    lt = torch.tensor(lens, dtype=torch.int32).cuda()
    v, m = torch.ops.orihime.sv_affine_forward(pad.cuda(), -2.0, -0.5, 0.6, lt)
    go, ge, gT = torch.ops.orihime.sv_affine_value_grad_params(pad.cuda(), -2.0, -0.5, 0.6, lt)
    assert torch.equal(out.value, v) and torch.equal(vals, v)
    assert torch.equal(out.grad_open, go) and torch.equal(out.grad_ext, ge) and torch.equal(out.grad_temp, gT)
    for k, mk in enumerate(ragged.unpack(out.map, off, l32)):
        assert torch.equal(mk, m[k, :int(lens[k, 0]), :int(lens[k, 1])]), k


def _check2(name, got, r32, r64, rel_floor=1e-4):
    got, r32, r64 = (np.asarray(x, np.float64) for x in (got, r32, r64))
    scale = max(float(np.abs(r64).max()), 1e-12)
    e64 = float(np.abs(got - r64).max())
    eref = float(np.abs(r32 - r64).max())
    bound = max(rel_floor * scale, eref)
    print(f"  {name:14s} ours-fp64 {e64:.2e}  ref32-fp64 {eref:.2e}  bound {bound:.2e}  scale {scale:.2e}")
    assert e64 <= bound, f"{name}: {e64:.3e} > {bound:.3e}"


SECOND = [
    (2, 24, 31, None, 0.7, 1),
    (4, 10, 12, [[8, 10], [10, 12], [0, 5], [7, 0]], 1.0, 2),
    (2, 64, 48, None, 0.3, 3),
    (1, 130, 300, None, 0.5, 4),
]


@pytest.mark.parametrize("lin", [False, True])
@pytest.mark.parametrize("B,L1,L2,lengths,T,seed", SECOND)
def test_sv_second_order_matches_oracle(lin, B, L1, L2, lengths, T, seed):
    o = torch.ops.orihime
    s, v = _gen((B, L1, L2), seed, 1.5), _gen((B, L1, L2), seed + 100)
    ln = None if lengths is None else torch.tensor(lengths, dtype=torch.int32)
    lnd = None if ln is None else ln.cuda()
    lnn = None if ln is None else ln.numpy()
    gaps = GAPS[lin]
    og = _oargs(lin, gaps)
    sn = s.numpy()
    hv = (o.sv_linear_marginals_hvp if lin else o.sv_affine_marginals_hvp)(s.cuda(), v.cuda(), *gaps, T, lnd)
    _check2("hvp", hv.cpu().numpy(), O.sv_hvp(sn, v.numpy(), lnn, *og, T),
            O.sv_hvp(sn, v.numpy(), lnn, *og, T, dtype=np.float64))
    fns = ((o.sv_linear_marginals_grad_gap, o.sv_linear_marginals_grad_temp) if lin else
           (o.sv_affine_marginals_grad_gap_open, o.sv_affine_marginals_grad_gap_ext,
            o.sv_affine_marginals_grad_temp))
    for p, fn in enumerate(fns):
        got = fn(s.cuda(), *gaps, T, lnd).cpu().numpy()
        _check2(f"dP/dtheta{p}", got, O.sv_param_grad(sn, lnn, *og, T, p, linear=lin),
                O.sv_param_grad(sn, lnn, *og, T, p, linear=lin, dtype=np.float64))
    bw = (o.sv_linear_marginals_backward if lin else o.sv_affine_marginals_backward)(
        s.cuda(), v.cuda(), *gaps, T, lnd)
    _check2("bw grad", bw[0].cpu().numpy(), O.sv_hvp(sn, v.numpy(), lnn, *og, T),
            O.sv_hvp(sn, v.numpy(), lnn, *og, T, dtype=np.float64))
    vn = v.numpy().astype(np.float64)
    # The temperature tangent comes from homogeneity in (s, go, ge, T) in the
    # same pass: T g_T = -sum(s * HG) - go * o - ge * e.  Errors D in the
    # returned HG and in the gap tangents o, e therefore move it by
    # -(sum(s * D) + go * Do + ge * De) / T; the check is that the scalar is
    # consistent with the identity given our other outputs (each bounded on
    # its own above and below).
    h64 = O.sv_hvp(sn, v.numpy(), lnn, *og, T, dtype=np.float64)
    dh = bw[0].cpu().numpy().astype(np.float64) - h64
    if lnn is not None:
        for b, (l1, l2) in enumerate(lnn.tolist()):
            dh[b, l1:, :] = 0.0
            dh[b, :, l2:] = 0.0
    r64s = [(vn * O.sv_param_grad(sn, lnn, *og, T, p, linear=lin, dtype=np.float64)).sum()
            for p in range(len(fns))]
    shift_T = -(sn.astype(np.float64) * dh).sum()
    for p, g in enumerate(gaps):
        shift_T -= g * (float(bw[1 + p].item()) - r64s[p])
    shift_T /= T
    for p in range(len(fns)):
        r64 = r64s[p]
        r32 = (vn * O.sv_param_grad(sn, lnn, *og, T, p, linear=lin)).sum()
        want = r64 + (shift_T if p == len(fns) - 1 else 0.0)
        got = float(bw[1 + p].item())
        print(f"  bw param {p}: got {got:.6e} fp64 {r64:.6e} identity shift {shift_T:.2e}")
        assert abs(got - want) <= max(abs(r32 - r64), 1e-4 * (1 + abs(r64))), p


@pytest.mark.parametrize("fam", ["svl", "sva"])
def test_sv_public_api_vs_golden(golden, fam):
    import orihime_b200 as ob
    lin = fam == "svl"
    fmap, fval, fent = ((ob.sv, ob.sv_value, ob.sv_entropy) if lin else
                        (ob.sv_affine, ob.sv_affine_value, ob.sv_affine_entropy))
    kw0 = (dict(gap_score=-1.0, temperature=0.7) if lin else
           dict(gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.7))
    for case in ("sq", "rect", "ragged", "unit", "row"):
        s = torch.from_numpy(golden[f"{case}/scores"]).cuda()
        cot = torch.from_numpy(golden[f"{case}/cot"]).cuda()
        ln = (torch.from_numpy(golden[f"{case}/lengths"]).to(torch.int32).cuda()
              if f"{case}/lengths" in golden.files else None)
        g = lambda k: golden[f"{case}/{fam}/{k}"]  # noqa: E731
        kw = dict(kw0, lengths=ln)
        np.testing.assert_allclose(fval(s, **kw).cpu().numpy(), g("value"), rtol=1e-5, atol=1e-5)
        x = s.clone().requires_grad_(True)
        (dx,) = torch.autograd.grad(-fval(x, **kw).mean(), x)
        np.testing.assert_allclose(dx.cpu().numpy(), g("dvalue"), atol=1e-5)
        x = s.clone().requires_grad_(True)
        (dm,) = torch.autograd.grad((fmap(x, **kw) * cot).sum(), x)
        np.testing.assert_allclose(dm.cpu().numpy(), g("dmap"), atol=1e-5)
        x = s.clone().requires_grad_(True)
        h = fent(x, **kw)
        np.testing.assert_allclose(h.detach().cpu().numpy(), g("entropy"), atol=2e-5)
        (de,) = torch.autograd.grad(h.sum(), x)
        np.testing.assert_allclose(de.cpu().numpy(), g("dentropy"), atol=1e-5)
        o = torch.ops.orihime
        if lin:
            bw = o.sv_linear_marginals_backward(s, cot, -1.0, 0.7, ln)
            names = ("gap_score", "temperature")
            jac = (o.sv_linear_marginals_grad_gap, o.sv_linear_marginals_grad_temp)
            args = (-1.0, 0.7)
        else:
            bw = o.sv_affine_marginals_backward(s, cot, -2.0, -0.5, 0.7, ln)
            names = ("gap_open_score", "gap_extend_score", "temperature")
            jac = (o.sv_affine_marginals_grad_gap_open, o.sv_affine_marginals_grad_gap_ext,
                   o.sv_affine_marginals_grad_temp)
            args = (-2.0, -0.5, 0.7)
        np.testing.assert_allclose(bw[0].cpu().numpy(), g("bw_pair_scores"), atol=1e-5)
        for k, name in enumerate(names):
            np.testing.assert_allclose(bw[1 + k].item(), g(f"bw_{name}"), atol=1e-4)
            np.testing.assert_allclose(jac[k](s, *args, ln).cpu().numpy(), g(f"sens_{name}"),
                                       atol=1e-4)


def test_sv_legacy_ops_equal_namespaced_ops():
    from orihime_b200 import _ops
    if len(_ops.LEGACY_DEFINED_HERE) != len(_ops.LEGACY_SCHEMAS):
        pytest.skip("the reference extension defined the legacy schemas; they stay its own")
    o = torch.ops.orihime
    s = _gen((3, 40, 57), 0, 1.5).cuda()
    v = _gen((3, 40, 57), 1).cuda()
    ln = torch.tensor([[40, 57], [13, 9], [40, 30]], dtype=torch.int32).cuda()
    eq = lambda a, b: all(torch.equal(x, y) for x, y in zip(a, b)) if isinstance(a, (list, tuple)) \
        else torch.equal(a, b)  # noqa: E731
    assert eq(o.soft_sv_affine_float(s, -2.0, -0.5, 0.7, ln), o.sv_affine_forward(s, -2.0, -0.5, 0.7, ln))
    assert eq(o.soft_sv_linear_float(s, -1.0, 0.7, ln), o.sv_linear_forward(s, -1.0, 0.7, ln))
    assert eq(o.soft_sv_affine_hvp(s, v, -2.0, -0.5, 0.7, ln), o.sv_affine_marginals_hvp(s, v, -2.0, -0.5, 0.7, ln))
    assert eq(o.soft_sv_linear_param_jacobian(s, 0, -1.0, 0.7, ln), o.sv_linear_marginals_grad_gap(s, -1.0, 0.7, ln))
    assert eq(o.soft_sv_affine_backward_full(s, v, -2.0, -0.5, 0.7, ln),
              o.sv_affine_marginals_backward(s, v, -2.0, -0.5, 0.7, ln))
    with pytest.raises(RuntimeError, match="param_type must be 0 or 1"):
        o.soft_sv_linear_param_jacobian(s, 2, -1.0, 0.7, ln)
