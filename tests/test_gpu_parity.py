"""CUDA path vs the oracle.

The oracle's float restatement reproduces the reference CPU kernels bit for
bit ("ref32"); its double instantiation is the truth ("fp64").

Parity bar: value relative error <= 1e-5 against ref32.  For the
marginal map the bar is absolute error <= 1e-5, measured against the FP64
truth: on long pairs an FP32 forward-backward (the reference included) drifts
further than that from the truth, so the map must be within
max(1e-5, |ref32 - fp64|) of fp64, i.e. at least as accurate as the reference.
dS/d(gap, temperature) follow the same rule with a 1e-4 relative floor.
Every comparison prints the measured errors.
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


def _gen(shape, seed, scale=1.5):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(*shape, generator=g) * scale).float()


def _emb_scores(B, N, M, d, seed, scale=3.0):
    """3 <e_i, f_j> / sqrt(d) with e, f ~ N(0, 1): the C2 score generator."""
    g = torch.Generator().manual_seed(seed)
    e = torch.randn(B, N, d, generator=g)
    f = torch.randn(B, M, d, generator=g)
    return (scale * torch.bmm(e, f.transpose(1, 2)) / d ** 0.5).float()


def _maxabs(a, b):
    a = np.asarray(a, np.float64)
    return float(np.abs(a - np.asarray(b, np.float64)).max()) if a.size else 0.0


def _check(name, got, r32, r64, floor, rel=False):
    """got must be within max(floor, |ref32 - fp64|) of fp64."""
    if rel:
        scale = np.maximum(np.abs(np.asarray(r64, np.float64)), 1e-6)
        e64 = float(np.max(np.abs(np.asarray(got, np.float64) - r64) / scale)) if np.size(got) else 0.0
        eref = float(np.max(np.abs(np.asarray(r32, np.float64) - r64) / scale)) if np.size(got) else 0.0
    else:
        e64, eref = _maxabs(got, r64), _maxabs(r32, r64)
    bound = max(floor, eref)
    print(f"  {name:10s} ours-fp64 {e64:.2e}  ref32-fp64 {eref:.2e}  bound {bound:.2e}")
    assert e64 <= bound, f"{name}: error vs fp64 {e64:.3e} > {bound:.3e} (ref32 {eref:.3e})"
    return e64


def _cmp(fam, s, ln, params, fp64=True):
    dev = torch.device("cuda")
    sd = s.to(dev).contiguous()
    lnd = None if ln is None else ln.to(dev)
    sn = s.numpy()
    lnn = None if ln is None else ln.numpy()
    if fam == "aff":
        v, m = torch.ops.orihime.sw_affine_forward(sd, *params, lnd)
        gg = torch.ops.orihime.sw_affine_value_grad_params(sd, *params, lnd)
        r32 = O.affine(sn, lnn, *params)
        r64 = O.affine(sn, lnn, *params, dtype=np.float64)
        keys = ("grad_open", "grad_ext", "grad_temp")
    else:
        v, m = torch.ops.orihime.sw_forward(sd, *params, lnd)
        gg = torch.ops.orihime.sw_value_grad_params(sd, *params, lnd)
        r32 = O.linear(sn, lnn, *params)
        r64 = O.linear(sn, lnn, *params, dtype=np.float64)
        keys = ("grad_gap", "grad_temp")
    torch.cuda.synchronize()
    v, m = v.cpu().numpy(), m.cpu().numpy()
    rel = np.abs(v - r32["value"]) / np.maximum(np.abs(r32["value"]), 1e-6)
    print(f"  value rel vs ref32 {rel.max() if rel.size else 0:.2e}")
    assert (rel.max() if rel.size else 0) <= VAL_RTOL
    _check("value", v, r32["value"], r64["value"], VAL_RTOL, rel=True)
    em = _check("map", m, r32["map"], r64["map"], MAP_ATOL)
    for got, key in zip(gg, keys):
        g = got.cpu().numpy()
        floor = 1e-4 * (1.0 + np.abs(r64[key]).max()) if g.size else 1e-4
        _check(key, g, r32[key], r64[key], floor)
    if ln is not None:
        for b, (l1, l2) in enumerate(lnn.tolist()):
            assert not m[b, l1:, :].any() and not m[b, :, l2:].any()
    return em


def _cmp_affine(s, ln, go, ge, T):
    return _cmp("aff", s, ln, (go, ge, T))


def _cmp_linear(s, ln, gap, T):
    return _cmp("lin", s, ln, (gap, T))


# ---- the reference's own test grid (tests/test_soft_sw_affine.py:140-193) ----

@pytest.mark.parametrize("B", [1, 4])
@pytest.mark.parametrize("shape", [(8, 10), (16, 16), (5, 20)])
@pytest.mark.parametrize("T", [0.1, 1.0, 2.0])
def test_affine_reference_grid(B, shape, T):
    _cmp_affine(_gen((B, *shape), 42), None, -2.0, -0.5, T)


@pytest.mark.parametrize("B", [1, 4])
@pytest.mark.parametrize("shape", [(8, 10), (16, 16), (5, 20)])
@pytest.mark.parametrize("T", [0.1, 1.0, 2.0])
def test_linear_reference_grid(B, shape, T):
    _cmp_linear(_gen((B, *shape), 42), None, -1.0, T)


# ---- shapes that exercise lanes, bands, chunks ----

@pytest.mark.parametrize("shape", [(1, 1), (1, 37), (37, 1), (3, 129), (129, 3), (70, 300),
                                   (300, 70), (33, 513), (600, 40)])
def test_affine_shapes(shape):
    _cmp_affine(_gen((3, *shape), 7), None, -2.0, -0.5, 0.7)


@pytest.mark.parametrize("shape", [(1, 1), (1, 37), (37, 1), (70, 300), (300, 70), (33, 513)])
def test_linear_shapes(shape):
    _cmp_linear(_gen((3, *shape), 8), None, -1.0, 0.7)


def test_affine_ragged_lengths():
    s = _gen((6, 150, 290), 9)
    ln = torch.tensor([[150, 290], [0, 10], [7, 0], [1, 1], [149, 131], [40, 257]], dtype=torch.int32)
    _cmp_affine(s, ln, -2.0, -0.5, 0.8)


def test_linear_ragged_lengths():
    s = _gen((5, 90, 200), 10)
    ln = torch.tensor([[90, 200], [0, 5], [3, 0], [45, 129], [90, 1]], dtype=torch.int32)
    _cmp_linear(s, ln, -1.0, 0.8)


def test_config1_linear_b8_128():
    """Config 1: linear B=8, 128x128, N(0,1) scores, gap -1, T 1."""
    g = torch.Generator().manual_seed(0)
    s = torch.randn(8, 128, 128, generator=g)
    _cmp_linear(s, None, -1.0, 1.0)


def test_config2_generator_256():
    """C2 score generator (3<e,f>/sqrt(64)), go -2, ge -0.5, T 0.5."""
    _cmp_affine(_emb_scores(2, 256, 256, 64, 1), None, -2.0, -0.5, 0.5)


def test_empty_batch_and_zero_lengths():
    dev = torch.device("cuda")
    v, m = torch.ops.orihime.sw_affine_forward(torch.zeros(0, 4, 5, device=dev), -2.0, -0.5, 1.0, None)
    assert v.shape == (0,) and m.shape == (0, 4, 5)
    v, m = torch.ops.orihime.sw_affine_forward(torch.zeros(2, 0, 5, device=dev), -2.0, -0.5, 1.0, None)
    assert torch.all(v == 0) and m.shape == (2, 0, 5)


# ---- size-independent properties at full sizes ----

def test_scale_invariance_bitwise():
    """S(2x) = 2 S(x) and the map is unchanged, bit for bit: scaling scores,
    gaps and temperature by a power of two leaves the scaled domain identical."""
    s = _emb_scores(4, 512, 384, 64, 3).cuda()
    v1, m1 = torch.ops.orihime.sw_affine_forward(s, -2.0, -0.5, 0.5, None)
    v2, m2 = torch.ops.orihime.sw_affine_forward(s * 2, -4.0, -1.0, 1.0, None)
    assert torch.equal(v2, 2 * v1)
    assert torch.equal(m1, m2)


@pytest.mark.parametrize("width, pairs", [
    (420, [[300, 420], [211, 300], [64, 399]]),   # 8 columns per lane, padded and cropped
    (200, [[300, 200], [211, 137], [64, 199]]),   # 4 columns per lane
])
def test_padding_invariance_bitwise(width, pairs):
    """A pair inside a padded batch (lengths) equals the cropped pair bit for
    bit when both run at the same columns per lane (the default depends on
    the padded width: swb_cols_per_lane)."""
    from orihime_b200 import _lib

    lib = _lib.load()
    s = _emb_scores(3, 300, width, 64, 4).cuda()
    ln = torch.tensor(pairs, dtype=torch.int32, device="cuda")
    v, m = torch.ops.orihime.sw_affine_forward(s, -2.0, -0.5, 0.5, ln)
    for b, (l1, l2) in enumerate(ln.tolist()):
        assert lib.swb_cols_per_lane(3, l2, -2.0, -0.5, 0.5) == lib.swb_cols_per_lane(3, width, -2.0, -0.5, 0.5)
        vc, mc = torch.ops.orihime.sw_affine_forward(s[b:b + 1, :l1, :l2].contiguous(), -2.0, -0.5,
                                                     0.5, None)
        assert torch.equal(vc[0], v[b])
        assert torch.equal(mc[0], m[b, :l1, :l2])


def test_deterministic_bitwise():
    s = _emb_scores(8, 257, 300, 64, 5).cuda()
    a = torch.ops.orihime.sw_affine_value_grad_params(s, -2.0, -0.5, 0.5, None)
    b = torch.ops.orihime.sw_affine_value_grad_params(s, -2.0, -0.5, 0.5, None)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    v1, m1 = torch.ops.orihime.sw_affine_forward(s, -2.0, -0.5, 0.5, None)
    v2, m2 = torch.ops.orihime.sw_affine_forward(s, -2.0, -0.5, 0.5, None)
    assert torch.equal(v1, v2) and torch.equal(m1, m2)


def test_config2_full_size_sampled_pairs():
    """Config 2 at full size (B=64, 1024x1024): properties on all pairs, the
    oracle on two sampled pairs."""
    s = _emb_scores(64, 1024, 1024, 64, 1)
    sd = s.cuda()
    v, m = torch.ops.orihime.sw_affine_forward(sd, -2.0, -0.5, 0.5, None)
    go, ge, gT = torch.ops.orihime.sw_affine_value_grad_params(sd, -2.0, -0.5, 0.5, None)
    assert torch.isfinite(v).all() and torch.isfinite(m).all()
    assert float(m.min()) >= 0.0 and float(m.max()) <= 1.0 + 1e-5
    # dS/dT identity holds by construction: (S - sum P s - go g_o - ge g_e) / T
    ps = (m * sd).sum(dim=(1, 2))
    gT_chk = (v - ps - (-2.0) * go - (-0.5) * ge) / 0.5
    torch.testing.assert_close(gT, gT_chk, rtol=1e-3, atol=1e-2)
    for b in (0, 37):
        sb = s[b:b + 1].numpy()
        r32 = O.affine(sb, None, -2.0, -0.5, 0.5)
        r64 = O.affine(sb, None, -2.0, -0.5, 0.5, dtype=np.float64)
        rel = abs(float(v[b]) - r32["value"][0]) / abs(r32["value"][0])
        print(f"  pair {b}: value rel vs ref32 {rel:.2e}")
        assert rel <= VAL_RTOL, rel
        _check("map", m[b:b + 1].cpu().numpy(), r32["map"], r64["map"], MAP_ATOL)


@pytest.mark.parametrize("fam", ["aff", "lin"])
def test_quiet_chunks_stay_within_tolerance(fam):
    """Long pairs where most adjoint chunks carry negligible flow: there the
    kernel writes zeros instead of recomputing, dropping values below ~2e-15.
    The map, value and gradients stay within the usual bounds of fp64; cells
    that the fp64 map puts below 1e-12 stay below 1e-12; two runs agree bit
    for bit (the skip decisions do not depend on timing)."""
    s = _emb_scores(2, 1200, 900, 64, 7)
    params = (-2.0, -0.5, 0.5) if fam == "aff" else (-1.0, 0.5)
    _cmp(fam, s, None, params)
    op = torch.ops.orihime.sw_affine_forward if fam == "aff" else torch.ops.orihime.sw_forward
    sd = s.cuda()
    _, m1 = op(sd, *params, None)
    _, m2 = op(sd, *params, None)
    assert torch.equal(m1, m2)
    r64 = (O.affine if fam == "aff" else O.linear)(s.numpy(), None, *params, dtype=np.float64)["map"]
    tiny = r64 < 1e-12
    print(f"  cells below 1e-12 in fp64: {tiny.mean():.2f}")
    assert tiny.mean() > 0.5   # the case does reach quiet regions
    assert float(m1.cpu().numpy()[tiny].max()) < 1e-12


@pytest.mark.parametrize("fam", ["aff", "lin"])
def test_quiet_chunks_with_unaligned_rows(fam):
    """Quiet chunks write their zero map rows in whole row pieces; with a
    padded width that is not a multiple of 4 the rows are not 16-byte aligned
    and the pieces are written element by element.  Ragged lengths put the
    pairs' right edges (pitch padding written as 0) inside those pieces."""
    s = _emb_scores(3, 1100, 1001, 64, 9)
    ln = torch.tensor([[1100, 1001], [1037, 998], [640, 733]], dtype=torch.int32)
    params = (-2.0, -0.5, 0.5) if fam == "aff" else (-1.0, 0.5)
    _cmp(fam, s, ln, params)


# ---- through the C ABI directly ----

def test_c_abi_direct_call():
    from orihime_b200 import _lib

    lib = _lib.load()
    s = _gen((2, 40, 150), 11).cuda()
    B, L1, L2 = s.shape
    out = [torch.empty(B, device="cuda") for _ in range(4)]
    mp = torch.empty_like(s)
    nb = lib.swb_sw_affine_workspace_bytes(B, L1, L2)
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    rc = lib.swb_sw_affine_forward(s.data_ptr(), None, B, L1, L2, -2.0, -0.5, 0.9,
                                   out[0].data_ptr(), mp.data_ptr(), out[1].data_ptr(),
                                   out[2].data_ptr(), out[3].data_ptr(), ws.data_ptr(), nb,
                                   torch.cuda.current_stream().cuda_stream, None)
    assert rc == 0
    torch.cuda.synchronize()
    o = O.affine(s.cpu().numpy(), None, -2.0, -0.5, 0.9)
    o64 = O.affine(s.cpu().numpy(), None, -2.0, -0.5, 0.9, dtype=np.float64)
    np.testing.assert_allclose(out[0].cpu().numpy(), o["value"], rtol=VAL_RTOL)
    _check("map", mp.cpu().numpy(), o["map"], o64["map"], MAP_ATOL)
    st = ctypes_status(lib, ws)
    assert st == 0


def ctypes_status(lib, ws):
    import ctypes

    st = ctypes.c_uint(0)
    rc = lib.swb_read_status(ws.data_ptr(), torch.cuda.current_stream().cuda_stream,
                             ctypes.byref(st))
    assert rc == 0
    return st.value


def test_bounded_wait_reports_timeout_and_context_survives():
    """Fault injection on the host side: band>0 waits on a word nobody writes,
    with a 2 ms bound.  The kernel must return, report the timeout in the status
    word, and leave the context usable."""
    from orihime_b200 import _lib

    lib = _lib.load()
    s = _gen((1, 20, 300), 12).cuda()  # 3 bands
    B, L1, L2 = s.shape
    outs = [torch.empty(B, device="cuda") for _ in range(4)]
    mp = torch.empty_like(s)
    nb = lib.swb_sw_affine_workspace_bytes(B, L1, L2)
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    opt = _lib.Options(0, 2_000_000, 1, None, 0)
    rc = lib.swb_sw_affine_forward(s.data_ptr(), None, B, L1, L2, -2.0, -0.5, 0.9,
                                   outs[0].data_ptr(), mp.data_ptr(), outs[1].data_ptr(),
                                   outs[2].data_ptr(), outs[3].data_ptr(), ws.data_ptr(), nb,
                                   torch.cuda.current_stream().cuda_stream, opt)
    assert rc == 0
    st = ctypes_status(lib, ws)
    assert st & _lib.STATUS_WAIT_TIMEOUT
    # the context still works
    _cmp_affine(_gen((1, 9, 9), 13), None, -2.0, -0.5, 1.0)


# ---- the reference's validation messages ----

def test_validation_messages():
    dev = torch.device("cuda")
    op = torch.ops.orihime.sw_affine_forward
    # CPU tensors never reach the CUDA kernels: without the reference's CPU
    # extension loaded the dispatcher refuses them outright.
    if not torch._C._dispatch_has_kernel_for_dispatch_key("orihime::sw_affine_forward", "CPU"):
        with pytest.raises(NotImplementedError, match="CPU"):
            op(torch.zeros(1, 3, 3), -2.0, -0.5, 1.0, None)
    with pytest.raises(RuntimeError, match="scores must be contiguous"):
        op(torch.zeros(1, 3, 4, device=dev).transpose(1, 2), -2.0, -0.5, 1.0, None)
    with pytest.raises(RuntimeError, match="scores must be float32"):
        op(torch.zeros(1, 3, 3, device=dev, dtype=torch.float64), -2.0, -0.5, 1.0, None)
    with pytest.raises(RuntimeError, match="scores must be 3D"):
        op(torch.zeros(3, 3, device=dev), -2.0, -0.5, 1.0, None)
    bad = torch.tensor([[5, 2]], dtype=torch.int32, device=dev)
    with pytest.raises(RuntimeError, match=r"lengths\[0,0\] must be between 0 and 4"):
        op(torch.zeros(1, 4, 4, device=dev), -2.0, -0.5, 1.0, bad)
    with pytest.raises(RuntimeError, match="lengths must be int32"):
        op(torch.zeros(1, 4, 4, device=dev), -2.0, -0.5, 1.0, bad.long())
    with pytest.raises(RuntimeError, match="gap_open must be a scalar tensor"):
        torch.ops.orihime.sw_affine_forward_t(torch.zeros(1, 4, 4, device=dev),
                                              torch.zeros(2, device=dev), torch.zeros(1, device=dev),
                                              torch.ones(1, device=dev),
                                              torch.tensor([[4, 4]], dtype=torch.int32, device=dev))


@pytest.mark.parametrize("shape", [(1, 1), (37, 1), (70, 300), (300, 70), (129, 65)])
@pytest.mark.parametrize("fam", ["aff", "lin"])
def test_two_columns_per_lane_variant(shape, fam):
    """The R=2 band layout (64-column bands) through the C ABI, vs the oracle."""
    from orihime_b200 import _lib

    lib = _lib.load()
    s = _gen((3, *shape), 21)
    sd = s.cuda()
    B, L1, L2 = s.shape
    outs = [torch.empty(B, device="cuda") for _ in range(4)]
    mp = torch.empty_like(sd)
    opt = _lib.Options(0, 0, 0, None, 2)
    st = torch.cuda.current_stream().cuda_stream
    if fam == "aff":
        nb = lib.swb_sw_affine_workspace_bytes(B, L1, L2)
        ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
        rc = lib.swb_sw_affine_forward(sd.data_ptr(), None, B, L1, L2, -2.0, -0.5, 0.8,
                                       outs[0].data_ptr(), mp.data_ptr(), outs[1].data_ptr(),
                                       outs[2].data_ptr(), outs[3].data_ptr(), ws.data_ptr(), nb,
                                       st, opt)
        r32 = O.affine(s.numpy(), None, -2.0, -0.5, 0.8)
        r64 = O.affine(s.numpy(), None, -2.0, -0.5, 0.8, dtype=np.float64)
    else:
        nb = lib.swb_sw_workspace_bytes(B, L1, L2)
        ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
        rc = lib.swb_sw_forward(sd.data_ptr(), None, B, L1, L2, -1.0, 0.8, outs[0].data_ptr(),
                                mp.data_ptr(), outs[1].data_ptr(), outs[3].data_ptr(),
                                ws.data_ptr(), nb, st, opt)
        r32 = O.linear(s.numpy(), None, -1.0, 0.8)
        r64 = O.linear(s.numpy(), None, -1.0, 0.8, dtype=np.float64)
    assert rc == 0
    torch.cuda.synchronize()
    np.testing.assert_allclose(outs[0].cpu().numpy(), r32["value"], rtol=VAL_RTOL)
    _check("map", mp.cpu().numpy(), r32["map"], r64["map"], MAP_ATOL)
