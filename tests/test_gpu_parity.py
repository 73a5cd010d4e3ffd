"""CUDA path vs the oracle (FP32 restatement, bit-identical to the reference CPU
kernels; FP64 truth reported beside it).

Tolerances (north star): value relative error <= 1e-5 and map absolute error
<= 1e-5 against the FP32 reference path; gradients of the value with respect
to the gap/temperature parameters within 1e-4 relative + 1e-4 absolute.
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


def _cmp_affine(s, ln, go, ge, T, val_rtol=VAL_RTOL, map_atol=MAP_ATOL, fp64=False):
    dev = torch.device("cuda")
    sd = s.to(dev).contiguous()
    lnd = None if ln is None else ln.to(dev)
    v, m = torch.ops.orihime.sw_affine_forward(sd, go, ge, T, lnd)
    gg = torch.ops.orihime.sw_affine_value_grad_params(sd, go, ge, T, lnd)
    torch.cuda.synchronize()
    sn = s.numpy()
    lnn = None if ln is None else ln.numpy()
    o = O.affine(sn, lnn, go, ge, T)
    rel = np.abs(v.cpu().numpy() - o["value"]) / np.maximum(np.abs(o["value"]), 1e-6)
    err_map = np.abs(m.cpu().numpy() - o["map"]).max() if sn.size else 0.0
    assert rel.max() <= val_rtol, f"value rel err {rel.max():.3e}"
    assert err_map <= map_atol, f"map abs err {err_map:.3e}"
    for got, key in zip(gg, ("grad_open", "grad_ext", "grad_temp")):
        np.testing.assert_allclose(got.cpu().numpy(), o[key], rtol=1e-4, atol=1e-4, err_msg=key)
    if ln is not None:
        mm = m.cpu().numpy()
        for b, (l1, l2) in enumerate(lnn.tolist()):
            assert not mm[b, l1:, :].any() and not mm[b, :, l2:].any()
    if fp64:
        o64 = O.affine(sn, lnn, go, ge, T, dtype=np.float64)
        return (np.abs(v.cpu().numpy() - o64["value"]).max(),
                np.abs(m.cpu().numpy() - o64["map"]).max())
    return rel.max(), err_map


def _cmp_linear(s, ln, gap, T, val_rtol=VAL_RTOL, map_atol=MAP_ATOL):
    dev = torch.device("cuda")
    sd = s.to(dev).contiguous()
    lnd = None if ln is None else ln.to(dev)
    v, m = torch.ops.orihime.sw_forward(sd, gap, T, lnd)
    gg = torch.ops.orihime.sw_value_grad_params(sd, gap, T, lnd)
    torch.cuda.synchronize()
    lnn = None if ln is None else ln.numpy()
    o = O.linear(s.numpy(), lnn, gap, T)
    rel = np.abs(v.cpu().numpy() - o["value"]) / np.maximum(np.abs(o["value"]), 1e-6)
    err_map = np.abs(m.cpu().numpy() - o["map"]).max() if s.numel() else 0.0
    assert rel.max() <= val_rtol, f"value rel err {rel.max():.3e}"
    assert err_map <= map_atol, f"map abs err {err_map:.3e}"
    for got, key in zip(gg, ("grad_gap", "grad_temp")):
        np.testing.assert_allclose(got.cpu().numpy(), o[key], rtol=1e-4, atol=1e-4, err_msg=key)
    return rel.max(), err_map


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
    """C2 score generator (3<e,f>/sqrt(64)), go -2, ge -0.5, T 0.5; FP64 error reported."""
    s = _emb_scores(2, 256, 256, 64, 1)
    ev, em = _cmp_affine(s, None, -2.0, -0.5, 0.5, fp64=True)
    print(f"C2@256 vs FP64: value abs err {ev:.3e}, map abs err {em:.3e}")


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


def test_padding_invariance_bitwise():
    """A pair inside a padded batch (lengths) equals the cropped pair bit for bit."""
    s = _emb_scores(3, 300, 420, 64, 4).cuda()
    ln = torch.tensor([[300, 420], [211, 137], [64, 399]], dtype=torch.int32, device="cuda")
    v, m = torch.ops.orihime.sw_affine_forward(s, -2.0, -0.5, 0.5, ln)
    for b, (l1, l2) in enumerate(ln.tolist()):
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
        o = O.affine(s[b:b + 1].numpy(), None, -2.0, -0.5, 0.5)
        rel = abs(float(v[b]) - o["value"][0]) / abs(o["value"][0])
        assert rel <= VAL_RTOL, rel
        err = np.abs(m[b].cpu().numpy() - o["map"][0]).max()
        assert err <= MAP_ATOL, err


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
    np.testing.assert_allclose(out[0].cpu().numpy(), o["value"], rtol=VAL_RTOL)
    assert np.abs(mp.cpu().numpy() - o["map"]).max() <= MAP_ATOL
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
    opt = _lib.Options(0, 2_000_000, 1)
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
    with pytest.raises(RuntimeError, match="scores must be a CUDA tensor"):
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
