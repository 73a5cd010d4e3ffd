"""swb_sw_affine_forward_static: the workspace-free entry point.

Compared with swb_sw_affine_forward (caller workspace) on two calls in a row
with different batches, so state left in the fixed scratch by the first call
must not leak into the second.  Kept in its own file, collected last, and
independent of the other test files.
"""

import ctypes

import pytest
import torch

from orihime_b200 import _lib

GO, GE, T = -2.0, -0.5, 0.7


def _scores(B, L1, L2, seed):
    g = torch.Generator().manual_seed(seed)
    e = torch.randn(B, L1, 32, generator=g)
    f = torch.randn(B, L2, 32, generator=g)
    return (2.0 * e @ f.transpose(1, 2) / 32 ** 0.5).float()


def _outputs(B, L1, L2):
    z = lambda *s: torch.full(s, float("nan"), dtype=torch.float32, device="cuda")
    return dict(value=z(B), map=z(B, L1, L2), go=z(B), ge=z(B), gt=z(B))


def _ptrs(o):
    return [o[k].data_ptr() for k in ("value", "map", "go", "ge", "gt")]


def _with_workspace(lib, s, lengths):
    B, L1, L2 = s.shape
    o = _outputs(B, L1, L2)
    wb = lib.swb_sw_affine_workspace_bytes(B, L1, L2)
    ws = torch.empty(wb, dtype=torch.uint8, device="cuda")
    rc = lib.swb_sw_affine_forward(s.data_ptr(), lengths.data_ptr() if lengths is not None else None,
                                   B, L1, L2, GO, GE, T, *_ptrs(o), ws.data_ptr(), wb,
                                   torch.cuda.current_stream().cuda_stream, None)
    _lib.check(rc, "swb_sw_affine_forward")
    torch.cuda.synchronize()
    return o


def _static(lib, s, lengths):
    B, L1, L2 = s.shape
    o = _outputs(B, L1, L2)
    rc = lib.swb_sw_affine_forward_static(
        s.data_ptr(), lengths.data_ptr() if lengths is not None else None, B, L1, L2, GO, GE, T,
        *_ptrs(o), torch.cuda.current_stream().cuda_stream, None)
    _lib.check(rc, "swb_sw_affine_forward_static")
    torch.cuda.synchronize()
    return o


def test_oversize_rejected_before_any_cuda_call():
    lib = _lib.load()
    limit = 32 * 1024 * 1024
    assert lib.swb_sw_affine_workspace_bytes(1, 4096, 4096) > limit
    f = ctypes.c_float
    rc = lib.swb_sw_affine_forward_static(None, None, 1, 4096, 4096, f(GO), f(GE), f(T), None,
                                          None, None, None, None, None, None)
    assert rc == _lib.ERR_WORKSPACE
    assert b"too small" in lib.swb_error_string(rc)
    # a batch whose workspace query is within the limit always fits
    assert lib.swb_sw_affine_workspace_bytes(8, 512, 512) <= limit


@pytest.mark.gpu
def test_static_matches_workspace_entry_point_twice():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    lib = _lib.load()
    # call 1: a batch near the scratch limit (default 4 columns per lane), full lengths
    s1 = _scores(12, 512, 512, 11).cuda()
    # call 2: a smaller ragged batch, different shape, per-pair lengths
    s2 = _scores(5, 300, 170, 12).cuda()
    ln2 = torch.tensor([[300, 170], [1, 90], [257, 3], [0, 40], [120, 129]],
                       dtype=torch.int32, device="cuda")
    cases = [(s1, None), (s2, ln2)]
    got = [_static(lib, s, ln) for s, ln in cases]
    want = [_with_workspace(lib, s, ln) for s, ln in cases]
    for g, w in zip(got, want):
        for k in ("value", "map", "go", "ge", "gt"):
            assert torch.isfinite(g[k]).all(), k
            torch.testing.assert_close(g[k], w[k], rtol=1e-5, atol=1e-6, msg=k)
    # pair 3 of call 2 is empty: value, map and gradients are exactly 0
    assert float(got[1]["value"][3]) == 0.0 and not got[1]["map"][3].any()


@pytest.mark.gpu
def test_static_timeout_shows_in_results_and_status():
    """A bounded cross-band wait that expires (injected on the host: bands
    after the first wait on a word nobody writes, for at most 2 ms) marks the
    affected pairs NaN and sets the shared scratch's status word, which
    swb_static_read_status reads; the next call starts clean."""
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    lib = _lib.load()
    s = _scores(3, 64, 300, 13).cuda()          # 300 columns: three bands of 128
    ln = torch.tensor([[64, 300], [64, 100], [20, 300]], dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    o = _outputs(3, 64, 300)
    opt = _lib.Options(0, 2_000_000, 1, None, 0, 0)
    rc = lib.swb_sw_affine_forward_static(s.data_ptr(), ln.data_ptr(), 3, 64, 300, GO, GE, T,
                                          *_ptrs(o), st, ctypes.byref(opt))
    _lib.check(rc, "swb_sw_affine_forward_static")
    torch.cuda.synchronize()
    status = ctypes.c_uint(0)
    _lib.check(lib.swb_static_read_status(st, ctypes.byref(status)), "swb_static_read_status")
    assert status.value & _lib.STATUS_WAIT_TIMEOUT
    # pairs 0 and 2 have bands that waited: NaN; pair 1 (one band) is unaffected
    for k in ("value", "go", "ge", "gt"):
        assert torch.isnan(o[k][0]) and torch.isnan(o[k][2]), k
        assert torch.isfinite(o[k][1]), k
    # the next call resets the scratch: correct results, status clear
    got = _static(lib, s, ln)
    want = _with_workspace(lib, s, ln)
    _lib.check(lib.swb_static_read_status(st, ctypes.byref(status)), "swb_static_read_status")
    assert status.value == 0
    for k in ("value", "map", "go", "ge", "gt"):
        torch.testing.assert_close(got[k], want[k], rtol=1e-5, atol=1e-6, msg=k)
