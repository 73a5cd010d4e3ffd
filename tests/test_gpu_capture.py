"""The padded drop-in ops inside CUDA graphs.

The reference reads `lengths` (and tensor parameters, `.item()`) on the host
in every call.  Here those reads are skipped while a stream is being
captured: lengths are range-checked on the device (a pair outside the padded
size comes back NaN), and the `_t` ops of the local families hand their
parameter tensors to the kernels as a device array, so a replay uses their
current values.  Eager calls keep the reference's host checks and messages.
"""

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    import orihime_b200  # noqa: F401


def _scores(B, L1, L2, seed):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(B, L1, L2, generator=g) * 1.5).cuda()


def _capture(fn):
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        fn()                     # warm-up outside the capture
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out = fn()
    return g, out


@pytest.mark.parametrize("fam", ["affine", "linear"])
def test_forward_with_lengths_replays_with_new_scores(fam):
    ops = torch.ops.orihime
    B, L1, L2 = 5, 70, 150
    x = _scores(B, L1, L2, 1)
    ln = torch.tensor([[70, 150], [33, 129], [0, 10], [70, 1], [12, 140]], dtype=torch.int32, device="cuda")
    call = ((lambda: ops.sw_affine_forward(x, -2.0, -0.5, 0.5, ln)) if fam == "affine"
            else (lambda: ops.sw_forward(x, -1.0, 0.5, ln)))
    g, (v, m) = _capture(call)
    for seed in (2, 3):
        x.copy_(_scores(B, L1, L2, seed))
        g.replay()
        torch.cuda.synchronize()
        ve, me = call()
        assert torch.equal(v, ve) and torch.equal(m, me)


@pytest.mark.parametrize("fam", ["affine", "linear"])
def test_forward_t_replays_with_new_parameter_values(fam):
    ops = torch.ops.orihime
    B, L1, L2 = 3, 60, 90
    x = _scores(B, L1, L2, 4)
    ln = torch.tensor([[60, 90], [17, 90], [60, 33]], dtype=torch.int32, device="cuda")
    if fam == "affine":
        go, ge, T = (torch.tensor(v, device="cuda") for v in (-2.0, -0.5, 0.5))
        call = lambda: ops.sw_affine_forward_t(x, go, ge, T, ln)  # noqa: E731
        eager = lambda: ops.sw_affine_forward(x, float(go), float(ge), float(T), ln)  # noqa: E731
        params = (go, ge, T)
    else:
        gp, T = (torch.tensor(v, device="cuda") for v in (-1.0, 0.5))
        call = lambda: ops.sw_forward_t(x, gp, T, ln)  # noqa: E731
        eager = lambda: ops.sw_forward(x, float(gp), float(T), ln)  # noqa: E731
        params = (gp, T)
    g, (v, m) = _capture(call)
    for new in ((-1.5, -0.25, 0.8), (-3.0, -1.0, 0.3)):
        for p, val in zip(params, new if fam == "affine" else (new[0], new[2])):
            p.fill_(val)
        g.replay()
        torch.cuda.synchronize()
        ve, me = eager()
        torch.testing.assert_close(v, ve, rtol=1e-6, atol=1e-7)
        torch.testing.assert_close(m, me, rtol=1e-6, atol=1e-7)


def test_bad_lengths_under_capture_give_nan_for_that_pair():
    ops = torch.ops.orihime
    x = _scores(3, 40, 50, 5)
    ln = torch.tensor([[40, 50], [39, 50], [20, 30]], dtype=torch.int32, device="cuda")
    g, (v, m) = _capture(lambda: ops.sw_affine_forward(x, -2.0, -0.5, 0.5, ln))
    ln[1, 0] = 41          # the replay reads the tensor's current values: pair 1 has L1 > 40
    g.replay()
    torch.cuda.synchronize()
    assert torch.isnan(v[1]) and torch.isfinite(v[0]) and torch.isfinite(v[2])
    # eagerly the same call raises the reference's message
    with pytest.raises(RuntimeError, match=r"lengths\[1,0\] must be between 0 and 40, got 41"):
        ops.sw_affine_forward(x, -2.0, -0.5, 0.5, ln)
