"""The checkpointed value op: the forward launches only the forward wavefront
and keeps sparse checkpoints; the backward runs the adjoint on them.

Its results equal the one-call forward + adjoint bit for bit whatever the
checkpoint stride: the adjoint rebuilds the skipped chunks' state with the
forward's own steps.  Memory between the two launches is reported per cell.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    import orihime_b200  # noqa: F401


def _emb(B, N, M, seed, d=64):
    g = torch.Generator().manual_seed(seed)
    e = torch.randn(B, N, d, generator=g)
    f = torch.randn(B, M, d, generator=g)
    return (3.0 * torch.bmm(e, f.transpose(1, 2)) / d ** 0.5).float().cuda()


@pytest.mark.parametrize("fam", ["sw_affine", "sw"])
@pytest.mark.parametrize("ck_every", [1, 2, 4, 16])
def test_checkpointed_adjoint_equals_one_call(fam, ck_every):
    from orihime_b200 import _ops

    s = _emb(4, 300, 211, 1)
    ln = torch.tensor([[300, 211], [77, 200], [0, 9], [299, 3]], dtype=torch.int32, device="cuda")
    params = (-2.0, -0.5, 0.5) if fam == "sw_affine" else (-1.0, 0.5)
    run = _ops.run_affine if fam == "sw_affine" else _ops.run_linear
    want = run(s, ln, *params)
    value, ws = _ops.run_checkpoint(fam, s, ln, params, ck_every)
    assert torch.equal(value, want[0])
    for _ in range(2):   # the adjoint can run more than once on one workspace
        got = _ops.run_adjoint(fam, s, ln, params, ck_every, ws)
        torch.cuda.synchronize()
        for g, w in zip(got, want):
            assert torch.equal(g, w)
    cells = 4 * 300 * 211
    print(f"  {fam} ck_every {ck_every}: workspace {ws.numel() / cells:.2f} B per padded cell")


def test_checkpoint_bytes_per_cell_at_stride_4():
    """The memory the value op keeps between forward and backward on a large
    batch: below 2 bytes per cell (the map it replaces is 4)."""
    from orihime_b200 import _lib

    lib = _lib.load()
    for B, L1, L2 in ((64, 1024, 1024), (4, 16384, 16384)):
        nb = lib.swb_sw_affine_checkpoint_workspace_bytes(B, L1, L2, 4)
        per = nb / (B * L1 * L2)
        print(f"  {B} x {L1} x {L2}: {per:.2f} B/cell kept between forward and backward")
        assert per < 2.0


@pytest.mark.parametrize("fam", ["sw_affine", "sw"])
def test_value_backward_uses_the_checkpointed_op(fam, monkeypatch):
    import orihime_b200 as ohm
    from orihime_b200 import _ops

    s = _emb(3, 120, 90, 2).requires_grad_(True)
    calls = {"checkpoint": 0, "adjoint": 0, "full": 0}
    real_c, real_a = _ops.run_checkpoint, _ops.run_adjoint
    real_f = _ops.run_affine if fam == "sw_affine" else _ops.run_linear
    monkeypatch.setattr(_ops, "run_checkpoint",
                        lambda *a, **k: calls.__setitem__("checkpoint", calls["checkpoint"] + 1) or real_c(*a, **k))
    monkeypatch.setattr(_ops, "run_adjoint",
                        lambda *a, **k: calls.__setitem__("adjoint", calls["adjoint"] + 1) or real_a(*a, **k))
    monkeypatch.setattr(_ops, "run_affine" if fam == "sw_affine" else "run_linear",
                        lambda *a, **k: calls.__setitem__("full", calls["full"] + 1) or real_f(*a, **k))
    if fam == "sw_affine":
        T = torch.tensor(0.5, device="cuda", requires_grad=True)
        v = ohm.sw_affine_value(s, gap_open_score=-2.0, gap_extend_score=-0.5, temperature=T)
    else:
        T = torch.tensor(0.5, device="cuda", requires_grad=True)
        v = ohm.sw_value(s, gap_score=-1.0, temperature=T)
    assert calls == {"checkpoint": 1, "adjoint": 0, "full": 0}     # forward only so far
    gv = torch.linspace(0.5, 1.5, 3, device="cuda")
    (v * gv).sum().backward()
    torch.cuda.synchronize()
    assert calls == {"checkpoint": 1, "adjoint": 1, "full": 0}
    monkeypatch.undo()
    params = (-2.0, -0.5, 0.5) if fam == "sw_affine" else (-1.0, 0.5)
    want = real_f(s.detach(), None, *params)
    assert torch.equal(v.detach(), want[0])
    assert torch.equal(s.grad, gv.view(-1, 1, 1) * want[1])
    assert torch.equal(T.grad.reshape(()), (gv * want[-1]).sum())


def test_c4_value_backward_peak_memory():
    """C4 (four 16384 x 16384 pairs, band mask |i - j| > 2048): value and its
    backward through the checkpointed op.  Between the two launches only the
    sparse checkpoints are kept; the peak is reported against one fp32
    three-state table and stays below the 21.7 GiB the eager value op took
    (map + workspace + masked copy)."""
    import orihime_b200 as ohm

    from test_gpu_configs import _c4_scores

    B, L, band = 4, 16384, 2048
    s = _c4_scores(B, L, band, 4).requires_grad_(True)
    i = torch.arange(L, device="cuda")
    mask = ((i[:, None] - i[None, :]).abs() > band).expand(B, L, L)
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    base = torch.cuda.memory_allocated()
    t0, t1, t2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    t0.record()
    v = ohm.sw_affine_value(s, gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.5, mask=mask)
    t1.record()
    v.sum().backward()
    t2.record()
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated() - base
    table = 3 * 4 * (L + 1) ** 2 * B
    print(f"  C4 value {t0.elapsed_time(t1):.0f} ms + backward {t1.elapsed_time(t2):.0f} ms; peak extra "
          f"{peak / 2**30:.1f} GiB (incl. the 4.3 GB score gradient); one three-state table "
          f"{table / 2**30:.1f} GiB")
    assert torch.isfinite(v).all() and torch.isfinite(s.grad).all()
    assert peak < 21.7 * 2**30
