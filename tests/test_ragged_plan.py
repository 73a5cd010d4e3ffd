"""Host-side ragged plan: packing helpers and the C ABI plan builder (CPU)."""

import ctypes

import numpy as np
import pytest
import torch

from orihime_b200 import _lib, ragged


def _plan(lengths, offsets, family=3):
    lib = _lib.load()
    ln = np.ascontiguousarray(np.asarray(lengths, np.int32).reshape(-1, 2))
    off = np.ascontiguousarray(np.asarray(offsets, np.int64))
    pb, wb = ctypes.c_size_t(0), ctypes.c_size_t(0)
    rc = lib.swb_ragged_plan(family, 4, ln.ctypes.data, off.ctypes.data, len(ln), None, 0,
                             ctypes.byref(pb), ctypes.byref(wb))
    if rc != 0:
        return rc, None
    buf = np.zeros(pb.value // 8 + 1, np.int64)
    rc = lib.swb_ragged_plan(family, 4, ln.ctypes.data, off.ctypes.data, len(ln), buf.ctypes.data,
                             buf.nbytes, ctypes.byref(pb), ctypes.byref(wb))
    return rc, buf


def test_pack_unpack_roundtrip():
    g = torch.Generator().manual_seed(0)
    mats = [torch.randn(a, b, generator=g) for a, b in [(3, 5), (0, 7), (9, 0), (1, 1), (17, 130)]]
    flat, off, ln = ragged.pack(mats)
    assert np.all(off % 4 == 0)
    assert ln.tolist() == [[3, 5], [0, 7], [9, 0], [1, 1], [17, 130]]
    for m, v in zip(mats, ragged.unpack(flat, off, ln)):
        assert torch.equal(m, v)


def test_plan_orders_longest_chain_first_and_places_bands():
    # the queue order is the pair's critical path L1 + 31 * bands (in
    # wavefront steps), then cells: a tall narrow pair goes before a wide
    # short one with more cells
    lengths = [[10, 20], [100, 300], [0, 5], [64, 129], [5, 600], [400, 30]]
    off, ln = ragged.layout(lengths)
    rc, buf = _plan(ln, off)
    assert rc == 0
    B = len(ln)
    hdr = buf[:10]
    pairs = buf[10:10 + 8 * B].reshape(B, 8)
    tasks = buf[10 + 8 * B:].view(np.int32)[:2 * hdr[2]].reshape(-1, 2)
    cells = [a * b for a, b in lengths]
    nb = [max(1, -(-b // 128)) for _, b in lengths]
    chain = [(a + 31 * n) if a * b > 0 else 0 for (a, b), n in zip(lengths, nb)]
    first_of_pair = []
    for p, _ in tasks:
        if p not in first_of_pair:
            first_of_pair.append(int(p))
    assert first_of_pair == sorted(range(B), key=lambda b: (-chain[b], -cells[b], b))
    assert first_of_pair[0] == 5 and first_of_pair[1] == 1  # 400 x 30 before 100 x 300
    assert hdr[2] == sum(nb)
    for p in range(B):
        assert pairs[p, 4] == nb[p]
        bands = [int(j) for q, j in tasks if q == p]
        assert bands == list(range(nb[p]))
        assert pairs[p, 0] == off[p]


@pytest.mark.parametrize("bad", ["misaligned", "overlap", "negative"])
def test_plan_rejects_bad_packing(bad):
    lengths = np.array([[4, 6], [3, 9]], np.int32)
    off, _ = ragged.layout(lengths)
    if bad == "misaligned":
        off = off + np.array([0, 2, 2])
    elif bad == "overlap":
        off[1] -= 4
    else:
        lengths[1, 0] = -1
    rc, _ = _plan(lengths, off)
    assert rc == _lib.ERR_ARG


def test_global_alignment_plan_uses_the_linear_layout():
    """Family 2 (global alignment, linear gap) places the same buffers as the
    linear model and records its own family code; an unknown family is refused."""
    lengths = [[40, 300], [0, 5], [17, 1], [129, 129]]
    off, _ = ragged.layout(lengths)
    rc1, lin = _plan(lengths, off, family=1)
    rc2, glob = _plan(lengths, off, family=2)
    assert rc1 == 0 and rc2 == 0
    assert np.array_equal(lin[1:7], glob[1:7])          # B, tasks, slots, ck, edge, push
    assert glob[7] & 0xff == 2 and lin[7] & 0xff == 1   # family word
    assert _plan(lengths, off, family=6)[0] != 0
    assert _plan(lengths, off, family=0)[0] != 0


def test_global_affine_plan_has_six_push_channels():
    """Family 4 (global alignment, affine gaps) places the affine checkpoints
    and edges with six push channels per row (left M, I, D; diagonal M, I, D)."""
    lengths = [[40, 300], [0, 5], [17, 1], [129, 129]]
    off, _ = ragged.layout(lengths)
    rc3, loc = _plan(lengths, off, family=3)
    rc4, glob = _plan(lengths, off, family=4)
    assert rc3 == 0 and rc4 == 0
    assert np.array_equal(loc[1:6], glob[1:6])          # B, tasks, slots, ck, edge
    assert glob[6] * 5 == loc[6] * 6                    # push floats: 6 vs 5 channels
    assert glob[7] & 0xff == 4
    rc5, sv = _plan(lengths, off, family=5)        # Saigo-Vert: the same six-channel layout
    assert rc5 == 0 and np.array_equal(sv[1:7], glob[1:7]) and sv[7] & 0xff == 5
