"""Packed ragged batches of soft Smith-Waterman (and soft Needleman-Wunsch) pairs.

The reference evaluates a batch of pairs of different lengths as one padded
[B, L1max, L2max] tensor (with ``lengths`` or a mask).  This module runs the
same DP over a *packed* batch: every pair's scores are stored at their own
size, one persistent kernel pair (forward + checkpointed adjoint) pulls band
tasks longest chain first, and the whole call can be captured in a CUDA graph.

Packing (``pack``): pair b is an L1_b x L2_b row-major block with row pitch
round_up(L2_b, 4) at element offset ``offsets[b]`` (a multiple of 4) of one
flat float32 buffer.  The map comes back in the same packing.

    flat, offsets, lengths = ragged.pack([s0, s1, ...])      # CPU or CUDA tensors
    plan = ragged.Plan(lengths, offsets, family="affine", device="cuda")
    out = plan.run(flat.cuda(), gap_open=-2.0, gap_ext=-0.5, temp=0.5)
    out.value, out.map, out.grad_open, out.grad_ext, out.grad_temp
    maps = ragged.unpack(out.map, offsets, lengths)

Families: "affine" and "linear" (local alignment), "global" (soft
Needleman-Wunsch, linear gap; parameters gap and temp as for "linear") and
"global_affine" (soft Needleman-Wunsch, affine gaps) and "saigo_vert"
(Saigo-Vert, affine gaps; its linear model is gap_open = gap_ext); the last
two take the parameters of "affine".
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib

_FAMILY = {"affine": 3, "linear": 1, "global": 2, "global_affine": 4, "saigo_vert": 5}
_AFFINE = ("affine", "global_affine", "saigo_vert")
_AFFINE_FN = {"affine": "swb_sw_affine_ragged", "global_affine": "swb_nw_affine_ragged",
              "saigo_vert": "swb_sv_affine_ragged"}


def pitch_of(L2: int) -> int:
    return (int(L2) + 3) & ~3


def layout(lengths) -> tuple[np.ndarray, np.ndarray]:
    """int64 offsets [B+1] and int32 lengths [B, 2] of the packing of ``lengths``."""
    ln = np.asarray(lengths, dtype=np.int64).reshape(-1, 2)
    sizes = ln[:, 0] * ((ln[:, 1] + 3) & ~3)
    offsets = np.zeros(len(ln) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offsets[1:])
    return offsets, ln.astype(np.int32)


def pack(mats: Sequence[torch.Tensor]) -> tuple[torch.Tensor, np.ndarray, np.ndarray]:
    """Pack 2-D float32 score matrices into (flat, offsets [B+1], lengths [B, 2])."""
    lengths = [(int(m.shape[0]), int(m.shape[1])) for m in mats]
    offsets, ln = layout(lengths)
    dev = mats[0].device if len(mats) else torch.device("cpu")
    flat = torch.zeros(int(offsets[-1]), dtype=torch.float32, device=dev)
    for b, m in enumerate(mats):
        L1, L2 = lengths[b]
        if L1 * L2 == 0:
            continue
        p = pitch_of(L2)
        view = flat[int(offsets[b]):int(offsets[b]) + L1 * p].view(L1, p)
        view[:, :L2] = m.to(device=dev, dtype=torch.float32)
    return flat, offsets, ln


def unpack(flat: torch.Tensor, offsets, lengths) -> list[torch.Tensor]:
    """Views [L1_b, L2_b] of each pair in a packed buffer."""
    out = []
    for b, (L1, L2) in enumerate(np.asarray(lengths).reshape(-1, 2).tolist()):
        p = pitch_of(L2)
        o = int(offsets[b])
        out.append(flat[o:o + L1 * p].view(L1, p)[:, :L2])
    return out


@dataclass
class Result:
    value: torch.Tensor      # [B]
    map: torch.Tensor        # packed, like the scores
    grad_open: torch.Tensor  # [B]  (linear: dS/dgap)
    grad_ext: Optional[torch.Tensor]
    grad_temp: torch.Tensor  # [B]


class Plan:
    """Launch plan of one packed batch layout (reusable across calls).

    Builds the host plan with the C ABI (validation, longest-chain-first task
    order, workspace placement), copies it to the device once and owns the
    workspace, so repeated calls allocate nothing and can be graph-captured.
    """

    def __init__(self, lengths, offsets, family: str = "affine", device="cuda",
                 cols_per_lane: int = 0):
        if family not in _FAMILY:
            raise ValueError(f"family must be one of {sorted(_FAMILY)}, got {family!r}")
        self.family = family
        self.lib = _lib.load()
        ln = np.ascontiguousarray(np.asarray(lengths, dtype=np.int32).reshape(-1, 2))
        off = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64).reshape(-1))
        B = ln.shape[0]
        if off.shape[0] != B + 1:
            raise ValueError(f"offsets must have B+1 = {B + 1} entries, got {off.shape[0]}")
        self.B = B
        self.lengths = ln
        self.offsets = off
        self.cells = int((ln[:, 0].astype(np.int64) * ln[:, 1]).sum())
        pb, wb = ctypes.c_size_t(0), ctypes.c_size_t(0)
        fam = _FAMILY[family]
        self.cols_per_lane = int(cols_per_lane)
        rc = self.lib.swb_ragged_plan(fam, self.cols_per_lane, ln.ctypes.data, off.ctypes.data, B,
                                      None, 0, ctypes.byref(pb), ctypes.byref(wb))
        if rc != _lib.OK:
            raise ValueError("invalid packed batch: lengths must be >= 0 and offsets multiples of 4 "
                             "with room for L1 * round_up(L2, 4) elements per pair")
        self.host_plan = np.zeros(pb.value // 8 + 1, dtype=np.int64)
        rc = self.lib.swb_ragged_plan(fam, self.cols_per_lane, ln.ctypes.data, off.ctypes.data, B,
                                      self.host_plan.ctypes.data, self.host_plan.nbytes,
                                      ctypes.byref(pb), ctypes.byref(wb))
        _lib.check(rc, "swb_ragged_plan")
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.dev_plan = torch.from_numpy(self.host_plan.view(np.uint8)).to(self.device)
        self.workspace_bytes = wb.value
        self.workspace = torch.empty(max(wb.value, 1), dtype=torch.uint8, device=self.device)
        self.map_elems = int(off[-1]) if B else 0

    def outputs(self) -> Result:
        dev = self.device
        e = lambda: torch.empty(self.B, dtype=torch.float32, device=dev)
        return Result(e(), torch.empty(self.map_elems, dtype=torch.float32, device=dev), e(),
                      e() if self.family in _AFFINE else None, e())

    def run(self, flat: torch.Tensor, *, gap_open: float = 0.0, gap_ext: float = 0.0,
            gap: float = 0.0, temp: float = 1.0, out: Optional[Result] = None,
            options: Optional[_lib.Options] = None) -> Result:
        """One forward + adjoint over the packed batch (asynchronous)."""
        if flat.device != self.device or flat.dtype != torch.float32 or not flat.is_contiguous():
            raise ValueError("scores must be a contiguous float32 tensor on the plan's device")
        if flat.numel() < self.map_elems:
            raise ValueError(f"scores has {flat.numel()} elements, the packing needs {self.map_elems}")
        if not (temp > 0):
            raise ValueError("temperature must be finite and strictly positive")
        out = out or self.outputs()
        st = torch.cuda.current_stream(self.device).cuda_stream
        hp = self.host_plan.ctypes.data
        dp = self.dev_plan.data_ptr()
        ws = self.workspace.data_ptr()
        with torch.cuda.device(self.device):
            if self.family in _AFFINE:
                fn = getattr(self.lib, _AFFINE_FN[self.family])
                rc = fn(
                    flat.data_ptr(), hp, dp, float(gap_open), float(gap_ext), float(temp),
                    out.value.data_ptr(), out.map.data_ptr(), out.grad_open.data_ptr(),
                    out.grad_ext.data_ptr(), out.grad_temp.data_ptr(), ws, self.workspace_bytes,
                    st, options)
            else:
                fn = self.lib.swb_nw_ragged if self.family == "global" else self.lib.swb_sw_ragged
                rc = fn(flat.data_ptr(), hp, dp, float(gap), float(temp), out.value.data_ptr(),
                        out.map.data_ptr(), out.grad_open.data_ptr(), out.grad_temp.data_ptr(), ws,
                        self.workspace_bytes, st, options)
        _lib.check(rc, "ragged soft alignment")
        return out

    def values(self, flat: torch.Tensor, *, gap_open: float = 0.0, gap_ext: float = 0.0,
               gap: float = 0.0, temp: float = 1.0, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """S per pair of the packed batch without map or gradients: the forward
        wavefront alone, about half the work of `run`, the same values bit for
        bit (asynchronous).  `out`: optional float32 [B] device tensor."""
        if flat.device != self.device or flat.dtype != torch.float32 or not flat.is_contiguous():
            raise ValueError("scores must be a contiguous float32 tensor on the plan's device")
        if flat.numel() < self.map_elems:
            raise ValueError(f"scores has {flat.numel()} elements, the packing needs {self.map_elems}")
        if not (temp > 0):
            raise ValueError("temperature must be finite and strictly positive")
        if out is None:
            out = torch.empty(self.B, dtype=torch.float32, device=self.device)
        st = torch.cuda.current_stream(self.device).cuda_stream
        hp = self.host_plan.ctypes.data
        dp = self.dev_plan.data_ptr()
        ws = self.workspace.data_ptr()
        with torch.cuda.device(self.device):
            if self.family in _AFFINE:
                fn = getattr(self.lib, _AFFINE_FN[self.family] + "_value")
                rc = fn(
                    flat.data_ptr(), hp, dp, float(gap_open), float(gap_ext), float(temp),
                    out.data_ptr(), ws, self.workspace_bytes, st)
            else:
                fn = (self.lib.swb_nw_ragged_value if self.family == "global"
                      else self.lib.swb_sw_ragged_value)
                rc = fn(flat.data_ptr(), hp, dp, float(gap), float(temp), out.data_ptr(), ws,
                        self.workspace_bytes, st)
        _lib.check(rc, "ragged soft alignment value")
        return out

    def status(self) -> int:
        st = ctypes.c_uint(0)
        rc = self.lib.swb_read_status(self.workspace.data_ptr(),
                                      torch.cuda.current_stream(self.device).cuda_stream,
                                      ctypes.byref(st))
        _lib.check(rc, "swb_read_status")
        return st.value

    def graph(self, flat: torch.Tensor, **params) -> tuple[torch.cuda.CUDAGraph, Result]:
        """Capture one call on static buffers; replay with ``g.replay()`` after
        writing new scores into ``flat``."""
        out = self.outputs()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.run(flat, out=out, **params)  # warm-up outside capture (device info, modules)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run(flat, out=out, **params)
        return g, out


def split_groups(lengths, parts: int) -> list[tuple[int, int]]:
    """Contiguous pair ranges [b0, b1) with about equal cells each (at most `parts`)."""
    ln = np.asarray(lengths, dtype=np.int64).reshape(-1, 2)
    B = ln.shape[0]
    if B == 0:
        return []
    parts = max(1, min(int(parts), B))
    cum = np.cumsum(ln[:, 0] * ln[:, 1])
    total = int(cum[-1])
    cuts, b0 = [], 0
    for k in range(1, parts):
        b = int(np.searchsorted(cum, total * k / parts, side="right"))
        b = min(max(b, b0 + 1), B - (parts - k))
        cuts.append((b0, b))
        b0 = b
    cuts.append((b0, B))
    return [c for c in cuts if c[1] > c[0]]


class StreamedPlan:
    """A packed batch run straight from pinned host memory, with the
    host-to-device copy overlapped with compute.

    The pairs are split into `parts` contiguous groups of about equal cell
    count, each with its own Plan.  A copy stream moves group k+1's scores
    while the compute stream runs group k; the compute stream waits only for
    its own group's copy.  The scores land in one device buffer in the same
    packing, and the map comes back as one packed device buffer.

        sp = ragged.StreamedPlan(lengths, offsets, parts=8, device="cuda")
        out = sp.run(host_flat_pinned, gap_open=-2.0, gap_ext=-0.5, temp=0.5)
    """

    def __init__(self, lengths, offsets, family: str = "affine", device="cuda", parts: int = 8,
                 cols_per_lane: int = 0):
        ln = np.asarray(lengths, dtype=np.int32).reshape(-1, 2)
        off = np.asarray(offsets, dtype=np.int64).reshape(-1)
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.family = family
        self.B = ln.shape[0]
        self.map_elems = int(off[-1]) if self.B else 0
        self.groups = split_groups(ln, parts)
        self.plans = []
        for b0, b1 in self.groups:
            sub_off = off[b0:b1 + 1] - off[b0]
            self.plans.append(Plan(ln[b0:b1], sub_off, family=family, device=self.device,
                                   cols_per_lane=cols_per_lane))
        self.offsets = off
        self.scores = torch.empty(max(self.map_elems, 1), dtype=torch.float32, device=self.device)
        self.copy_stream = torch.cuda.Stream(self.device)
        self.events = [torch.cuda.Event() for _ in self.groups]

    def outputs(self) -> Result:
        dev = self.device
        e = lambda: torch.empty(self.B, dtype=torch.float32, device=dev)
        return Result(e(), torch.empty(self.map_elems, dtype=torch.float32, device=dev), e(),
                      e() if self.family in _AFFINE else None, e())

    def run(self, host_flat: torch.Tensor, *, out: Optional[Result] = None, **params) -> Result:
        """Copy `host_flat` (pinned, packed like `offsets`) group by group and
        run each group as soon as its scores are on the device (asynchronous)."""
        if host_flat.device.type != "cpu" or host_flat.dtype != torch.float32:
            raise ValueError("host_flat must be a float32 CPU tensor (pinned for overlap)")
        if host_flat.numel() < self.map_elems:
            raise ValueError(f"host_flat has {host_flat.numel()} elements, the packing needs {self.map_elems}")
        out = out or self.outputs()
        compute = torch.cuda.current_stream(self.device)
        # the copy stream must not overwrite scores a previous call still reads
        self.copy_stream.wait_stream(compute)
        for k, ((b0, b1), plan) in enumerate(zip(self.groups, self.plans)):
            e0, e1 = int(self.offsets[b0]), int(self.offsets[b1])
            with torch.cuda.stream(self.copy_stream):
                self.scores[e0:e1].copy_(host_flat[e0:e1], non_blocking=True)
                self.events[k].record(self.copy_stream)
            compute.wait_event(self.events[k])
            sub = Result(out.value[b0:b1], out.map[e0:e1], out.grad_open[b0:b1],
                         None if out.grad_ext is None else out.grad_ext[b0:b1], out.grad_temp[b0:b1])
            plan.run(self.scores[e0:e1], out=sub, **params)
        return out

    def status(self) -> int:
        st = 0
        for p in self.plans:
            st |= p.status()
        return st


# ---------------------------------------------------------------------------
# one pair list across several GPUs
# ---------------------------------------------------------------------------

def pair_cost(lengths, cols_per_lane: int = 4) -> np.ndarray:
    """Work of each pair for load balancing: the cells its bands compute, i.e.
    the band count times the band's wavefront steps (L1 + 31) times the band
    width, which counts the partly dead last band and the fill and drain of
    every band, not just L1 * L2."""
    ln = np.asarray(lengths, dtype=np.int64).reshape(-1, 2)
    w = 32 * int(cols_per_lane or 4)
    nb = np.maximum(1, (ln[:, 1] + w - 1) // w)
    cost = nb * (ln[:, 0] + 31) * w
    return np.where((ln[:, 0] > 0) & (ln[:, 1] > 0), cost, 0)


def lpt_partition(lengths, parts: int, cost=None) -> list[np.ndarray]:
    """Pair indices of each of `parts` shards, longest processing time first:
    pairs in decreasing cost, each to the shard with the least cost so far
    (ties: the lowest shard).  Deterministic, so every rank computes the same
    partition from the same lengths.  Each shard's indices are ascending."""
    import heapq

    c = pair_cost(lengths) if cost is None else np.asarray(cost, dtype=np.float64)
    parts = max(1, int(parts))
    heap = [(0, g) for g in range(parts)]
    buckets = [[] for _ in range(parts)]
    for b in np.argsort(-c, kind="stable"):
        load, g = heapq.heappop(heap)
        buckets[g].append(int(b))
        heapq.heappush(heap, (load + int(c[b]), g))
    return [np.array(sorted(x), dtype=np.int64) for x in buckets]


def shard_scores(flat: torch.Tensor, offsets, lengths, idx, device=None) -> tuple[torch.Tensor, np.ndarray, np.ndarray]:
    """The packed buffer of pairs `idx` of a packed batch: (flat, offsets,
    lengths) of the shard in the same packing, copied to `device`."""
    off = np.asarray(offsets, dtype=np.int64)
    ln = np.asarray(lengths).reshape(-1, 2)
    sub_off, sub_ln = layout(ln[idx])
    dev = flat.device if device is None else torch.device(device)
    out = torch.empty(max(int(sub_off[-1]), 1), dtype=torch.float32, device=dev)
    for k, b in enumerate(np.asarray(idx).tolist()):
        n = int(sub_off[k + 1] - sub_off[k])
        if n:
            out[int(sub_off[k]):int(sub_off[k]) + n].copy_(flat[int(off[b]):int(off[b]) + n],
                                                            non_blocking=True)
    return out, sub_off, sub_ln


class ShardedPlan:
    """One packed batch split across GPUs by LPT on the pairs' computed cells
    (`pair_cost`), one persistent forward + adjoint launch per GPU and no
    collective on the data path: pairs are independent.

    Single process, several devices:

        sp = ragged.ShardedPlan(lengths, devices=["cuda:0", "cuda:1"])
        flats = sp.scatter(flat_host)            # each shard's packed scores on its device
        outs = sp.run(flats, gap_open=-2.0, gap_ext=-0.5, temp=0.5)
        values = sp.gather_values(outs)          # [B], in the batch's pair order

    One process per GPU (torchrun): every rank builds the same partition and
    runs only its shard (``rank``/``world``); ``all_gather_values`` assembles
    the values of all ranks with one all_gather (optional, for reporting).
    """

    def __init__(self, lengths, offsets=None, family: str = "affine", devices=None,
                 rank: Optional[int] = None, world: Optional[int] = None, cols_per_lane: int = 0):
        ln = np.asarray(lengths, dtype=np.int32).reshape(-1, 2)
        self.B = ln.shape[0]
        self.lengths = ln
        self.offsets = layout(ln)[0] if offsets is None else np.asarray(offsets, dtype=np.int64)
        self.family = family
        if world is not None:
            self.world, self.rank = int(world), int(rank or 0)
            self.devices = [torch.device(devices) if devices is not None else
                            torch.device("cuda", torch.cuda.current_device())]
            self.local = [self.rank]
        else:
            devs = devices or ["cuda"]
            self.devices = [torch.device(d) for d in devs]
            self.world, self.rank = len(self.devices), 0
            self.local = list(range(self.world))
        self.shards = lpt_partition(ln, self.world, pair_cost(ln, cols_per_lane or 4))
        self.plans = {}
        for k, g in enumerate(self.local):
            idx = self.shards[g]
            sub_off, sub_ln = layout(ln[idx])
            self.plans[g] = Plan(sub_ln, sub_off, family=family, device=self.devices[k],
                                 cols_per_lane=cols_per_lane)

    def cost(self) -> list[int]:
        """Computed cells of each shard (the LPT loads)."""
        c = pair_cost(self.lengths)
        return [int(c[idx].sum()) for idx in self.shards]

    def scatter(self, flat: torch.Tensor) -> dict:
        """Each local shard's packed scores on its device, from the whole
        batch's packed buffer (host or device)."""
        return {g: shard_scores(flat, self.offsets, self.lengths, self.shards[g],
                                self.plans[g].device)[0] for g in self.local}

    def run(self, flats: dict, **params) -> dict:
        """One forward + adjoint per local shard, asynchronous on each
        device's current stream; returns {shard: Result}."""
        return {g: self.plans[g].run(flats[g], **params) for g in self.local}

    def gather_values(self, outs: dict, device=None) -> torch.Tensor:
        """Values of the local shards, in the batch's pair order ([B])."""
        dev = torch.device(device) if device is not None else self.devices[0]
        v = torch.full((self.B,), float("nan"), dtype=torch.float32, device=dev)
        for g, r in outs.items():
            v[torch.as_tensor(self.shards[g], device=dev)] = r.value.to(dev)
        return v

    def all_gather_values(self, value_local: torch.Tensor, group=None) -> torch.Tensor:
        """[B] values of every rank's shard from this rank's [len(shard)]
        values (a collective: every rank calls it)."""
        return all_gather_values(value_local, self.shards, self.B, group)


def all_gather_values(value_local: torch.Tensor, shards, B: int, group=None) -> torch.Tensor:
    """Assemble per-pair values computed shard by shard on the ranks of a
    process group: one all_gather of equally padded blocks, then a scatter
    into the batch's pair order.  `shards[g]` are rank g's pair indices."""
    import torch.distributed as dist

    n = max(len(x) for x in shards)
    pad = torch.zeros(n, dtype=value_local.dtype, device=value_local.device)
    pad[:value_local.numel()] = value_local
    blocks = [torch.empty_like(pad) for _ in range(len(shards))]
    dist.all_gather(blocks, pad, group=group)
    out = torch.empty(B, dtype=value_local.dtype, device=value_local.device)
    for g, blk in enumerate(blocks):
        idx = torch.as_tensor(shards[g], device=value_local.device)
        out[idx] = blk[:len(shards[g])]
    return out


# ---------------------------------------------------------------------------
# columns per lane chosen per length bucket
# ---------------------------------------------------------------------------

# Length buckets of the autotuner: L2 in octaves from 32 (the band width is
# 32 x columns per lane, so L2 sets the dead columns of a pair's last band)
# times L1 below / from 256 (a band's 31 fill and drain steps weigh more on
# short pairs).  Key "l2lo:l1lo", e.g. "512:256".
L2_EDGES = (0, 64, 128, 256, 512, 1024)
L1_EDGES = (0, 256)

# Columns per lane per bucket, measured on a B200 (the local families in the
# linear domain, 2048 pairs per bucket filling the GPU, N(0, 1) * 1.5 scores at
# T 0.5): used when no tuned table is cached for this GPU.
DEFAULT_COLS = {"0:0": 2, "0:256": 2, "64:0": 4, "64:256": 2, "128:0": 8, "128:256": 2,
                "256:0": 8, "256:256": 4, "512:0": 8, "512:256": 8, "1024:0": 8, "1024:256": 8}


def bucket_of(L1: int, L2: int) -> str:
    l2 = max(e for e in L2_EDGES if L2 >= e)
    l1 = max(e for e in L1_EDGES if L1 >= e)
    return f"{l2}:{l1}"


def _cache_path(device) -> str:
    import os
    import re

    name = torch.cuda.get_device_name(device) if torch.cuda.is_available() else "cpu"
    d = os.environ.get("ORIHIME_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "orihime_b200"))
    return os.path.join(d, "cols_" + re.sub(r"[^A-Za-z0-9]+", "_", name) + ".json")


def cols_table(device=None) -> dict:
    """Columns per lane per bucket: the environment variable
    ORIHIME_B200_COLS (a JSON object, or "bucket=R,..." pairs, or a path to a
    JSON file) overrides; else the table `tune` cached for this GPU; else
    DEFAULT_COLS.  Buckets missing from a table take DEFAULT_COLS' entry."""
    import json
    import os

    table = dict(DEFAULT_COLS)
    spec = os.environ.get("ORIHIME_B200_COLS")
    if spec:
        if os.path.exists(spec):
            table.update(json.load(open(spec)))
        elif spec.lstrip().startswith("{"):
            table.update(json.loads(spec))
        else:
            for kv in spec.split(","):
                k, v = kv.split("=")
                table[k.strip()] = int(v)
        return table
    try:
        path = _cache_path(device)
        if os.path.exists(path):
            table.update(json.load(open(path))["table"])
    except Exception:
        pass
    return table


def tune(family: str = "affine", device="cuda", pairs: int = 2048, reps: int = 5,
         choices=(2, 4, 8), save: bool = True, seed: int = 0) -> dict:
    """Time every length bucket at each columns-per-lane choice on this GPU
    and keep the fastest: per bucket, `pairs` pairs with lengths log-uniform
    in the bucket (N(0, 1) * 1.5 scores, gap_open -2, gap_ext -0.5 or gap -1,
    T 0.5), one packed plan per choice, CUDA-graph replays timed with CUDA
    events.  The table is cached as JSON per GPU name (see cols_table)."""
    import json
    import os

    dev = torch.device(device)
    rng = np.random.default_rng(seed)
    params = dict(gap_open=-2.0, gap_ext=-0.5, temp=0.5) if family in _AFFINE else dict(gap=-1.0, temp=0.5)
    table, times = {}, {}
    l2e = list(L2_EDGES) + [2049]
    l1e = list(L1_EDGES) + [2049]
    for a2, b2 in zip(l2e[:-1], l2e[1:]):
        for a1, b1 in zip(l1e[:-1], l1e[1:]):
            key = f"{a2}:{a1}"
            lo2, lo1 = max(a2, 16), max(a1, 16)
            ln = np.stack([np.exp(rng.uniform(np.log(lo1), np.log(b1), pairs)),
                           np.exp(rng.uniform(np.log(lo2), np.log(b2), pairs))], 1)
            ln = np.clip(np.floor(ln), [lo1, lo2], [b1 - 1, b2 - 1]).astype(np.int64)
            off, ln32 = layout(ln)
            g = torch.Generator(device=dev)
            g.manual_seed(seed + a2 * 7 + a1)
            flat = torch.randn(int(off[-1]), generator=g, device=dev) * 1.5
            best = None
            for R in choices:
                plan = Plan(ln32, off, family=family, device=dev, cols_per_lane=R)
                gr, _ = plan.graph(flat, **params)
                for _ in range(2):
                    gr.replay()
                torch.cuda.synchronize(dev)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    gr.replay()
                e1.record()
                torch.cuda.synchronize(dev)
                ms = e0.elapsed_time(e1) / reps
                times[f"{key}:R{R}"] = ms
                if best is None or ms < best[1]:
                    best = (R, ms)
                del gr, plan
            table[key] = best[0]
    if save:
        path = _cache_path(dev)
        os.makedirs(os.path.dirname(path), exist_ok=True)
        json.dump({"gpu": torch.cuda.get_device_name(dev), "family": family, "table": table,
                   "ms": times}, open(path, "w"), indent=1)
    return {"table": table, "ms": times}


class MixedPlan:
    """A packed batch run with a columns-per-lane choice per pair (the bucket
    table of cols_table, or `table`): one Plan per choice over its pairs, all
    on the batch's own packed score and map buffers (the original offsets,
    no copies), launched on parallel streams that join before `run` returns
    (graph-capturable); per-pair outputs are scattered into [B] arrays.  Same
    interface as Plan.  The local families ("affine", "linear") in the
    linear domain take 2, 4 or 8; the others 2 or 4."""

    def __init__(self, lengths, offsets, family: str = "affine", device="cuda", table=None):
        ln = np.ascontiguousarray(np.asarray(lengths, dtype=np.int32).reshape(-1, 2))
        off = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64).reshape(-1))
        self.B = ln.shape[0]
        self.lengths, self.offsets, self.family = ln, off, family
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.table = dict(table) if table is not None else cols_table(self.device)
        local = family in ("affine", "linear")
        cols = np.array([self.table.get(bucket_of(int(a), int(b)), 4) for a, b in ln.tolist()], dtype=np.int64)
        if not local:
            cols = np.where(cols == 8, 4, cols)
        self.cols = cols
        self.cells = int((ln[:, 0].astype(np.int64) * ln[:, 1]).sum())
        self.map_elems = int(off[-1]) if self.B else 0
        self.subs = []   # (R, pair indices, index tensor, Plan)
        for R in sorted(set(cols.tolist())):
            idx = np.nonzero(cols == R)[0]
            sub_off = np.concatenate([off[idx], [off[idx[-1] + 1]]])
            plan = Plan(ln[idx], sub_off, family=family, device=self.device, cols_per_lane=int(R))
            self.subs.append((int(R), idx, torch.as_tensor(idx, device=self.device), plan))
        self.streams = [torch.cuda.Stream(self.device) for _ in self.subs[1:]]
        self.workspace_bytes = sum(p.workspace_bytes for *_, p in self.subs)

    def computed_cells(self) -> int:
        """Cells the bands compute (dead columns and fill/drain included)."""
        w = 32 * self.cols
        nb = np.maximum(1, (self.lengths[:, 1] + w - 1) // w)
        c = nb * (self.lengths[:, 0] + 31) * w
        return int(np.where((self.lengths[:, 0] > 0) & (self.lengths[:, 1] > 0), c, 0).sum())

    def outputs(self) -> Result:
        dev = self.device
        e = lambda: torch.empty(self.B, dtype=torch.float32, device=dev)  # noqa: E731
        return Result(e(), torch.empty(self.map_elems, dtype=torch.float32, device=dev), e(),
                      e() if self.family in _AFFINE else None, e())

    def _fanout(self, fns):
        """Run fns[k] on stream k (the current stream for k = 0, side streams
        forked from it for the others) and join them back."""
        main = torch.cuda.current_stream(self.device)
        for s in self.streams:
            s.wait_stream(main)
        for k, fn in enumerate(fns):
            with torch.cuda.stream(main if k == 0 else self.streams[k - 1]):
                fn()
        for s in self.streams:
            main.wait_stream(s)

    def run(self, flat: torch.Tensor, *, out: Optional[Result] = None, **params) -> Result:
        """One forward + adjoint over the batch (asynchronous): the sub-plans
        write their pairs' cells into out.map and their per-pair outputs are
        scattered into out's [B] arrays."""
        out = out or self.outputs()
        dev = self.device
        e = lambda n: torch.empty(n, dtype=torch.float32, device=dev)  # noqa: E731
        # per-pair outputs of each sub-plan, allocated on the current stream
        subs_out = [Result(e(len(idx)), out.map, e(len(idx)), e(len(idx)) if out.grad_ext is not None else None,
                           e(len(idx))) for _, idx, _, _ in self.subs]
        self._fanout([lambda p=plan, o=o: p.run(flat, out=o, **params)
                      for (_, _, _, plan), o in zip(self.subs, subs_out)])
        for (R, idx, it, plan), r in zip(self.subs, subs_out):
            out.value.index_copy_(0, it, r.value)
            out.grad_open.index_copy_(0, it, r.grad_open)
            if out.grad_ext is not None:
                out.grad_ext.index_copy_(0, it, r.grad_ext)
            out.grad_temp.index_copy_(0, it, r.grad_temp)
        return out

    def values(self, flat: torch.Tensor, *, out: Optional[torch.Tensor] = None, **params) -> torch.Tensor:
        """S per pair without map or gradients (the forward wavefront alone)."""
        if out is None:
            out = torch.empty(self.B, dtype=torch.float32, device=self.device)
        vals = [torch.empty(len(idx), dtype=torch.float32, device=self.device) for _, idx, _, _ in self.subs]
        self._fanout([lambda p=plan, v=v: p.values(flat, out=v, **params)
                      for (_, _, _, plan), v in zip(self.subs, vals)])
        for (R, idx, it, plan), v in zip(self.subs, vals):
            out.index_copy_(0, it, v)
        return out

    def status(self) -> int:
        st = 0
        for *_, p in self.subs:
            st |= p.status()
        return st

    def graph(self, flat: torch.Tensor, **params) -> tuple[torch.cuda.CUDAGraph, Result]:
        """Capture one call on static buffers; replay with ``g.replay()``."""
        out = self.outputs()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.run(flat, out=out, **params)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run(flat, out=out, **params)
        return g, out


def _signature(lengths, family) -> str:
    """A coarse key of a batch for the tuning cache: the family, the pair
    count's power of two and the cells per length bucket as a share of the
    batch, in tenths."""
    ln = np.asarray(lengths, dtype=np.int64).reshape(-1, 2)
    cells = ln[:, 0] * ln[:, 1]
    tot = max(int(cells.sum()), 1)
    share = {}
    for (a, b), c in zip(ln.tolist(), cells.tolist()):
        k = bucket_of(a, b)
        share[k] = share.get(k, 0) + c
    hist = ",".join(f"{k}={round(10 * v / tot)}" for k, v in sorted(share.items()) if round(10 * v / tot))
    return f"{family}|B{int(np.log2(max(len(ln), 1)))}|{hist}"


def autotune_plan(lengths, offsets, family: str = "affine", device="cuda", flat=None, reps: int = 3,
                  use_cache: bool = True, **params):
    """The fastest launch configuration for this batch on this GPU, chosen by
    timing: one Plan per columns-per-lane choice (2, 4 and, for the local
    families, 8) and the MixedPlan of the bucket table, each captured in a
    CUDA graph and replayed on `flat` (the batch's packed scores; N(0, 1) *
    1.5 if None) with CUDA events.  The choice is cached per GPU and batch
    signature (see cols_table for the cache folder).  Returns (plan, report)
    where report = {"choice": ..., "ms": {candidate: ms}, "cached": bool}."""
    import json
    import os

    dev = torch.device(device)
    if dev.type == "cuda" and dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    ln = np.asarray(lengths, dtype=np.int32).reshape(-1, 2)
    local = family in ("affine", "linear")
    cands = {f"R{r}": (lambda r=r: Plan(ln, offsets, family=family, device=dev, cols_per_lane=r))
             for r in ((2, 4, 8) if local else (2, 4))}
    cands["mixed"] = lambda: MixedPlan(ln, offsets, family=family, device=dev)
    sig = _signature(ln, family)
    path = _cache_path(dev).replace("cols_", "plans_")
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except Exception:
            cache = {}
    if use_cache and sig in cache and cache[sig]["choice"] in cands:
        return cands[cache[sig]["choice"]](), dict(cache[sig], cached=True)
    if not params:
        params = dict(gap_open=-2.0, gap_ext=-0.5, temp=0.5) if family in _AFFINE else dict(gap=-1.0, temp=0.5)
    if flat is None:
        g = torch.Generator(device=dev)
        g.manual_seed(0)
        off = np.asarray(offsets, dtype=np.int64)
        flat = torch.randn(max(int(off[-1]), 1), generator=g, device=dev) * 1.5
    times, best = {}, None
    for name, make in cands.items():
        plan = make()
        gr, _ = plan.graph(flat, **params)
        gr.replay()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            gr.replay()
        e1.record()
        torch.cuda.synchronize(dev)
        times[name] = e0.elapsed_time(e1) / reps
        if best is None or times[name] < times[best[0]]:
            best = (name, plan)
        del gr
        if best[1] is not plan:
            del plan
    report = {"choice": best[0], "ms": times, "signature": sig}
    if use_cache:
        cache[sig] = report
        os.makedirs(os.path.dirname(path), exist_ok=True)
        json.dump(cache, open(path, "w"), indent=1)
    return best[1], dict(report, cached=False)
