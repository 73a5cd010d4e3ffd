"""Benchmark: fwd+bwd GCUPS of soft Smith-Waterman (affine gaps) over a packed
ragged batch on B200, against the padded plain launch on the same GPU and the
reference's own CPU implementation.

Workload (one "step"): 4096 pairs whose lengths N, M are drawn independently
log-uniform in [32, 2048] (seed 3), pair scores 3 <e_i, f_j> / sqrt(64) with
e, f ~ N(0, 1) in d = 64 (seeded per pair), gap_open -2, gap_ext -0.5, T 0.5.
One step = one forward + checkpointed adjoint over the whole packed batch
(value, marginal map and dS/d(params) for every pair).  Inputs (3.9 GB of
scores) are larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU (torchrun): the job is N x 4096 pairs drawn the same way (seed 3),
split across the ranks by LPT on each pair's computed cells (weak scaling:
about 4096 pairs per GPU); each rank runs its shard, no collective touches
the data path, and rank 0 prints the line with the max-over-ranks time and
the whole job's cells; the values are gathered once after timing.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd GCUPS, soft SW-affine ragged batch, vs padded plain on same B200"
GO, GE, T = -2.0, -0.5, 0.5
NPAIRS, LMIN, LMAX, D = 4096, 32, 2048, 64
MUFU_PER_CELL = 21      # algorithmic MUFU ops per cell, forward 11 + adjoint 10
MUFU_PER_CELL_BWD = 10  # adjoint kernel alone
BYTES_PER_CELL = 8      # compulsory HBM bytes per cell (score read + map write)
E2E_PARTS = 8           # pair groups of the end-to-end pipeline


def workload_lengths(seed: int, n: int = NPAIRS) -> np.ndarray:
    rng = np.random.default_rng(seed)
    ln = np.exp(rng.uniform(np.log(LMIN), np.log(LMAX), size=(n, 2)))
    return np.rint(ln).astype(np.int64)


def shard_of(world: int, rank: int, pairs: int = NPAIRS):
    """This rank's pairs of the whole job: N x `pairs` pairs (seed 3) split
    across the N ranks by LPT on their computed cells.  Returns (lengths,
    global pair indices, all shards); one rank gets the whole batch."""
    from orihime_b200 import ragged

    lengths = workload_lengths(3, pairs * world)
    shards = ragged.lpt_partition(lengths, world)
    return lengths[shards[rank]], shards[rank], shards


def make_scores(torch, lengths, offsets, seed, device, index=None):
    """Packed scores 3 <e_i, f_j> / sqrt(64) (e, f ~ N(0, 1) in 64 dimensions),
    built on the device pair by pair; pair b is seeded by its index in the
    whole job (`index[b]`, default b)."""
    from orihime_b200 import ragged

    flat = torch.zeros(int(offsets[-1]), dtype=torch.float32, device=device)
    g = torch.Generator(device=device)
    for b, (L1, L2) in enumerate(lengths.tolist()):
        g.manual_seed(seed * 100003 + (int(index[b]) if index is not None else b))
        e = torch.randn(L1, D, generator=g, device=device)
        f = torch.randn(L2, D, generator=g, device=device)
        p = ragged.pitch_of(L2)
        flat[int(offsets[b]):int(offsets[b]) + L1 * p].view(L1, p)[:, :L2] = 3.0 * (e @ f.T) / D ** 0.5
    return flat


class ClockSampler:
    """SM clock, power and clock-event reasons sampled during the timed region
    (read only; no setting is changed).  NVML is polled every 10 ms on the
    device matched by PCI bus id; without NVML, nvidia-smi is polled (about
    one sample per 0.2 s)."""

    _BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
             ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.source = None
        self._stop = threading.Event()
        self._th = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.index)
        bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
        except Exception:
            nv = h = None

        def run_nvml():
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            while not self._stop.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append([str(sm), str(mx), f"{pw:.1f}"]
                                        + ["Active" if bits & b else "Not Active" for _, b in self._BITS])
                except Exception:
                    pass
                self._stop.wait(0.01)

        def run_smi():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True,
                                         text=True, timeout=5).stdout.strip()
                    if out:
                        self.samples.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self.source = "nvml" if h is not None else "nvidia-smi"
        self._th = threading.Thread(target=run_nvml if h is not None else run_smi, daemon=True)
        self._th.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._th.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = [n for n, _ in self._BITS]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 3 + k and "Active" in s[3 + k] and "Not" not in s[3 + k]})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples), "source": self.source}


def dist_init(torch, backend: str = "nccl"):
    """One process per GPU (torchrun env).  `backend` "gloo" runs the same
    host logic on CPU ranks (tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(torch, world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(torch, world, x: float) -> float:
    if world == 1:
        return x
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def mufu_peak(torch, lib) -> float:
    """Measured ex2 throughput (ops/s) of this GPU: the MUFU roofline denominator."""
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, iters = sms * 8, 4096
    scratch = torch.empty(blocks * 256, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        lib.swb_mufu_probe(scratch.data_ptr(), blocks, iters, st)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        lib.swb_mufu_probe(scratch.data_ptr(), blocks, iters, st)
        b.record()
        torch.cuda.synchronize()
        best = max(best, blocks * 256 * iters * 8 / (a.elapsed_time(b) * 1e-3))
    return best


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(p))
    except Exception:
        return {}


# ---------------------------------------------------------------------------
# reference CPU arm
# ---------------------------------------------------------------------------

def reference_cpu_sample(lengths, seed, budget_cells=2.0e8, chunk=None):
    """A bounded sample of the workload for the reference CPU kernels: every
    k-th pair (by index) until about `budget_cells` cells, grouped into padded
    chunks of similar size as the reference's batched API expects."""
    import torch

    idx = np.arange(len(lengths))
    cells = lengths[:, 0] * lengths[:, 1]
    order = idx[np.argsort(-cells, kind="stable")]
    step = max(1, int(cells.sum() / budget_cells))
    pick = np.sort(order[::step])
    chunks, cur = [], []
    chunk = chunk or min(64, max(8, os.cpu_count() or 8))
    cap = 4e9 / 40  # padded cells per chunk: scores, map and the 3-plane alpha/beta in RAM
    for b in sorted(pick, key=lambda b: -cells[b]):
        if cur:
            L1m = max(int(lengths[x, 0]) for x in cur + [b])
            L2m = max(int(lengths[x, 1]) for x in cur + [b])
            if (len(cur) + 1) * L1m * L2m > cap:
                chunks.append(cur)
                cur = []
        cur.append(b)
        if len(cur) == chunk:
            chunks.append(cur)
            cur = []
    if cur:
        chunks.append(cur)
    data = []
    for ch in chunks:
        L1m = int(max(lengths[b, 0] for b in ch))
        L2m = int(max(lengths[b, 1] for b in ch))
        s = np.zeros((len(ch), L1m, L2m), np.float32)
        for k, b in enumerate(ch):
            g = torch.Generator().manual_seed(seed * 100003 + int(b))
            L1, L2 = int(lengths[b, 0]), int(lengths[b, 1])
            e = torch.randn(L1, D, generator=g)
            f = torch.randn(L2, D, generator=g)
            s[k, :L1, :L2] = (3.0 * (e @ f.T) / D ** 0.5).numpy()
        ln = np.array([[lengths[b, 0], lengths[b, 1]] for b in ch], np.int32)
        data.append((s, ln))
    return data, int(cells[pick].sum()), len(pick)


def run_reference(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O

    if not O.ref_available():
        try:
            O.build(ref=True)
        except Exception:
            pass
    lengths = workload_lengths(3)
    data, cells, npairs = reference_cpu_sample(lengths, 3)
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    if O.ref_available():
        kind, fn = "reference", lambda s, ln: O.ref_affine(s, ln, GO, GE, T)
    else:
        kind, fn = "port", lambda s, ln: O.affine(s, ln, GO, GE, T)
        threads = 1

    def step():
        for s, ln in data:
            fn(s, ln)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    gcups = cells / dt / 1e9
    sample = (f"{npairs} of the {NPAIRS} pairs (every k-th by size, {cells:.3g} cells) in padded "
              f"chunks of up to {min(64, max(8, threads))}; reference CPU kernels (src/sw_affine/kernels_cpu.cpp) forward+backward")
    line = {"impl": "reference", "metric": METRIC, "value": gcups, "unit": "GCUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"ragged batch: {NPAIRS} affine pairs, N,M log-uniform "
                                   f"[{LMIN},{LMAX}], go {GO} ge {GE} T {T}", "sample": sample},
            "cpu_baseline": {"value": gcups, "unit": "GCUPS", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": gcups, "unit": "GCUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# second-order ops (not the contract line: a measurement and profiling case)
# ---------------------------------------------------------------------------

def second_order(args):
    """The second-order ops at the training-step shapes: `--pairs` pairs
    (default 256) of 512 x 512, scores <e_i, f_j> / sqrt(128) with N(0, 1)
    embeddings.  Times the HVP, dP/dT and the map's full VJP (the HVP pass
    with the parameter tangents) through the C ABI with buffers allocated
    once, CUDA events on the launching stream, `--warmup` untimed and
    `--steps` timed calls each; prints one JSON line."""
    import torch

    import orihime_b200  # noqa: F401
    from orihime_b200 import _lib

    lib = _lib.load()
    B = args.pairs if args.pairs != NPAIRS else 256
    N, d = 512, 128
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    e = torch.randn(B, N, d, generator=g, device="cuda")
    f = torch.randn(B, N, d, generator=g, device="cuda")
    s = (torch.bmm(e, f.transpose(1, 2)) / d ** 0.5).contiguous()
    v = torch.randn(B, N, N, generator=g, device="cuda")
    del e, f
    out = torch.empty_like(s)
    gt = torch.zeros(B, 4, device="cuda")
    nbytes = int(lib.swb_sw_affine_aux_workspace_bytes_for(B, N, N, GO, GE, T))
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    P = lambda t: t.data_ptr()  # noqa: E731
    calls = {
        "hvp": lambda: lib.swb_sw_affine_hvp(P(s), P(v), None, B, N, N, GO, GE, T, P(out), None,
                                             P(ws), nbytes, st),
        "grad_temp": lambda: lib.swb_sw_affine_param_jacobian(P(s), None, B, N, N, GO, GE, T, 2,
                                                              P(out), P(ws), nbytes, st),
        "marginals_backward": lambda: lib.swb_sw_affine_hvp(P(s), P(v), None, B, N, N, GO, GE, T,
                                                            P(out), P(gt), P(ws), nbytes, st),
    }
    cells = B * N * N
    res = {}
    for name, fn in calls.items():
        for _ in range(max(args.warmup, 1)):
            if fn() != 0:
                raise RuntimeError(f"{name} failed")
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / args.steps
        res[name] = {"ms": round(ms, 3), "gcups": round(cells / ms / 1e6, 2)}
    print(json.dumps({"second_order": res, "pairs": B, "shape": [N, N], "workspace_bytes": nbytes,
                      "params": {"gap_open": GO, "gap_ext": GE, "temp": T}}))
    return 0


# ---------------------------------------------------------------------------
# global alignment (soft Needleman-Wunsch, linear gap): a measurement case
# ---------------------------------------------------------------------------

def global_alignment(args):
    """Soft Needleman-Wunsch (linear gap, then affine gaps with gap_open -2,
    gap_ext -0.5) at three workloads: 64 pairs of
    1024 x 1024 (scores 3 <e_i, f_j> / sqrt(64), gap -1, T 0.5) for the
    forward + adjoint (value, map, dS/dgap, dS/dT) and the value alone;
    256 pairs of 512 x 512 (N(0, 1) embeddings, d = 128) for the HVP, dP/dT
    and the map's full VJP; and the contract line's ragged batch (4096
    pairs) as one packed plan, forward + adjoint and value alone.  Through the C ABI with buffers allocated once,
    CUDA events on the launching stream, `--warmup` untimed and `--steps`
    timed calls each.  The reference's CPU kernels (src/nw/kernels_cpu.cpp)
    run 2 of the 64 pairs on all host threads for the CPU line.  Prints one
    JSON line."""
    import torch

    import orihime_b200  # noqa: F401
    from orihime_b200 import _lib

    lib = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    P = lambda t: t.data_ptr()  # noqa: E731
    gap, temp = -1.0, 0.5

    def timed(fn):
        for _ in range(max(args.warmup, 1)):
            if fn() != 0:
                raise RuntimeError("global-alignment call failed")
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / args.steps

    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    B, N, d = 64, 1024, 64
    e = torch.randn(B, N, d, generator=g, device="cuda")
    f = torch.randn(B, N, d, generator=g, device="cuda")
    s = (3.0 * torch.bmm(e, f.transpose(1, 2)) / d ** 0.5).contiguous()
    del e, f
    val, amap = torch.empty(B, device="cuda"), torch.empty_like(s)
    gg, gT = torch.empty(B, device="cuda"), torch.empty(B, device="cuda")
    nb = int(lib.swb_nw_workspace_bytes(B, N, N))
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    nbv = int(lib.swb_nw_value_workspace_bytes(B, N, N))
    wsv = torch.empty(nbv, dtype=torch.uint8, device="cuda")
    cells = B * N * N
    res = {}
    ms = timed(lambda: lib.swb_nw_forward(P(s), None, B, N, N, gap, temp, P(val), P(amap), P(gg),
                                          P(gT), P(ws), nb, st, None))
    res["forward_adjoint"] = {"ms": round(ms, 3), "gcups": round(cells / ms / 1e6, 2)}
    ms = timed(lambda: lib.swb_nw_value(P(s), None, B, N, N, gap, temp, P(val), P(wsv), nbv, st))
    res["value_only"] = {"ms": round(ms, 3), "gcups": round(cells / ms / 1e6, 2)}
    sample = s[:2].cpu().numpy()
    del s, amap, ws, wsv

    B5, N5, d5 = 256, 512, 128
    g.manual_seed(5)
    e = torch.randn(B5, N5, d5, generator=g, device="cuda")
    f = torch.randn(B5, N5, d5, generator=g, device="cuda")
    s5 = (torch.bmm(e, f.transpose(1, 2)) / d5 ** 0.5).contiguous()
    v5 = torch.randn(B5, N5, N5, generator=g, device="cuda")
    del e, f
    out, gt = torch.empty_like(s5), torch.zeros(B5, 4, device="cuda")
    nx = int(lib.swb_nw_aux_workspace_bytes(B5, N5, N5))
    wx = torch.empty(nx, dtype=torch.uint8, device="cuda")
    c5 = B5 * N5 * N5
    for name, fn in (
            ("hvp", lambda: lib.swb_nw_hvp(P(s5), P(v5), None, B5, N5, N5, gap, temp, P(out), None,
                                           P(wx), nx, st)),
            ("grad_temp", lambda: lib.swb_nw_param_jacobian(P(s5), None, B5, N5, N5, gap, temp, 1,
                                                            P(out), P(wx), nx, st)),
            ("marginals_backward", lambda: lib.swb_nw_hvp(P(s5), P(v5), None, B5, N5, N5, gap, temp,
                                                          P(out), P(gt), P(wx), nx, st))):
        ms = timed(fn)
        res[name] = {"ms": round(ms, 3), "gcups": round(c5 / ms / 1e6, 2), "shape": [B5, N5, N5]}
    del s5, v5, out, wx

    # the bench's ragged batch (4096 pairs, log-uniform 32..2048, seed 3) as one packed plan
    from orihime_b200 import ragged
    lengths = workload_lengths(3)
    offsets, ln32 = ragged.layout(lengths)
    flat = make_scores(torch, lengths, offsets, 3, "cuda")
    plan = ragged.Plan(ln32, offsets, family="global", device="cuda")
    outr = plan.outputs()
    vals = torch.empty(plan.B, device="cuda")
    rcells = plan.cells
    ms = timed(lambda: (plan.run(flat, gap=gap, temp=temp, out=outr), 0)[1])
    res["ragged_forward_adjoint"] = {"ms": round(ms, 3), "gcups": round(rcells / ms / 1e6, 2),
                                     "pairs": plan.B, "cells": rcells}
    ms = timed(lambda: (plan.values(flat, gap=gap, temp=temp, out=vals), 0)[1])
    res["ragged_value_only"] = {"ms": round(ms, 3), "gcups": round(rcells / ms / 1e6, 2)}
    del flat, plan, outr

    # affine gaps: the same three workloads
    aff = {}
    go, ge = -2.0, -0.5
    g.manual_seed(1)
    e = torch.randn(B, N, d, generator=g, device="cuda")
    f = torch.randn(B, N, d, generator=g, device="cuda")
    s = (3.0 * torch.bmm(e, f.transpose(1, 2)) / d ** 0.5).contiguous()
    del e, f
    amap = torch.empty_like(s)
    go_, ge_ = torch.empty(B, device="cuda"), torch.empty(B, device="cuda")
    nb = int(lib.swb_nw_affine_workspace_bytes(B, N, N))
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    nbv = int(lib.swb_nw_affine_value_workspace_bytes(B, N, N))
    wsv = torch.empty(nbv, dtype=torch.uint8, device="cuda")
    ms = timed(lambda: lib.swb_nw_affine_forward(P(s), None, B, N, N, go, ge, temp, P(val), P(amap),
                                                 P(go_), P(ge_), P(gT), P(ws), nb, st, None))
    aff["forward_adjoint"] = {"ms": round(ms, 3), "gcups": round(cells / ms / 1e6, 2)}
    ms = timed(lambda: lib.swb_nw_affine_value(P(s), None, B, N, N, go, ge, temp, P(val), P(wsv),
                                               nbv, st))
    aff["value_only"] = {"ms": round(ms, 3), "gcups": round(cells / ms / 1e6, 2)}
    del s, amap, ws, wsv
    g.manual_seed(5)
    e = torch.randn(B5, N5, d5, generator=g, device="cuda")
    f = torch.randn(B5, N5, d5, generator=g, device="cuda")
    s5 = (torch.bmm(e, f.transpose(1, 2)) / d5 ** 0.5).contiguous()
    v5 = torch.randn(B5, N5, N5, generator=g, device="cuda")
    del e, f
    out = torch.empty_like(s5)
    nx = int(lib.swb_nw_affine_aux_workspace_bytes(B5, N5, N5))
    wx = torch.empty(nx, dtype=torch.uint8, device="cuda")
    for name, fn in (
            ("hvp", lambda: lib.swb_nw_affine_hvp(P(s5), P(v5), None, B5, N5, N5, go, ge, temp,
                                                  P(out), None, P(wx), nx, st)),
            ("grad_temp", lambda: lib.swb_nw_affine_param_jacobian(P(s5), None, B5, N5, N5, go, ge,
                                                                   temp, 2, P(out), P(wx), nx, st)),
            ("marginals_backward", lambda: lib.swb_nw_affine_hvp(P(s5), P(v5), None, B5, N5, N5, go,
                                                                 ge, temp, P(out), P(gt), P(wx), nx,
                                                                 st))):
        ms = timed(fn)
        aff[name] = {"ms": round(ms, 3), "gcups": round(c5 / ms / 1e6, 2), "shape": [B5, N5, N5]}
    del s5, v5, out, wx
    flat = make_scores(torch, lengths, offsets, 3, "cuda")
    plan = ragged.Plan(ln32, offsets, family="global_affine", device="cuda")
    outr = plan.outputs()
    ms = timed(lambda: (plan.run(flat, gap_open=go, gap_ext=ge, temp=temp, out=outr), 0)[1])
    aff["ragged_forward_adjoint"] = {"ms": round(ms, 3), "gcups": round(rcells / ms / 1e6, 2)}
    ms = timed(lambda: (plan.values(flat, gap_open=go, gap_ext=ge, temp=temp, out=vals), 0)[1])
    aff["ragged_value_only"] = {"ms": round(ms, 3), "gcups": round(rcells / ms / 1e6, 2)}
    del flat, plan, outr
    res["affine"] = dict(aff, params={"gap_open": go, "gap_ext": ge, "temp": temp})

    line = {"global_alignment": res, "shape": [B, N, N], "params": {"gap": gap, "temp": temp}}
    try:
        from oracle import oracle as O   # the reference's CPU kernels, as a baseline
        if O.ref_available():
            torch.set_num_threads(os.cpu_count() or 1)
            t0 = time.perf_counter()
            O.ref_nw(sample, None, gap, temp)
            sec = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": round(sample.size / sec / 1e9, 4), "unit": "GCUPS",
                                    "cores": torch.get_num_threads(), "kind": "reference",
                                    "sample": "2 of the 64 pairs of 1024 x 1024, forward + backward"}
    except ImportError:
        pass
    print(json.dumps(line))
    return 0


def saigo_vert(args):
    """Saigo-Vert local alignment, affine gaps (gap_open -2, gap_ext -0.5,
    T 0.5), through the C ABI: the contract line's ragged batch (4096 pairs)
    as one packed plan (family 5), forward + adjoint and value alone; 64
    pairs of 1024 x 1024 (scores 3 <e_i, f_j> / sqrt(64)) padded; and the
    HVP / dP/dT / map VJP at 256 x 512 x 512.  CUDA events on the launching
    stream, `--warmup` untimed and `--steps` timed calls each.  The
    reference's CPU kernels (src/sv_affine/kernels_cpu.cpp) run 2 of the 64
    pairs on all host threads for the CPU line.  Prints one JSON line."""
    import torch

    import orihime_b200  # noqa: F401
    from orihime_b200 import _lib, ragged

    lib = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    P = lambda t: t.data_ptr()  # noqa: E731
    go, ge, temp = -2.0, -0.5, 0.5

    def timed(fn):
        for _ in range(max(args.warmup, 1)):
            if fn() != 0:
                raise RuntimeError("Saigo-Vert call failed")
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / args.steps

    res = {}
    lengths = workload_lengths(3)
    offsets, ln32 = ragged.layout(lengths)
    flat = make_scores(torch, lengths, offsets, 3, "cuda")
    plan = ragged.Plan(ln32, offsets, family="saigo_vert", device="cuda")
    outr = plan.outputs()
    vals = torch.empty(plan.B, device="cuda")
    rc = plan.cells
    ms = timed(lambda: (plan.run(flat, gap_open=go, gap_ext=ge, temp=temp, out=outr), 0)[1])
    res["ragged_forward_adjoint"] = {"ms": round(ms, 3), "gcups": round(rc / ms / 1e6, 2),
                                     "pairs": plan.B, "cells": rc}
    ms = timed(lambda: (plan.values(flat, gap_open=go, gap_ext=ge, temp=temp, out=vals), 0)[1])
    res["ragged_value_only"] = {"ms": round(ms, 3), "gcups": round(rc / ms / 1e6, 2)}
    del flat, plan, outr

    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    B, N, d = 64, 1024, 64
    e = torch.randn(B, N, d, generator=g, device="cuda")
    f = torch.randn(B, N, d, generator=g, device="cuda")
    s = (3.0 * torch.bmm(e, f.transpose(1, 2)) / d ** 0.5).contiguous()
    del e, f
    val, amap = torch.empty(B, device="cuda"), torch.empty_like(s)
    go_, ge_, gT = (torch.empty(B, device="cuda") for _ in range(3))
    nb = int(lib.swb_sv_affine_workspace_bytes(B, N, N))
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    nbv = int(lib.swb_sv_affine_value_workspace_bytes(B, N, N))
    wsv = torch.empty(nbv, dtype=torch.uint8, device="cuda")
    cells = B * N * N
    ms = timed(lambda: lib.swb_sv_affine_forward(P(s), None, B, N, N, go, ge, temp, P(val), P(amap),
                                                 P(go_), P(ge_), P(gT), P(ws), nb, st, None))
    res["forward_adjoint"] = {"ms": round(ms, 3), "gcups": round(cells / ms / 1e6, 2),
                              "shape": [B, N, N]}
    ms = timed(lambda: lib.swb_sv_affine_value(P(s), None, B, N, N, go, ge, temp, P(val), P(wsv),
                                               nbv, st))
    res["value_only"] = {"ms": round(ms, 3), "gcups": round(cells / ms / 1e6, 2)}
    sample = s[:2].cpu().numpy()
    del s, amap, ws, wsv

    B5, N5, d5 = 256, 512, 128
    g.manual_seed(5)
    e = torch.randn(B5, N5, d5, generator=g, device="cuda")
    f = torch.randn(B5, N5, d5, generator=g, device="cuda")
    s5 = (torch.bmm(e, f.transpose(1, 2)) / d5 ** 0.5).contiguous()
    v5 = torch.randn(B5, N5, N5, generator=g, device="cuda")
    del e, f
    out, gt = torch.empty_like(s5), torch.zeros(B5, 4, device="cuda")
    nx = int(lib.swb_sv_affine_aux_workspace_bytes(B5, N5, N5))
    wx = torch.empty(nx, dtype=torch.uint8, device="cuda")
    c5 = B5 * N5 * N5
    for name, fn in (
            ("hvp", lambda: lib.swb_sv_affine_hvp(P(s5), P(v5), None, B5, N5, N5, go, ge, temp,
                                                  P(out), None, P(wx), nx, st)),
            ("grad_temp", lambda: lib.swb_sv_affine_param_jacobian(P(s5), None, B5, N5, N5, go, ge,
                                                                   temp, 2, P(out), P(wx), nx, st)),
            ("marginals_backward", lambda: lib.swb_sv_affine_hvp(P(s5), P(v5), None, B5, N5, N5, go,
                                                                 ge, temp, P(out), P(gt), P(wx), nx,
                                                                 st))):
        ms = timed(fn)
        res[name] = {"ms": round(ms, 3), "gcups": round(c5 / ms / 1e6, 2), "shape": [B5, N5, N5]}
    del s5, v5, out, wx

    line = {"saigo_vert": res, "params": {"gap_open": go, "gap_ext": ge, "temp": temp}}
    try:
        from oracle import oracle as O   # the reference's CPU kernels, as a baseline
        if O.ref_available():
            torch.set_num_threads(os.cpu_count() or 1)
            t0 = time.perf_counter()
            O.ref_sv(sample, None, go, ge, temp)
            sec = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": round(sample.size / sec / 1e9, 4), "unit": "GCUPS",
                                    "cores": torch.get_num_threads(), "kind": "reference",
                                    "sample": "2 of the 64 pairs of 1024 x 1024, forward + backward"}
    except ImportError:
        pass
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

TRAFFIC_PROFILES = {4: "lbwd_kernel_affine_r4_dram.md", 8: "lfwd_lbwd_kernels_affine_r8_1024pairs.md"}


def profile_traffic(cols):
    """DRAM bytes per useful cell of one adjoint launch with `cols` columns
    per lane, from the committed ncu summary of that kernel (its line
    'dram_bytes_per_cell: X'), and the summary's path; (None, None) when no
    capture of that kernel is committed."""
    name = TRAFFIC_PROFILES.get(cols)
    if name is None:
        return None, None
    path = os.path.join(ROOT, "profiles", name)
    try:
        txt = open(path).read()
    except OSError:
        return None, None
    val = None
    for line in txt.splitlines():
        if line.strip().startswith("dram_bytes_per_cell:"):
            val = float(line.split(":", 1)[1].split()[0])
    return val, f"profiles/{name}"


def time_steps(torch, fn, steps, stream=None):
    """Milliseconds of `steps` calls of fn, CUDA events on the current stream."""
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--pairs", type=int, default=NPAIRS, help="pairs per GPU (profiling cases)")
    ap.add_argument("--cols-per-lane", type=int, default=0, help="band columns per lane (2, 4 or 8; 0 = timed choice)")
    ap.add_argument("--quick", action="store_true",
                    help="timed steps only: no e2e, plain, CPU legs (profiling cases)")
    ap.add_argument("--global-alignment", action="store_true",
                    help="time the soft Needleman-Wunsch (global alignment) ops instead")
    ap.add_argument("--saigo-vert", action="store_true",
                    help="time the Saigo-Vert (affine gaps) ops instead")
    ap.add_argument("--second-order", action="store_true",
                    help="time the second-order ops at the training-step shapes instead")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.global_alignment:
        return global_alignment(args)
    if args.second_order:
        return second_order(args)
    if args.saigo_vert:
        return saigo_vert(args)

    import torch

    import orihime_b200
    from orihime_b200 import _lib, ragged

    world, rank, local = dist_init(torch)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _lib.load()

    # one pair list for the whole job, LPT-sharded over the ranks (one rank:
    # the whole batch); no collective touches the data
    lengths, gidx, shards = shard_of(world, rank, args.pairs)
    offsets, ln32 = ragged.layout(lengths)
    cells = int((lengths[:, 0] * lengths[:, 1]).sum())
    flat = make_scores(torch, lengths, offsets, 3, dev, index=gidx)
    params = dict(gap_open=GO, gap_ext=GE, temp=T)
    # launch configuration: columns per lane chosen by timing the candidates
    # (2, 4, 8 for every pair, or per length bucket) on this batch and GPU
    if args.cols_per_lane:
        plan = ragged.Plan(ln32, offsets, family="affine", device=dev, cols_per_lane=args.cols_per_lane)
        tuning = {"choice": f"R{args.cols_per_lane}", "fixed": True}
    else:
        plan, tuning = ragged.autotune_plan(ln32, offsets, "affine", dev, flat=flat, **params)
    cols = int(tuning["choice"][1:]) if tuning["choice"].startswith("R") else 0
    if cols:
        plan_cols = np.full(len(lengths), cols)
    else:
        plan_cols = plan.cols
    w = 32 * plan_cols
    computed = int((np.maximum(1, (lengths[:, 1] + w - 1) // w) * (lengths[:, 0] + 31) * w).sum())
    # the eager leg records the forward / adjoint split inside one uniform plan
    eplan = plan if isinstance(plan, ragged.Plan) else ragged.Plan(ln32, offsets, family="affine",
                                                                   device=dev, cols_per_lane=4)

    # ---- headline: the packed plan captured in a CUDA graph, replayed ----
    graph, gout = plan.graph(flat, **params)
    for _ in range(max(args.warmup, 3)):
        graph.replay()
    torch.cuda.synchronize()
    if plan.status() != 0:
        raise RuntimeError("kernel reported a bounded-wait timeout")
    with ClockSampler(local) as clk:
        barrier(torch, world)
        torch.cuda.synchronize()
        total_ms = time_steps(torch, graph.replay, args.steps)
        barrier(torch, world)
    total_ms = max_over_ranks(torch, world, total_ms)
    ms = total_ms / args.steps
    job = workload_lengths(3, args.pairs * world)
    all_cells = int((job[:, 0] * job[:, 1]).sum())   # every shard's cells: the whole job
    gcups_all = all_cells / (ms * 1e-3) / 1e9
    if world > 1:   # the job's values in pair order (one all_gather, outside the timed region)
        vals = ragged.all_gather_values(gout.value, shards, sum(len(x) for x in shards))
    else:
        vals = gout.value
    if not bool(torch.isfinite(vals).all()):
        raise RuntimeError("non-finite values")

    # ---- the same step through plan.run (no graph), with the forward /
    # adjoint split recorded by the library between the two kernels ----
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    for trio in ev:           # create the underlying CUDA events before timing
        for e_ in trio:
            e_.record()
    torch.cuda.synchronize()
    opts = [_lib.Options(0, 0, 0, trio[1].cuda_event, 0, 0) for trio in ev]
    out = eplan.outputs()
    for _ in range(2):
        eplan.run(flat, out=out, **params)
    torch.cuda.synchronize()
    barrier(torch, world)
    for k in range(args.steps):
        ev[k][0].record()
        eplan.run(flat, out=out, options=opts[k], **params)
        ev[k][2].record()
    torch.cuda.synchronize()
    barrier(torch, world)
    per_step = sorted(ev[k][0].elapsed_time(ev[k][2]) for k in range(args.steps))
    eager_ms = max_over_ranks(torch, world, float(np.mean(per_step)))
    kernel_split = {
        "fwd_ms": float(np.mean([ev[k][0].elapsed_time(ev[k][1]) for k in range(args.steps)])),
        "bwd_ms": float(np.mean([ev[k][1].elapsed_time(ev[k][2]) for k in range(args.steps)])),
        "note": "plan.run without a graph; fwd_ms includes the per-call workspace memsets",
    }
    del graph, gout, out

    if args.quick:
        if rank == 0:
            print(json.dumps({"quick": True, "pairs": args.pairs, "cols_per_lane": args.cols_per_lane,
                              "cells": cells, "ms_per_step": ms, "eager_ms_per_step": eager_ms,
                              "gcups": gcups_all, "kernel_ms": kernel_split}))
        return 0

    # ---- dense posteriors: the same lengths with N(0, 1) scores at T = 1
    # (few cells are negligible, so the adjoint's quiet-chunk skip rarely
    # applies) ----
    g = torch.Generator(device=dev)
    g.manual_seed(11 + rank)
    dense = torch.randn(flat.numel(), generator=g, device=dev)
    dgraph, _ = plan.graph(dense, gap_open=GO, gap_ext=GE, temp=1.0)
    for _ in range(2):
        dgraph.replay()
    torch.cuda.synchronize()
    barrier(torch, world)
    dense_ms = max_over_ranks(torch, world, time_steps(torch, dgraph.replay, args.steps)) / args.steps
    barrier(torch, world)
    dense_line = {"value": all_cells / (dense_ms * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": dense_ms,
                  "workload": "the same lengths, scores N(0, 1), gap_open -2, gap_ext -0.5, T 1.0 (CUDA graph)"}
    del dgraph, dense

    # ---- e2e through the public API: pinned host scores in, values out ----
    # StreamedPlan copies the batch in E2E_PARTS pair groups on a copy stream
    # and starts each group's kernels as soon as its scores have arrived.
    host = torch.empty(flat.numel(), dtype=torch.float32, pin_memory=True)
    host.copy_(flat.cpu())
    host_val = torch.empty(plan.B, dtype=torch.float32, pin_memory=True)
    del plan, eplan
    torch.cuda.empty_cache()
    splan = ragged.StreamedPlan(ln32, offsets, family="affine", device=dev, parts=E2E_PARTS,
                                cols_per_lane=cols or 4)
    sout = splan.outputs()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(2):
        splan.run(host, gap_open=GO, gap_ext=GE, temp=T, out=sout)
        host_val.copy_(sout.value, non_blocking=True)
    torch.cuda.synchronize()
    barrier(torch, world)
    e0.record()
    for _ in range(args.steps):
        splan.run(host, gap_open=GO, gap_ext=GE, temp=T, out=sout)
        host_val.copy_(sout.value, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    if splan.status() != 0:
        raise RuntimeError("kernel reported a bounded-wait timeout")
    e2e_ms = max_over_ranks(torch, world, e0.elapsed_time(e1)) / args.steps
    # the copy floor: the same bytes as one pinned host -> device copy, no compute
    reps = 3
    splan.scores.copy_(host, non_blocking=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        splan.scores.copy_(host, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    copy_ms = max_over_ranks(torch, world, e0.elapsed_time(e1)) / reps
    e2e = {"value": all_cells / (e2e_ms * 1e-3) / 1e9, "unit": "GCUPS",
           "h2d_bytes_per_step": flat.numel() * 4, "d2h_bytes_per_step": splan.B * 4,
           "ms_per_step": e2e_ms, "pipeline": f"{len(splan.groups)} pair groups, copy/compute overlapped",
           "copy_floor": {"ms": copy_ms, "h2d_gbs": flat.numel() * 4 / (copy_ms * 1e-3) / 1e9,
                          "frac": copy_ms / e2e_ms,
                          "how": "one pinned host -> device copy of the step's scores, CUDA events"}}
    del splan, sout, host

    # ---- the plain padded drop-in over the same pairs ----
    plain = None if args.no_plain else plain_padded(torch, lengths, offsets, flat, ms, cells)

    line = None
    if rank == 0:
        peak = mufu_peak(torch, lib)
        bwd_ms = kernel_split.get("bwd_ms")
        hbm = measured_peaks().get("hbm_gbs")
        roof = None
        if bwd_ms:
            achieved = MUFU_PER_CELL_BWD * cells / (bwd_ms * 1e-3)
            tpc, tsrc = profile_traffic(cols or 4)
            roof = {"bound": "mufu", "achieved": achieved / 1e9, "peak": peak / 1e9,
                    "unit": "Gop/s", "frac": achieved / peak,
                    "traffic": None if tpc is None else tpc * cells,
                    "traffic_source": tsrc,
                    "kernel": f"lbwd_kernel<3,{cols or 4},1,0> (checkpointed adjoint, scaled linear domain)",
                    "algorithmic": (f"{MUFU_PER_CELL_BWD} ex2/lg2 per cell (the log-domain adjoint's "
                                    f"count) x {cells} cells"),
                    "peak_source": "measured in-bench (swb_mufu_probe: ex2.approx throughput)",
                    "step_frac": (MUFU_PER_CELL * cells / (ms * 1e-3)) / peak,
                    "hbm_frac_of_measured": (None if not hbm else
                                             (BYTES_PER_CELL * cells / (ms * 1e-3)) / (hbm * 1e9)),
                    "note": ("the linear-domain kernels issue about 1 ex2 per cell instead of the "
                             "21 the log-sum-exp recurrence needs, so they can exceed this roofline; "
                             "the fraction is throughput relative to the MUFU bound of the reference's "
                             "formulation")}
        cpu = None if args.no_cpu_baseline else cpu_baseline(lengths)
        clocks = clk.summary()
        line = {"metric": METRIC, "value": gcups_all, "unit": "GCUPS", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"ragged batch: {args.pairs * world} affine pairs, N,M log-uniform "
                                       f"[{LMIN},{LMAX}] (seed 3), scores 3<e,f>/sqrt(64)"
                                       + (f", LPT-sharded over {world} GPUs" if world > 1 else ""),
                           "cells": all_cells, "cells_rank0": cells,
                           "gap_open": GO, "gap_ext": GE, "temp": T,
                           "timed": "CUDA graph replay of the packed plan (forward + adjoint)",
                           "launch": {"columns_per_lane": tuning["choice"],
                                      "tuning_ms": tuning.get("ms"),
                                      "how": "ragged.autotune_plan: candidates timed on this batch"
                                             if not tuning.get("fixed") else "--cols-per-lane",
                                      "computed_over_useful_cells": computed / cells},
                           "l2": "inputs (3.9 GB) larger than L2; no flush",
                           "parallelism": (f"LPT shards x{world} of one pair list, no collective on "
                                           "the data path" if world > 1 else "one GPU")},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": 2 * args.steps, "clocks": clocks,
                "eager_ms_per_step": eager_ms, "kernel_ms": kernel_split,
                "step_ms_spread_eager": [per_step[0], per_step[-1]],
                "dense_posteriors": dense_line, "plain_padded": plain}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def plain_padded(torch, lengths, offsets, flat, ragged_ms, cells_all, chunk=64):
    """The plain padded drop-in (torch.ops.orihime.sw_affine_forward) over
    ALL pairs of the batch: pairs grouped by size in chunks of `chunk`, each
    chunk padded to its own largest L1 x L2, the kernel times of
    the chunks summed.  Two variants: masked (cells outside each pair at the
    mask sentinel, as ohm.sw_affine(mask=...) passes them: the whole padded
    area is computed) and lengths (the kernel skips cells outside each
    pair)."""
    from orihime_b200 import operator as op
    from orihime_b200 import ragged

    dev = flat.device
    # grouping with little padding: by L2 in half-octave buckets, then by L1
    # (2.2x padded cells on this batch; sorting by L1 alone pads 4.1x)
    order = np.lexsort((lengths[:, 0], np.floor(np.log2(lengths[:, 1]) * 2)))[::-1]
    res = {"masked": 0.0, "lengths": 0.0}
    padded_cells = 0
    for c0 in range(0, len(order), chunk):
        pick = order[c0:c0 + chunk]
        L1m = int(lengths[pick, 0].max())
        L2m = int(lengths[pick, 1].max())
        padded_cells += len(pick) * L1m * L2m
        x = torch.zeros(len(pick), L1m, L2m, device=dev)
        mask = torch.ones(len(pick), L1m, L2m, dtype=torch.bool, device=dev)
        for k, b in enumerate(pick):
            L1, L2 = int(lengths[b, 0]), int(lengths[b, 1])
            p = ragged.pitch_of(L2)
            x[k, :L1, :L2] = flat[int(offsets[b]):int(offsets[b]) + L1 * p].view(L1, p)[:, :L2]
            mask[k, :L1, :L2] = False
        xm = op.normalize_mask(x.masked_fill(mask, float("-inf")), T).contiguous()
        ln = torch.tensor([[int(lengths[b, 0]), int(lengths[b, 1])] for b in pick], dtype=torch.int32,
                          device=dev)
        for name, fn in (("masked", lambda: torch.ops.orihime.sw_affine_forward(xm, GO, GE, T, None)),
                         ("lengths", lambda: torch.ops.orihime.sw_affine_forward(x, GO, GE, T, ln))):
            fn()
            torch.cuda.synchronize()
            res[name] += time_steps(torch, fn, 1)
        del x, mask, xm
    torch.cuda.empty_cache()
    ragged_gcups = cells_all / (ragged_ms * 1e-3) / 1e9
    out = {"sample": (f"all {len(order)} pairs grouped by size (L2 half-octave, then L1) in padded chunks of {chunk} "
                      f"({padded_cells:.4g} padded cells for {cells_all:.4g} useful)")}
    for name in ("masked", "lengths"):
        out[name] = {"ms": res[name], "gcups_useful": cells_all / (res[name] * 1e-3) / 1e9}
    out["ragged_over_plain_masked"] = ragged_gcups / out["masked"]["gcups_useful"]
    out["ragged_over_plain_lengths"] = ragged_gcups / out["lengths"]["gcups_useful"]
    return out


def cpu_baseline(lengths):
    """The reference CPU kernels on a bounded sample of the workload (this host's cores)."""
    import torch

    from oracle import oracle as O

    if not O.ref_available():
        try:
            O.build(ref=True)
        except Exception:
            pass
    data, cells, npairs = reference_cpu_sample(lengths, 3, budget_cells=2e8)
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    if O.ref_available():
        kind, fn = "reference", lambda s, ln: O.ref_affine(s, ln, GO, GE, T)
    else:
        kind, fn = "port", lambda s, ln: O.affine(s, ln, GO, GE, T)
        threads = 1
    t0 = time.perf_counter()
    for s, ln in data:
        fn(s, ln)
    dt = time.perf_counter() - t0
    return {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": threads, "kind": kind,
            "sample": f"{npairs} pairs ({cells:.3g} cells) of the workload, padded chunks of "
                      f"up to {min(64, max(8, threads))}, "
                      f"{dt:.1f} s"}


if __name__ == "__main__":
    sys.exit(main())
