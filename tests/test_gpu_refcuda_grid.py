"""Our public map and value against the reference's CUDA path on the
reference's own benchmark shapes (the 22 cases of its rectangular-production
grid, benchmarks/grid_cases.json and benchmarks/grid.py of
megure-labs/orihime), all six families, on the same GPU.

Inputs follow that harness: uniform scores in [-0.5, 0.5) seeded per case,
its parameters per family, full lengths except the ragged case.  The
reference runs its legacy float op, which is what its public map and value
both run (forward and backward); ours runs the public functions under
no_grad: map = forward + adjoint, value = the forward wavefront alone.
Timing: CUDA events, 3 warm-up calls, iterations for ~20 ms, median of 3.

The reference extension (``make -C oracle refcuda``) must load before
orihime_b200, so the comparison runs in a child process; the table is
printed.  Bar: values within rel 1e-4 of the reference path (uniform scores
at T ~ 0.7 are well conditioned)."""

import json
import os
import statistics
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu

# (id, batch, L1, L2, explicit lengths or None)
CASES = [
    ("rect-b1-64x64", 1, 64, 64, None), ("rect-b1-128x128", 1, 128, 128, None),
    ("rect-b1-256x256", 1, 256, 256, None), ("rect-b1-512x512", 1, 512, 512, None),
    ("rect-b1-1024x1024", 1, 1024, 1024, None), ("rect-b1-2048x2048", 1, 2048, 2048, None),
    ("rect-b1-128x2048", 1, 128, 2048, None), ("rect-b1-2048x128", 1, 2048, 128, None),
    ("rect-b1-512x2048", 1, 512, 2048, None), ("rect-b1-2048x512", 1, 2048, 512, None),
    ("rect-b1-511x1023", 1, 511, 1023, None), ("rect-b1-1023x511", 1, 1023, 511, None),
    ("rect-b1-1023x2047", 1, 1023, 2047, None), ("rect-b1-2047x1023", 1, 2047, 1023, None),
    ("rect-b8-64x64", 8, 64, 64, None), ("rect-b32-64x64", 32, 64, 64, None),
    ("rect-b128-64x64", 128, 64, 64, None), ("rect-b8-128x128", 8, 128, 128, None),
    ("rect-b32-128x128", 32, 128, 128, None), ("rect-b8-256x256", 8, 256, 256, None),
    ("rect-b4-512x512", 4, 512, 512, None),
    ("rect-b4-2048x2048-ragged", 4, 2048, 2048, [[2048, 2048], [1537, 997], [511, 2047], [127, 257]]),
]
# family: (public name, legacy reference op, parameters)
FAMILIES = {
    "sw": ("sw", "soft_sw_float", dict(gap_score=-0.75, temperature=0.73)),
    "sw_affine": ("sw_affine", "soft_sw_affine_float",
                  dict(gap_open_score=-1.25, gap_extend_score=-0.25, temperature=0.73)),
    "sv": ("sv", "soft_sv_linear_float", dict(gap_score=-0.75, temperature=0.73)),
    "sv_affine": ("sv_affine", "soft_sv_affine_float",
                  dict(gap_open_score=-2.0, gap_extend_score=-0.5, temperature=1.0)),
    "nw": ("nw", "soft_nw_float", dict(gap_score=-0.75, temperature=0.73)),
    "nw_affine": ("nw_affine", "soft_nw_affine_float",
                  dict(gap_open_score=-1.25, gap_extend_score=-0.25, temperature=0.73)),
}


def _time(torch, fn, target_ms=20.0):
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    fn()
    e1.record()
    e1.synchronize()
    probe = max(e0.elapsed_time(e1), 1e-3)
    it = max(3, min(200, int(target_ms / probe) + 1))
    samples = []
    for _ in range(3):
        e0.record()
        for _ in range(it):
            fn()
        e1.record()
        e1.synchronize()
        samples.append(e0.elapsed_time(e1) / it)
    return statistics.median(samples)


def _worker():
    sys.path.insert(0, ROOT)
    import torch
    from oracle import oracle as O

    torch.ops.load_library(O.ref_cuda_path())
    import orihime_b200 as ohm   # takes over the namespaced ops; the legacy ones stay the reference's

    ops = torch.ops.orihime
    rows = []
    for fam, (pub, legacy, params) in FAMILIES.items():
        ref_op = getattr(ops, legacy)
        fmap, fval = getattr(ohm, pub), getattr(ohm, f"{pub}_value")
        vals = list(params.values())
        for k, (cid, B, L1, L2, explicit) in enumerate(CASES):
            g = torch.Generator(device="cpu").manual_seed(0x5A17 + k)
            x = (torch.rand((B, L1, L2), generator=g) - 0.5).cuda()
            ln = [[L1, L2]] * B if explicit is None else explicit
            lengths = torch.tensor(ln, dtype=torch.int32, device="cuda")
            cells = sum(a * b for a, b in ln)
            with torch.no_grad():
                rv, _ = ref_op(x, *vals, lengths)[:2]
                ov = fval(x, **params, lengths=lengths)
                rel = float(((ov - rv).abs() / rv.abs().clamp_min(1e-6)).max())
                tr = _time(torch, lambda: ref_op(x, *vals, lengths))
                tm = _time(torch, lambda: fmap(x, **params, lengths=lengths))
                tv = _time(torch, lambda: fval(x, **params, lengths=lengths))
            rows.append(dict(family=fam, case=cid, cells=cells, ref_ms=tr, map_ms=tm, value_ms=tv,
                             map_speedup=tr / tm, value_speedup=tr / tv, value_rel=rel))
            del x
    print("RESULT " + json.dumps(rows))


def test_grid_against_reference_cuda_path():
    import torch
    from oracle import oracle as O

    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    if O.ref_cuda_path() is None:
        pytest.skip("reference CUDA extension not built (make -C oracle refcuda)")
    r = subprocess.run([sys.executable, __file__, "worker"], capture_output=True, text=True,
                       timeout=1500, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    rows = json.loads(r.stdout.split("RESULT ", 1)[1])
    assert len(rows) == len(CASES) * len(FAMILIES)
    print(f"\n  {'family':10s} {'case':26s} {'ref ms':>9s} {'map ms':>9s} {'value ms':>9s} {'map x':>7s} {'value x':>7s}")
    for c in rows:
        print(f"  {c['family']:10s} {c['case']:26s} {c['ref_ms']:9.3f} {c['map_ms']:9.3f} {c['value_ms']:9.3f} "
              f"{c['map_speedup']:7.1f} {c['value_speedup']:7.1f}")
        assert c["value_rel"] <= 1e-4, c


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "worker":
    _worker()
