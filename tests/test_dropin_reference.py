"""The drop-in mechanics with the reference's unchanged Python package (CPU).

The reference package with its CPU extension is built from the reference
sources by tests/golden/make_golden.py (``build_reference``; about two
minutes on 8 cores, once).  A child process imports it, then this package,
and checks what a user of the reference sees:

* no schema is defined twice: this package registers kernels on the
  reference's own schemas, which stay as the reference declared them;
* the CUDA and AutogradCUDA kernels of the replaced ops are present, and the
  reference loader's cached "CUDA dispatch available" answer is refreshed,
  so its wrappers accept CUDA tensors (a CPU-only build otherwise refuses
  them, orihime/_ops.py:161-170);
* the reference's CPU results are bit-identical before and after the import;
* the public functions and named operations have the reference's
  signatures and field names.

The numerical side of the drop-in (the same public calls on CUDA tensors
against the reference's recorded outputs) is tests/test_gpu_public_api.py.
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import inspect, json, sys
sys.path.insert(0, PKG)
sys.path.insert(1, ROOT)
import torch
import orihime as ref
import orihime._ops as ref_loader

torch.manual_seed(0)
s = torch.randn(3, 9, 11) * 1.5
ln = torch.tensor([[9, 11], [4, 7], [0, 3]], dtype=torch.int32)
kw = dict(gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.7)
before = [ref.sw_affine(s, lengths=ln, **kw), ref.sw_affine_value(s, lengths=ln, **kw),
          ref.sw(s, gap_score=-1.0, temperature=0.7), ref.ops.sw_affine.sensitivity(s, **kw)["temperature"]]
flag_before = ref_loader._cuda_dispatch_available

import orihime_b200 as ob

after = [ref.sw_affine(s, lengths=ln, **kw), ref.sw_affine_value(s, lengths=ln, **kw),
         ref.sw(s, gap_score=-1.0, temperature=0.7), ref.ops.sw_affine.sensitivity(s, **kw)["temperature"]]
has = torch._C._dispatch_has_kernel_for_dispatch_key
ops = list(ob._ops.SCHEMAS)
schemas_equal = all(
    str(getattr(torch.ops.orihime, n).default._schema) == str(torch._C.parse_schema("orihime::" + ob._ops.SCHEMAS[n]))
    for n in ops)


def sig(f):
    return [(p.name, str(p.kind), repr(p.default)) for p in inspect.signature(f).parameters.values()]


funcs = [n for n in ob.__all__ if n != "ops"]
fields = {}
for n in ("sw", "sw_affine", "nw", "nw_affine", "sv", "sv_affine"):
    a, b = getattr(ref.ops, n), getattr(ob.ops, n)
    fields[n] = [list(a.backward_fields) == list(b.backward_fields),
                 list(a.sensitivity_fields) == list(b.sensitivity_fields)]
print(json.dumps({
    "defined_here": ob._ops.DEFINED_HERE,
    "cuda": {n: has("orihime::" + n, "CUDA") for n in ops},
    "autograd_cuda": {n: has("orihime::" + n, "AutogradCUDA") for n in
                      ("sw_forward", "sw_forward_t", "sw_affine_forward", "sw_affine_forward_t")},
    "flag_before": flag_before, "flag_after": ref_loader._cuda_dispatch_available,
    "cpu_unchanged": all(torch.equal(x, y) for x, y in zip(before, after)),
    "schemas_equal": schemas_equal,
    "signatures": {n: sig(getattr(ref, n)) == sig(getattr(ob, n)) for n in funcs},
    "fields": fields,
}))
'''


def _reference_package():
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    try:
        import make_golden
    finally:
        sys.path.pop(0)
    if os.path.exists(os.path.join(make_golden.WORK, "orihime", "_C.so")):
        return make_golden.WORK
    if not os.path.isdir(os.path.join(make_golden.REF, "orihime")):
        pytest.skip("reference sources not present (ORIHIME_REFERENCE)")
    return make_golden.build_reference()


def test_reference_package_then_this_one():
    pkg = _reference_package()
    code = f"PKG = {pkg!r}\nROOT = {ROOT!r}\n" + CHILD
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["defined_here"] == []
    assert all(out["cuda"].values()), [k for k, v in out["cuda"].items() if not v]
    assert all(out["autograd_cuda"].values()), out["autograd_cuda"]
    assert out["flag_before"] is False and out["flag_after"] is True
    assert out["cpu_unchanged"]
    assert out["schemas_equal"]
    assert all(out["signatures"].values()), [k for k, v in out["signatures"].items() if not v]
    assert all(all(v) for v in out["fields"].values()), out["fields"]
