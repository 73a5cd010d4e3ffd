"""The raw tier (orihime_b200.raw, the reference's orihime.raw): no-graph
parameter VJPs with a type-stable contract and the named kernel bindings
(checks in tests/_raw_checks.py)."""

import os
import subprocess
import sys

import pytest
import torch

import orihime_b200 as ohm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FAMILIES = ("sw", "sw_affine", "nw", "nw_affine", "sv_linear", "sv_affine")


def test_modules_and_fields():
    assert ohm.raw.__all__ == ["VJPFields", "sw", "sw_affine", "sv_linear", "sv_affine", "nw", "nw_affine"]
    assert ohm.raw.sw_affine.vjp_fields == ("gap_open_score", "gap_extend_score", "temperature")
    assert ohm.raw.sv_linear.vjp_fields == ("gap_score", "temperature")
    for f in FAMILIES:
        mod = getattr(ohm.raw, f)
        for name in ("vjp_fields", "vjp_one", "vjp", "forward", "forward_t", "value_grad_params",
                     "marginals_backward", "marginals_hvp"):
            assert name in mod.__all__ and hasattr(mod, name), (f, name)


@pytest.mark.parametrize("family", FAMILIES)
def test_contract_errors_before_dispatch(family):
    import _raw_checks as C

    C.check_errors(family, "cpu")


def test_values_on_oracle_cpu_kernels():
    code = ("import sys; sys.path.insert(0, 'tests'); import _oracle_cpu_ops; import _raw_checks as C; "
            "[C.check_values(f, 'cpu') for f in ('sw', 'sw_affine')]; print('raw ok')")
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0 and "raw ok" in res.stdout, res.stdout[-3000:] + res.stderr[-3000:]


@pytest.mark.gpu
@pytest.mark.parametrize("family", FAMILIES)
def test_values_on_cuda(family):
    import _raw_checks as C

    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    C.check_values(family, "cuda")
    C.check_errors(family, "cuda")
