"""torch.compile over the public functions: fullgraph and graph-break
compiles of map, value and entropy, reverse mode, dynamic tensor parameters
and masks, as the reference's tests/test_compile.py exercises them (checks in
tests/_compile_checks.py).

The CPU test runs the checks under aot_eager in a child process whose
local-alignment ops have CPU kernels computed by the fp64 oracle
(tests/_oracle_cpu_ops.py).  The GPU tests run aot_eager on all six families
and the default inductor on the local families."""

import os
import subprocess
import sys

import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FAMILIES = ("sw", "sw_affine", "nw", "nw_affine", "sv_linear", "sv_affine")


def test_compile_on_oracle_cpu_kernels():
    code = ("import sys; sys.path.insert(0, 'tests'); import _oracle_cpu_ops; "
            "import _compile_checks as C; "
            "print('checks', C.run_all(('sw', 'sw_affine'), 'cpu', backends=('aot_eager',)))")
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=900)
    assert res.returncode == 0, res.stdout[-3000:] + res.stderr[-3000:]
    assert "checks 18" in res.stdout, res.stdout[-2000:]


@pytest.mark.gpu
@pytest.mark.parametrize("family", FAMILIES)
def test_compile_aot_eager(family):
    import _compile_checks as C

    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    assert C.run_all((family,), "cuda", backends=("aot_eager",)) == 9


@pytest.mark.gpu
@pytest.mark.parametrize("family", ("sw", "sw_affine"))
def test_compile_default_inductor(family):
    import _compile_checks as C

    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    assert C.run_all((family,), "cuda", backends=("inductor",)) == 9
