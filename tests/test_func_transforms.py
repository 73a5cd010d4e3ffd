"""torch.func over the public functions: jvp, vjp, jacrev and vmap of map,
value and entropy, as the reference's tests/test_func_compat.py exercises
them (checks in tests/_func_checks.py).

The CPU test runs the checks in a child process whose local-alignment ops
have CPU kernels computed by the fp64 oracle (tests/_oracle_cpu_ops.py): it
covers the autograd / transform plumbing without a GPU.  The GPU tests run
the same checks on the CUDA kernels for all six families."""

import os
import subprocess
import sys

import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FAMILIES = ("sw", "sw_affine", "nw", "nw_affine", "sv_linear", "sv_affine")


def test_transforms_on_oracle_cpu_kernels():
    code = ("import sys; sys.path.insert(0, 'tests'); import _oracle_cpu_ops; "
            "import _func_checks as C; n = C.run_all(('sw', 'sw_affine'), 'cpu'); "
            "[C.check_masked_and_ragged(f, 'cpu') for f in ('sw', 'sw_affine')]; print('checks', n)")
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=900)
    assert res.returncode == 0, res.stdout[-3000:] + res.stderr[-3000:]
    assert "checks 50" in res.stdout, res.stdout[-2000:]


@pytest.mark.gpu
@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("observable", ("map", "value", "entropy"))
def test_transforms_match_eager_and_finite_differences(family, observable):
    import _func_checks as C

    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    for chk in (C.check_jvp, C.check_vjp, C.check_jacrev, C.check_vmap, C.check_eager_backward,
                C.check_parameter_vmap_guard, C.check_forward_mode_under_vmap_raises):
        chk(family, observable, "cuda")
    C.check_vmap(family, observable, "cuda", batch=1)


@pytest.mark.gpu
@pytest.mark.parametrize("family", FAMILIES)
def test_transforms_with_mask_and_lengths_and_entropy_directions(family):
    import _func_checks as C

    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    C.check_masked_and_ragged(family, "cuda")
    C.check_entropy_parameter_directions_raise(family, "cuda")
