"""Test infrastructure: CPU kernels for the local-alignment ops, computed by
the fp64 oracle, so that the autograd and torch.func plumbing of the public
functions (orihime_b200.operator) can be exercised without a GPU.

The package itself has no CPU path; these registrations exist only in the
child process of tests/test_func_transforms.py that imports this module.
Scores are read as float64 by the oracle and results returned as float32.
"""

from __future__ import annotations

import numpy as np
import torch

import orihime_b200  # noqa: F401  (defines the op schemas)
from oracle import oracle as O

_LIB = torch.library.Library("orihime", "IMPL")
_OWN = torch.library.Library("orihime_b200", "IMPL")


def _np(t):
    return None if t is None else t.detach().cpu().numpy()


def _t(a, like):
    return torch.as_tensor(np.asarray(a, dtype=np.float32), device=like.device)


def _affine(scores, go, ge, T, lengths):
    return O.affine(_np(scores), _np(lengths), go, ge, T, dtype=np.float64)


def _linear(scores, gap, T, lengths):
    return O.linear(_np(scores), _np(lengths), gap, T, dtype=np.float64)


def _reg(lib, name, fn):
    lib.impl(name, fn, "CPU")


# ---- soft Smith-Waterman, affine gaps ----
_reg(_LIB, "sw_affine_forward",
     lambda s, go, ge, T, ln: [_t((r := _affine(s, go, ge, T, ln))["value"], s), _t(r["map"], s)])
_reg(_LIB, "sw_affine_value_grad_params",
     lambda s, go, ge, T, ln: tuple(_t((r := _affine(s, go, ge, T, ln))[k], s)
                                    for k in ("grad_open", "grad_ext", "grad_temp")))
_reg(_LIB, "sw_affine_marginals_hvp",
     lambda s, v, go, ge, T, ln: _t(O.affine_hvp(_np(s), _np(v), _np(ln), go, ge, T, dtype=np.float64), s))
for _k, _name in enumerate(("gap_open", "gap_ext", "temp")):
    _reg(_LIB, f"sw_affine_marginals_grad_{_name}",
         lambda s, go, ge, T, ln, k=_k: _t(O.affine_param_grad(_np(s), _np(ln), go, ge, T, k,
                                                               dtype=np.float64), s))
_reg(_OWN, "sw_affine_value", lambda s, go, ge, T, ln: _t(_affine(s, go, ge, T, ln)["value"], s))
_reg(_OWN, "sw_affine_forward_with_grads",
     lambda s, go, ge, T, ln: tuple(_t((r := _affine(s, go, ge, T, ln))[k], s)
                                    for k in ("value", "map", "grad_open", "grad_ext", "grad_temp")))

# ---- soft Smith-Waterman, linear gap ----
_reg(_LIB, "sw_forward",
     lambda s, g, T, ln: [_t((r := _linear(s, g, T, ln))["value"], s), _t(r["map"], s)])
_reg(_LIB, "sw_value_grad_params",
     lambda s, g, T, ln: tuple(_t((r := _linear(s, g, T, ln))[k], s) for k in ("grad_gap", "grad_temp")))
_reg(_LIB, "sw_marginals_hvp",
     lambda s, v, g, T, ln: _t(O.linear_hvp(_np(s), _np(v), _np(ln), g, T, dtype=np.float64), s))
for _k, _name in enumerate(("gap", "temp")):
    _reg(_LIB, f"sw_marginals_grad_{_name}",
         lambda s, g, T, ln, k=_k: _t(O.linear_param_grad(_np(s), _np(ln), g, T, k, dtype=np.float64), s))
_reg(_OWN, "sw_value", lambda s, g, T, ln: _t(_linear(s, g, T, ln)["value"], s))
_reg(_OWN, "sw_forward_with_grads",
     lambda s, g, T, ln: tuple(_t((r := _linear(s, g, T, ln))[k], s)
                               for k in ("value", "map", "grad_gap", "grad_temp")))
