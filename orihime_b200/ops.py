"""Named operations ``ops.<name>`` with the reference's finite surface
(orihime/_public_ops.py:79-263, installed for the alignment families at
:270-313): per family, ``forward`` (map / value / entropy), ``backward``
(a map cotangent contracted against the pair scores and each scalar
parameter) and ``sensitivity`` (dP/dtheta per scalar parameter).

Field names are the public map function's own argument names, so
``ops.sw_affine.backward(x, grad_map=g, gap_open_score=-2.0, ...)`` returns
``{"pair_scores": ..., "gap_open_score": ..., "gap_extend_score": ...,
"temperature": ...}``.  ``output=`` selects one field (the tensor itself) or
a sequence of them (a dict), with the reference's messages for bad
selections.  The evaluations run under ``no_grad`` and call this package's
kernels: the scores' field is the map's vector-Jacobian product (HVP
kernel), a parameter's field is the cotangent contracted with the map's
parameter sensitivity.
"""

from __future__ import annotations

from importlib import import_module
from inspect import signature
from typing import Any, Callable, Sequence

import torch
from torch import Tensor

# the modules themselves (the package re-exports their functions under the same names)
_sw = import_module(".sw", __package__)
_nw = import_module(".nw", __package__)
_sv = import_module(".sv", __package__)

FORWARD_FIELDS = ("map", "value", "entropy")


def _select(output, allowed: tuple[str, ...]) -> tuple[tuple[str, ...], bool]:
    """(fields, single) for an ``output=`` argument (orihime/_public_ops.py:35-58)."""
    if output is None:
        return allowed, False
    if isinstance(output, str):
        fields, single = (output,), True
    elif isinstance(output, Sequence):
        fields, single = tuple(output), False
    else:
        raise TypeError("output must be None, a field name, or a sequence of names")
    if not fields:
        raise ValueError("output must select at least one field")
    if not all(isinstance(f, str) for f in fields):
        raise TypeError("output field names must be strings")
    if len(set(fields)) != len(fields):
        raise ValueError("output must not contain duplicate field names")
    for f in fields:
        if f not in allowed:
            raise ValueError(f"unknown output field {f!r}; expected one of {allowed!r}")
    return fields, single


def _result(fields, single, evaluate: Callable[[str], Tensor]):
    if single:
        return evaluate(fields[0])
    return {f: evaluate(f) for f in fields}


class PublicOperation:
    """forward / backward / sensitivity of one alignment family."""

    def __init__(self, name: str, operator, map_fn, value_fn, entropy_fn):
        self.name = name
        self._op = operator
        self._fns = {"map": map_fn, "value": value_fn, "entropy": entropy_fn}
        self._sig = signature(map_fn)
        names = tuple(self._sig.parameters)
        nparams = len(operator.params)
        self.input_fields = names[:1]
        self.parameter_fields = names[1:1 + nparams]
        self.backward_fields = (*self.input_fields, *self.parameter_fields)
        self.sensitivity_fields = self.parameter_fields
        # public field -> the operator's own name for it
        self._internal = dict(zip(self.backward_fields, (operator.primary_name, *operator.params)))

    def _bind(self, args, kwargs):
        b = self._sig.bind(*args, **kwargs)
        b.apply_defaults()
        v = b.arguments
        primary = v[self.input_fields[0]]
        if not isinstance(primary, Tensor):
            raise TypeError(f"{self.input_fields[0]} must be a tensor")
        params = tuple(v[f] for f in self.parameter_fields)
        return primary, params, v

    def forward(self, *args: Any, output=None, **kwargs: Any):
        """Selected map, value and entropy outputs."""
        fields, single = _select(output, FORWARD_FIELDS)
        return _result(fields, single, lambda f: self._fns[f](*args, **kwargs))

    def backward(self, *args: Any, grad_map: Tensor, output=None, **kwargs: Any):
        """A map cotangent contracted against the selected inputs and parameters."""
        fields, single = _select(output, self.backward_fields)
        primary, params, v = self._bind(args, kwargs)
        extra = dict(lengths=v.get("lengths"), mask=v.get("mask"), dtype=v.get("dtype"))

        def evaluate(field: str) -> Tensor:
            with torch.no_grad():
                r = self._op.vjp(primary, *params, grad_map=grad_map, wrt=self._internal[field], **extra)
            if field not in self.parameter_fields:
                return r
            orig = v[field]
            if isinstance(orig, Tensor):
                return r.to(device=orig.device, dtype=orig.dtype).reshape(orig.shape)
            return r.reshape(())

        return _result(fields, single, evaluate)

    def sensitivity(self, *args: Any, output=None, **kwargs: Any):
        """dP/dtheta [B, L1, L2] for the selected scalar parameters."""
        fields, single = _select(output, self.sensitivity_fields)
        primary, params, v = self._bind(args, kwargs)
        extra = dict(lengths=v.get("lengths"), mask=v.get("mask"), dtype=v.get("dtype"))

        def evaluate(field: str) -> Tensor:
            with torch.no_grad():
                return self._op.sensitivity(primary, *params, wrt=self._internal[field], **extra)

        return _result(fields, single, evaluate)

    def __repr__(self) -> str:
        return f"<orihime_b200.ops.{self.name}>"


sw = PublicOperation("sw", _sw._sw_operator, _sw.sw, _sw.sw_value, _sw.sw_entropy)
sw_affine = PublicOperation("sw_affine", _sw._sw_affine_operator, _sw.sw_affine, _sw.sw_affine_value,
                            _sw.sw_affine_entropy)
nw = PublicOperation("nw", _nw._nw_operator, _nw.nw, _nw.nw_value, _nw.nw_entropy)
nw_affine = PublicOperation("nw_affine", _nw._nw_affine_operator, _nw.nw_affine, _nw.nw_affine_value,
                            _nw.nw_affine_entropy)
sv = PublicOperation("sv", _sv._sv_linear_operator, _sv.sv, _sv.sv_value, _sv.sv_entropy)
sv_affine = PublicOperation("sv_affine", _sv._sv_affine_operator, _sv.sv_affine, _sv.sv_affine_value,
                            _sv.sv_affine_entropy)

__all__ = ["sw", "sw_affine", "nw", "nw_affine", "sv", "sv_affine", "PublicOperation"]
