"""Shared machinery of the raw tier (orihime/raw/_base.py): no-graph
parameter VJPs with a type-stable contract, and the named kernel bindings.

vjp_one(pair_scores, wrt=field, cotangent=g, <params>, lengths) contracts a
map cotangent with the map's sensitivity to one scalar parameter; vjp(...)
returns a dict for a tuple of fields.  The cotangent must already be a
contiguous FP32 tensor with the map's shape and device (TypeError /
ValueError otherwise, before any kernel runs).  A float parameter's VJP has
shape [1], a tensor parameter's the parameter's own shape, dtype and device.

The kernel bindings call torch.ops.orihime.<family>_* directly;
marginals_backward and marginals_hvp first check the user's vector with the
same contract, raising RuntimeError as the op bodies do.
"""

from __future__ import annotations

from inspect import Parameter, Signature
from typing import Callable, Optional, TypeAlias

import torch
from torch import Tensor

from .. import operator as _op

VJPFields: TypeAlias = tuple[str, ...]

# public parameter names and the ops' own names, per family
_PARAMS = {
    "sw": (("gap_score", "temperature"), ("gap", "temp")),
    "sw_affine": (("gap_open_score", "gap_extend_score", "temperature"), ("gap_open", "gap_ext", "temp")),
    "nw": (("gap_score", "temperature"), ("gap", "temp")),
    "nw_affine": (("gap_open_score", "gap_extend_score", "temperature"), ("gap_open", "gap_ext", "temp")),
    "sv_linear": (("gap_score", "temperature"), ("gap", "temp")),
    "sv_affine": (("gap_open_score", "gap_extend_score", "temperature"), ("gap_open", "gap_ext", "temp")),
}
_DEFAULTS = {"gap_score": 0.0, "gap_open_score": 0.0, "gap_extend_score": 0.0, "temperature": 1.0}


def check_vector(primary: Tensor, vector, *, name: str, primary_name: str,
                 error_type: Optional[type] = RuntimeError) -> Tensor:
    """A derivative vector must match the primary's shape and device and be
    contiguous FP32 (orihime/operator.py:176-221); error_type None keeps the
    TypeError / ValueError split of the raw VJPs."""
    if not isinstance(primary, Tensor):
        raise TypeError(f"{primary_name} must be a tensor")

    def fail(message, default):
        raise (error_type or default)(message)

    if not isinstance(vector, Tensor):
        fail(f"{name} must be a tensor", TypeError)
    if vector.shape != primary.shape:
        fail(f"{name} must have same shape as {primary_name}; got {tuple(vector.shape)} and "
             f"{tuple(primary.shape)}", ValueError)
    if vector.dtype != torch.float32:
        fail(f"{name} must have dtype torch.float32, got {vector.dtype}", TypeError)
    if vector.device != primary.device:
        fail(f"{name} must be on same device as {primary_name}; got {vector.device} and "
             f"{primary.device}", ValueError)
    if not vector.is_contiguous():
        fail(f"{name} must be contiguous", ValueError)
    return vector


class RawFamily:
    """The raw tier of one family."""

    def __init__(self, family: str):
        self.family = family
        self.vjp_fields, self._internal = _PARAMS[family]
        self.operator = _op.OPERATORS[family]

    def _field(self, wrt) -> str:
        if not isinstance(wrt, str):
            raise TypeError("wrt must be a string")
        if wrt not in self.vjp_fields:
            raise ValueError(f"invalid wrt field {wrt!r}; expected one of {self.vjp_fields!r}")
        return wrt

    def vjp_one(self, pair_scores, wrt, cotangent, params, lengths) -> Tensor:
        field = self._field(wrt)
        check_vector(pair_scores, cotangent, name="cotangent", primary_name="map", error_type=None)
        k = self.vjp_fields.index(field)
        with torch.no_grad():
            r = self.operator.vjp(pair_scores, *params, grad_map=cotangent, wrt=self._internal[k],
                                  lengths=lengths)
        p = params[k]
        if isinstance(p, Tensor):
            return r.reshape(p.shape).to(device=p.device, dtype=p.dtype)
        return r.reshape(1)

    def vjp(self, pair_scores, wrt, cotangent, params, lengths) -> dict:
        if not isinstance(wrt, tuple):
            raise TypeError("wrt must be a tuple of field names")
        if len(set(wrt)) != len(wrt):
            raise ValueError("wrt must not contain duplicates")
        fields = tuple(self._field(f) for f in wrt)
        check_vector(pair_scores, cotangent, name="cotangent", primary_name="map", error_type=None)
        return {f: self.vjp_one(pair_scores, f, cotangent, params, lengths) for f in fields}

    def public(self, which: str) -> Callable:
        """vjp_one / vjp with the reference's keyword signature."""
        impl = getattr(self, which)
        names = self.vjp_fields

        def fn(pair_scores, *, wrt, cotangent, lengths=None, **params):
            unknown = set(params) - set(names)
            if unknown:
                raise TypeError(f"{which}() got unexpected keyword arguments {sorted(unknown)}")
            vals = tuple(params.get(n, _DEFAULTS[n]) for n in names)
            return impl(pair_scores, wrt, cotangent, vals, lengths)

        kw = [Parameter("wrt", Parameter.KEYWORD_ONLY), Parameter("cotangent", Parameter.KEYWORD_ONLY)]
        kw += [Parameter(n, Parameter.KEYWORD_ONLY, default=_DEFAULTS[n]) for n in names]
        kw += [Parameter("lengths", Parameter.KEYWORD_ONLY, default=None)]
        fn.__signature__ = Signature([Parameter("pair_scores", Parameter.POSITIONAL_OR_KEYWORD), *kw])
        fn.__name__ = fn.__qualname__ = which
        fn.__doc__ = (f"{'One selected' if which == 'vjp_one' else 'Selected'} {self.family} parameter "
                      "VJP(s) of a map cotangent (no graph); the cotangent must be contiguous FP32 with "
                      "the map's shape and device.")
        return fn

    def bindings(self) -> dict:
        """The named kernel bindings: forward, forward_t, value_grad_params,
        marginals_backward, marginals_hvp and marginals_grad_<param>."""
        ops, f, n = torch.ops.orihime, self.family, len(self._internal)
        out = {}

        def split(args, lengths):
            """(params, lengths): lengths may also come positionally, after the parameters."""
            if len(args) == n + 1 and lengths is None:
                return args[:n], args[n]
            return args, lengths

        def plain(opname):
            op = getattr(ops, f"{f}_{opname}")

            def fn(scores, *args, lengths=None):
                params, lengths = split(args, lengths)
                return op(scores, *params, lengths)
            return fn

        for name in ("forward", "forward_t", "value_grad_params"):
            out[name] = plain(name)
        for p in self._internal:
            out[f"marginals_grad_{p}"] = plain(f"marginals_grad_{p}")
        mb, hv = getattr(ops, f"{f}_marginals_backward"), getattr(ops, f"{f}_marginals_hvp")

        def marginals_backward(scores, grad_marginals, *args, lengths=None):
            check_vector(scores, grad_marginals, name="cotangent", primary_name="scores")
            params, lengths = split(args, lengths)
            return mb(scores, grad_marginals, *params, lengths)

        def marginals_hvp(scores, v, *args, lengths=None):
            check_vector(scores, v, name="tangent", primary_name="scores")
            params, lengths = split(args, lengths)
            return hv(scores, v, *params, lengths)

        out["marginals_backward"] = marginals_backward
        out["marginals_hvp"] = marginals_hvp
        for name, fn in out.items():
            fn.__name__ = fn.__qualname__ = name
        return out


def module_globals(family: str) -> dict:
    """The public names of one family's raw module."""
    raw = RawFamily(family)
    g = {"vjp_fields": raw.vjp_fields, "vjp_one": raw.public("vjp_one"), "vjp": raw.public("vjp")}
    g.update(raw.bindings())
    g["__all__"] = ["vjp_fields", "vjp_one", "vjp", *raw.bindings()]
    return g
