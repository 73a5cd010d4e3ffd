"""Host-side mirror of orihime's Operator engine for the soft Smith-Waterman path.

Follows orihime/operator.py: input contract and error messages
(:1948-2074), FP32 numerical domain |score|/T <= 80 (:249-331), boolean or
-inf masks normalised to a finite exclusion sentinel (:334-386, :2178-2206),
autocast computing in FP32 (:2095-2101), and the three observables:

* ``map``     = dS/dscores (marginals); backward = Hessian-vector product
                plus parameter sensitivities (ops/sw_affine.py:149-198);
* ``value``   = S; backward = grad * map, dS/dtheta (:1324-1410);
* ``entropy`` = dS/dT (ops/sw_affine.py:144); backward = grad * dP/dT
                through the scores only (:1126-1190).

Every native call goes to ``torch.ops.orihime.*`` (CUDA implementations in
``_ops``); there is no CPU fallback in this package.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Optional, Sequence, Union

import torch
from torch import Tensor

Param = Union[float, int, Tensor]

MAX_ABS_SCORE_TEMPERATURE_RATIO = 80.0   # orihime/operator.py:27
MASK_SENTINEL_MAGNITUDE = 1.0e4          # orihime/operator.py:28
MASK_EXCLUSION_RATIO = 200.0             # orihime/operator.py:32


# ---------------------------------------------------------------------------
# validation
# ---------------------------------------------------------------------------

def _validate_scalar_parameter_shape(value: Param, name: str) -> None:
    if not isinstance(value, Tensor):
        return
    if value.ndim == 0 or (value.ndim == 1 and value.shape[0] == 1):
        return
    raise ValueError(f"{name} must be a scalar tensor with shape [] or [1], got shape {tuple(value.shape)}")


def _validate_temperature(value: Param) -> None:
    _validate_scalar_parameter_shape(value, "temperature")
    message = "temperature must be finite and strictly positive"
    if isinstance(value, Tensor):
        if not value.is_floating_point():
            raise TypeError("temperature tensor must have a floating-point dtype")
        if not bool((torch.isfinite(value) & (value > 0)).all()):
            raise RuntimeError(message)
        return
    try:
        scalar = float(value)
    except (TypeError, ValueError) as exc:
        raise TypeError("temperature must be a real number or tensor") from exc
    if not math.isfinite(scalar) or scalar <= 0:
        raise ValueError(f"{message}, got {scalar}")


def _as_float(value: Param) -> float:
    return float(value.detach().reshape(()).item()) if isinstance(value, Tensor) else float(value)


def _validate_domain(name: str, x: Tensor, params: Sequence[Param], param_names: Sequence[str]) -> None:
    limit = MAX_ABS_SCORE_TEMPERATURE_RATIO
    T = params[param_names.index("temp")]
    _validate_temperature(T)
    Tf = _as_float(T)
    message = ("orihime's supported FP32 numerical domain requires every finite "
               f"|score or cost| / temperature to be <= {limit:g}")
    if bool(torch.isposinf(x).any()):
        raise RuntimeError(f"{name} contains an unsupported infinity; use -inf score masks")
    ok = ~torch.isnan(x) & (torch.isneginf(x) | (x == -MASK_SENTINEL_MAGNITUDE) | (x.abs() <= limit * Tf))
    if not bool(ok.all()):
        raise RuntimeError(f"{message}; {name} is out of domain")
    for pname, value in zip(param_names, params):
        if pname == "temp":
            continue
        _validate_scalar_parameter_shape(value, pname)
        v = _as_float(value)
        if isinstance(value, Tensor):
            if not value.is_floating_point():
                raise TypeError(f"{pname} tensor must have a floating-point dtype")
            if not (math.isfinite(v) and abs(v) <= limit * Tf):
                raise RuntimeError(f"{message}; {pname} is out of domain")
        else:
            if not math.isfinite(v):
                raise ValueError(f"{message}; {pname} must be finite")
            if abs(v) > limit * Tf:
                raise ValueError(f"{message}; {pname} is out of domain")


def _validate_and_normalize(name: str, x: Tensor, params: Sequence[Param],
                            param_names: Sequence[str]) -> Tensor:
    """_validate_domain then normalize_mask, with the full-tensor questions of
    both answered by one fused device pass (swb_scan_scores) for fp32 CUDA
    inputs: the same checks in the same order with the same messages, the
    same sentinel values, one host synchronisation instead of three or four."""
    if not (x.is_cuda and x.dtype == torch.float32 and x.numel() > 0):
        _validate_domain(name, x, params, param_names)
        return normalize_mask(x, _as_float(params[param_names.index("temp")]))
    from . import _ops as ops_mod

    limit = MAX_ABS_SCORE_TEMPERATURE_RATIO
    T = params[param_names.index("temp")]
    _validate_temperature(T)
    Tf = _as_float(T)
    message = ("orihime's supported FP32 numerical domain requires every finite "
               f"|score or cost| / temperature to be <= {limit:g}")
    flags, amax = ops_mod.scan_scores(x.detach().contiguous(), limit * Tf, MASK_SENTINEL_MAGNITUDE)
    if flags & ops_mod.SCAN_POSINF:
        raise RuntimeError(f"{name} contains an unsupported infinity; use -inf score masks")
    if flags & ops_mod.SCAN_DOMAIN:
        raise RuntimeError(f"{message}; {name} is out of domain")
    for pname, value in zip(param_names, params):
        if pname == "temp":
            continue
        _validate_scalar_parameter_shape(value, pname)
        v = _as_float(value)
        if isinstance(value, Tensor):
            if not value.is_floating_point():
                raise TypeError(f"{pname} tensor must have a floating-point dtype")
            if not (math.isfinite(v) and abs(v) <= limit * Tf):
                raise RuntimeError(f"{message}; {pname} is out of domain")
        else:
            if not math.isfinite(v):
                raise ValueError(f"{message}; {pname} must be finite")
            if abs(v) > limit * Tf:
                raise ValueError(f"{message}; {pname} is out of domain")
    if not flags & ops_mod.SCAN_NEGINF:
        return x
    path_len = float(sum(x.shape[1:]))
    offset = (path_len * MAX_ABS_SCORE_TEMPERATURE_RATIO + MASK_EXCLUSION_RATIO) * Tf
    retained = amax.view(-1, *([1] * (x.ndim - 1)))
    retained = torch.where(torch.isfinite(retained), retained, retained.new_zeros(()))
    sentinel = (retained - offset).to(dtype=x.dtype)
    return torch.where(torch.isneginf(x), sentinel, x)


def normalize_mask(x: Tensor, temp: float) -> Tensor:
    """-inf cells -> amax - (sum(shape[1:]) * 80 + 200) * T, per batch item
    (orihime/operator.py:334-386).  The sentinel carries no gradient."""
    neg = torch.isneginf(x)
    if not bool(neg.any()):
        return x
    dims = tuple(range(1, x.ndim))
    path_len = float(sum(x.shape[1:]))
    offset = (path_len * MAX_ABS_SCORE_TEMPERATURE_RATIO + MASK_EXCLUSION_RATIO) * temp
    retained = x.detach().amax(dim=dims, keepdim=True)
    retained = torch.where(torch.isfinite(retained), retained, retained.new_zeros(()))
    sentinel = (retained - offset).to(dtype=x.dtype)
    return torch.where(neg, sentinel, x)


# ---------------------------------------------------------------------------
# family adapters (orihime/ops/sw.py, orihime/ops/sw_affine.py)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class Family:
    name: str
    params: tuple[str, ...]
    forward: Callable            # (scores, *floats, lengths) -> [value, map]
    grads: Callable              # (scores, *floats, lengths) -> per-param dS/dtheta [B] each
    hvp: Callable                # (scores, v, *floats, lengths) -> [B, L1, L2]
    sens: tuple[Callable, ...]   # per param: (scores, *floats, lengths) -> dP/dtheta
    value: Callable = None       # (scores, *floats, lengths) -> [B], forward wavefront only
    full: Callable = None        # (scores, *floats, lengths) -> (value, map, *dS/dtheta), one call


def _ops():
    return torch.ops.orihime


SW = Family(
    "sw", ("gap", "temp"),
    forward=lambda *a: _ops().sw_forward(*a),
    grads=lambda *a: _ops().sw_value_grad_params(*a),
    hvp=lambda *a: _ops().sw_marginals_hvp(*a),
    sens=(lambda *a: _ops().sw_marginals_grad_gap(*a),
          lambda *a: _ops().sw_marginals_grad_temp(*a)),
    value=lambda *a: torch.ops.orihime_b200.sw_value(*a),
    full=lambda *a: torch.ops.orihime_b200.sw_forward_with_grads(*a),
)

SW_AFFINE = Family(
    "sw_affine", ("gap_open", "gap_ext", "temp"),
    forward=lambda *a: _ops().sw_affine_forward(*a),
    grads=lambda *a: _ops().sw_affine_value_grad_params(*a),
    hvp=lambda *a: _ops().sw_affine_marginals_hvp(*a),
    sens=(lambda *a: _ops().sw_affine_marginals_grad_gap_open(*a),
          lambda *a: _ops().sw_affine_marginals_grad_gap_ext(*a),
          lambda *a: _ops().sw_affine_marginals_grad_temp(*a)),
    value=lambda *a: torch.ops.orihime_b200.sw_affine_value(*a),
    full=lambda *a: torch.ops.orihime_b200.sw_affine_forward_with_grads(*a),
)

NW = Family(
    "nw", ("gap", "temp"),
    forward=lambda *a: _ops().nw_forward(*a),
    grads=lambda *a: _ops().nw_value_grad_params(*a),
    hvp=lambda *a: _ops().nw_marginals_hvp(*a),
    sens=(lambda *a: _ops().nw_marginals_grad_gap(*a),
          lambda *a: _ops().nw_marginals_grad_temp(*a)),
    value=lambda *a: torch.ops.orihime_b200.nw_value(*a),
    full=lambda *a: torch.ops.orihime_b200.nw_forward_with_grads(*a),
)

NW_AFFINE = Family(
    "nw_affine", ("gap_open", "gap_ext", "temp"),
    forward=lambda *a: _ops().nw_affine_forward(*a),
    # (value, dS/dgo, dS/dge, dS/dT): src/nw_affine/torch_cuda.cpp:688-702
    grads=lambda *a: _ops().nw_affine_value_grad_params(*a)[1:],
    hvp=lambda *a: _ops().nw_affine_marginals_hvp(*a),
    sens=(lambda *a: _ops().nw_affine_marginals_grad_gap_open(*a),
          lambda *a: _ops().nw_affine_marginals_grad_gap_ext(*a),
          lambda *a: _ops().nw_affine_marginals_grad_temp(*a)),
    value=lambda *a: torch.ops.orihime_b200.nw_affine_value(*a),
    full=lambda *a: torch.ops.orihime_b200.nw_affine_forward_with_grads(*a),
)

SV_LINEAR = Family(
    "sv_linear", ("gap", "temp"),
    forward=lambda *a: _ops().sv_linear_forward(*a),
    grads=lambda *a: _ops().sv_linear_value_grad_params(*a),
    hvp=lambda *a: _ops().sv_linear_marginals_hvp(*a),
    sens=(lambda *a: _ops().sv_linear_marginals_grad_gap(*a),
          lambda *a: _ops().sv_linear_marginals_grad_temp(*a)),
    value=lambda *a: torch.ops.orihime_b200.sv_linear_value(*a),
    full=lambda *a: torch.ops.orihime_b200.sv_linear_forward_with_grads(*a),
)

SV_AFFINE = Family(
    "sv_affine", ("gap_open", "gap_ext", "temp"),
    forward=lambda *a: _ops().sv_affine_forward(*a),
    grads=lambda *a: _ops().sv_affine_value_grad_params(*a),
    hvp=lambda *a: _ops().sv_affine_marginals_hvp(*a),
    sens=(lambda *a: _ops().sv_affine_marginals_grad_gap_open(*a),
          lambda *a: _ops().sv_affine_marginals_grad_gap_ext(*a),
          lambda *a: _ops().sv_affine_marginals_grad_temp(*a)),
    value=lambda *a: torch.ops.orihime_b200.sv_affine_value(*a),
    full=lambda *a: torch.ops.orihime_b200.sv_affine_forward_with_grads(*a),
)


# ---------------------------------------------------------------------------
# autograd functions
# ---------------------------------------------------------------------------

def _param_grad(total: Tensor, like: Param) -> Optional[Tensor]:
    if isinstance(like, Tensor) and like.requires_grad:
        return total.reshape(like.shape).to(device=like.device, dtype=like.dtype)
    return None


class _ValueFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fam, lengths, scores, *params):
        vals = [_as_float(p) for p in params]
        needs_params = any(isinstance(p, Tensor) and p.requires_grad for p in params)
        if needs_params:
            # one forward + adjoint gives the value, the map and dS/dtheta
            value, smap, *grads = fam.full(scores, *vals, lengths)
        else:
            value, smap = fam.forward(scores, *vals, lengths)
            grads = None
        ctx.fam, ctx.params = fam, params
        ctx.save_for_backward(smap)
        ctx.param_grads = grads
        return value

    @staticmethod
    def backward(ctx, gv):
        (smap,) = ctx.saved_tensors
        gs = gv.view(-1, 1, 1) * smap if ctx.needs_input_grad[2] else None
        out = [None, None, gs]
        for k, p in enumerate(ctx.params):
            g = None
            if ctx.param_grads is not None and isinstance(p, Tensor) and p.requires_grad:
                g = _param_grad((gv * ctx.param_grads[k]).sum(), p)
            out.append(g)
        return tuple(out)


# Checkpoint stride of the checkpointed value op: the forward keeps the DP
# state of every CHECKPOINT_EVERY-th chunk of 4 wavefront steps (about 5 / k
# bytes per computed cell at k = CHECKPOINT_EVERY), and the adjoint recomputes
# the chunks in between.  4 keeps ~1.3 B/cell, a third of the map's 4 B/cell.
CHECKPOINT_EVERY = 4


class _CheckpointedValueFn(torch.autograd.Function):
    """value with a deferred adjoint (local families, gaps <= 0): forward
    runs only the forward wavefront and keeps its sparse checkpoints in a
    workspace; backward runs the checkpointed adjoint on them and scales the
    map and dS/dtheta by the value's cotangent.  Nothing of size [B, L1, L2]
    is kept between the two."""

    @staticmethod
    def forward(ctx, fam, lengths, ws_value, scores, *params):
        value, ws = ws_value
        ctx.fam, ctx.params, ctx.lengths, ctx.ws = fam, params, lengths, ws
        ctx.vals = [_as_float(p) for p in params]
        ctx.save_for_backward(scores)
        return value

    @staticmethod
    def backward(ctx, gv):
        from . import _ops as ops_mod

        (scores,) = ctx.saved_tensors
        _, smap, *grads = ops_mod.run_adjoint(ctx.fam.name, scores, ctx.lengths, ctx.vals,
                                              CHECKPOINT_EVERY, ctx.ws)
        gs = gv.view(-1, 1, 1) * smap if ctx.needs_input_grad[3] else None
        out = [None, None, None, gs]
        for k, p in enumerate(ctx.params):
            g = None
            if isinstance(p, Tensor) and p.requires_grad:
                g = _param_grad((gv * grads[k]).sum(), p)
            out.append(g)
        return tuple(out)


def _checkpointed_value(fam, lengths, scores, params):
    """The checkpointed value op, or None where it does not apply (another
    family, a positive gap, under stream capture)."""
    if fam.name not in ("sw", "sw_affine") or torch.cuda.is_current_stream_capturing():
        return None
    from . import _ops as ops_mod

    vals = [_as_float(p) for p in params]
    got = ops_mod.run_checkpoint(fam.name, scores.detach(), lengths, vals, CHECKPOINT_EVERY)
    if got is None:
        return None
    return _CheckpointedValueFn.apply(fam, lengths, got, scores, *params)


class _MapFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fam, lengths, scores, *params):
        vals = [_as_float(p) for p in params]
        _, smap = fam.forward(scores, *vals, lengths)
        ctx.fam, ctx.params, ctx.vals, ctx.lengths = fam, params, vals, lengths
        ctx.save_for_backward(scores)
        return smap

    @staticmethod
    def backward(ctx, gm):
        (scores,) = ctx.saved_tensors
        gm = gm.contiguous()
        gs = ctx.fam.hvp(scores, gm, *ctx.vals, ctx.lengths) if ctx.needs_input_grad[2] else None
        out = [None, None, gs]
        for k, p in enumerate(ctx.params):
            g = None
            if isinstance(p, Tensor) and p.requires_grad:
                field = ctx.fam.sens[k](scores, *ctx.vals, ctx.lengths)
                g = _param_grad((gm * field).sum(), p)
            out.append(g)
        return tuple(out)


class _EntropyFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fam, lengths, scores, *params):
        vals = [_as_float(p) for p in params]
        grads = fam.grads(scores, *vals, lengths)
        ctx.fam, ctx.vals, ctx.lengths, ctx.nparams = fam, vals, lengths, len(params)
        ctx.save_for_backward(scores)
        return grads[-1]

    @staticmethod
    def backward(ctx, ge):
        (scores,) = ctx.saved_tensors
        gs = None
        if ctx.needs_input_grad[2]:
            field = ctx.fam.sens[-1](scores, *ctx.vals, ctx.lengths)
            gs = ge.view(-1, 1, 1) * field
        return (None, None, gs) + (None,) * ctx.nparams


# ---------------------------------------------------------------------------
# the operator
# ---------------------------------------------------------------------------

class Operator:
    """One soft alignment family (Smith-Waterman or Needleman-Wunsch) with map /
    value / entropy observables."""

    def __init__(self, fam: Family, primary_name: str = "pair_scores"):
        self.fam = fam
        self.name = fam.name
        self.params = fam.params
        self.primary_name = primary_name

    # -- input contract (orihime/operator.py:1948-2074, :2178-2206) --
    def _prepare(self, primary, params, lengths, mask, dtype):
        name = self.primary_name
        if not isinstance(primary, Tensor):
            raise TypeError(f"{name} must be a tensor")
        if mask is not None:
            if not isinstance(mask, Tensor) or mask.dtype != torch.bool:
                got = mask.dtype if isinstance(mask, Tensor) else type(mask).__name__
                raise TypeError(f"mask must be a boolean tensor flagging excluded cells; got {got}")
            if tuple(mask.shape) != tuple(primary.shape):
                raise ValueError(f"mask shape {tuple(mask.shape)} must match {name} shape {tuple(primary.shape)}")
            if mask.device != primary.device:
                raise ValueError(f"mask must be on the same device as {name}, got {mask.device} and {primary.device}")
            primary = primary.masked_fill(mask, float("-inf"))
        if len(params) != len(self.params):
            raise TypeError(f"{self.name} expects parameters {self.params}")
        if dtype is not None and dtype != torch.float32:
            raise TypeError(f"dtype must be torch.float32 or None, got {dtype}")
        if dtype is None and torch.is_autocast_enabled(primary.device.type):
            dtype = torch.float32
        if dtype is not None and primary.dtype != dtype:
            primary = primary.to(dtype)
            params = tuple(p.to(dtype) if isinstance(p, Tensor) and p.is_floating_point() else p
                           for p in params)
        if primary.ndim != 3:
            raise ValueError(f"{name} must have shape [B, L1, L2], got {tuple(primary.shape)}")
        if primary.shape[0] == 0:
            raise ValueError(f"{self.name} does not support an empty leading batch (B=0)")
        if not primary.is_floating_point():
            raise TypeError(f"{name} must have a floating-point dtype")
        if primary.dtype != torch.float32:
            raise TypeError(f"{name} must have dtype torch.float32 outside autocast; got {primary.dtype}")
        for pname, p in zip(self.params, params):
            _validate_scalar_parameter_shape(p, pname)
            if isinstance(p, Tensor):
                if not p.is_floating_point():
                    raise TypeError(f"{pname} tensor must have a floating-point dtype")
                if p.device != primary.device:
                    raise ValueError(f"{pname} tensor must be on the same device as {name}, got {p.device} and {primary.device}")
                if p.dtype != torch.float32:
                    raise TypeError(f"{pname} tensor must have dtype torch.float32 outside autocast; got {p.dtype}")
        if lengths is not None:
            if not isinstance(lengths, Tensor):
                raise TypeError("lengths must be a tensor or None")
            if tuple(lengths.shape) != (primary.shape[0], 2):
                raise ValueError(f"lengths must have shape [B, 2], got {tuple(lengths.shape)}")
            if lengths.dtype != torch.int32:
                raise TypeError(f"lengths must have dtype torch.int32, got {lengths.dtype}")
            if lengths.device != primary.device:
                raise ValueError("lengths must be on the same device as the primary input, got "
                                 f"{lengths.device} and {primary.device}")
            if not lengths.is_contiguous():
                raise ValueError("lengths must be contiguous")
            lim = torch.tensor(primary.shape[1:], device=lengths.device, dtype=torch.int32)
            if not bool(((lengths >= 0) & (lengths <= lim)).all()):
                raise RuntimeError("lengths entries must lie within the padded input shape")
        primary = _validate_and_normalize(name, primary, params, self.params)
        if not primary.is_contiguous():
            primary = primary.contiguous()
        if lengths is None:
            B, L1, L2 = primary.shape
            lengths = torch.tensor([[L1, L2]] * B, dtype=torch.int32, device=primary.device)
        return primary, params, lengths

    def __call__(self, primary, *params, lengths=None, mask=None, dtype=None) -> Tensor:
        x, params, lengths = self._prepare(primary, params, lengths, mask, dtype)
        return _MapFn.apply(self.fam, lengths, x, *params)

    def value(self, primary, *params, lengths=None, mask=None, dtype=None) -> Tensor:
        x, params, lengths = self._prepare(primary, params, lengths, mask, dtype)
        needs_grad = torch.is_grad_enabled() and (
            x.requires_grad or any(isinstance(p, Tensor) and p.requires_grad for p in params))
        if not needs_grad:
            # no gradient can flow: the forward wavefront alone (same values,
            # no marginal map, about half the work)
            return self.fam.value(x, *[_as_float(p) for p in params], lengths)
        v = _checkpointed_value(self.fam, lengths, x, params)
        if v is not None:
            return v
        return _ValueFn.apply(self.fam, lengths, x, *params)

    def entropy(self, primary, *params, lengths=None, mask=None, dtype=None) -> Tensor:
        x, params, lengths = self._prepare(primary, params, lengths, mask, dtype)
        return _EntropyFn.apply(self.fam, lengths, x, *params)

    # -- named ops tier (orihime/operator.py:2312-2400) --
    def vjp(self, primary, *params, grad_map, wrt, lengths=None, mask=None, dtype=None) -> Tensor:
        x, params, lengths = self._prepare(primary, params, lengths, mask, dtype)
        vals = [_as_float(p) for p in params]
        if wrt == self.primary_name:
            return self.fam.hvp(x, grad_map.contiguous(), *vals, lengths)
        k = self.params.index(wrt)
        return (grad_map * self.fam.sens[k](x, *vals, lengths)).sum()

    def sensitivity(self, primary, *params, wrt, lengths=None, mask=None, dtype=None) -> Tensor:
        x, params, lengths = self._prepare(primary, params, lengths, mask, dtype)
        vals = [_as_float(p) for p in params]
        return self.fam.sens[self.params.index(wrt)](x, *vals, lengths)
