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
from torch.autograd.function import once_differentiable

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

def _param_grad(total: Tensor, meta, needed: bool) -> Optional[Tensor]:
    """dS/dtheta summed over the batch, shaped like the parameter tensor
    (meta = its shape, dtype, device), or None for a float parameter."""
    if needed and meta is not None:
        shape, dtype, device = meta
        return total.reshape(shape).to(device=device, dtype=dtype)
    return None


def _param_meta(params):
    return [(p.shape, p.dtype, p.device) if isinstance(p, Tensor) else None for p in params]


# ---------------------------------------------------------------------------
# autograd Functions (eager autograd and torch.func: vjp, jvp, jacrev, vmap)
# ---------------------------------------------------------------------------
# Each observable is one torch.autograd.Function in the setup_context form,
# which torch.func can transform (the reference registers its observables the
# same way, orihime/operator.py:1288-1570):
# * vjp / jacrev: backward is written with torch ops and the native ops,
#   whose vmap rules fold a mapped cotangent into the native batch;
# * jvp: a forward-mode rule per observable -- value: <map, ds> + sum_k
#   dS/dtheta_k dtheta_k; map: HVP(ds) + sum_k dP/dtheta_k dtheta_k;
#   entropy: <dP/dT, ds> (its parameter directions are not available, as in
#   the reference);
# * vmap: the mapped dimension is folded into the native batch and the
#   Function runs once over vmap_size * B pairs; a mapped scalar parameter is
#   an error, with the native ops' message.
# Eager calls run the value-dependent part of the input contract (lengths
# range, temperature, numerical domain, -inf masks) before the Function, so
# the mask normalisation is ordinary autograd.  Under a transform the inputs
# may be wrapped tensors that cannot be inspected, so forward runs it on the
# plain tensors and its -inf cells get zero derivatives (their sentinel is a
# constant).  forward returns the normalised scores and the -inf mask as
# extra, non-differentiable outputs: setup_context may save only inputs and
# outputs.

_PUBLIC_PARAM = {"gap": "gap_score", "gap_open": "gap_open_score", "gap_ext": "gap_extend_score",
                 "temp": "temperature"}


def _interpreters() -> tuple:
    return tuple(torch._C._functorch.get_interpreter_stack() or ())


def _transforms_active() -> bool:
    return bool(_interpreters())


def _vmap_active() -> bool:
    vm = torch._C._functorch.TransformType.Vmap
    return any(i.key() == vm for i in _interpreters())


def _strip(t):
    """t without its grad-tracking wrappers: the native ops read storage,
    which those wrappers do not expose.  Batching wrappers stay; the native
    ops' vmap rules fold them."""
    if isinstance(t, Tensor):
        f = torch._C._functorch
        while f.is_gradtrackingtensor(t):
            t = f.get_unwrapped(t)
    return t


def _no_forward_mode_under_vmap(op, observable: str) -> None:
    if _vmap_active():
        raise NotImplementedError(
            f"{op.name}{observable} has no batched forward-mode rule: its jvp function runs once per "
            "call and cannot take mapped tangents (torch.func.jacfwd, or vmap over jvp); use "
            "torch.func.jacrev or vmap over vjp")


def _entropy_direction_error(op, pname: str) -> NotImplementedError:
    return NotImplementedError(
        f"{op.name}_entropy is differentiable only w.r.t. its primary {op.primary_name} input in "
        f"this release; the entropy gradient w.r.t. parameter {_PUBLIC_PARAM.get(pname, pname)} "
        "(a second derivative involving temperature) is not available -- see "
        "DERIVATIVE_COVERAGE.md. Detach the parameter or use finite differences.")


def _checked(op, x: Tensor, params, lengths):
    """The value-dependent part of the input contract on plain tensors:
    lengths within the padded shape, the temperature, the FP32 numerical
    domain and -inf masks.  Returns (normalised scores, the -inf cells or
    None)."""
    if lengths is not None:
        lim = torch.tensor(x.shape[1:], device=lengths.device, dtype=torch.int32)
        if not bool(((lengths >= 0) & (lengths <= lim)).all()):
            raise RuntimeError("lengths entries must lie within the padded input shape")
    xn = _validate_and_normalize(op.primary_name, x, params, op.params)
    neg = torch.isneginf(x) if xn is not x else None
    return (xn if xn.is_contiguous() else xn.contiguous()), neg


def _fold_vmap(fn, info, in_dims, op, validate, lengths, scores, params):
    """vmap rule shared by the observables: fold the mapped dimension of the
    scores (and lengths) into the native batch, run fn once, unfold."""
    for pname, d in zip(op.params, in_dims[4:]):
        if d is not None:
            raise RuntimeError(f"orihime::{op.name}_forward_t does not support mapping scalar argument "
                               f"{pname!r}; keep scalar parameters unbatched")
    V = info.batch_size
    ld, sd = in_dims[2], in_dims[3]
    s = scores.movedim(sd, 0) if sd is not None else scores.unsqueeze(0).expand(V, *scores.shape)
    B = s.shape[1]
    s = s.reshape(V * B, *s.shape[2:]).contiguous()
    if lengths is not None:
        ln = lengths.movedim(ld, 0) if ld is not None else lengths.unsqueeze(0).expand(V, *lengths.shape)
        lengths = ln.reshape(V * B, 2).contiguous()
    out = fn.apply(op, validate, lengths, s, *params)
    out = tuple(o.reshape(V, B, *o.shape[1:]) for o in out)
    return out, tuple(0 for _ in out)


def _saved(ctx):
    """(scores, lengths, -inf mask or None) saved by setup_context."""
    saved = ctx.saved_tensors
    scores = saved[0]
    lengths = saved[1] if ctx.has_lengths else None
    neg = saved[-1] if ctx.has_neg else None
    return scores, lengths, neg


def _save_inputs(ctx, inputs, output, nlead: int):
    """Save the scores the native ops need (the input, or the normalised
    copy forward returned), the lengths and the -inf mask, for backward and
    for jvp; output[:nlead] are the observable's own outputs."""
    op, validate, lengths, scores, *params = inputs
    extra = output[nlead:]
    if validate:
        scores = extra[0]
    neg = extra[1] if validate and len(extra) > 1 else None
    ctx.op, ctx.validate = op, validate
    ctx.vals = [_as_float(p) for p in params]
    ctx.pmeta = _param_meta(params)
    ctx.has_lengths, ctx.has_neg = lengths is not None, neg is not None
    tensors = (scores,) + ((lengths,) if lengths is not None else ()) + ((neg,) if neg is not None else ())
    return tensors, extra


class _ValueFn(torch.autograd.Function):
    """value S [B]; backward: cotangent x map, and cotangent . dS/dtheta."""

    @staticmethod
    def forward(op, validate, lengths, scores, *params):
        neg = None
        if validate:
            scores, neg = _checked(op, scores, params, lengths)
        vals = [_as_float(p) for p in params]
        value, smap, *grads = op.fam.full(scores, *vals, lengths)
        if neg is not None:
            smap = smap.masked_fill(neg, 0.0)
        return (value, smap, *grads)

    @staticmethod
    def setup_context(ctx, inputs, output):
        value, smap, *grads = output
        ctx.mark_non_differentiable(smap, *grads)
        ctx.save_for_backward(smap, *grads)
        ctx.save_for_forward(smap, *grads)
        ctx.pmeta = _param_meta(inputs[4:])
        ctx.op = inputs[0]

    @staticmethod
    @once_differentiable
    def backward(ctx, gv, *_):
        smap, *grads = ctx.saved_tensors
        gs = gv.reshape(-1, 1, 1) * smap if ctx.needs_input_grad[3] else None
        out = [None, None, None, gs]
        for k, meta in enumerate(ctx.pmeta):
            out.append(_param_grad((gv * grads[k]).sum(), meta, ctx.needs_input_grad[4 + k]))
        return tuple(out)

    @staticmethod
    def jvp(ctx, _op, _validate, _lengths, t_scores, *t_params):
        _no_forward_mode_under_vmap(ctx.op, "_value")
        smap, *grads = ctx.saved_tensors
        t = None
        if t_scores is not None:
            t = (smap * t_scores).sum(dim=(1, 2))
        for g, tp in zip(grads, t_params):
            if tp is not None:
                d = g * tp.reshape(())
                t = d if t is None else t + d
        if t is None:
            t = torch.zeros_like(grads[0])
        return (t, None, *(None for _ in grads))

    @staticmethod
    def vmap(info, in_dims, op, validate, lengths, scores, *params):
        return _fold_vmap(_ValueFn, info, in_dims, op, validate, lengths, scores, params)


# Checkpoint stride of the checkpointed value op: the forward keeps the DP
# state of every CHECKPOINT_EVERY-th chunk of 4 wavefront steps (about 3.7 / k
# bytes per computed cell at k = CHECKPOINT_EVERY), and the adjoint recomputes
# the chunks in between.  4 keeps ~0.93 B/cell, under a quarter of the map's
# 4 B/cell.
CHECKPOINT_EVERY = 4


class _CheckpointedValueFn(torch.autograd.Function):
    """value with a deferred adjoint (local families, gaps <= 0, eager calls):
    forward runs only the forward wavefront and keeps its sparse checkpoints
    in a workspace; backward runs the checkpointed adjoint on them and scales
    the map and dS/dtheta by the value's cotangent.  Nothing of size
    [B, L1, L2] is kept between the two."""

    @staticmethod
    def forward(ctx, fam, lengths, ws_value, scores, *params):
        value, ws = ws_value
        ctx.fam, ctx.lengths, ctx.ws = fam, lengths, ws
        ctx.vals = [_as_float(p) for p in params]
        ctx.pmeta = _param_meta(params)
        ctx.save_for_backward(scores)
        return value

    @staticmethod
    @once_differentiable
    def backward(ctx, gv):
        from . import _ops as ops_mod

        (scores,) = ctx.saved_tensors
        _, smap, *grads = ops_mod.run_adjoint(ctx.fam.name, scores, ctx.lengths, ctx.vals,
                                              CHECKPOINT_EVERY, ctx.ws)
        gs = gv.view(-1, 1, 1) * smap if ctx.needs_input_grad[3] else None
        out = [None, None, None, gs]
        for k, meta in enumerate(ctx.pmeta):
            out.append(_param_grad((gv * grads[k]).sum(), meta, ctx.needs_input_grad[4 + k]))
        return tuple(out)


def _checkpointed_value(fam, lengths, scores, params):
    """The checkpointed value op, or None where it does not apply (another
    family, a positive gap, a tensor off CUDA, under stream capture)."""
    if (fam.name not in ("sw", "sw_affine") or not scores.is_cuda
            or torch.cuda.is_current_stream_capturing()):
        return None
    from . import _ops as ops_mod

    vals = [_as_float(p) for p in params]
    got = ops_mod.run_checkpoint(fam.name, scores.detach(), lengths, vals, CHECKPOINT_EVERY)
    if got is None:
        return None
    return _CheckpointedValueFn.apply(fam, lengths, got, scores, *params)


class _MapFn(torch.autograd.Function):
    """map dS/dscores; backward: HVP of the cotangent and cotangent . dP/dtheta."""

    @staticmethod
    def forward(op, validate, lengths, scores, *params):
        neg = None
        if validate:
            scores, neg = _checked(op, scores, params, lengths)
        vals = [_as_float(p) for p in params]
        _, smap = op.fam.forward(scores, *vals, lengths)
        if neg is not None:
            smap = smap.masked_fill(neg, 0.0)
        # the normalised scores may be the input itself: return a view of it
        extra = (scores.view_as(scores),) if validate else ()
        if neg is not None:
            extra += (neg,)
        return (smap, *extra)

    @staticmethod
    def setup_context(ctx, inputs, output):
        tensors, extra = _save_inputs(ctx, inputs, output, 1)
        if extra:
            ctx.mark_non_differentiable(*extra)
        ctx.save_for_backward(*tensors)
        ctx.save_for_forward(*tensors)

    @staticmethod
    @once_differentiable
    def backward(ctx, gm, *_):
        scores, lengths, neg = _saved(ctx)
        fam, vals = ctx.op.fam, ctx.vals
        sc = _strip(scores)
        g = _strip(gm)
        if neg is not None:
            g = g.masked_fill(neg, 0.0)
        g = g.contiguous()
        gs = None
        if ctx.needs_input_grad[3]:
            gs = fam.hvp(sc, g, *vals, lengths)
            if neg is not None:
                gs = gs.masked_fill(neg, 0.0)
        out = [None, None, None, gs]
        for k, meta in enumerate(ctx.pmeta):
            need = ctx.needs_input_grad[4 + k]
            total = (g * fam.sens[k](sc, *vals, lengths)).sum() if need else None
            out.append(_param_grad(total, meta, need))
        return tuple(out)

    @staticmethod
    def jvp(ctx, _op, _validate, _lengths, t_scores, *t_params):
        _no_forward_mode_under_vmap(ctx.op, "")
        scores, lengths, neg = _saved(ctx)
        fam, vals = ctx.op.fam, ctx.vals
        sc = _strip(scores)
        t = None
        if t_scores is not None:
            d = _strip(t_scores)
            if neg is not None:
                d = d.masked_fill(neg, 0.0)
            t = fam.hvp(sc, d.contiguous(), *vals, lengths)
        for k, tp in enumerate(t_params):
            if tp is not None:
                d = fam.sens[k](sc, *vals, lengths) * _strip(tp).reshape(())
                t = d if t is None else t + d
        if t is None:
            t = torch.zeros_like(sc)
        elif neg is not None:
            t = t.masked_fill(neg, 0.0)
        return (t,) + (None,) * (1 + ctx.has_neg if ctx.validate else 0)

    @staticmethod
    def vmap(info, in_dims, op, validate, lengths, scores, *params):
        return _fold_vmap(_MapFn, info, in_dims, op, validate, lengths, scores, params)


class _EntropyFn(torch.autograd.Function):
    """entropy dS/dT [B]; backward: cotangent x dP/dT through the scores only
    (a parameter direction raises, as in the reference)."""

    @staticmethod
    def forward(op, validate, lengths, scores, *params):
        neg = None
        if validate:
            scores, neg = _checked(op, scores, params, lengths)
        vals = [_as_float(p) for p in params]
        ent = op.fam.grads(scores, *vals, lengths)[-1]
        extra = (scores.view_as(scores),) if validate else ()
        if neg is not None:
            extra += (neg,)
        return (ent, *extra)

    @staticmethod
    def setup_context(ctx, inputs, output):
        tensors, extra = _save_inputs(ctx, inputs, output, 1)
        if extra:
            ctx.mark_non_differentiable(*extra)
        ctx.save_for_backward(*tensors)
        ctx.save_for_forward(*tensors)

    @staticmethod
    @once_differentiable
    def backward(ctx, ge, *_):
        for k, pname in enumerate(ctx.op.params):
            if ctx.needs_input_grad[4 + k] and ctx.pmeta[k] is not None:
                raise _entropy_direction_error(ctx.op, pname)
        scores, lengths, neg = _saved(ctx)
        gs = None
        if ctx.needs_input_grad[3]:
            field = ctx.op.fam.sens[-1](_strip(scores), *ctx.vals, lengths)
            gs = _strip(ge).reshape(-1, 1, 1) * field
            if neg is not None:
                gs = gs.masked_fill(neg, 0.0)
        return (None, None, None, gs) + (None,) * len(ctx.pmeta)

    @staticmethod
    def jvp(ctx, _op, _validate, _lengths, t_scores, *t_params):
        for pname, tp in zip(ctx.op.params, t_params):
            if tp is not None:
                raise _entropy_direction_error(ctx.op, pname)
        _no_forward_mode_under_vmap(ctx.op, "_entropy")
        scores, lengths, neg = _saved(ctx)
        sc = _strip(scores)
        if t_scores is None:
            t = sc.new_zeros(sc.shape[0])
        else:
            d = _strip(t_scores)
            if neg is not None:
                d = d.masked_fill(neg, 0.0)
            t = (ctx.op.fam.sens[-1](sc, *ctx.vals, lengths) * d).sum(dim=(1, 2))
        return (t,) + (None,) * (1 + ctx.has_neg if ctx.validate else 0)

    @staticmethod
    def vmap(info, in_dims, op, validate, lengths, scores, *params):
        return _fold_vmap(_EntropyFn, info, in_dims, op, validate, lengths, scores, params)


# ---------------------------------------------------------------------------
# the operator
# ---------------------------------------------------------------------------

# Operator of each family by name (the compile path's ops look them up).
OPERATORS: dict = {}


class Operator:
    """One soft alignment family (Smith-Waterman, Needleman-Wunsch or
    Saigo-Vert) with map / value / entropy observables."""

    def __init__(self, fam: Family, primary_name: str = "pair_scores"):
        self.fam = fam
        self.name = fam.name
        self.params = fam.params
        self.primary_name = primary_name
        OPERATORS[fam.name] = self

    # -- input contract (orihime/operator.py:1948-2074, :2178-2206) --
    def _prepare_shapes(self, primary, params, lengths, mask, dtype):
        """The checks that read no tensor values (types, shapes, dtypes,
        devices) and the mask and dtype conversions: safe on tensors that a
        torch.func transform wraps."""
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
        return primary, params, lengths

    def _prepare(self, primary, params, lengths, mask, dtype):
        """The whole input contract.  lengths stays None when the caller gave
        none: the ops take that as full lengths, with no host round trip."""
        primary, params, lengths = self._prepare_shapes(primary, params, lengths, mask, dtype)
        primary, _ = _checked(self, primary, params, lengths)
        return primary, params, lengths

    def _compiled(self, kind, primary, params, lengths, mask, dtype) -> Tensor:
        """While Dynamo traces: the observable as one opaque op (_pt2)."""
        from . import _pt2

        x, params, lengths = self._prepare_shapes(primary, params, lengths, mask, dtype)
        return _pt2.observable(kind, self, x, lengths, params)

    def __call__(self, primary, *params, lengths=None, mask=None, dtype=None) -> Tensor:
        if torch.compiler.is_compiling():
            return self._compiled("map", primary, params, lengths, mask, dtype)
        if _transforms_active():
            x, params, lengths = self._prepare_shapes(primary, params, lengths, mask, dtype)
            return _MapFn.apply(self, True, lengths, x, *params)[0]
        x, params, lengths = self._prepare(primary, params, lengths, mask, dtype)
        return _MapFn.apply(self, False, lengths, x, *params)[0]

    def value(self, primary, *params, lengths=None, mask=None, dtype=None) -> Tensor:
        if torch.compiler.is_compiling():
            return self._compiled("value", primary, params, lengths, mask, dtype)
        if _transforms_active():
            x, params, lengths = self._prepare_shapes(primary, params, lengths, mask, dtype)
            return _ValueFn.apply(self, True, lengths, x, *params)[0]
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
        return _ValueFn.apply(self, False, lengths, x, *params)[0]

    def entropy(self, primary, *params, lengths=None, mask=None, dtype=None) -> Tensor:
        if torch.compiler.is_compiling():
            return self._compiled("entropy", primary, params, lengths, mask, dtype)
        if _transforms_active():
            x, params, lengths = self._prepare_shapes(primary, params, lengths, mask, dtype)
            return _EntropyFn.apply(self, True, lengths, x, *params)[0]
        x, params, lengths = self._prepare(primary, params, lengths, mask, dtype)
        return _EntropyFn.apply(self, False, lengths, x, *params)[0]

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
