"""torch.compile path of the public observables (map, value, entropy).

Under Dynamo the public functions cannot run their value-dependent input
contract (lengths range, temperature, numerical domain, -inf mask
normalisation: host reads of tensor values) or read tensor parameters as
floats.  So while compiling, each observable is one opaque custom op whose
kernel does that work at run time and whose fake impl gives only the output
shapes; its backward is another opaque op (or plain tensor arithmetic).  Both
trace with fullgraph=True under aot_eager and inductor.  This is the role of
the reference's PT2 mirror library (orihime/_pt2_ops.py:107-270).

Parameters travel in three fixed slots (a family has two or three): slot k
holds a Python float in f<k> or a tensor in t<k> (then f<k> is unused), so
the run-time checks see each parameter as the caller passed it and raise the
same errors.  The value op returns (value, map, stacked dS/dtheta), the map
and entropy ops (observable, normalised scores, -inf cells): extra outputs
the backward needs, which the public functions drop.
"""

from __future__ import annotations

from typing import Optional

import torch
from torch import Tensor

from . import operator as _op

_SLOTS = 3


def _params(family, fs, ts):
    n = len(_op.OPERATORS[family].params)
    return [ts[k] if ts[k] is not None else fs[k] for k in range(n)]


def _slots(params):
    fs = [0.0] * _SLOTS
    ts = [None] * _SLOTS
    for k, p in enumerate(params):
        if isinstance(p, Tensor):
            ts[k] = p
        else:
            fs[k] = float(p)
    return fs, ts


def _run_checked(family, scores, lengths, fs, ts):
    op = _op.OPERATORS[family]
    params = _params(family, fs, ts)
    xn, neg = _op._checked(op, scores, params, lengths)
    if neg is None:
        neg = torch.zeros(scores.shape, dtype=torch.bool, device=scores.device)
    return op, [_op._as_float(p) for p in params], xn, neg


def _vals(family, fs, ts):
    return [_op._as_float(p) for p in _params(family, fs, ts)]


def _save(ctx, inputs):
    family, _, lengths, f0, f1, f2, t0, t1, t2 = inputs
    ctx.family, ctx.fs = family, [f0, f1, f2]
    ctx.tslot = [t is not None for t in (t0, t1, t2)]
    ctx.tmeta = [(t.shape, t.dtype, t.device) if t is not None else None for t in (t0, t1, t2)]
    ctx.has_lengths = lengths is not None
    return lengths, [t for t in (t0, t1, t2) if t is not None]


def _restore(ctx, tensors):
    it = iter(tensors)
    return [next(it) if s else None for s in ctx.tslot]


def _param_grads(ctx, per_param):
    """Gradients of the three tensor slots from per-parameter totals."""
    out = []
    for k in range(_SLOTS):
        meta = ctx.tmeta[k]
        out.append(None if meta is None else per_param(k).reshape(meta[0]).to(device=meta[2], dtype=meta[1]))
    return out


# ---- value ------------------------------------------------------------------

@torch.library.custom_op("orihime_b200::pt2_value", mutates_args=())
def pt2_value(family: str, scores: Tensor, lengths: Optional[Tensor], f0: float, f1: float, f2: float,
              t0: Optional[Tensor], t1: Optional[Tensor],
              t2: Optional[Tensor]) -> tuple[Tensor, Tensor, Tensor]:
    op, vals, xn, neg = _run_checked(family, scores, lengths, [f0, f1, f2], [t0, t1, t2])
    value, smap, *grads = op.fam.full(xn, *vals, lengths)
    return value, smap.masked_fill(neg, 0.0), torch.stack(grads)


@pt2_value.register_fake
def _(family, scores, lengths, f0, f1, f2, t0, t1, t2):
    B = scores.shape[0]
    n = len(_op.OPERATORS[family].params)
    return scores.new_empty([B]), scores.new_empty(scores.shape), scores.new_empty([n, B])


def _value_setup(ctx, inputs, output):
    _save(ctx, inputs)
    _, smap, gstack = output
    ctx.save_for_backward(smap, gstack)


def _value_backward(ctx, gv, _gmap, _gg):
    smap, gstack = ctx.saved_tensors
    gs = gv.reshape(-1, 1, 1) * smap
    return (None, gs, None, None, None, None,
            *_param_grads(ctx, lambda k: (gv * gstack[k]).sum()))


pt2_value.register_autograd(_value_backward, setup_context=_value_setup)


# ---- map --------------------------------------------------------------------

@torch.library.custom_op("orihime_b200::pt2_map", mutates_args=())
def pt2_map(family: str, scores: Tensor, lengths: Optional[Tensor], f0: float, f1: float, f2: float,
            t0: Optional[Tensor], t1: Optional[Tensor],
            t2: Optional[Tensor]) -> tuple[Tensor, Tensor, Tensor]:
    op, vals, xn, neg = _run_checked(family, scores, lengths, [f0, f1, f2], [t0, t1, t2])
    _, smap = op.fam.forward(xn, *vals, lengths)
    return smap.masked_fill(neg, 0.0), xn.clone(), neg


@pt2_map.register_fake
def _(family, scores, lengths, f0, f1, f2, t0, t1, t2):
    return (scores.new_empty(scores.shape), scores.new_empty(scores.shape),
            scores.new_empty(scores.shape, dtype=torch.bool))


@torch.library.custom_op("orihime_b200::pt2_map_vjp", mutates_args=())
def pt2_map_vjp(family: str, scores: Tensor, lengths: Optional[Tensor], f0: float, f1: float,
                f2: float, t0: Optional[Tensor], t1: Optional[Tensor], t2: Optional[Tensor],
                neg: Tensor, grad: Tensor) -> tuple[Tensor, Tensor]:
    op = _op.OPERATORS[family]
    vals = _vals(family, [f0, f1, f2], [t0, t1, t2])
    g = grad.masked_fill(neg, 0.0).contiguous()
    gs = op.fam.hvp(scores, g, *vals, lengths).masked_fill(neg, 0.0)
    pg = torch.stack([(g * sens(scores, *vals, lengths)).sum() for sens in op.fam.sens])
    return gs, pg


@pt2_map_vjp.register_fake
def _(family, scores, lengths, f0, f1, f2, t0, t1, t2, neg, grad):
    return scores.new_empty(scores.shape), scores.new_empty([len(_op.OPERATORS[family].params)])


def _map_setup(ctx, inputs, output):
    lengths, tensors = _save(ctx, inputs)
    _, xn, neg = output
    ctx.save_for_backward(xn, neg, lengths, *tensors)


def _map_backward(ctx, gm, _gx, _gn):
    xn, neg, lengths, *tensors = ctx.saved_tensors
    ts = _restore(ctx, tensors)
    gs, pg = pt2_map_vjp(ctx.family, xn, lengths if ctx.has_lengths else None, *ctx.fs, *ts, neg, gm)
    return (None, gs, None, None, None, None, *_param_grads(ctx, lambda k: pg[k]))


pt2_map.register_autograd(_map_backward, setup_context=_map_setup)


# ---- entropy ----------------------------------------------------------------

@torch.library.custom_op("orihime_b200::pt2_entropy", mutates_args=())
def pt2_entropy(family: str, scores: Tensor, lengths: Optional[Tensor], f0: float, f1: float,
                f2: float, t0: Optional[Tensor], t1: Optional[Tensor],
                t2: Optional[Tensor]) -> tuple[Tensor, Tensor, Tensor]:
    op, vals, xn, neg = _run_checked(family, scores, lengths, [f0, f1, f2], [t0, t1, t2])
    ent = op.fam.grads(xn, *vals, lengths)[-1]
    return ent.clone(), xn.clone(), neg


@pt2_entropy.register_fake
def _(family, scores, lengths, f0, f1, f2, t0, t1, t2):
    return (scores.new_empty([scores.shape[0]]), scores.new_empty(scores.shape),
            scores.new_empty(scores.shape, dtype=torch.bool))


@torch.library.custom_op("orihime_b200::pt2_entropy_vjp", mutates_args=())
def pt2_entropy_vjp(family: str, scores: Tensor, lengths: Optional[Tensor], f0: float, f1: float,
                    f2: float, t0: Optional[Tensor], t1: Optional[Tensor], t2: Optional[Tensor],
                    neg: Tensor, grad: Tensor) -> Tensor:
    op = _op.OPERATORS[family]
    vals = _vals(family, [f0, f1, f2], [t0, t1, t2])
    field = op.fam.sens[-1](scores, *vals, lengths)
    return (grad.reshape(-1, 1, 1) * field).masked_fill(neg, 0.0)


@pt2_entropy_vjp.register_fake
def _(family, scores, lengths, f0, f1, f2, t0, t1, t2, neg, grad):
    return scores.new_empty(scores.shape)


def _entropy_setup(ctx, inputs, output):
    lengths, tensors = _save(ctx, inputs)
    _, xn, neg = output
    ctx.save_for_backward(xn, neg, lengths, *tensors)
    ctx.tgrad = [t is not None and t.requires_grad for t in inputs[6:9]]


def _entropy_backward(ctx, ge, _gx, _gn):
    op = _op.OPERATORS[ctx.family]
    for name, req in zip(op.params, ctx.tgrad):
        if req:
            raise _op._entropy_direction_error(op, name)
    xn, neg, lengths, *tensors = ctx.saved_tensors
    ts = _restore(ctx, tensors)
    gs = pt2_entropy_vjp(ctx.family, xn, lengths if ctx.has_lengths else None, *ctx.fs, *ts, neg, ge)
    return (None, gs, None, None, None, None, None, None, None)


pt2_entropy.register_autograd(_entropy_backward, setup_context=_entropy_setup)


# ---- entry point used by operator.Operator while compiling ---------------------

def observable(kind: str, op, x: Tensor, lengths: Optional[Tensor], params) -> Tensor:
    fs, ts = _slots(params)
    fn = {"value": pt2_value, "map": pt2_map, "entropy": pt2_entropy}[kind]
    return fn(op.name, x, lengths, *fs, *ts)[0]
