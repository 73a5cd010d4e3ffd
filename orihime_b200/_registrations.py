"""Meta (fake) shapes, FP32 autocast and vmap batch-folding rules of the soft
Smith-Waterman and soft Needleman-Wunsch ops, for the ops that orihime_b200
defined itself, and of its own value-only ops (`orihime_b200::sw_value`,
`sw_affine_value`, `nw_value`).

The reference registers the same three things for its ops:
- fake impls: `orihime/_compile.py:25-140`;
- autocast: `orihime/_compile.py:323-452`;
- vmap rules: `orihime/_ops.py:178-211` and `:371-406`.

When the reference extension defined the schemas first, its Python package
makes these registrations itself, so nothing is registered here; a second
registration would make its import fail.

* **Fake impls** describe output shapes without running a kernel, so
  `torch.compile`, `torch.export` and FX tracing can trace the ops.
* **Autocast** casts floating inputs to float32 under `torch.autocast("cuda")`:
  the recurrences accumulate long chains of log-sum-exps and need fp32.
* **vmap rules** fold the mapped dimension into the native batch B of the
  batch-aligned arguments (`scores`, `v`, `grad_marginals`, `lengths`), run
  one launch over vmap_size * B pairs and unfold the outputs. A mapped scalar
  parameter is an error, as in the reference. `*_marginals_backward` returns
  batch-summed parameter gradients ([1] each); its rule takes the per-pair
  parameter tangents of the same single pass and sums them per mapped element.
"""

from __future__ import annotations

import torch

from . import _ops

_BATCH_ARGS = frozenset({"scores", "v", "grad_marginals", "lengths"})
_NPARAMS = {"sw": 2, "sw_affine": 3, "nw": 2, "nw_affine": 3, "sv_linear": 2, "sv_affine": 3}


def _fam(name: str) -> str:
    for f in ("sw_affine", "nw_affine", "sv_affine", "sv_linear", "nw"):
        if name.startswith(f):
            return f
    return "sw"


# ---- fake impls -------------------------------------------------------------

def _fake_forward(scores, *rest):
    B, L1, L2 = scores.shape
    return [scores.new_empty([B]), scores.new_empty([B, L1, L2])]


def _fake_grad_params(n):
    def fake(scores, *rest):
        return tuple(scores.new_empty([scores.size(0)]) for _ in range(n))
    return fake


def _fake_map(scores, *rest):
    return scores.new_empty(scores.shape)


def _fake_backward(n):
    def fake(scores, *rest):
        return (scores.new_empty(scores.shape), *(scores.new_empty([1]) for _ in range(n)))
    return fake


def _fake_value(scores, *rest):
    return scores.new_empty([scores.size(0)])


def _fake_forward_with_grads(n):
    def fake(scores, *rest):
        B, L1, L2 = scores.shape
        return (scores.new_empty([B]), scores.new_empty([B, L1, L2]),
                *(scores.new_empty([B]) for _ in range(n)))
    return fake


def _fake_for(name: str):
    n = _NPARAMS[_fam(name)]
    if name.endswith("_forward_with_grads"):
        return _fake_forward_with_grads(n)
    if name.endswith("_value"):
        return _fake_value
    if name.endswith("_forward") or name.endswith("_forward_t"):
        return _fake_forward
    if name.endswith("_value_grad_params"):
        # nw_affine's also returns the value first (src/nw_affine/registry.cpp:45)
        return _fake_grad_params(n + 1 if name.startswith("nw_affine") else n)
    if name.endswith("_marginals_backward"):
        return _fake_backward(n)
    return _fake_map


# ---- vmap batch folding -----------------------------------------------------

def _vmap_rule(name: str, namespace: str = "orihime"):
    op = getattr(getattr(torch.ops, namespace), name).default
    argn = [a.name for a in op._schema.arguments]
    bidx = [k for k, n in enumerate(argn) if n in _BATCH_ARGS]
    fam = _fam(name)
    backward = name.endswith("_marginals_backward")

    def rule(info, in_dims, *args):
        for k, d in enumerate(in_dims):
            if d is not None and k not in bidx:
                raise RuntimeError(f"{namespace}::{name} does not support mapping scalar argument "
                                   f"{argn[k]!r}; keep scalar parameters unbatched")
        V = info.batch_size
        nb = None
        args = list(args)
        for k in bidx:
            x = args[k]
            if not isinstance(x, torch.Tensor):
                continue
            x = x.movedim(in_dims[k], 0) if in_dims[k] is not None else x.unsqueeze(0).expand(V, *x.shape)
            if x.ndim < 2:
                raise RuntimeError(f"{namespace}::{name} batch argument {argn[k]!r} has no native batch "
                                   "dimension")
            if nb is None:
                nb = x.shape[1]
            elif x.shape[1] != nb:
                raise RuntimeError(f"{namespace}::{name} received inconsistent native batch sizes "
                                   f"{nb} and {x.shape[1]}")
            args[k] = x.reshape(V * nb, *x.shape[2:]).contiguous()
        if nb is None:
            raise RuntimeError(f"{namespace}::{name} requires a mapped batch-aligned tensor")

        def unfold(t):
            return t.reshape(V, nb, *t.shape[1:])

        if backward:
            a = dict(zip(argn, args))
            params = tuple(a[n] for n in argn[2:-1])
            out, gt = _ops.marginals_backward_per_pair(fam, a["scores"], a["grad_marginals"], params,
                                                       a["lengths"])
            sums = gt.reshape(V, nb, 4).sum(1)
            res = (unfold(out), *(sums[:, k:k + 1].contiguous() for k in range(_NPARAMS[fam])))
            return res, tuple(0 for _ in res)
        res = op(*args)
        if isinstance(res, (list, tuple)):
            outs = [unfold(t) for t in res]
            dims = [0] * len(outs)
            return (outs, dims) if isinstance(res, list) else (tuple(outs), tuple(dims))
        return unfold(res), 0

    return rule


def register(names, namespace: str = "orihime") -> None:
    """Fake impls, FP32 autocast and vmap rules for the ops in `names`."""
    for name in names:
        qual = f"{namespace}::{name}"
        torch.library.register_fake(qual)(_fake_for(name))
        torch.library.register_autocast(qual, "cuda", torch.float32)
        torch.library.register_vmap(qual, _vmap_rule(name, namespace))
