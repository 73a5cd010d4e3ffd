"""CUDA implementations of the ``torch.ops.orihime`` soft Smith-Waterman ops
(linear and affine gaps) and soft Needleman-Wunsch ops (global alignment,
linear gap).

This module is the drop-in seam.  The reference registers its CUDA kernels
with ``TORCH_LIBRARY_IMPL(orihime, CUDA / AutogradCUDA, m)``
(src/sw/torch_cuda.cpp:803-830, src/sw_affine/torch_cuda.cpp:917-946,
src/nw/torch_cuda.cpp:795-821); here the same operator names get
implementations that call the B200 kernels through the C ABI (``_lib``).

* If the reference's own extension is already loaded in the process, its
  schemas exist and only the CUDA / AutogradCUDA kernels are replaced.
* Otherwise the schemas are defined here, character for character as in
  src/sw/registry.cpp:38-44, src/sw_affine/registry.cpp:35-42 and
  src/nw/registry.cpp:45-51.

Validation mirrors the reference op bodies (same conditions, same messages)
so that error-path tests read the same.  Like the reference, the value ops
read ``lengths`` on the host to range-check them.
"""

from __future__ import annotations

from typing import Optional

import torch

from . import _lib

_LIB = _lib.load()  # fail loudly at import if the CUDA library is missing

SCHEMAS = {
    # src/sw/registry.cpp:38-44
    "sw_forward": "sw_forward(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor[]",
    "sw_forward_t": "sw_forward_t(Tensor scores, Tensor gap, Tensor temp, Tensor lengths) -> Tensor[]",
    "sw_value_grad_params": "sw_value_grad_params(Tensor scores, float gap, float temp, Tensor? lengths) -> (Tensor, Tensor)",
    "sw_marginals_backward": "sw_marginals_backward(Tensor scores, Tensor grad_marginals, float gap, float temp, Tensor? lengths) -> (Tensor, Tensor, Tensor)",
    "sw_marginals_hvp": "sw_marginals_hvp(Tensor scores, Tensor v, float gap, float temp, Tensor? lengths) -> Tensor",
    "sw_marginals_grad_gap": "sw_marginals_grad_gap(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor",
    "sw_marginals_grad_temp": "sw_marginals_grad_temp(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor",
    # src/sw_affine/registry.cpp:35-42
    "sw_affine_forward": "sw_affine_forward(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor[]",
    "sw_affine_forward_t": "sw_affine_forward_t(Tensor scores, Tensor gap_open, Tensor gap_ext, Tensor temp, Tensor lengths) -> Tensor[]",
    "sw_affine_value_grad_params": "sw_affine_value_grad_params(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> (Tensor, Tensor, Tensor)",
    "sw_affine_marginals_backward": "sw_affine_marginals_backward(Tensor scores, Tensor grad_marginals, float gap_open, float gap_ext, float temp, Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor)",
    "sw_affine_marginals_hvp": "sw_affine_marginals_hvp(Tensor scores, Tensor v, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    "sw_affine_marginals_grad_gap_open": "sw_affine_marginals_grad_gap_open(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    "sw_affine_marginals_grad_gap_ext": "sw_affine_marginals_grad_gap_ext(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    "sw_affine_marginals_grad_temp": "sw_affine_marginals_grad_temp(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    # src/nw/registry.cpp:45-47
    "nw_forward": "nw_forward(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor[]",
    "nw_forward_t": "nw_forward_t(Tensor scores, Tensor gap, Tensor temp, Tensor lengths) -> Tensor[]",
    "nw_value_grad_params": "nw_value_grad_params(Tensor scores, float gap, float temp, Tensor? lengths) -> (Tensor, Tensor)",
    # src/nw_affine/registry.cpp:43-45
    "nw_affine_forward": "nw_affine_forward(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor[]",
    "nw_affine_forward_t": "nw_affine_forward_t(Tensor scores, Tensor gap_open, Tensor gap_ext, Tensor temp, Tensor lengths) -> Tensor[]",
    "nw_affine_value_grad_params": "nw_affine_value_grad_params(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor)",
    # src/nw_affine/registry.cpp:46-50
    "nw_affine_marginals_backward": "nw_affine_marginals_backward(Tensor scores, Tensor grad_marginals, float gap_open, float gap_ext, float temp, Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor)",
    "nw_affine_marginals_hvp": "nw_affine_marginals_hvp(Tensor scores, Tensor v, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    "nw_affine_marginals_grad_gap_open": "nw_affine_marginals_grad_gap_open(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    "nw_affine_marginals_grad_gap_ext": "nw_affine_marginals_grad_gap_ext(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    "nw_affine_marginals_grad_temp": "nw_affine_marginals_grad_temp(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    # src/sv_linear/registry.cpp:28-34
    "sv_linear_forward": "sv_linear_forward(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor[]",
    "sv_linear_forward_t": "sv_linear_forward_t(Tensor scores, Tensor gap, Tensor temp, Tensor lengths) -> Tensor[]",
    "sv_linear_value_grad_params": "sv_linear_value_grad_params(Tensor scores, float gap, float temp, Tensor? lengths) -> (Tensor, Tensor)",
    "sv_linear_marginals_backward": "sv_linear_marginals_backward(Tensor scores, Tensor grad_marginals, float gap, float temp, Tensor? lengths) -> (Tensor, Tensor, Tensor)",
    "sv_linear_marginals_hvp": "sv_linear_marginals_hvp(Tensor scores, Tensor v, float gap, float temp, Tensor? lengths) -> Tensor",
    "sv_linear_marginals_grad_gap": "sv_linear_marginals_grad_gap(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor",
    "sv_linear_marginals_grad_temp": "sv_linear_marginals_grad_temp(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor",
    # src/sv_affine/registry.cpp:37-44
    "sv_affine_forward": "sv_affine_forward(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor[]",
    "sv_affine_forward_t": "sv_affine_forward_t(Tensor scores, Tensor gap_open, Tensor gap_ext, Tensor temp, Tensor lengths) -> Tensor[]",
    "sv_affine_value_grad_params": "sv_affine_value_grad_params(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> (Tensor, Tensor, Tensor)",
    "sv_affine_marginals_backward": "sv_affine_marginals_backward(Tensor scores, Tensor grad_marginals, float gap_open, float gap_ext, float temp, Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor)",
    "sv_affine_marginals_hvp": "sv_affine_marginals_hvp(Tensor scores, Tensor v, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    "sv_affine_marginals_grad_gap_open": "sv_affine_marginals_grad_gap_open(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    "sv_affine_marginals_grad_gap_ext": "sv_affine_marginals_grad_gap_ext(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    "sv_affine_marginals_grad_temp": "sv_affine_marginals_grad_temp(Tensor scores, float gap_open, float gap_ext, float temp, Tensor? lengths) -> Tensor",
    # src/nw/registry.cpp:48-51
    "nw_marginals_backward": "nw_marginals_backward(Tensor scores, Tensor grad_marginals, float gap, float temp, Tensor? lengths) -> (Tensor, Tensor, Tensor)",
    "nw_marginals_hvp": "nw_marginals_hvp(Tensor scores, Tensor v, float gap, float temp, Tensor? lengths) -> Tensor",
    "nw_marginals_grad_gap": "nw_marginals_grad_gap(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor",
    "nw_marginals_grad_temp": "nw_marginals_grad_temp(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor",
}

_INT32_MAX = 2**31 - 1


def _op_exists(name: str) -> bool:
    try:
        torch._C._dispatch_find_schema_or_throw(f"orihime::{name}", "")
        return True
    except RuntimeError:
        return False


_DEF_LIB = torch.library.Library("orihime", "FRAGMENT")
DEFINED_HERE = []
for _name, _schema in SCHEMAS.items():
    if not _op_exists(_name):
        _DEF_LIB.define(_schema)
        DEFINED_HERE.append(_name)

_IMPL_LIB = torch.library.Library("orihime", "IMPL")


# ---------------------------------------------------------------------------
# validation (src/common/torch_utils.h:31-110, src/sw*/torch_cuda.cpp:35-110)
# ---------------------------------------------------------------------------

_SCALAR_NAMES = {
    torch.float32: "Float", torch.float64: "Double", torch.float16: "Half",
    torch.bfloat16: "BFloat16", torch.int32: "Int", torch.int64: "Long", torch.bool: "Bool",
    torch.int16: "Short", torch.int8: "Char", torch.uint8: "Byte",
}


def _stype(t: torch.Tensor) -> str:
    return _SCALAR_NAMES.get(t.dtype, str(t.dtype))


def check_input_cuda(x: torch.Tensor, name: str) -> None:
    if not x.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not x.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    if x.dtype != torch.float32:
        raise RuntimeError(f"{name} must be float32, got {_stype(x)}")


def _checked_dim(v: int, what: str) -> int:
    if v < 0:
        raise RuntimeError(f"{what} must be non-negative, got {v}")
    if v > _INT32_MAX:
        raise RuntimeError(f"{what} exceeds CUDA int index range: {v}")
    return int(v)


def check_shape(scores: torch.Tensor, family: str) -> tuple[int, int, int]:
    """3-D check plus the reference's index-range guards (torch_cuda.cpp:35-67)."""
    if scores.dim() != 3:
        raise RuntimeError("scores must be 3D (B, L1, L2)")
    B = _checked_dim(scores.size(0), "scores.size(0)")
    L1 = _checked_dim(scores.size(1), "scores.size(1)")
    L2 = _checked_dim(scores.size(2), "scores.size(2)")
    if L1 > _INT32_MAX - L2:
        raise RuntimeError(f"{family} dimensions too large: L1 + L2 exceeds CUDA int index range")
    return B, L1, L2


def _capturing() -> bool:
    """A CUDA graph is being captured on the current stream: no host
    synchronisation is allowed, so range checks move to the device."""
    return torch.cuda.is_available() and torch.cuda.is_current_stream_capturing()


def resolve_lengths(lengths, B: int, L1: int, L2: int, device) -> Optional[torch.Tensor]:
    """Validate [B, 2] int32 lengths (validate_sw_affine_lengths_cuda), or
    None for full lengths: the C ABI takes a null lengths pointer as the
    padded shape, so no default tensor is copied to the device.

    The value range check reads the lengths on the host, as the reference
    does (same messages).  While a CUDA graph is being captured that read is
    not allowed: the kernels then check the range on the device, clamp, and
    return NaN for the pairs concerned (status bit SWB_STATUS_BAD_LENGTHS)."""
    if lengths is None:
        return None
    if not lengths.is_cuda:
        raise RuntimeError("lengths must be a CUDA tensor")
    if not lengths.is_contiguous():
        raise RuntimeError("lengths must be contiguous")
    if not (lengths.dim() == 2 and lengths.size(0) == B and lengths.size(1) == 2):
        raise RuntimeError(
            "Expected lengths.dim() == 2 && lengths.size(0) == B && lengths.size(1) == 2 "
            "to be true, but got false."
        )
    if lengths.dtype != torch.int32:
        raise RuntimeError("lengths must be int32")
    if lengths.device != device:
        raise RuntimeError(f"lengths must be on same device as scores, got {lengths.device} vs {device}")
    if _capturing():
        return lengths
    host = lengths.cpu().tolist()
    for b, (l1, l2) in enumerate(host):
        if not (0 <= l1 <= L1):
            raise RuntimeError(f"lengths[{b},0] must be between 0 and {L1}, got {l1}")
        if not (0 <= l2 <= L2):
            raise RuntimeError(f"lengths[{b},1] must be between 0 and {L2}, got {l2}")
    return lengths


def _scalar_param(t: torch.Tensor, name: str) -> float:
    if t.numel() != 1:
        raise RuntimeError(f"{name} must be a scalar tensor")
    return float(t.detach().cpu().reshape(()).item())


def _device_params(scores, *params):
    """Under stream capture, the `_t` ops' tensor parameters as one float32
    device array the kernels read at each replay (no .item()): returns
    (options, placeholder floats).  Local families only (the linear-domain
    kernels): the placeholders choose that domain, and the kernels mark every
    pair NaN if a replayed value is not valid there (a positive gap or a
    temperature that is not finite and > 0)."""
    for t, n in zip(params, ("parameter",) * len(params)):
        if t.numel() != 1:
            raise RuntimeError(f"{n} must be a scalar tensor")
    arr = torch.stack([t.detach().reshape(()).to(device=scores.device, dtype=torch.float32)
                       for t in params]).contiguous()
    opt = _lib.Options(0, 0, 0, None, 0, _lib.DOMAIN_LINEAR, arr.data_ptr())
    opt._keep = arr   # the array must live as long as the captured graph uses it
    return opt, [-1.0] * (len(params) - 1) + [1.0]


# ---------------------------------------------------------------------------
# kernel calls
# ---------------------------------------------------------------------------

def _stream(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t):
    return None if t is None else t.data_ptr()


def run_affine(scores, lengths, go, ge, temp, options=None, family="sw_affine"):
    """value, map, grad_open, grad_ext, grad_temp for a validated padded batch;
    family "sw_affine" (local) or "nw_affine" (global alignment)."""
    B, L1, L2 = scores.shape
    dev = scores.device
    value = torch.empty(B, dtype=torch.float32, device=dev)
    amap = torch.empty_like(scores)
    g_open = torch.empty(B, dtype=torch.float32, device=dev)
    g_ext = torch.empty(B, dtype=torch.float32, device=dev)
    g_T = torch.empty(B, dtype=torch.float32, device=dev)
    if B == 0:
        return value, amap, g_open, g_ext, g_T
    name = {"sw_affine": "swb_sw_affine_forward", "nw_affine": "swb_nw_affine_forward",
            "sv_affine": "swb_sv_affine_forward"}[family]
    nbytes = getattr(_LIB, name.replace("_forward", "_workspace_bytes"))(B, L1, L2)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        rc = getattr(_LIB, name)(
            _ptr(scores), _ptr(lengths), B, L1, L2, float(go), float(ge), float(temp),
            _ptr(value), _ptr(amap), _ptr(g_open), _ptr(g_ext), _ptr(g_T), _ptr(ws), nbytes,
            _stream(dev), options)
    _lib.check(rc, name)
    return value, amap, g_open, g_ext, g_T


def run_linear(scores, lengths, gap, temp, options=None, family="sw"):
    """value, map, grad_gap, grad_temp for a validated padded batch; family
    "sw" (local) or "nw" (global alignment)."""
    B, L1, L2 = scores.shape
    dev = scores.device
    value = torch.empty(B, dtype=torch.float32, device=dev)
    amap = torch.empty_like(scores)
    g_gap = torch.empty(B, dtype=torch.float32, device=dev)
    g_T = torch.empty(B, dtype=torch.float32, device=dev)
    if B == 0:
        return value, amap, g_gap, g_T
    nw = family == "nw"
    nbytes = (_LIB.swb_nw_workspace_bytes if nw else _LIB.swb_sw_workspace_bytes)(B, L1, L2)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    fn = _LIB.swb_nw_forward if nw else _LIB.swb_sw_forward
    with torch.cuda.device(dev):
        rc = fn(_ptr(scores), _ptr(lengths), B, L1, L2, float(gap), float(temp), _ptr(value),
                _ptr(amap), _ptr(g_gap), _ptr(g_T), _ptr(ws), nbytes, _stream(dev), options)
    _lib.check(rc, "swb_nw_forward" if nw else "swb_sw_forward")
    return value, amap, g_gap, g_T


SCAN_POSINF, SCAN_DOMAIN, SCAN_NEGINF = 1, 2, 4


def scan_scores(x, limit, sentinel):
    """One device pass over a contiguous fp32 CUDA tensor [B, ...]: (flags,
    amax[B]).  flags: SCAN_POSINF if some cell is +inf, SCAN_DOMAIN if some
    cell is NaN or finite with |x| > limit and not -sentinel, SCAN_NEGINF if
    some cell is -inf; amax: each item's largest cell.  Reading the flags
    synchronises the stream once."""
    B = x.shape[0]
    per = x.numel() // B if B else 0
    words = torch.empty(1 + 2 * B, dtype=torch.int32, device=x.device)
    amax = words[1 + B:].view(torch.float32)
    with torch.cuda.device(x.device):
        rc = _LIB.swb_scan_scores(_ptr(x), B, per, float(limit), float(sentinel), _ptr(words), _ptr(amax),
                                  _stream(x.device))
    _lib.check(rc, "swb_scan_scores")
    return int(words[0].item()) if B else 0, amax


def run_value(fam, scores, lengths, params):
    """S per pair of a validated padded batch, forward wavefront only (no map,
    no gradients); equal bit for bit to the value of run_affine / run_linear."""
    B, L1, L2 = scores.shape
    dev = scores.device
    value = torch.empty(B, dtype=torch.float32, device=dev)
    if B == 0:
        return value
    if fam == "sv_linear":   # the Saigo-Vert affine model with gap_open = gap_ext = gap
        fam, params = "sv_affine", (params[0], params[0], params[1])
    name = {"sw": "swb_sw_value", "sw_affine": "swb_sw_affine_value", "nw": "swb_nw_value",
            "nw_affine": "swb_nw_affine_value", "sv_affine": "swb_sv_affine_value"}[fam]
    nbytes = int(getattr(_LIB, name + "_workspace_bytes")(B, L1, L2))
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        rc = getattr(_LIB, name)(_ptr(scores), _ptr(lengths), B, L1, L2, *map(float, params),
                                 _ptr(value), _ptr(ws), nbytes, _stream(dev))
    _lib.check(rc, name)
    return value


# ---- checkpointed value: forward now, adjoint in the backward ---------------

def run_checkpoint(fam, scores, lengths, params, ck_every):
    """Forward wavefront only (local families, gaps <= 0): value [B] and the
    workspace holding the checkpoints the adjoint needs later, or None when
    the parameters need the log-domain kernels (a positive gap)."""
    B, L1, L2 = scores.shape
    dev = scores.device
    value = torch.empty(B, dtype=torch.float32, device=dev)
    affine = fam == "sw_affine"
    if any(float(p) > 0 for p in params[:-1]) or B == 0:
        return None
    nbytes = int((_LIB.swb_sw_affine_checkpoint_workspace_bytes if affine
                  else _LIB.swb_sw_checkpoint_workspace_bytes)(B, L1, L2, ck_every))
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        if affine:
            rc = _LIB.swb_sw_affine_checkpoint(_ptr(scores), _ptr(lengths), B, L1, L2, *map(float, params),
                                               int(ck_every), _ptr(value), _ptr(ws), nbytes, _stream(dev))
        else:
            rc = _LIB.swb_sw_checkpoint(_ptr(scores), _ptr(lengths), B, L1, L2, *map(float, params),
                                        int(ck_every), _ptr(value), _ptr(ws), nbytes, _stream(dev))
    _lib.check(rc, "swb_sw_checkpoint")
    return value, ws


def run_adjoint(fam, scores, lengths, params, ck_every, ws):
    """The checkpointed adjoint on a run_checkpoint workspace: (value, map,
    dS/dparameters...)."""
    B, L1, L2 = scores.shape
    dev = scores.device
    e = lambda: torch.empty(B, dtype=torch.float32, device=dev)  # noqa: E731
    value, amap = e(), torch.empty_like(scores)
    nbytes = ws.numel()
    with torch.cuda.device(dev):
        if fam == "sw_affine":
            go, ge, gT = e(), e(), e()
            rc = _LIB.swb_sw_affine_adjoint(_ptr(scores), _ptr(lengths), B, L1, L2, *map(float, params),
                                            int(ck_every), _ptr(value), _ptr(amap), _ptr(go), _ptr(ge),
                                            _ptr(gT), _ptr(ws), nbytes, _stream(dev))
            grads = (go, ge, gT)
        else:
            gg, gT = e(), e()
            rc = _LIB.swb_sw_adjoint(_ptr(scores), _ptr(lengths), B, L1, L2, *map(float, params),
                                     int(ck_every), _ptr(value), _ptr(amap), _ptr(gg), _ptr(gT), _ptr(ws),
                                     nbytes, _stream(dev))
            grads = (gg, gT)
    _lib.check(rc, "swb_sw_adjoint")
    return (value, amap, *grads)


def _prep(scores, lengths, family):
    check_input_cuda(scores, "scores")
    B, L1, L2 = check_shape(scores, family)
    return resolve_lengths(lengths, B, L1, L2, scores.device)


# ---- affine ----------------------------------------------------------------

def sw_affine_forward(scores, gap_open, gap_ext, temp, lengths):
    """orihime::sw_affine_forward -> [value [B], marginals [B, L1, L2]]
    (src/sw_affine/torch_cuda.cpp:820 -> :419 -> :128-206)."""
    ln = _prep(scores, lengths, "sw_affine")
    v, m, *_ = run_affine(scores, ln, gap_open, gap_ext, temp)
    return [v, m]


def sw_affine_forward_t(scores, gap_open, gap_ext, temp, lengths):
    """orihime::sw_affine_forward_t (src/sw_affine/torch_cuda.cpp:830 -> :126-206)."""
    check_input_cuda(scores, "scores")
    if scores.dim() != 3:
        raise RuntimeError("scores must be 3D (B, L1, L2)")
    if _capturing():
        opt, (go, ge, T) = _device_params(scores, gap_open, gap_ext, temp)
        B, L1, L2 = check_shape(scores, "sw_affine")
        ln = resolve_lengths(lengths, B, L1, L2, scores.device)
        v, m, *_ = run_affine(scores, ln, go, ge, T, options=opt)
        return [v, m]
    go = _scalar_param(gap_open, "gap_open")
    ge = _scalar_param(gap_ext, "gap_ext")
    T = _scalar_param(temp, "temperature")
    B, L1, L2 = check_shape(scores, "sw_affine")
    ln = resolve_lengths(lengths, B, L1, L2, scores.device)
    v, m, *_ = run_affine(scores, ln, go, ge, T)
    return [v, m]


def sw_affine_value_grad_params(scores, gap_open, gap_ext, temp, lengths):
    """orihime::sw_affine_value_grad_params -> (dS/dgo, dS/dge, dS/dT), each [B]
    (src/sw_affine/torch_cuda.cpp:842 -> soft_sw_affine_cuda_with_grads :446)."""
    ln = _prep(scores, lengths, "sw_affine")
    _, _, go, ge, gT = run_affine(scores, ln, gap_open, gap_ext, temp)
    return go, ge, gT


# ---- linear ----------------------------------------------------------------

def sw_forward(scores, gap, temp, lengths):
    """orihime::sw_forward -> [value [B], marginals [B, L1, L2]] (src/sw/torch_cuda.cpp:364-402)."""
    ln = _prep(scores, lengths, "sw")
    v, m, *_ = run_linear(scores, ln, gap, temp)
    return [v, m]


def sw_forward_t(scores, gap, temp, lengths):
    """orihime::sw_forward_t (src/sw/torch_cuda.cpp:124-210)."""
    check_input_cuda(scores, "scores")
    if scores.dim() != 3:
        raise RuntimeError("scores must be 3D (B, L1, L2)")
    if _capturing():
        opt, (g, T) = _device_params(scores, gap, temp)
        B, L1, L2 = check_shape(scores, "sw")
        ln = resolve_lengths(lengths, B, L1, L2, scores.device)
        v, m, *_ = run_linear(scores, ln, g, T, options=opt)
        return [v, m]
    g = _scalar_param(gap, "gap")
    T = _scalar_param(temp, "temperature")
    B, L1, L2 = check_shape(scores, "sw")
    ln = resolve_lengths(lengths, B, L1, L2, scores.device)
    v, m, *_ = run_linear(scores, ln, g, T)
    return [v, m]


def sw_value_grad_params(scores, gap, temp, lengths):
    """orihime::sw_value_grad_params -> (dS/dgap, dS/dT), each [B] (src/sw/torch_cuda.cpp:404-450)."""
    ln = _prep(scores, lengths, "sw")
    _, _, gg, gT = run_linear(scores, ln, gap, temp)
    return gg, gT


# ---- global alignment (Needleman-Wunsch, linear gap) -----------------------

def nw_forward(scores, gap, temp, lengths):
    """orihime::nw_forward -> [value [B], marginals [B, L1, L2]]
    (src/nw/torch_cuda.cpp:716 -> soft_nw_cuda_float :364)."""
    ln = _prep(scores, lengths, "nw")
    v, m, *_ = run_linear(scores, ln, gap, temp, family="nw")
    return [v, m]


def nw_forward_t(scores, gap, temp, lengths):
    """orihime::nw_forward_t (src/nw/torch_cuda.cpp:726 -> SoftNWCUDAFunction :110-200)."""
    check_input_cuda(scores, "scores")
    if scores.dim() != 3:
        raise RuntimeError("scores must be 3D (B, L1, L2)")
    g = _scalar_param(gap, "gap")
    T = _scalar_param(temp, "temperature")
    B, L1, L2 = check_shape(scores, "nw")
    ln = resolve_lengths(lengths, B, L1, L2, scores.device)
    v, m, *_ = run_linear(scores, ln, g, T, family="nw")
    return [v, m]


def nw_value_grad_params(scores, gap, temp, lengths):
    """orihime::nw_value_grad_params -> (dS/dgap, dS/dT), each [B]
    (src/nw/torch_cuda.cpp:736 -> soft_nw_cuda_with_grads :384)."""
    ln = _prep(scores, lengths, "nw")
    _, _, gg, gT = run_linear(scores, ln, gap, temp, family="nw")
    return gg, gT


# ---- global alignment with affine gaps (Needleman-Wunsch affine) -------------

def nw_affine_forward(scores, gap_open, gap_ext, temp, lengths):
    """orihime::nw_affine_forward -> [value [B], marginals [B, L1, L2]]
    (src/nw_affine/torch_cuda.cpp:667 -> soft_nw_affine_cuda_float :364)."""
    ln = _prep(scores, lengths, "nw_affine")
    v, m, *_ = run_affine(scores, ln, gap_open, gap_ext, temp, family="nw_affine")
    return [v, m]


def nw_affine_forward_t(scores, gap_open, gap_ext, temp, lengths):
    """orihime::nw_affine_forward_t (src/nw_affine/torch_cuda.cpp:677 -> :352)."""
    check_input_cuda(scores, "scores")
    if scores.dim() != 3:
        raise RuntimeError("scores must be 3D (B, L1, L2)")
    go = _scalar_param(gap_open, "gap_open")
    ge = _scalar_param(gap_ext, "gap_ext")
    T = _scalar_param(temp, "temperature")
    B, L1, L2 = check_shape(scores, "nw_affine")
    ln = resolve_lengths(lengths, B, L1, L2, scores.device)
    v, m, *_ = run_affine(scores, ln, go, ge, T, family="nw_affine")
    return [v, m]


def nw_affine_value_grad_params(scores, gap_open, gap_ext, temp, lengths):
    """orihime::nw_affine_value_grad_params -> (value, dS/dgo, dS/dge, dS/dT), each [B]
    (src/nw_affine/torch_cuda.cpp:688-702 -> soft_nw_affine_cuda_with_grads :387)."""
    ln = _prep(scores, lengths, "nw_affine")
    v, _, go, ge, gT = run_affine(scores, ln, gap_open, gap_ext, temp, family="nw_affine")
    return v, go, ge, gT


# ---- second-order ops --------------------------------------------------------

def _check_like(scores, other, name, msg_shape):
    check_input_cuda(other, name)
    if scores.dim() != 3:
        raise RuntimeError("scores must be 3D")
    if other.shape != scores.shape:
        raise RuntimeError(msg_shape)
    if other.device != scores.device:
        raise RuntimeError(f"{name} must be on same device as scores, got {other.device} vs {scores.device}")


# Largest workspace one second-order call takes at once; a batch needing more
# is processed in pair groups (results identical: pairs are independent).
# Fewer, larger groups are faster: the log-domain HVP at 4096 pairs of
# 512 x 512 takes 31 ms in groups of 3060 pairs (64 GiB) and 34 ms in groups
# of 765 (16 GiB).  Half the free device memory still bounds it.
AUX_BUDGET_MAX = 64 << 30


_AUX = {  # family -> (workspace bytes, HVP, parameter Jacobian) entry points
    "sw": ("swb_sw_aux_workspace_bytes", "swb_sw_hvp", "swb_sw_param_jacobian"),
    "sw_affine": ("swb_sw_affine_aux_workspace_bytes", "swb_sw_affine_hvp",
                  "swb_sw_affine_param_jacobian"),
    "nw": ("swb_nw_aux_workspace_bytes", "swb_nw_hvp", "swb_nw_param_jacobian"),
    "nw_affine": ("swb_nw_affine_aux_workspace_bytes", "swb_nw_affine_hvp",
                  "swb_nw_affine_param_jacobian"),
    "sv_affine": ("swb_sv_affine_aux_workspace_bytes", "swb_sv_affine_hvp",
                  "swb_sv_affine_param_jacobian"),
}


# Local families: the workspace the call with given parameters launches (the
# linear-domain tangent kernels' checkpoints, about 7 B per cell, when every
# gap is <= 0), instead of the larger log-domain field table.
_AUX_FOR = {"sw": "swb_sw_aux_workspace_bytes_for", "sw_affine": "swb_sw_affine_aux_workspace_bytes_for"}


def _aux_plan(fam, B, L1, L2, dev, params):
    """(pairs per group, workspace bytes) for a second-order call with these
    parameters.  The log-domain kernels' field table is about 100 (affine) /
    50 (linear) bytes per cell, so large batches are split to stay within
    min(AUX_BUDGET_MAX, max(2 GiB, half the free device memory))."""
    if fam in _AUX_FOR:
        f = getattr(_LIB, _AUX_FOR[fam])
        vals = [float(p) for p in params]
        fn = lambda b, l1, l2: f(b, l1, l2, *vals)  # noqa: E731
    else:
        fn = getattr(_LIB, _AUX[fam][0])
    nbytes = int(fn(B, L1, L2))
    # the free-memory query is a host call; under stream capture use the floor
    free = 0 if _capturing() else torch.cuda.mem_get_info(dev)[0]
    budget = min(AUX_BUDGET_MAX, max(2 << 30, free // 2))
    g = B
    if nbytes > budget:
        g = max(1, min(B, B * budget // nbytes))
        while g > 1 and int(fn(g, L1, L2)) > budget:
            g = max(1, g // 2)
    last = B - (B - 1) // g * g
    return g, max(int(fn(g, L1, L2)), int(fn(last, L1, L2)))


def _groups(B, g):
    for b0 in range(0, B, g):
        yield b0, min(B, b0 + g)


def run_hvp(fam, scores, v, lengths, params, want_grads=False):
    """H.v of the map (and optionally the per-pair tangents of dS/dparams, S)."""
    B, L1, L2 = scores.shape
    dev = scores.device
    out = torch.empty_like(scores)
    gt = torch.zeros(B, 4, dtype=torch.float32, device=dev) if want_grads else None
    if B == 0:
        return out, gt
    g, nbytes = _aux_plan(fam, B, L1, L2, dev, params)
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    fn = getattr(_LIB, _AUX[fam][1])
    with torch.cuda.device(dev):
        for b0, b1 in _groups(B, g):
            ln = None if lengths is None else lengths[b0:b1]
            rc = fn(_ptr(scores[b0:b1]), _ptr(v[b0:b1]), _ptr(ln), b1 - b0, L1, L2, *map(float, params),
                    _ptr(out[b0:b1]), _ptr(None if gt is None else gt[b0:b1]), _ptr(ws), nbytes,
                    _stream(dev))
            _lib.check(rc, _AUX[fam][1])
    return out, gt


def run_param_jacobian(fam, scores, lengths, params, which):
    B, L1, L2 = scores.shape
    dev = scores.device
    out = torch.empty_like(scores)
    if B == 0:
        return out
    g, nbytes = _aux_plan(fam, B, L1, L2, dev, params)
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    fn = getattr(_LIB, _AUX[fam][2])
    with torch.cuda.device(dev):
        for b0, b1 in _groups(B, g):
            ln = None if lengths is None else lengths[b0:b1]
            rc = fn(_ptr(scores[b0:b1]), _ptr(ln), b1 - b0, L1, L2, *map(float, params), int(which),
                    _ptr(out[b0:b1]), _ptr(ws), nbytes, _stream(dev))
            _lib.check(rc, _AUX[fam][2])
    return out


def sw_affine_marginals_hvp(scores, v, gap_open, gap_ext, temp, lengths):
    """orihime::sw_affine_marginals_hvp (src/sw_affine/torch_cuda.cpp:866 -> :508)."""
    check_input_cuda(scores, "scores")
    _check_like(scores, v, "tangent", "scores and tangent must have same shape")
    ln = _prep(scores, lengths, "sw_affine")
    return run_hvp("sw_affine", scores, v, ln, (gap_open, gap_ext, temp))[0]


def _affine_param(which):
    def op(scores, gap_open, gap_ext, temp, lengths):
        ln = _prep(scores, lengths, "sw_affine")
        return run_param_jacobian("sw_affine", scores, ln, (gap_open, gap_ext, temp), which)
    op.__doc__ = (f"orihime::sw_affine_marginals_grad_* param {which} "
                  "(src/sw_affine/torch_cuda.cpp:878-910 -> :580)")
    return op


def marginals_backward_per_pair(fam, scores, grad_marginals, params, lengths):
    """Validated map VJP with per-pair parameter tangents: (grad_scores,
    gt[B][4]).  gt[b] holds the tangents along G of pair b's parameter
    gradients (affine: go, ge, T, S; linear: gap, T, 0, S); the
    marginals_backward ops sum them over the batch."""
    check_input_cuda(scores, "scores")
    if scores.dim() != 3:
        raise RuntimeError("scores must be 3D (B, L1, L2)")
    if grad_marginals.shape != scores.shape:
        raise RuntimeError("grad_alignment must have same shape as scores")
    if not grad_marginals.is_cuda:
        raise RuntimeError("grad_alignment must be a CUDA tensor")
    if grad_marginals.device != scores.device:
        raise RuntimeError(f"grad_alignment must be on same device as scores, got "
                           f"{grad_marginals.device} vs {scores.device}")
    g = grad_marginals.contiguous().to(torch.float32)
    ln = _prep(scores, lengths, fam)
    if fam == "sv_linear":   # via the affine model: tangent of dS/dgap = open + ext
        gap, temp = params
        out, gt = run_hvp("sv_affine", scores, g, ln, (gap, gap, temp), want_grads=True)
        return out, torch.stack([gt[:, 0] + gt[:, 1], gt[:, 2], torch.zeros_like(gt[:, 0]), gt[:, 3]], 1)
    return run_hvp(fam, scores, g, ln, params, want_grads=True)


def sw_affine_marginals_backward(scores, grad_marginals, gap_open, gap_ext, temp, lengths):
    """orihime::sw_affine_marginals_backward -> (grad_scores, d/dgo [1], d/dge [1], d/dT [1])
    (src/sw_affine/torch_cuda.cpp:854 -> soft_sw_affine_backward_full_cuda :681-811).

    One tangent pass along the cotangent G: grad_scores = H.G (the Hessian is
    symmetric) and sum(G * dP/dtheta) = d/dG (dS/dtheta), the tangents of the
    parameter gradients, summed over the batch."""
    out, gt = marginals_backward_per_pair("sw_affine", scores, grad_marginals,
                                          (gap_open, gap_ext, temp), lengths)
    tot = gt[:, :3].sum(0)
    return out, tot[0:1].clone(), tot[1:2].clone(), tot[2:3].clone()


def sw_marginals_hvp(scores, v, gap, temp, lengths):
    """orihime::sw_marginals_hvp (src/sw/torch_cuda.cpp:766 -> soft_sw_regular_hvp_cuda :453)."""
    check_input_cuda(scores, "scores")
    _check_like(scores, v, "tangent", "scores and tangent must have same shape")
    ln = _prep(scores, lengths, "sw")
    return run_hvp("sw", scores, v, ln, (gap, temp))[0]


def _linear_param(which):
    def op(scores, gap, temp, lengths):
        ln = _prep(scores, lengths, "sw")
        return run_param_jacobian("sw", scores, ln, (gap, temp), which)
    op.__doc__ = f"orihime::sw_marginals_grad_* param {which} (src/sw/torch_cuda.cpp:777-796 -> soft_sw_regular_param_jacobian_cuda :519)"
    return op


def sw_marginals_backward(scores, grad_marginals, gap, temp, lengths):
    """orihime::sw_marginals_backward -> (grad_scores, d/dgap [1], d/dT [1])
    (src/sw/torch_cuda.cpp:755 -> soft_sw_backward_full_cuda :612)."""
    out, gt = marginals_backward_per_pair("sw", scores, grad_marginals, (gap, temp), lengths)
    tot = gt[:, :2].sum(0)
    return out, tot[0:1].clone(), tot[1:2].clone()


def nw_marginals_hvp(scores, v, gap, temp, lengths):
    """orihime::nw_marginals_hvp (src/nw/torch_cuda.cpp:758 -> soft_nw_hvp_cuda :442)."""
    check_input_cuda(scores, "scores")
    _check_like(scores, v, "tangent", "scores and tangent must have same shape")
    ln = _prep(scores, lengths, "nw")
    return run_hvp("nw", scores, v, ln, (gap, temp))[0]


def _nw_param(which):
    def op(scores, gap, temp, lengths):
        ln = _prep(scores, lengths, "nw")
        return run_param_jacobian("nw", scores, ln, (gap, temp), which)
    op.__doc__ = (f"orihime::nw_marginals_grad_* param {which} "
                  "(src/nw/torch_cuda.cpp:769-790 -> soft_nw_param_jacobian_cuda :509)")
    return op


def nw_marginals_backward(scores, grad_marginals, gap, temp, lengths):
    """orihime::nw_marginals_backward -> (grad_scores, d/dgap [1], d/dT [1])
    (src/nw/torch_cuda.cpp:747 -> soft_nw_backward_full_cuda :603); one
    tangent pass along the cotangent, as for the local alignment."""
    out, gt = marginals_backward_per_pair("nw", scores, grad_marginals, (gap, temp), lengths)
    tot = gt[:, :2].sum(0)
    return out, tot[0:1].clone(), tot[1:2].clone()


def nw_affine_marginals_hvp(scores, v, gap_open, gap_ext, temp, lengths):
    """orihime::nw_affine_marginals_hvp (src/nw_affine/torch_cuda.cpp:716 -> soft_nw_affine_hvp_cuda :435)."""
    check_input_cuda(scores, "scores")
    _check_like(scores, v, "tangent", "scores and tangent must have same shape")
    ln = _prep(scores, lengths, "nw_affine")
    return run_hvp("nw_affine", scores, v, ln, (gap_open, gap_ext, temp))[0]


def _nw_affine_param(which):
    def op(scores, gap_open, gap_ext, temp, lengths):
        ln = _prep(scores, lengths, "nw_affine")
        return run_param_jacobian("nw_affine", scores, ln, (gap_open, gap_ext, temp), which)
    op.__doc__ = (f"orihime::nw_affine_marginals_grad_* param {which} "
                  "(src/nw_affine/torch_cuda.cpp:727-755 -> soft_nw_affine_param_jacobian_cuda :484)")
    return op


def nw_affine_marginals_backward(scores, grad_marginals, gap_open, gap_ext, temp, lengths):
    """orihime::nw_affine_marginals_backward -> (grad_scores, d/dgo [1], d/dge [1], d/dT [1])
    (src/nw_affine/torch_cuda.cpp:704 -> soft_nw_affine_backward_full_cuda :555); one
    tangent pass along the cotangent."""
    out, gt = marginals_backward_per_pair("nw_affine", scores, grad_marginals,
                                          (gap_open, gap_ext, temp), lengths)
    tot = gt[:, :3].sum(0)
    return out, tot[0:1].clone(), tot[1:2].clone(), tot[2:3].clone()


# ---- Saigo-Vert (local; affine, and linear as affine with one gap) -------------
# src/sv_affine/torch_cuda.cpp and src/sv_linear/torch_cuda.cpp bodies; the
# linear model runs the affine kernels with gap_open = gap_ext = gap and
# reports dS/dgap = dS/dgap_open + dS/dgap_ext.

def sv_affine_forward(scores, gap_open, gap_ext, temp, lengths):
    """orihime::sv_affine_forward -> [value [B], marginals [B, L1, L2]]."""
    ln = _prep(scores, lengths, "sv_affine")
    v, m, *_ = run_affine(scores, ln, gap_open, gap_ext, temp, family="sv_affine")
    return [v, m]


def sv_affine_forward_t(scores, gap_open, gap_ext, temp, lengths):
    """orihime::sv_affine_forward_t (tensor parameters)."""
    check_input_cuda(scores, "scores")
    if scores.dim() != 3:
        raise RuntimeError("scores must be 3D (B, L1, L2)")
    go = _scalar_param(gap_open, "gap_open")
    ge = _scalar_param(gap_ext, "gap_ext")
    T = _scalar_param(temp, "temperature")
    B, L1, L2 = check_shape(scores, "sv_affine")
    ln = resolve_lengths(lengths, B, L1, L2, scores.device)
    v, m, *_ = run_affine(scores, ln, go, ge, T, family="sv_affine")
    return [v, m]


def sv_affine_value_grad_params(scores, gap_open, gap_ext, temp, lengths):
    """orihime::sv_affine_value_grad_params -> (dS/dgo, dS/dge, dS/dT), each [B]."""
    ln = _prep(scores, lengths, "sv_affine")
    _, _, go, ge, gT = run_affine(scores, ln, gap_open, gap_ext, temp, family="sv_affine")
    return go, ge, gT


def sv_affine_marginals_hvp(scores, v, gap_open, gap_ext, temp, lengths):
    check_input_cuda(scores, "scores")
    _check_like(scores, v, "tangent", "scores and tangent must have same shape")
    ln = _prep(scores, lengths, "sv_affine")
    return run_hvp("sv_affine", scores, v, ln, (gap_open, gap_ext, temp))[0]


def _sv_affine_param(which):
    def op(scores, gap_open, gap_ext, temp, lengths):
        ln = _prep(scores, lengths, "sv_affine")
        return run_param_jacobian("sv_affine", scores, ln, (gap_open, gap_ext, temp), which)
    op.__doc__ = f"orihime::sv_affine_marginals_grad_* param {which}"
    return op


def sv_affine_marginals_backward(scores, grad_marginals, gap_open, gap_ext, temp, lengths):
    out, gt = marginals_backward_per_pair("sv_affine", scores, grad_marginals,
                                          (gap_open, gap_ext, temp), lengths)
    tot = gt[:, :3].sum(0)
    return out, tot[0:1].clone(), tot[1:2].clone(), tot[2:3].clone()


def sv_linear_forward(scores, gap, temp, lengths):
    """orihime::sv_linear_forward -> [value [B], marginals [B, L1, L2]]."""
    ln = _prep(scores, lengths, "sv_linear")
    v, m, *_ = run_affine(scores, ln, gap, gap, temp, family="sv_affine")
    return [v, m]


def sv_linear_forward_t(scores, gap, temp, lengths):
    check_input_cuda(scores, "scores")
    if scores.dim() != 3:
        raise RuntimeError("scores must be 3D (B, L1, L2)")
    g = _scalar_param(gap, "gap")
    T = _scalar_param(temp, "temperature")
    B, L1, L2 = check_shape(scores, "sv_linear")
    ln = resolve_lengths(lengths, B, L1, L2, scores.device)
    v, m, *_ = run_affine(scores, ln, g, g, T, family="sv_affine")
    return [v, m]


def sv_linear_value_grad_params(scores, gap, temp, lengths):
    """orihime::sv_linear_value_grad_params -> (dS/dgap, dS/dT), each [B]."""
    ln = _prep(scores, lengths, "sv_linear")
    _, _, go, ge, gT = run_affine(scores, ln, gap, gap, temp, family="sv_affine")
    return go + ge, gT


def sv_linear_marginals_hvp(scores, v, gap, temp, lengths):
    check_input_cuda(scores, "scores")
    _check_like(scores, v, "tangent", "scores and tangent must have same shape")
    ln = _prep(scores, lengths, "sv_linear")
    return run_hvp("sv_affine", scores, v, ln, (gap, gap, temp))[0]


def _sv_linear_param(which):
    def op(scores, gap, temp, lengths):
        ln = _prep(scores, lengths, "sv_linear")
        if which == 1:
            return run_param_jacobian("sv_affine", scores, ln, (gap, gap, temp), 2)
        return (run_param_jacobian("sv_affine", scores, ln, (gap, gap, temp), 0) +
                run_param_jacobian("sv_affine", scores, ln, (gap, gap, temp), 1))
    op.__doc__ = f"orihime::sv_linear_marginals_grad_* param {which} (gap = open + ext directions)"
    return op


def sv_linear_marginals_backward(scores, grad_marginals, gap, temp, lengths):
    out, gt = marginals_backward_per_pair("sv_linear", scores, grad_marginals, (gap, temp), lengths)
    tot = gt[:, :2].sum(0)
    return out, tot[0:1].clone(), tot[1:2].clone()


IMPLS = {
    "sv_affine_forward": sv_affine_forward,
    "sv_affine_forward_t": sv_affine_forward_t,
    "sv_affine_value_grad_params": sv_affine_value_grad_params,
    "sv_affine_marginals_hvp": sv_affine_marginals_hvp,
    "sv_affine_marginals_grad_gap_open": _sv_affine_param(0),
    "sv_affine_marginals_grad_gap_ext": _sv_affine_param(1),
    "sv_affine_marginals_grad_temp": _sv_affine_param(2),
    "sv_affine_marginals_backward": sv_affine_marginals_backward,
    "sv_linear_forward": sv_linear_forward,
    "sv_linear_forward_t": sv_linear_forward_t,
    "sv_linear_value_grad_params": sv_linear_value_grad_params,
    "sv_linear_marginals_hvp": sv_linear_marginals_hvp,
    "sv_linear_marginals_grad_gap": _sv_linear_param(0),
    "sv_linear_marginals_grad_temp": _sv_linear_param(1),
    "sv_linear_marginals_backward": sv_linear_marginals_backward,
    "nw_affine_marginals_hvp": nw_affine_marginals_hvp,
    "nw_affine_marginals_grad_gap_open": _nw_affine_param(0),
    "nw_affine_marginals_grad_gap_ext": _nw_affine_param(1),
    "nw_affine_marginals_grad_temp": _nw_affine_param(2),
    "nw_affine_marginals_backward": nw_affine_marginals_backward,
    "nw_marginals_hvp": nw_marginals_hvp,
    "nw_marginals_grad_gap": _nw_param(0),
    "nw_marginals_grad_temp": _nw_param(1),
    "nw_marginals_backward": nw_marginals_backward,
    "sw_marginals_hvp": sw_marginals_hvp,
    "sw_marginals_grad_gap": _linear_param(0),
    "sw_marginals_grad_temp": _linear_param(1),
    "sw_marginals_backward": sw_marginals_backward,
    "sw_affine_marginals_hvp": sw_affine_marginals_hvp,
    "sw_affine_marginals_grad_gap_open": _affine_param(0),
    "sw_affine_marginals_grad_gap_ext": _affine_param(1),
    "sw_affine_marginals_grad_temp": _affine_param(2),
    "sw_affine_marginals_backward": sw_affine_marginals_backward,
    "sw_forward": sw_forward,
    "sw_forward_t": sw_forward_t,
    "sw_value_grad_params": sw_value_grad_params,
    "sw_affine_forward": sw_affine_forward,
    "sw_affine_forward_t": sw_affine_forward_t,
    "sw_affine_value_grad_params": sw_affine_value_grad_params,
    "nw_forward": nw_forward,
    "nw_forward_t": nw_forward_t,
    "nw_value_grad_params": nw_value_grad_params,
    "nw_affine_forward": nw_affine_forward,
    "nw_affine_forward_t": nw_affine_forward_t,
    "nw_affine_value_grad_params": nw_affine_value_grad_params,
}

for _name, _fn in IMPLS.items():
    _IMPL_LIB.impl(_name, _fn, "CUDA")


# ---------------------------------------------------------------------------
# AutogradCUDA kernels of the forward ops
# ---------------------------------------------------------------------------
# The reference makes sw_forward(_t) / sw_affine_forward(_t) differentiable
# with a C++ autograd Function registered at AutogradCUDA
# (src/sw_affine/torch_cuda.cpp:938-946, src/sw/torch_cuda.cpp:820-830);
# backward = value cotangent x map + HVP of the map cotangent, plus the
# parameter gradients for the tensor-parameter (_t) variants.  An AutogradCUDA
# kernel runs before the CUDA kernel, so these registrations are what make
# the B200 kernels the ones that run when the reference extension is loaded
# too.  Forward redispatches below autograd to the CUDA kernels above.

def _below(op, *args):
    with torch._C._AutoDispatchBelowAutograd():
        return op(*args)


def _pgrad(g, like):
    return g.reshape(like.shape).to(dtype=like.dtype) if like.requires_grad else None


class _ForwardFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fam, tensor_params, scores, lengths, *params):
        name = f"{fam}_forward" + ("_t" if tensor_params else "")
        v, m = _below(getattr(torch.ops.orihime, name), scores, *params, lengths)
        ctx.fam, ctx.tensor_params, ctx.lengths = fam, tensor_params, lengths
        # the parameter values the backward ops take as floats; under stream
        # capture a host read is not allowed, so the backward reads them
        ctx.vals = (None if tensor_params and _capturing() else
                    tuple(_scalar_param(p, "param") if tensor_params else float(p) for p in params))
        ctx.params = params
        ctx.save_for_backward(scores, m)
        return v, m

    @staticmethod
    def backward(ctx, gv, gm):
        scores, m = ctx.saved_tensors
        fam, vals, ln = ctx.fam, ctx.vals, ctx.lengths
        if vals is None:
            vals = tuple(_scalar_param(p, "param") for p in ctx.params)
        ops = torch.ops.orihime
        gs = torch.zeros_like(scores) if ctx.needs_input_grad[2] else None
        pg = [None] * len(ctx.params)
        want_p = ctx.tensor_params and any(ctx.needs_input_grad[4:])
        if gv is not None:
            if gs is not None:
                gs = gs + gv.view(-1, 1, 1) * m
            if want_p:
                grads = _below(getattr(ops, f"{fam}_value_grad_params"), scores, *vals, ln)
                if fam == "nw_affine":   # (value, grads...): src/nw_affine/torch_cuda.cpp:696
                    grads = grads[1:]
                pg = [(gv * g).sum() for g in grads]
        if gm is not None:
            gmc = gm.contiguous()
            if want_p:
                mb = _below(getattr(ops, f"{fam}_marginals_backward"), scores, gmc, *vals, ln)
                if gs is not None:
                    gs = gs + mb[0]
                pg = [mb[1 + k].reshape(()) if pg[k] is None else pg[k] + mb[1 + k].reshape(())
                      for k in range(len(pg))]
            elif gs is not None:
                gs = gs + _below(getattr(ops, f"{fam}_marginals_hvp"), scores, gmc, *vals, ln)
        out = [None, None, gs, None]
        for k, p in enumerate(ctx.params):
            out.append(_pgrad(pg[k], p) if (ctx.tensor_params and pg[k] is not None
                                             and ctx.needs_input_grad[4 + k]) else None)
        return tuple(out)


def _autograd_forward(fam, tensor_params):
    def kernel(scores, *rest):
        *params, lengths = rest
        v, m = _ForwardFn.apply(fam, tensor_params, scores, lengths, *params)
        return [v, m]
    return kernel


for _name, _fam, _t in (("sw_forward", "sw", False), ("sw_forward_t", "sw", True),
                        ("sw_affine_forward", "sw_affine", False),
                        ("sw_affine_forward_t", "sw_affine", True),
                        ("nw_forward", "nw", False), ("nw_forward_t", "nw", True),
                        ("nw_affine_forward", "nw_affine", False),
                        ("nw_affine_forward_t", "nw_affine", True),
                        ("sv_affine_forward", "sv_affine", False),
                        ("sv_affine_forward_t", "sv_affine", True),
                        ("sv_linear_forward", "sv_linear", False),
                        ("sv_linear_forward_t", "sv_linear", True)):
    _IMPL_LIB.impl(_name, _autograd_forward(_fam, _t), "AutogradCUDA")


# ---------------------------------------------------------------------------
# legacy soft_sw* / soft_nw* ops (src/sw/registry.cpp:30-35,
# src/sw_affine/registry.cpp:27-32, src/nw/registry.cpp:34-39,
# src/nw_affine/registry.cpp:35-40)
# ---------------------------------------------------------------------------
# The reference keeps 36 older schemas beside the namespaced ones; its Python
# package no longer calls them.  Each is one of the namespaced op bodies under
# another name (src/sw*/torch_cuda.cpp:803-830, :917-946,
# src/nw*/torch_cuda.cpp:795-821, :763-786).  They are defined
# and given CUDA kernels only when orihime_b200 defines the schemas itself:
# with the reference extension loaded first, they stay the reference's own.

LEGACY_SCHEMAS = {
    "soft_sw": "soft_sw(Tensor scores, Tensor gap, Tensor temperature, Tensor lengths) -> Tensor[]",
    "soft_sw_float": "soft_sw_float(Tensor scores, float gap, float temperature, Tensor? lengths) -> Tensor[]",
    "soft_sw_with_grads": "soft_sw_with_grads(Tensor scores, float gap, float temperature, Tensor? lengths) "
                          "-> (Tensor, Tensor, Tensor, Tensor)",
    "soft_sw_hvp": "soft_sw_hvp(Tensor scores, Tensor tangent, float gap, float temperature, Tensor? lengths) "
                   "-> Tensor",
    "soft_sw_param_jacobian": "soft_sw_param_jacobian(Tensor scores, int param_type, float gap, "
                              "float temperature, Tensor? lengths) -> Tensor",
    "soft_sw_backward_full": "soft_sw_backward_full(Tensor scores, Tensor grad_alignment, float gap, "
                             "float temperature, Tensor? lengths) -> (Tensor, Tensor, Tensor)",
    "soft_sw_affine": "soft_sw_affine(Tensor scores, Tensor gap_open, Tensor gap_ext, Tensor temperature, "
                      "Tensor lengths) -> Tensor[]",
    "soft_sw_affine_float": "soft_sw_affine_float(Tensor scores, float gap_open, float gap_ext, "
                            "float temperature, Tensor? lengths) -> Tensor[]",
    "soft_sw_affine_with_grads": "soft_sw_affine_with_grads(Tensor scores, float gap_open, float gap_ext, "
                                 "float temperature, Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor, Tensor)",
    "soft_sw_affine_hvp": "soft_sw_affine_hvp(Tensor scores, Tensor tangent, float gap_open, float gap_ext, "
                          "float temperature, Tensor? lengths) -> Tensor",
    "soft_sw_affine_param_jacobian": "soft_sw_affine_param_jacobian(Tensor scores, int param_type, "
                                     "float gap_open, float gap_ext, float temperature, Tensor? lengths) -> Tensor",
    "soft_sw_affine_backward_full": "soft_sw_affine_backward_full(Tensor scores, Tensor grad_alignment, "
                                    "float gap_open, float gap_ext, float temperature, Tensor? lengths) "
                                    "-> (Tensor, Tensor, Tensor, Tensor)",
    "soft_nw": "soft_nw(Tensor scores, Tensor gap, Tensor temperature, Tensor lengths) -> Tensor[]",
    "soft_nw_float": "soft_nw_float(Tensor scores, float gap, float temperature, Tensor? lengths) -> Tensor[]",
    "soft_nw_with_grads": "soft_nw_with_grads(Tensor scores, float gap, float temperature, Tensor? lengths) "
                          "-> (Tensor, Tensor, Tensor, Tensor)",
    "soft_nw_hvp": "soft_nw_hvp(Tensor scores, Tensor tangent, float gap, float temperature, Tensor? lengths) "
                   "-> Tensor",
    "soft_nw_param_jacobian": "soft_nw_param_jacobian(Tensor scores, int param_type, float gap, "
                              "float temperature, Tensor? lengths) -> Tensor",
    "soft_nw_backward_full": "soft_nw_backward_full(Tensor scores, Tensor grad_alignment, float gap, "
                             "float temperature, Tensor? lengths) -> (Tensor, Tensor, Tensor)",
    "soft_nw_affine": "soft_nw_affine(Tensor scores, Tensor gap_open, Tensor gap_ext, Tensor temperature, "
                      "Tensor lengths) -> Tensor[]",
    "soft_nw_affine_float": "soft_nw_affine_float(Tensor scores, float gap_open, float gap_ext, "
                            "float temperature, Tensor? lengths) -> Tensor[]",
    "soft_nw_affine_with_grads": "soft_nw_affine_with_grads(Tensor scores, float gap_open, float gap_ext, "
                                 "float temperature, Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor, Tensor)",
    "soft_nw_affine_hvp": "soft_nw_affine_hvp(Tensor scores, Tensor tangent, float gap_open, float gap_ext, "
                          "float temperature, Tensor? lengths) -> Tensor",
    "soft_nw_affine_param_jacobian": "soft_nw_affine_param_jacobian(Tensor scores, int param_type, "
                                     "float gap_open, float gap_ext, float temperature, Tensor? lengths) -> Tensor",
    "soft_nw_affine_backward_full": "soft_nw_affine_backward_full(Tensor scores, Tensor grad_alignment, "
                                    "float gap_open, float gap_ext, float temperature, Tensor? lengths) "
                                    "-> (Tensor, Tensor, Tensor, Tensor)",
    # src/sv_linear/registry.cpp:20-25, src/sv_affine/registry.cpp:29-34
    "soft_sv_linear": "soft_sv_linear(Tensor scores, Tensor gap, Tensor temperature, Tensor lengths) -> Tensor[]",
    "soft_sv_linear_float": "soft_sv_linear_float(Tensor scores, float gap, float temperature, "
                            "Tensor? lengths) -> Tensor[]",
    "soft_sv_linear_with_grads": "soft_sv_linear_with_grads(Tensor scores, float gap, float temperature, "
                                 "Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor)",
    "soft_sv_linear_hvp": "soft_sv_linear_hvp(Tensor scores, Tensor tangent, float gap, float temperature, "
                          "Tensor? lengths) -> Tensor",
    "soft_sv_linear_param_jacobian": "soft_sv_linear_param_jacobian(Tensor scores, int param_type, float gap, "
                                     "float temperature, Tensor? lengths) -> Tensor",
    "soft_sv_linear_backward_full": "soft_sv_linear_backward_full(Tensor scores, Tensor grad_alignment, "
                                    "float gap, float temperature, Tensor? lengths) -> (Tensor, Tensor, Tensor)",
    "soft_sv_affine": "soft_sv_affine(Tensor scores, Tensor gap_open, Tensor gap_ext, Tensor temperature, "
                      "Tensor lengths) -> Tensor[]",
    "soft_sv_affine_float": "soft_sv_affine_float(Tensor scores, float gap_open, float gap_ext, "
                            "float temperature, Tensor? lengths) -> Tensor[]",
    "soft_sv_affine_with_grads": "soft_sv_affine_with_grads(Tensor scores, float gap_open, float gap_ext, "
                                 "float temperature, Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor, Tensor)",
    "soft_sv_affine_hvp": "soft_sv_affine_hvp(Tensor scores, Tensor tangent, float gap_open, float gap_ext, "
                          "float temperature, Tensor? lengths) -> Tensor",
    "soft_sv_affine_param_jacobian": "soft_sv_affine_param_jacobian(Tensor scores, int param_type, "
                                     "float gap_open, float gap_ext, float temperature, Tensor? lengths) -> Tensor",
    "soft_sv_affine_backward_full": "soft_sv_affine_backward_full(Tensor scores, Tensor grad_alignment, "
                                    "float gap_open, float gap_ext, float temperature, Tensor? lengths) "
                                    "-> (Tensor, Tensor, Tensor, Tensor)",
}
LEGACY_DEFINED_HERE = []
if DEFINED_HERE:
    for _name, _schema in LEGACY_SCHEMAS.items():
        if not _op_exists(_name):
            _DEF_LIB.define(_schema)
            LEGACY_DEFINED_HERE.append(_name)


def _legacy_with_grads_linear(scores, gap, temperature, lengths):
    ln = _prep(scores, lengths, "sw")
    return tuple(run_linear(scores, ln, gap, temperature))


def _legacy_with_grads_nw(scores, gap, temperature, lengths):
    ln = _prep(scores, lengths, "nw")
    return tuple(run_linear(scores, ln, gap, temperature, family="nw"))


def _legacy_with_grads_sv_affine(scores, gap_open, gap_ext, temperature, lengths):
    ln = _prep(scores, lengths, "sv_affine")
    return tuple(run_affine(scores, ln, gap_open, gap_ext, temperature, family="sv_affine"))


def _legacy_with_grads_sv_linear(scores, gap, temperature, lengths):
    ln = _prep(scores, lengths, "sv_linear")
    v, m, go, ge, gT = run_affine(scores, ln, gap, gap, temperature, family="sv_affine")
    return v, m, go + ge, gT


def _legacy_sv_linear_jacobian(scores, param_type, gap, temperature, lengths):
    if not 0 <= int(param_type) < 2:
        raise RuntimeError("param_type must be 0 or 1")
    return _sv_linear_param(int(param_type))(scores, gap, temperature, lengths)


def _legacy_with_grads_nw_affine(scores, gap_open, gap_ext, temperature, lengths):
    ln = _prep(scores, lengths, "nw_affine")
    return tuple(run_affine(scores, ln, gap_open, gap_ext, temperature, family="nw_affine"))


def _legacy_with_grads_affine(scores, gap_open, gap_ext, temperature, lengths):
    ln = _prep(scores, lengths, "sw_affine")
    return tuple(run_affine(scores, ln, gap_open, gap_ext, temperature))


def _legacy_jacobian(fam, nparams):
    # messages of src/sw/torch_cuda.cpp:528, src/sw_affine/torch_cuda.cpp:591, src/nw/torch_cuda.cpp:519
    msg = "param_type must be 0 or 1" if nparams == 2 else "param_type must be 0, 1, or 2"

    def op(scores, param_type, *rest):
        if not 0 <= int(param_type) < nparams:
            raise RuntimeError(msg)
        *params, lengths = rest
        ln = _prep(scores, lengths, fam)
        return run_param_jacobian(fam, scores, ln, tuple(params), int(param_type))
    return op


LEGACY_IMPLS = {
    "soft_sw_float": sw_forward,
    "soft_sw": sw_forward_t,
    "soft_sw_with_grads": _legacy_with_grads_linear,
    "soft_sw_hvp": sw_marginals_hvp,
    "soft_sw_param_jacobian": _legacy_jacobian("sw", 2),
    "soft_sw_backward_full": sw_marginals_backward,
    "soft_sw_affine_float": sw_affine_forward,
    "soft_sw_affine": sw_affine_forward_t,
    "soft_sw_affine_with_grads": _legacy_with_grads_affine,
    "soft_sw_affine_hvp": sw_affine_marginals_hvp,
    "soft_sw_affine_param_jacobian": _legacy_jacobian("sw_affine", 3),
    "soft_sw_affine_backward_full": sw_affine_marginals_backward,
    "soft_nw_float": nw_forward,
    "soft_nw": nw_forward_t,
    "soft_nw_with_grads": _legacy_with_grads_nw,
    "soft_nw_hvp": nw_marginals_hvp,
    "soft_nw_param_jacobian": _legacy_jacobian("nw", 2),
    "soft_nw_backward_full": nw_marginals_backward,
    "soft_nw_affine_float": nw_affine_forward,
    "soft_nw_affine": nw_affine_forward_t,
    "soft_nw_affine_with_grads": _legacy_with_grads_nw_affine,
    "soft_nw_affine_hvp": nw_affine_marginals_hvp,
    "soft_nw_affine_param_jacobian": _legacy_jacobian("nw_affine", 3),
    "soft_nw_affine_backward_full": nw_affine_marginals_backward,
    "soft_sv_linear_float": sv_linear_forward,
    "soft_sv_linear": sv_linear_forward_t,
    "soft_sv_linear_with_grads": _legacy_with_grads_sv_linear,
    "soft_sv_linear_hvp": sv_linear_marginals_hvp,
    "soft_sv_linear_param_jacobian": _legacy_sv_linear_jacobian,
    "soft_sv_linear_backward_full": sv_linear_marginals_backward,
    "soft_sv_affine_float": sv_affine_forward,
    "soft_sv_affine": sv_affine_forward_t,
    "soft_sv_affine_with_grads": _legacy_with_grads_sv_affine,
    "soft_sv_affine_hvp": sv_affine_marginals_hvp,
    "soft_sv_affine_param_jacobian": _legacy_jacobian("sv_affine", 3),
    "soft_sv_affine_backward_full": sv_affine_marginals_backward,
}
for _name in LEGACY_DEFINED_HERE:
    _IMPL_LIB.impl(_name, LEGACY_IMPLS[_name], "CUDA")
for _name, _fam, _t in (("soft_sw_float", "sw", False), ("soft_sw", "sw", True),
                        ("soft_sw_affine_float", "sw_affine", False), ("soft_sw_affine", "sw_affine", True),
                        ("soft_nw_float", "nw", False), ("soft_nw", "nw", True),
                        ("soft_nw_affine_float", "nw_affine", False),
                        ("soft_nw_affine", "nw_affine", True),
                        ("soft_sv_linear_float", "sv_linear", False), ("soft_sv_linear", "sv_linear", True),
                        ("soft_sv_affine_float", "sv_affine", False), ("soft_sv_affine", "sv_affine", True)):
    if _name in LEGACY_DEFINED_HERE:   # differentiable like the reference (AutogradCUDA)
        _IMPL_LIB.impl(_name, _autograd_forward(_fam, _t), "AutogradCUDA")


# ---------------------------------------------------------------------------
# build-owned ops (namespace orihime_b200, no reference counterpart)
# ---------------------------------------------------------------------------
# Value only: the forward wavefront without map or gradients, for scoring
# under no_grad (the reference's forward ops always run forward + backward).

OWN_SCHEMAS = {
    "sw_value": "sw_value(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor",
    "sw_affine_value": "sw_affine_value(Tensor scores, float gap_open, float gap_ext, float temp, "
                       "Tensor? lengths) -> Tensor",
    "nw_value": "nw_value(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor",
    "nw_affine_value": "nw_affine_value(Tensor scores, float gap_open, float gap_ext, float temp, "
                       "Tensor? lengths) -> Tensor",
    "sv_linear_value": "sv_linear_value(Tensor scores, float gap, float temp, Tensor? lengths) -> Tensor",
    "sv_affine_value": "sv_affine_value(Tensor scores, float gap_open, float gap_ext, float temp, "
                       "Tensor? lengths) -> Tensor",
    # value, map and dS/dparameters from ONE forward + adjoint call (the
    # reference's forward op and its value_grad_params op each run both passes)
    "sw_forward_with_grads": "sw_forward_with_grads(Tensor scores, float gap, float temp, "
                             "Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor)",
    "sw_affine_forward_with_grads": "sw_affine_forward_with_grads(Tensor scores, float gap_open, "
                                    "float gap_ext, float temp, Tensor? lengths) -> "
                                    "(Tensor, Tensor, Tensor, Tensor, Tensor)",
    "nw_forward_with_grads": "nw_forward_with_grads(Tensor scores, float gap, float temp, "
                             "Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor)",
    "nw_affine_forward_with_grads": "nw_affine_forward_with_grads(Tensor scores, float gap_open, "
                                    "float gap_ext, float temp, Tensor? lengths) -> "
                                    "(Tensor, Tensor, Tensor, Tensor, Tensor)",
    "sv_linear_forward_with_grads": "sv_linear_forward_with_grads(Tensor scores, float gap, float temp, "
                                    "Tensor? lengths) -> (Tensor, Tensor, Tensor, Tensor)",
    "sv_affine_forward_with_grads": "sv_affine_forward_with_grads(Tensor scores, float gap_open, "
                                    "float gap_ext, float temp, Tensor? lengths) -> "
                                    "(Tensor, Tensor, Tensor, Tensor, Tensor)",
}
_OWN_LIB = torch.library.Library("orihime_b200", "DEF")
for _name, _schema in OWN_SCHEMAS.items():
    _OWN_LIB.define(_schema)


def _own_sw_value(scores, gap, temp, lengths):
    ln = _prep(scores, lengths, "sw")
    return run_value("sw", scores, ln, (gap, temp))


def _own_sw_affine_value(scores, gap_open, gap_ext, temp, lengths):
    ln = _prep(scores, lengths, "sw_affine")
    return run_value("sw_affine", scores, ln, (gap_open, gap_ext, temp))


def _own_nw_value(scores, gap, temp, lengths):
    ln = _prep(scores, lengths, "nw")
    return run_value("nw", scores, ln, (gap, temp))


_OWN_LIB.impl("sw_value", _own_sw_value, "CUDA")
_OWN_LIB.impl("sw_affine_value", _own_sw_affine_value, "CUDA")
def _own_nw_affine_value(scores, gap_open, gap_ext, temp, lengths):
    ln = _prep(scores, lengths, "nw_affine")
    return run_value("nw_affine", scores, ln, (gap_open, gap_ext, temp))


_OWN_LIB.impl("nw_value", _own_nw_value, "CUDA")
def _own_sv_linear_value(scores, gap, temp, lengths):
    ln = _prep(scores, lengths, "sv_linear")
    return run_value("sv_linear", scores, ln, (gap, temp))


def _own_sv_affine_value(scores, gap_open, gap_ext, temp, lengths):
    ln = _prep(scores, lengths, "sv_affine")
    return run_value("sv_affine", scores, ln, (gap_open, gap_ext, temp))


_OWN_LIB.impl("nw_affine_value", _own_nw_affine_value, "CUDA")
_OWN_LIB.impl("sv_linear_value", _own_sv_linear_value, "CUDA")
_OWN_LIB.impl("sv_affine_value", _own_sv_affine_value, "CUDA")


def _own_linear_with_grads(fam):
    def impl(scores, gap, temp, lengths):
        ln = _prep(scores, lengths, fam)
        if fam == "sv_linear":   # the Saigo-Vert affine model with gap_open = gap_ext = gap
            v, m, go, ge, gT = run_affine(scores, ln, gap, gap, temp, family="sv_affine")
            return v, m, go + ge, gT
        v, m, gg, gT = run_linear(scores, ln, gap, temp, family=fam)
        return v, m, gg, gT
    return impl


def _own_affine_with_grads(fam):
    def impl(scores, gap_open, gap_ext, temp, lengths):
        ln = _prep(scores, lengths, fam)
        return run_affine(scores, ln, gap_open, gap_ext, temp, family=fam)
    return impl


for _fam_name in ("sw", "nw", "sv_linear"):
    _OWN_LIB.impl(f"{_fam_name}_forward_with_grads", _own_linear_with_grads(_fam_name), "CUDA")
for _fam_name in ("sw_affine", "nw_affine", "sv_affine"):
    _OWN_LIB.impl(f"{_fam_name}_forward_with_grads", _own_affine_with_grads(_fam_name), "CUDA")

# Meta shapes, FP32 autocast and vmap rules for the ops defined here (when the
# reference extension defined them, its own Python package registers these).
from . import _registrations  # noqa: E402

_registrations.register(DEFINED_HERE)
_registrations.register(list(OWN_SCHEMAS), namespace="orihime_b200")


def _tell_reference_loader() -> None:
    """The reference's loader looks up a CUDA kernel for ``orihime::sw_forward``
    once, when its extension loads, and keeps the answer
    (orihime/_ops.py:42-47, :92); a build of it without CUDA keeps False and
    then refuses CUDA tensors (:161-170).  Once the kernels above are
    registered on its schemas, the answer is True."""
    import sys

    ref = sys.modules.get("orihime._ops")
    if ref is None or getattr(ref, "_cuda_dispatch_available", None) is not False:
        return
    if torch._C._dispatch_has_kernel_for_dispatch_key("orihime::sw_forward", "CUDA"):
        ref._cuda_dispatch_available = True


_tell_reference_loader()
