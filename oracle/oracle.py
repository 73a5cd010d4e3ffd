"""TEST INFRASTRUCTURE ONLY: the CPU oracle for the soft Smith-Waterman path.

Two libraries sit behind this module, both built by ``oracle/Makefile``:

* ``_oracle.so`` -- our C restatement of the reference recurrences
  (``sw_oracle_impl.h``), in float (``_f32``: operation-for-operation mirror of
  the reference CPU kernels) and double (``_f64``: the FP64 truth).
* ``_ref/libref_swcpu.so`` -- the reference's own CPU kernels
  (``src/sw/kernels_cpu.cpp``, ``src/sw_affine/kernels_cpu.cpp``), compiled
  from their sources.  Present wherever the Makefile's ``ref`` target ran.
* ``_ref/libref_swcuda.so`` -- the reference's own CUDA extension (target
  ``refcuda``); ``ref_cuda_path()`` gives its path for a GPU test that loads it.

Only ``tests/``, ``bench.py``'s CPU legs and ``__graft_entry__.smoke()`` may
import this module.  The product never does.

All arrays use the reference's padded layout: scores ``[B, L1, L2]`` C-order,
lengths ``[B, 2]`` int32 (or ``None`` for full lengths).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "_oracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libref_swcpu.so")

_F = ctypes.c_float
_D = ctypes.c_double
_I = ctypes.c_int
_P = ctypes.c_void_p


# Root of the reference sources (megure-labs/orihime) that the oracle libraries are
# compiled from: the environment variable ORIHIME_REFERENCE, default
# /root/reference.  On a machine without those sources only the prebuilt
# libraries under _ref/ are used.
REFERENCE = os.environ.get("ORIHIME_REFERENCE", "/root/reference")


def build(ref: bool = True) -> None:
    """Compile the oracle (and the reference CPU kernels and CUDA extension
    when their sources exist under ``REFERENCE``)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    if ref and os.path.isdir(os.path.join(REFERENCE, "src")):
        for target in ("ref", "refcuda"):
            subprocess.run(["make", "-s", "-C", _HERE, target, f"REF={REFERENCE}"], check=True)


def ref_cuda_path() -> Optional[str]:
    p = os.path.join(_HERE, "_ref", "libref_swcuda.so")
    return p if os.path.exists(p) else None


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_ORACLE_SO):
            build(ref=False)
        _lib = ctypes.CDLL(_ORACLE_SO)
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(_REF_SO)
    return _ref


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_P)


def _prep(scores, lengths, dtype):
    s = np.ascontiguousarray(scores, dtype=dtype)
    assert s.ndim == 3, "scores must be [B, L1, L2]"
    ln = None if lengths is None else np.ascontiguousarray(lengths, dtype=np.int32)
    return s, ln


def _scal(dtype):
    return _F if dtype == np.float32 else _D


def _sfx(dtype):
    return "_f32" if dtype == np.float32 else "_f64"


# ---------------------------------------------------------------------------
# our restatement
# ---------------------------------------------------------------------------

def affine(scores, lengths, gap_open, gap_ext, temp, dtype=np.float32) -> dict:
    """value [B], map [B,L1,L2], grad_open/grad_ext/grad_temp [B]."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = {k: np.zeros(B, dtype) for k in ("value", "grad_open", "grad_ext", "grad_temp")}
    out["map"] = np.zeros_like(s)
    fn = getattr(lib(), "oracle_sw_affine_forward" + _sfx(dtype))
    sc = _scal(dtype)
    rc = fn(_ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap_open), sc(gap_ext), sc(temp),
            _ptr(out["value"]), _ptr(out["map"]), _ptr(out["grad_open"]),
            _ptr(out["grad_ext"]), _ptr(out["grad_temp"]))
    assert rc == 0
    return out


def affine_hvp(scores, v, lengths, gap_open, gap_ext, temp, dtype=np.float32) -> np.ndarray:
    s, ln = _prep(scores, lengths, dtype)
    vv = np.ascontiguousarray(v, dtype=dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_sw_affine_hvp" + _sfx(dtype))(
        _ptr(s), _ptr(vv), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap_open), sc(gap_ext),
        sc(temp), _ptr(out))
    assert rc == 0
    return out


def affine_param_grad(scores, lengths, gap_open, gap_ext, temp, param: int,
                      dtype=np.float32) -> np.ndarray:
    """d(map)/d(theta); param 0 = gap_open, 1 = gap_ext, 2 = temperature."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_sw_affine_param_grad" + _sfx(dtype))(
        _ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap_open), sc(gap_ext), sc(temp),
        _I(param), _ptr(out))
    assert rc == 0
    return out


def linear(scores, lengths, gap, temp, dtype=np.float32) -> dict:
    """value [B], map [B,L1,L2], grad_gap/grad_temp [B]."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = {k: np.zeros(B, dtype) for k in ("value", "grad_gap", "grad_temp")}
    out["map"] = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_sw_linear_forward" + _sfx(dtype))(
        _ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap), sc(temp), _ptr(out["value"]),
        _ptr(out["map"]), _ptr(out["grad_gap"]), _ptr(out["grad_temp"]))
    assert rc == 0
    return out


def linear_hvp(scores, v, lengths, gap, temp, dtype=np.float32) -> np.ndarray:
    s, ln = _prep(scores, lengths, dtype)
    vv = np.ascontiguousarray(v, dtype=dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_sw_linear_hvp" + _sfx(dtype))(
        _ptr(s), _ptr(vv), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap), sc(temp), _ptr(out))
    assert rc == 0
    return out


def linear_param_grad(scores, lengths, gap, temp, param: int, dtype=np.float32) -> np.ndarray:
    """d(map)/d(theta); param 0 = gap, 1 = temperature."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_sw_linear_param_grad" + _sfx(dtype))(
        _ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap), sc(temp), _I(param), _ptr(out))
    assert rc == 0
    return out


def nw(scores, lengths, gap, temp, dtype=np.float32) -> dict:
    """Global alignment (Needleman-Wunsch, linear gap): value [B], map,
    grad_gap/grad_temp [B]."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = {k: np.zeros(B, dtype) for k in ("value", "grad_gap", "grad_temp")}
    out["map"] = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_nw_linear_forward" + _sfx(dtype))(
        _ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap), sc(temp), _ptr(out["value"]),
        _ptr(out["map"]), _ptr(out["grad_gap"]), _ptr(out["grad_temp"]))
    assert rc == 0
    return out


def nw_hvp(scores, v, lengths, gap, temp, dtype=np.float32) -> np.ndarray:
    s, ln = _prep(scores, lengths, dtype)
    vv = np.ascontiguousarray(v, dtype=dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_nw_linear_hvp" + _sfx(dtype))(
        _ptr(s), _ptr(vv), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap), sc(temp), _ptr(out))
    assert rc == 0
    return out


def nw_param_grad(scores, lengths, gap, temp, param: int, dtype=np.float32) -> np.ndarray:
    """d(map)/d(theta) of the global alignment; param 0 = gap, 1 = temperature."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_nw_linear_param_grad" + _sfx(dtype))(
        _ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap), sc(temp), _I(param), _ptr(out))
    assert rc == 0
    return out


def nw_affine(scores, lengths, gap_open, gap_ext, temp, dtype=np.float32) -> dict:
    """Global alignment with affine gaps: value [B], map, grad_open/grad_ext/
    grad_temp [B]."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = {k: np.zeros(B, dtype) for k in ("value", "grad_open", "grad_ext", "grad_temp")}
    out["map"] = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_nw_affine_forward" + _sfx(dtype))(
        _ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap_open), sc(gap_ext), sc(temp),
        _ptr(out["value"]), _ptr(out["map"]), _ptr(out["grad_open"]), _ptr(out["grad_ext"]),
        _ptr(out["grad_temp"]))
    assert rc == 0
    return out


def nw_affine_hvp(scores, v, lengths, gap_open, gap_ext, temp, dtype=np.float32) -> np.ndarray:
    s, ln = _prep(scores, lengths, dtype)
    vv = np.ascontiguousarray(v, dtype=dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_nw_affine_hvp" + _sfx(dtype))(
        _ptr(s), _ptr(vv), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap_open), sc(gap_ext), sc(temp),
        _ptr(out))
    assert rc == 0
    return out


def nw_affine_param_grad(scores, lengths, gap_open, gap_ext, temp, param: int,
                         dtype=np.float32) -> np.ndarray:
    """d(map)/d(theta); param 0 = gap_open, 1 = gap_ext, 2 = temperature."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_nw_affine_param_grad" + _sfx(dtype))(
        _ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap_open), sc(gap_ext), sc(temp), _I(param),
        _ptr(out))
    assert rc == 0
    return out


def sv(scores, lengths, gap_open, gap_ext, temp, linear=False, dtype=np.float32) -> dict:
    """Saigo-Vert local alignment: value [B], map, grad_open/grad_ext/grad_temp
    [B]; linear=True (go = ge = gap) reports dS/dgap as grad_open."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = {k: np.zeros(B, dtype) for k in ("value", "grad_open", "grad_ext", "grad_temp")}
    out["map"] = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_sv_forward" + _sfx(dtype))(
        _ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap_open), sc(gap_ext), sc(temp), _I(int(linear)),
        _ptr(out["value"]), _ptr(out["map"]), _ptr(out["grad_open"]), _ptr(out["grad_ext"]),
        _ptr(out["grad_temp"]))
    assert rc == 0
    return out


def sv_hvp(scores, v, lengths, gap_open, gap_ext, temp, dtype=np.float32) -> np.ndarray:
    s, ln = _prep(scores, lengths, dtype)
    vv = np.ascontiguousarray(v, dtype=dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    rc = getattr(lib(), "oracle_sv_hvp" + _sfx(dtype))(
        _ptr(s), _ptr(vv), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap_open), sc(gap_ext), sc(temp),
        _ptr(out))
    assert rc == 0
    return out


def sv_param_grad(scores, lengths, gap_open, gap_ext, temp, param: int, linear=False,
                  dtype=np.float32) -> np.ndarray:
    """d(map)/d(theta); affine: 0 = gap_open, 1 = gap_ext, 2 = temperature;
    linear (go = ge = gap): 0 = gap, 1 = temperature."""
    s, ln = _prep(scores, lengths, dtype)
    B, L1, L2 = s.shape
    out = np.zeros_like(s)
    sc = _scal(dtype)
    pt = ((3, 2)[param]) if linear else param
    rc = getattr(lib(), "oracle_sv_param_grad" + _sfx(dtype))(
        _ptr(s), _ptr(ln), _I(B), _I(L1), _I(L2), sc(gap_open), sc(gap_ext), sc(temp),
        _I(int(linear)), _I(pt), _ptr(out))
    assert rc == 0
    return out


# ---------------------------------------------------------------------------
# the reference's own CPU kernels (src/sw*/kernels_cpu.cpp,
# src/nw*/kernels_cpu.cpp, src/sv_*/kernels_cpu.cpp), float32 only
# ---------------------------------------------------------------------------

def _full_lengths(B, L1, L2, ln):
    if ln is not None:
        return ln
    return np.tile(np.array([[L1, L2]], np.int32), (B, 1))


def ref_affine(scores, lengths, gap_open, gap_ext, temp) -> dict:
    """sw_affine_forward_cpu + sw_affine_backward_cpu (kernels_cpu.cpp:94, :201)."""
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = 3 * (L1 + 1) * (L2 + 1)
    alpha = np.empty((B, n_alpha), np.float32)
    beta = np.empty((B, n_alpha), np.float32)
    out = {k: np.zeros(B, np.float32) for k in ("value", "grad_open", "grad_ext", "grad_temp")}
    out["map"] = np.zeros_like(s)
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap_open), _F(gap_ext), _F(temp))
    r.sw_affine_forward_cpu(_ptr(s), _ptr(alpha), _ptr(out["value"]), _ptr(ln), *a)
    r.sw_affine_backward_cpu(_ptr(alpha), _ptr(s), _ptr(out["value"]), _ptr(beta),
                             _ptr(out["map"]), _ptr(out["grad_open"]), _ptr(out["grad_ext"]),
                             _ptr(out["grad_temp"]), _ptr(ln), *a)
    return out


def ref_affine_hvp(scores, v, lengths, gap_open, gap_ext, temp) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    vv = np.ascontiguousarray(v, dtype=np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = 3 * (L1 + 1) * (L2 + 1)
    alpha = np.empty((B, n_alpha), np.float32)
    da = np.empty((B, n_alpha), np.float32)
    dbe = np.empty((B, n_alpha), np.float32)
    part = np.zeros(B, np.float32)
    dpart = np.zeros(B, np.float32)
    out = np.zeros_like(s)
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap_open), _F(gap_ext), _F(temp))
    r.sw_affine_forward_cpu(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    r.sw_affine_hvp_cpu(_ptr(alpha), _ptr(s), _ptr(part), _ptr(vv), _ptr(da), _ptr(dpart),
                        _ptr(dbe), _ptr(out), _ptr(ln), *a)
    return out


def ref_affine_param_grad(scores, lengths, gap_open, gap_ext, temp, param: int) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    base = ref_affine(s, ln, gap_open, gap_ext, temp)
    n_alpha = 3 * (L1 + 1) * (L2 + 1)
    alpha = np.empty((B, n_alpha), np.float32)
    part = np.zeros(B, np.float32)
    U = np.empty((B, n_alpha), np.float32)
    be = np.empty((B, n_alpha), np.float32)
    W = np.empty((B, n_alpha), np.float32)
    out = np.zeros_like(s)
    dS = np.ascontiguousarray(base[("grad_open", "grad_ext", "grad_temp")[param]])
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap_open), _F(gap_ext), _F(temp))
    r.sw_affine_forward_cpu(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    r.sw_affine_param_grad_cpu(_ptr(alpha), _ptr(s), _ptr(part), _ptr(dS), _ptr(U), _ptr(be),
                               _ptr(W), _ptr(out), _ptr(ln), *a, _I(param))
    return out


def ref_linear(scores, lengths, gap, temp) -> dict:
    """sw_regular_forward_cpu + sw_regular_backward_cpu (src/sw/kernels_cpu.cpp:70, :154)."""
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = (L1 + 1) * (L2 + 1)
    alpha = np.empty((B, n_alpha), np.float32)
    beta = np.empty((B, n_alpha), np.float32)
    out = {k: np.zeros(B, np.float32) for k in ("value", "grad_gap", "grad_temp")}
    out["map"] = np.zeros_like(s)
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap), _F(temp))
    r.sw_regular_forward_cpu(_ptr(s), _ptr(alpha), _ptr(out["value"]), _ptr(ln), *a)
    r.sw_regular_backward_cpu(_ptr(alpha), _ptr(s), _ptr(out["value"]), _ptr(beta),
                              _ptr(out["map"]), _ptr(out["grad_gap"]), _ptr(out["grad_temp"]),
                              _ptr(ln), *a)
    return out


def ref_linear_hvp(scores, v, lengths, gap, temp) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    vv = np.ascontiguousarray(v, dtype=np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = (L1 + 1) * (L2 + 1)
    alpha, da, be, dbe = (np.empty((B, n_alpha), np.float32) for _ in range(4))
    part = np.zeros(B, np.float32)
    dpart = np.zeros(B, np.float32)
    out = np.zeros_like(s)
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap), _F(temp))
    r.sw_regular_forward_cpu(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    r.sw_regular_hvp_cpu(_ptr(alpha), _ptr(s), _ptr(part), _ptr(vv), _ptr(da), _ptr(dpart),
                         _ptr(be), _ptr(dbe), _ptr(out), _ptr(ln), *a)
    return out


def ref_linear_param_grad(scores, lengths, gap, temp, param: int) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    base = ref_linear(s, ln, gap, temp)
    n_alpha = (L1 + 1) * (L2 + 1)
    alpha, U, be, W = (np.empty((B, n_alpha), np.float32) for _ in range(4))
    part = np.zeros(B, np.float32)
    out = np.zeros_like(s)
    dS = np.ascontiguousarray(base[("grad_gap", "grad_temp")[param]])
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap), _F(temp))
    r.sw_regular_forward_cpu(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    r.sw_regular_param_grad_cpu(_ptr(alpha), _ptr(s), _ptr(part), _ptr(dS), _ptr(U), _ptr(be),
                                _ptr(W), _ptr(out), _ptr(ln), *a, _I(param))
    return out


def ref_nw(scores, lengths, gap, temp) -> dict:
    """nw_forward_cpu + nw_backward_cpu (src/nw/kernels_cpu.cpp:77, :156)."""
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = (L1 + 1) * (L2 + 1)
    alpha = np.empty((B, n_alpha), np.float32)
    beta = np.empty((B, n_alpha), np.float32)
    out = {k: np.zeros(B, np.float32) for k in ("value", "grad_gap", "grad_temp")}
    out["map"] = np.zeros_like(s)
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap), _F(temp))
    r.nw_forward_cpu(_ptr(s), _ptr(alpha), _ptr(out["value"]), _ptr(ln), *a)
    r.nw_backward_cpu(_ptr(alpha), _ptr(s), _ptr(out["value"]), _ptr(beta), _ptr(out["map"]),
                      _ptr(out["grad_gap"]), _ptr(out["grad_temp"]), _ptr(ln), *a)
    return out


def ref_nw_hvp(scores, v, lengths, gap, temp) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    vv = np.ascontiguousarray(v, dtype=np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = (L1 + 1) * (L2 + 1)
    alpha, da, be, dbe = (np.empty((B, n_alpha), np.float32) for _ in range(4))
    part = np.zeros(B, np.float32)
    dpart = np.zeros(B, np.float32)
    out = np.zeros_like(s)
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap), _F(temp))
    r.nw_forward_cpu(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    r.nw_hvp_cpu(_ptr(alpha), _ptr(s), _ptr(part), _ptr(vv), _ptr(da), _ptr(dpart), _ptr(be),
                 _ptr(dbe), _ptr(out), _ptr(ln), *a)
    return out


def ref_nw_param_grad(scores, lengths, gap, temp, param: int) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    base = ref_nw(s, ln, gap, temp)
    n_alpha = (L1 + 1) * (L2 + 1)
    alpha, U, be, W = (np.empty((B, n_alpha), np.float32) for _ in range(4))
    part = np.zeros(B, np.float32)
    out = np.zeros_like(s)
    dS = np.ascontiguousarray(base[("grad_gap", "grad_temp")[param]])
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap), _F(temp))
    r.nw_forward_cpu(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    r.nw_param_grad_cpu(_ptr(alpha), _ptr(s), _ptr(part), _ptr(dS), _ptr(U), _ptr(be), _ptr(W),
                        _ptr(out), _ptr(ln), *a, _I(param))
    return out


def ref_nw_affine(scores, lengths, gap_open, gap_ext, temp) -> dict:
    """nw_affine_forward_cpu + nw_affine_backward_cpu (src/nw_affine/kernels_cpu.cpp:100, :193)."""
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = 3 * (L1 + 1) * (L2 + 1)
    alpha = np.empty((B, n_alpha), np.float32)
    beta = np.empty((B, n_alpha), np.float32)
    out = {k: np.zeros(B, np.float32) for k in ("value", "grad_open", "grad_ext", "grad_temp")}
    out["map"] = np.zeros_like(s)
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap_open), _F(gap_ext), _F(temp))
    r.nw_affine_forward_cpu(_ptr(s), _ptr(alpha), _ptr(out["value"]), _ptr(ln), *a)
    r.nw_affine_backward_cpu(_ptr(alpha), _ptr(s), _ptr(out["value"]), _ptr(beta), _ptr(out["map"]),
                             _ptr(out["grad_open"]), _ptr(out["grad_ext"]), _ptr(out["grad_temp"]),
                             _ptr(ln), *a)
    return out


def ref_nw_affine_hvp(scores, v, lengths, gap_open, gap_ext, temp) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    vv = np.ascontiguousarray(v, dtype=np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = 3 * (L1 + 1) * (L2 + 1)
    alpha, da, be, dbe = (np.empty((B, n_alpha), np.float32) for _ in range(4))
    part = np.zeros(B, np.float32)
    dpart = np.zeros(B, np.float32)
    out = np.zeros_like(s)
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap_open), _F(gap_ext), _F(temp))
    r.nw_affine_forward_cpu(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    r.nw_affine_hvp_cpu(_ptr(alpha), _ptr(s), _ptr(part), _ptr(vv), _ptr(da), _ptr(dpart), _ptr(be),
                        _ptr(dbe), _ptr(out), _ptr(ln), *a)
    return out


def ref_nw_affine_param_grad(scores, lengths, gap_open, gap_ext, temp, param: int) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = 3 * (L1 + 1) * (L2 + 1)
    alpha, U, be, W = (np.empty((B, n_alpha), np.float32) for _ in range(4))
    part = np.zeros(B, np.float32)
    dS = np.zeros(B, np.float32)
    out = np.zeros_like(s)
    r = ref_lib()
    a = (_I(B), _I(L1), _I(L2), _F(gap_open), _F(gap_ext), _F(temp))
    r.nw_affine_forward_cpu(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    r.nw_affine_param_grad_cpu(_ptr(alpha), _ptr(s), _ptr(part), _ptr(dS), _ptr(U), _ptr(be), _ptr(W),
                               _ptr(out), _ptr(ln), *a, _I(param))
    return out


def _ref_sv_prefix(linear):
    return "sv_linear" if linear else "sv_affine"


def ref_sv(scores, lengths, gap_open, gap_ext, temp, linear=False) -> dict:
    """sv_{affine,linear}_forward_cpu + _backward_cpu (src/sv_*/kernels_cpu.cpp)."""
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = 3 * (L1 + 1) * (L2 + 1)
    alpha = np.empty((B, n_alpha), np.float32)
    beta = np.empty((B, n_alpha), np.float32)
    out = {k: np.zeros(B, np.float32) for k in ("value", "grad_open", "grad_ext", "grad_temp")}
    out["map"] = np.zeros_like(s)
    r = ref_lib()
    pre = _ref_sv_prefix(linear)
    prm = (_F(gap_open), _F(temp)) if linear else (_F(gap_open), _F(gap_ext), _F(temp))
    a = (_I(B), _I(L1), _I(L2), *prm)
    getattr(r, pre + "_forward_cpu")(_ptr(s), _ptr(alpha), _ptr(out["value"]), _ptr(ln), *a)
    grads = ((out["grad_open"], out["grad_temp"]) if linear
             else (out["grad_open"], out["grad_ext"], out["grad_temp"]))
    getattr(r, pre + "_backward_cpu")(_ptr(alpha), _ptr(s), _ptr(out["value"]), _ptr(beta),
                                      _ptr(out["map"]), *map(_ptr, grads), _ptr(ln), *a)
    return out


def ref_sv_hvp(scores, v, lengths, gap_open, gap_ext, temp, linear=False) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    vv = np.ascontiguousarray(v, dtype=np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    n_alpha = 3 * (L1 + 1) * (L2 + 1)
    alpha, da, dbe = (np.empty((B, n_alpha), np.float32) for _ in range(3))
    part = np.zeros(B, np.float32)
    dpart = np.zeros(B, np.float32)
    out = np.zeros_like(s)
    r = ref_lib()
    pre = _ref_sv_prefix(linear)
    prm = (_F(gap_open), _F(temp)) if linear else (_F(gap_open), _F(gap_ext), _F(temp))
    a = (_I(B), _I(L1), _I(L2), *prm)
    getattr(r, pre + "_forward_cpu")(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    getattr(r, pre + "_hvp_cpu")(_ptr(alpha), _ptr(s), _ptr(part), _ptr(vv), _ptr(da), _ptr(dpart),
                                 _ptr(dbe), _ptr(out), _ptr(ln), *a)
    return out


def ref_sv_param_grad(scores, lengths, gap_open, gap_ext, temp, param: int, linear=False) -> np.ndarray:
    s, ln = _prep(scores, lengths, np.float32)
    B, L1, L2 = s.shape
    ln = _full_lengths(B, L1, L2, ln)
    base = ref_sv(s, ln, gap_open, gap_ext, temp, linear)
    key = (("grad_open", "grad_temp") if linear else ("grad_open", "grad_ext", "grad_temp"))[param]
    n_alpha = 3 * (L1 + 1) * (L2 + 1)
    alpha, U, be, W = (np.empty((B, n_alpha), np.float32) for _ in range(4))
    part = np.zeros(B, np.float32)
    out = np.zeros_like(s)
    dS = np.ascontiguousarray(base[key])
    r = ref_lib()
    pre = _ref_sv_prefix(linear)
    prm = (_F(gap_open), _F(temp)) if linear else (_F(gap_open), _F(gap_ext), _F(temp))
    a = (_I(B), _I(L1), _I(L2), *prm)
    getattr(r, pre + "_forward_cpu")(_ptr(s), _ptr(alpha), _ptr(part), _ptr(ln), *a)
    getattr(r, pre + "_param_grad_cpu")(_ptr(alpha), _ptr(s), _ptr(part), _ptr(dS), _ptr(U), _ptr(be),
                                        _ptr(W), _ptr(out), _ptr(ln), *a, _I(param))
    return out
