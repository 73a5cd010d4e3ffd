"""ctypes binding of the CUDA library ``_swb.so`` (C ABI: include/orihime_b200.h).

The library is required: there is no CPU or pure-PyTorch fallback.  Importing
the op layer on a machine without the built library raises ImportError with
the build command.
"""

from __future__ import annotations

import ctypes
import os

_SO = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_swb.so")

ABI_VERSION = 2

DOMAIN_AUTO, DOMAIN_LOG, DOMAIN_LINEAR = 0, 1, 2

OK = 0
ERR_ARG = -1
ERR_WORKSPACE = -2
ERR_CUDA = -3

STATUS_WAIT_TIMEOUT = 1
STATUS_BAD_LENGTHS = 2
STATUS_BAD_PARAMS = 4


class Options(ctypes.Structure):
    """Mirror of ``swb_options``."""

    _fields_ = [
        ("max_ctas", ctypes.c_int),
        ("spin_limit_ns", ctypes.c_ulonglong),
        ("fault_inject", ctypes.c_int),
        ("split_event", ctypes.c_void_p),
        ("cols_per_lane", ctypes.c_int),
        ("domain", ctypes.c_int),
        ("params_device", ctypes.c_void_p),
    ]


_lib = None


def path() -> str:
    return _SO


def load() -> ctypes.CDLL:
    """Load (once) and return the CUDA library, or raise ImportError."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_SO):
        raise ImportError(
            f"orihime_b200 CUDA library not found at {_SO}; build it with "
            "`python orihime_b200/build.py` (needs nvcc)"
        )
    lib = ctypes.CDLL(_SO)
    vp, sz, i, f = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_float
    lib.swb_abi_version.restype = i
    lib.swb_error_string.restype = ctypes.c_char_p
    lib.swb_error_string.argtypes = [i]
    lib.swb_sw_affine_workspace_bytes.restype = sz
    lib.swb_sw_affine_workspace_bytes.argtypes = [i, i, i]
    lib.swb_sw_workspace_bytes.restype = sz
    lib.swb_sw_workspace_bytes.argtypes = [i, i, i]
    lib.swb_sw_affine_forward.restype = i
    lib.swb_sw_affine_forward.argtypes = [vp, vp, i, i, i, f, f, f, vp, vp, vp, vp, vp, vp, sz,
                                          vp, ctypes.POINTER(Options)]
    lib.swb_sw_affine_forward_static.restype = i
    lib.swb_sw_affine_forward_static.argtypes = [vp, vp, i, i, i, f, f, f, vp, vp, vp, vp, vp,
                                                 vp, ctypes.POINTER(Options)]
    lib.swb_sw_forward.restype = i
    lib.swb_sw_forward.argtypes = [vp, vp, i, i, i, f, f, vp, vp, vp, vp, vp, sz, vp,
                                   ctypes.POINTER(Options)]
    lib.swb_read_status.restype = i
    lib.swb_read_status.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_uint)]
    lib.swb_static_read_status.restype = i
    lib.swb_static_read_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint)]
    ll = ctypes.c_longlong
    lib.swb_ragged_plan.restype = i
    lib.swb_ragged_plan.argtypes = [i, i, vp, vp, i, vp, sz, ctypes.POINTER(sz), ctypes.POINTER(sz)]
    lib.swb_sw_affine_ragged.restype = i
    lib.swb_sw_affine_ragged.argtypes = [vp, vp, vp, f, f, f, vp, vp, vp, vp, vp, vp, sz, vp,
                                         ctypes.POINTER(Options)]
    lib.swb_sw_ragged.restype = i
    lib.swb_sw_ragged.argtypes = [vp, vp, vp, f, f, vp, vp, vp, vp, vp, sz, vp,
                                  ctypes.POINTER(Options)]
    del ll
    lib.swb_sw_affine_aux_workspace_bytes.restype = sz
    lib.swb_sw_affine_aux_workspace_bytes.argtypes = [i, i, i]
    lib.swb_sw_aux_workspace_bytes.restype = sz
    lib.swb_sw_aux_workspace_bytes.argtypes = [i, i, i]
    lib.swb_sw_affine_aux_workspace_bytes_for.restype = sz
    lib.swb_sw_affine_aux_workspace_bytes_for.argtypes = [i, i, i, f, f, f]
    lib.swb_sw_aux_workspace_bytes_for.restype = sz
    lib.swb_sw_aux_workspace_bytes_for.argtypes = [i, i, i, f, f]
    lib.swb_sw_affine_value_workspace_bytes.restype = sz
    lib.swb_sw_affine_value_workspace_bytes.argtypes = [i, i, i]
    lib.swb_sw_value_workspace_bytes.restype = sz
    lib.swb_sw_value_workspace_bytes.argtypes = [i, i, i]
    lib.swb_scan_scores.restype = i
    lib.swb_scan_scores.argtypes = [vp, i, ctypes.c_longlong, f, f, vp, vp, vp]
    lib.swb_sw_affine_ragged_value.restype = i
    lib.swb_sw_affine_ragged_value.argtypes = [vp, vp, vp, f, f, f, vp, vp, sz, vp]
    lib.swb_sw_ragged_value.restype = i
    lib.swb_sw_ragged_value.argtypes = [vp, vp, vp, f, f, vp, vp, sz, vp]
    lib.swb_sw_affine_value.restype = i
    lib.swb_sw_affine_value.argtypes = [vp, vp, i, i, i, f, f, f, vp, vp, sz, vp]
    lib.swb_sw_value.restype = i
    lib.swb_sw_value.argtypes = [vp, vp, i, i, i, f, f, vp, vp, sz, vp]
    lib.swb_sw_affine_hvp.restype = i
    lib.swb_sw_affine_hvp.argtypes = [vp, vp, vp, i, i, i, f, f, f, vp, vp, vp, sz, vp]
    lib.swb_sw_affine_param_jacobian.restype = i
    lib.swb_sw_affine_param_jacobian.argtypes = [vp, vp, i, i, i, f, f, f, i, vp, vp, sz, vp]
    lib.swb_sw_hvp.restype = i
    lib.swb_sw_hvp.argtypes = [vp, vp, vp, i, i, i, f, f, vp, vp, vp, sz, vp]
    lib.swb_sw_param_jacobian.restype = i
    lib.swb_sw_param_jacobian.argtypes = [vp, vp, i, i, i, f, f, i, vp, vp, sz, vp]
    lib.swb_nw_workspace_bytes.restype = sz
    lib.swb_nw_workspace_bytes.argtypes = [i, i, i]
    lib.swb_nw_forward.restype = i
    lib.swb_nw_forward.argtypes = [vp, vp, i, i, i, f, f, vp, vp, vp, vp, vp, sz, vp,
                                   ctypes.POINTER(Options)]
    lib.swb_nw_value_workspace_bytes.restype = sz
    lib.swb_nw_value_workspace_bytes.argtypes = [i, i, i]
    lib.swb_nw_value.restype = i
    lib.swb_nw_value.argtypes = [vp, vp, i, i, i, f, f, vp, vp, sz, vp]
    lib.swb_nw_aux_workspace_bytes.restype = sz
    lib.swb_nw_aux_workspace_bytes.argtypes = [i, i, i]
    lib.swb_nw_hvp.restype = i
    lib.swb_nw_hvp.argtypes = [vp, vp, vp, i, i, i, f, f, vp, vp, vp, sz, vp]
    lib.swb_nw_param_jacobian.restype = i
    lib.swb_nw_param_jacobian.argtypes = [vp, vp, i, i, i, f, f, i, vp, vp, sz, vp]
    lib.swb_nw_ragged.restype = i
    lib.swb_nw_ragged.argtypes = [vp, vp, vp, f, f, vp, vp, vp, vp, vp, sz, vp, ctypes.POINTER(Options)]
    lib.swb_nw_ragged_value.restype = i
    lib.swb_nw_ragged_value.argtypes = [vp, vp, vp, f, f, vp, vp, sz, vp]
    lib.swb_nw_affine_workspace_bytes.restype = sz
    lib.swb_nw_affine_workspace_bytes.argtypes = [i, i, i]
    lib.swb_nw_affine_forward.restype = i
    lib.swb_nw_affine_forward.argtypes = [vp, vp, i, i, i, f, f, f, vp, vp, vp, vp, vp, vp, sz,
                                          vp, ctypes.POINTER(Options)]
    lib.swb_nw_affine_value_workspace_bytes.restype = sz
    lib.swb_nw_affine_value_workspace_bytes.argtypes = [i, i, i]
    lib.swb_nw_affine_value.restype = i
    lib.swb_nw_affine_value.argtypes = [vp, vp, i, i, i, f, f, f, vp, vp, sz, vp]
    lib.swb_nw_affine_ragged.restype = i
    lib.swb_nw_affine_ragged.argtypes = [vp, vp, vp, f, f, f, vp, vp, vp, vp, vp, vp, sz, vp,
                                         ctypes.POINTER(Options)]
    lib.swb_nw_affine_ragged_value.restype = i
    lib.swb_nw_affine_ragged_value.argtypes = [vp, vp, vp, f, f, f, vp, vp, sz, vp]
    lib.swb_nw_affine_aux_workspace_bytes.restype = sz
    lib.swb_nw_affine_aux_workspace_bytes.argtypes = [i, i, i]
    lib.swb_nw_affine_hvp.restype = i
    lib.swb_nw_affine_hvp.argtypes = [vp, vp, vp, i, i, i, f, f, f, vp, vp, vp, sz, vp]
    lib.swb_nw_affine_param_jacobian.restype = i
    lib.swb_nw_affine_param_jacobian.argtypes = [vp, vp, i, i, i, f, f, f, i, vp, vp, sz, vp]
    lib.swb_sv_affine_workspace_bytes.restype = sz
    lib.swb_sv_affine_workspace_bytes.argtypes = [i, i, i]
    lib.swb_sv_affine_forward.restype = i
    lib.swb_sv_affine_forward.argtypes = [vp, vp, i, i, i, f, f, f, vp, vp, vp, vp, vp, vp, sz,
                                          vp, ctypes.POINTER(Options)]
    lib.swb_sv_affine_value_workspace_bytes.restype = sz
    lib.swb_sv_affine_value_workspace_bytes.argtypes = [i, i, i]
    lib.swb_sv_affine_value.restype = i
    lib.swb_sv_affine_value.argtypes = [vp, vp, i, i, i, f, f, f, vp, vp, sz, vp]
    lib.swb_sv_affine_ragged.restype = i
    lib.swb_sv_affine_ragged.argtypes = [vp, vp, vp, f, f, f, vp, vp, vp, vp, vp, vp, sz, vp,
                                         ctypes.POINTER(Options)]
    lib.swb_sv_affine_ragged_value.restype = i
    lib.swb_sv_affine_ragged_value.argtypes = [vp, vp, vp, f, f, f, vp, vp, sz, vp]
    lib.swb_sv_affine_aux_workspace_bytes.restype = sz
    lib.swb_sv_affine_aux_workspace_bytes.argtypes = [i, i, i]
    lib.swb_sv_affine_hvp.restype = i
    lib.swb_sv_affine_hvp.argtypes = [vp, vp, vp, i, i, i, f, f, f, vp, vp, vp, sz, vp]
    lib.swb_sv_affine_param_jacobian.restype = i
    lib.swb_sv_affine_param_jacobian.argtypes = [vp, vp, i, i, i, f, f, f, i, vp, vp, sz, vp]
    lib.swb_sw_affine_checkpoint_workspace_bytes.restype = sz
    lib.swb_sw_affine_checkpoint_workspace_bytes.argtypes = [i, i, i, i]
    lib.swb_sw_checkpoint_workspace_bytes.restype = sz
    lib.swb_sw_checkpoint_workspace_bytes.argtypes = [i, i, i, i]
    lib.swb_sw_affine_checkpoint.restype = i
    lib.swb_sw_affine_checkpoint.argtypes = [vp, vp, i, i, i, f, f, f, i, vp, vp, sz, vp]
    lib.swb_sw_affine_adjoint.restype = i
    lib.swb_sw_affine_adjoint.argtypes = [vp, vp, i, i, i, f, f, f, i, vp, vp, vp, vp, vp, vp, sz, vp]
    lib.swb_sw_checkpoint.restype = i
    lib.swb_sw_checkpoint.argtypes = [vp, vp, i, i, i, f, f, i, vp, vp, sz, vp]
    lib.swb_sw_adjoint.restype = i
    lib.swb_sw_adjoint.argtypes = [vp, vp, i, i, i, f, f, i, vp, vp, vp, vp, vp, sz, vp]
    lib.swb_cols_per_lane.restype = i
    lib.swb_cols_per_lane.argtypes = [i, i, f, f, f]
    lib.swb_mufu_probe.restype = i
    lib.swb_mufu_probe.argtypes = [vp, i, i, vp]
    got = lib.swb_abi_version()
    if got != ABI_VERSION:
        raise ImportError(f"orihime_b200 library ABI {got} != expected {ABI_VERSION}; rebuild it")
    _lib = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc != OK:
        msg = load().swb_error_string(rc).decode()
        raise RuntimeError(f"{what} failed: {msg} (code {rc})")
