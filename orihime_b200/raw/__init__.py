"""The low-level tier (orihime/raw/__init__.py): per family, no-graph
parameter VJPs (vjp_fields, vjp_one, vjp) and the named kernel bindings
(forward, forward_t, value_grad_params, marginals_backward, marginals_hvp,
marginals_grad_<param>)."""

from ._base import VJPFields
from . import nw as nw
from . import nw_affine as nw_affine
from . import sv_affine as sv_affine
from . import sv_linear as sv_linear
from . import sw as sw
from . import sw_affine as sw_affine

__all__ = ["VJPFields", "sw", "sw_affine", "sv_linear", "sv_affine", "nw", "nw_affine"]
