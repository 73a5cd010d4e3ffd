"""orihime_b200: B200-native (sm_100a) soft Smith-Waterman and soft
Needleman-Wunsch for megure-labs/orihime.

Importing the package registers CUDA implementations of the
``torch.ops.orihime`` soft Smith-Waterman operators (linear and affine gaps)
soft Needleman-Wunsch operators (global alignment, linear and affine gaps)
and Saigo-Vert operators (linear and affine gaps), and
exposes the public functions with orihime's signatures, plus the named
operations ``ops.<family>.forward / backward / sensitivity``.
"""

from . import _lib as _lib
from . import _ops as _ops
from .nw import nw, nw_affine, nw_affine_entropy, nw_affine_value, nw_entropy, nw_value
from .sv import (sv, sv_affine, sv_affine_entropy, sv_affine_value, sv_entropy, sv_linear,
                 sv_linear_entropy, sv_linear_value, sv_value)
from .sw import sw, sw_affine, sw_affine_entropy, sw_affine_value, sw_entropy, sw_value
from . import ops as ops
from . import _pt2 as _pt2
from . import raw as raw

__version__ = "0.1.0"

__all__ = ["sw", "sw_value", "sw_entropy", "sw_affine", "sw_affine_value", "sw_affine_entropy",
           "nw", "nw_value", "nw_entropy", "nw_affine", "nw_affine_value", "nw_affine_entropy",
           "sv", "sv_value", "sv_entropy", "sv_affine", "sv_affine_value", "sv_affine_entropy", "ops"]
