"""Raw tier of the soft Needleman-Wunsch, affine gaps operator (orihime/raw/nw_affine.py): vjp_fields,
vjp_one, vjp and the named kernel bindings."""

from ._base import module_globals

globals().update(module_globals("nw_affine"))
