"""Raw tier of the soft Smith-Waterman, affine gaps operator (orihime/raw/sw_affine.py): vjp_fields,
vjp_one, vjp and the named kernel bindings."""

from ._base import module_globals

globals().update(module_globals("sw_affine"))
