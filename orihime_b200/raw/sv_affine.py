"""Raw tier of the Saigo-Vert, affine gaps operator (orihime/raw/sv_affine.py): vjp_fields,
vjp_one, vjp and the named kernel bindings."""

from ._base import module_globals

globals().update(module_globals("sv_affine"))
