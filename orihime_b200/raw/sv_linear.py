"""Raw tier of the Saigo-Vert, linear gap operator (orihime/raw/sv_linear.py): vjp_fields,
vjp_one, vjp and the named kernel bindings."""

from ._base import module_globals

globals().update(module_globals("sv_linear"))
