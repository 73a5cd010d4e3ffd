"""Raw tier of the soft Needleman-Wunsch, linear gap operator (orihime/raw/nw.py): vjp_fields,
vjp_one, vjp and the named kernel bindings."""

from ._base import module_globals

globals().update(module_globals("nw"))
