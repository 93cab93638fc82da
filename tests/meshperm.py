"""Renumbering of a mesh for the general-mesh tests: the same cells, nodes and ghosts
under other ids, and each cell's faces starting at another corner (the case generator
``tnsgpu.cases.renumbered_mesh``)."""
from tnsgpu.cases import renumbered_mesh as permute_mesh  # noqa: F401
