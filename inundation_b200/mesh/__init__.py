"""Mesh geometry, active-set block topology and synthetic scenario meshes."""

from .geometry import MeshGeometry, build_geometry, edge_bed_steps, hilbert_permutation, hilbert_reorder, with_bed

__all__ = [
    "MeshGeometry",
    "build_geometry",
    "edge_bed_steps",
    "hilbert_permutation",
    "hilbert_reorder",
    "with_bed",
]
