"""This package's geometry builder against the reference's, on the golden fixtures.

``tests/golden/geometry.npz`` holds the reference's ``build_geometry`` and
``hilbert_reorder`` outputs (``inundation/mesh/geometry.py``) for a quad
valley (bed datum 0 and 300 m), a seeded 2000-cell Voronoi mesh and a small
mixed-degree mesh with clockwise cells. Every array must be identical, bit
for bit: the edge numbering and CSR order fix the gather order of the step.
Also the reference's checks on the packed signed CSR
(``tests/unit/test_inundation_signed_csr.py``) and the per-edge bed steps
(``tests/unit/test_mesh_edge_dz.py``).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from inundation_b200.mesh.geometry import MeshGeometry, build_geometry, edge_bed_steps, hilbert_reorder

GOLDEN = np.load(Path(__file__).parent / "golden" / "geometry.npz")
FIELDS = (
    "origin", "centroid", "area", "zb", "cell_vertices", "cell_vertex_ptr", "cell_bbox", "edge_len", "edge_nx",
    "edge_ny", "edge_dzL", "edge_dzR", "edge_cellL", "edge_cellR", "edge_sideL", "edge_sideR", "cell_edge_ptr",
    "cell_edge_idx", "cell_nbr_idx", "cell_edge_side", "cell_edge_idx_signed",
)
MESHES = ["valley", "valley300", "voronoi", "mixed"]


def build(name: str) -> tuple[MeshGeometry, MeshGeometry, np.ndarray]:
    offsets = GOLDEN[f"{name}_in_offsets"]
    raw = build_geometry(
        GOLDEN[f"{name}_in_verts"],
        GOLDEN[f"{name}_in_faces"],
        offsets if offsets.size else None,
        zb_from_file=GOLDEN[f"{name}_in_zb"],
    )
    ordered, perm = hilbert_reorder(raw, verbose=False)
    return raw, ordered, perm


def assert_identical(geom: MeshGeometry, prefix: str) -> None:
    for f in FIELDS:
        want = GOLDEN[f"{prefix}{f}"]
        got = np.asarray(getattr(geom, f))
        assert got.dtype == want.dtype, f"{f}: dtype {got.dtype} != {want.dtype}"
        assert got.shape == want.shape, f"{f}: shape {got.shape} != {want.shape}"
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), f"{f} differs from the reference"
    n, e, v, d = GOLDEN[f"{prefix}NEV"].tolist()
    assert (geom.N, geom.E, geom.V, geom.max_degree) == (n, e, v, d)


@pytest.mark.parametrize("name", MESHES)
def test_build_matches_the_reference_bit_for_bit(name: str) -> None:
    raw, ordered, perm = build(name)
    assert_identical(raw, f"{name}_raw_")
    assert_identical(ordered, f"{name}_hil_")
    np.testing.assert_array_equal(perm, GOLDEN[f"{name}_perm"])


def signed_csr_consistent(geom: MeshGeometry) -> None:
    cell = np.repeat(np.arange(geom.N), np.diff(geom.cell_edge_ptr))
    edge, side = geom.cell_edge_idx.astype(np.int64), geom.cell_edge_side.astype(np.int64)
    assert np.array_equal(geom.cell_edge_idx_signed.astype(np.int64), (edge << 1) | side)
    owner = np.where(side == 1, geom.edge_cellR[edge], geom.edge_cellL[edge])
    assert np.array_equal(owner, cell)
    left = np.bincount(edge[side == 0], minlength=geom.E)
    right = np.bincount(edge[side == 1], minlength=geom.E)
    assert (left == 1).all()
    inner = geom.edge_cellR != -1
    assert (right[inner] == 1).all() and (right[~inner] == 0).all()


@pytest.mark.parametrize("name", MESHES)
def test_signed_csr_is_consistent(name: str) -> None:
    raw, ordered, _ = build(name)
    signed_csr_consistent(raw)
    signed_csr_consistent(ordered)


def test_interior_normals_point_from_left_to_right() -> None:
    _, g, _ = build("voronoi")
    inner = g.edge_cellR >= 0
    step = g.centroid[g.edge_cellR[inner]].astype(np.float64) - g.centroid[g.edge_cellL[inner]]
    assert (step[:, 0] * g.edge_nx[inner] + step[:, 1] * g.edge_ny[inner] >= -1e-3).all()
    assert np.allclose(np.hypot(g.edge_nx, g.edge_ny), 1.0, atol=1e-6)


def test_bed_steps_are_exact_and_one_side_sits_on_the_face() -> None:
    _, g, _ = build("valley300")
    zb = g.zb.astype(np.float64)
    wall = g.edge_cellR < 0
    zl = zb[g.edge_cellL]
    zr = np.where(wall, zl, zb[np.where(wall, 0, g.edge_cellR)])
    face = np.maximum(zl, zr)
    np.testing.assert_array_equal(g.edge_dzL.astype(np.float64), face - zl)
    np.testing.assert_array_equal(g.edge_dzR.astype(np.float64), face - zr)
    assert (np.minimum(g.edge_dzL, g.edge_dzR) == 0.0).all()
    assert (g.edge_dzL[wall] == 0.0).all() and (g.edge_dzR[wall] == 0.0).all()


def test_bed_steps_far_from_the_datum() -> None:
    zb = np.array([1000.0, 1000.0 + 2.0**-13, 999.5], dtype=np.float32)
    dzl, dzr = edge_bed_steps(zb, np.array([0, 1, 2], np.int32), np.array([1, 2, -1], np.int32))
    np.testing.assert_array_equal(dzl, np.array([2.0**-13, 0.0, 0.0], np.float32))
    np.testing.assert_array_equal(dzr, np.array([0.0, 0.5 + 2.0**-13, 0.0], np.float32))


def test_sliver_cells_are_refused() -> None:
    verts = np.array([[0, 0], [1, 0], [2, 0], [0, 1]], dtype=np.float64)
    faces = np.array([[0, 1, 2], [0, 1, 3]], dtype=np.int32)
    with pytest.raises(ValueError, match="area"):
        build_geometry(verts, faces, zb_from_file=np.zeros(2, np.float32))


def test_rejects_bad_bed_and_roughness() -> None:
    verts = np.array([[0, 0], [1, 0], [0, 1]], dtype=np.float64)
    faces = np.array([[0, 1, 2]], dtype=np.int32)
    with pytest.raises(ValueError, match="finite"):
        build_geometry(verts, faces, zb_from_file=np.array([np.nan], np.float32))
    with pytest.raises(ValueError, match="manning"):
        build_geometry(verts, faces, zb_from_file=np.zeros(1, np.float32), manning_n_from_file=np.zeros(1, np.float32))
