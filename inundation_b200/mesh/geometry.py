"""Unstructured polygon-mesh geometry in the form the shallow-water step reads.

``MeshGeometry`` carries the same fields, dtypes and conventions as the
reference's ``inundation/mesh/geometry.py:37-117``: coordinates relative to the
mesh's lower-left corner; per-cell area and centroid; per-edge length, unit
normal pointing from the left to the right cell, bed steps ``(dzL, dzR)``;
``edge_cellR == -1`` on a wall; and the per-cell signed CSR
``(edge << 1) | is_right`` in the order of each cell's sides.

The arrays must match the reference bit for bit, because the edge numbering,
the per-cell CSR order and the float32 values fix the summation order and the
rounding of every flux sum. The steps that decide them therefore follow the
reference's algorithm: shoelace sums grouped by polygon degree
(``geometry.py:130-170,330-373``), half-edge matching by a sorted vertex-pair
key (``:173-202``), normal orientation by the centroid step (``:205-238``),
float64 bed steps (``:241-254``), the CSR ordered by (cell, side)
(``:445-468``), Skilling's Hilbert transform of order 10 (``:505-552``) and the
edge sort by ``min(cellL, cellR)`` (``:642-670``).
"""

from __future__ import annotations

from dataclasses import dataclass, replace
from typing import Any

import numpy as np
from numpy.typing import NDArray

from ..tuning import MIN_CELL_AREA

_EDGE_LENGTH_EPS = 1e-30
_CENTROID_EPS = 1e-20


@dataclass
class MeshGeometry:
    """Precomputed mesh arrays (field-for-field the reference's ``MeshGeometry``)."""

    origin: NDArray[np.float64]
    centroid: NDArray[np.float32]
    area: NDArray[np.float32]
    zb: NDArray[np.float32]
    cell_vertices: NDArray[np.float32]
    cell_vertex_ptr: NDArray[np.int32]
    cell_bbox: NDArray[np.float32]
    edge_len: NDArray[np.float32]
    edge_nx: NDArray[np.float32]
    edge_ny: NDArray[np.float32]
    edge_dzL: NDArray[np.float32]
    edge_dzR: NDArray[np.float32]
    edge_cellL: NDArray[np.int32]
    edge_cellR: NDArray[np.int32]
    edge_sideL: NDArray[np.int32]
    edge_sideR: NDArray[np.int32]
    cell_edge_ptr: NDArray[np.int32]
    cell_edge_idx: NDArray[np.int32]
    cell_nbr_idx: NDArray[np.int32]
    cell_edge_side: NDArray[np.int32]
    cell_edge_idx_signed: NDArray[np.int32]
    N: int
    E: int
    V: int
    max_degree: int = 3
    manning_n: NDArray[np.float32] | None = None

    @property
    def world_centroid(self) -> NDArray[np.float64]:
        return self.centroid.astype(np.float64) + self.origin


def _shoelace(xy: NDArray[np.float64]) -> tuple[NDArray[np.float64], NDArray[np.float64]]:
    """Per-row cross terms and signed area of polygons given as ``(n, d, 2)``."""
    x, y = xy[:, :, 0], xy[:, :, 1]
    cross = x * np.roll(y, -1, axis=1) - np.roll(x, -1, axis=1) * y
    return cross, 0.5 * np.sum(cross, axis=1)


def _centroids(xy: NDArray[np.float64], cross: NDArray[np.float64], signed_area: NDArray[np.float64]) -> NDArray[np.float64]:
    x, y = xy[:, :, 0], xy[:, :, 1]
    with np.errstate(divide="ignore", invalid="ignore"):
        six = 6.0 * signed_area
        cx = np.sum((x + np.roll(x, -1, axis=1)) * cross, axis=1) / six
        cy = np.sum((y + np.roll(y, -1, axis=1)) * cross, axis=1) / six
    return np.column_stack([cx, cy])


def _cell_area_centroid(
    verts: NDArray[np.float64], faces: NDArray[np.int32], offsets: NDArray[np.int32]
) -> tuple[NDArray[np.float32], NDArray[np.float64]]:
    """Area (float32) and centroid (float64) per cell; clockwise cells are re-oriented in ``faces``.

    A mesh of one polygon degree recomputes a reversed cell's area from the
    reversed ring and falls back on the vertex mean for a zero-area cell; a
    mixed mesh keeps the magnitude of the first sum. Both follow the two
    branches of the reference (geometry.py:330-373 and 130-170).
    """
    degrees = np.diff(offsets)
    n = degrees.size
    uniform = n > 0 and int(degrees.min()) == int(degrees.max())
    area = np.empty(n, dtype=np.float32)
    centroid = np.empty((n, 2), dtype=np.float64)
    for degree in np.unique(degrees).tolist():
        cells = np.flatnonzero(degrees == degree)
        slots = offsets[cells, None].astype(np.int64) + np.arange(degree)
        ring = faces[slots]
        xy = verts[ring]
        cross, signed = _shoelace(xy)
        cw = signed < 0
        if cw.any():
            ring[cw] = ring[cw, ::-1]
            faces[slots] = ring
            xy = verts[ring]
            if uniform:
                cross, signed = _shoelace(xy)
            else:
                cross, _ = _shoelace(xy)
                signed = np.abs(signed)
        area[cells] = np.maximum(signed, 1e-30)
        c = _centroids(xy, cross, signed)
        if uniform:
            degenerate = np.abs(signed) < _CENTROID_EPS
            if degenerate.any():
                c[degenerate] = xy[degenerate].mean(axis=1)
        centroid[cells] = c
    return area, centroid


def _pair_sides(
    faces: NDArray[np.int32], offsets: NDArray[np.int32], n_verts: int
) -> tuple[NDArray[np.int64], NDArray[np.int64], NDArray[np.int64]]:
    """Match polygon sides that share a vertex pair.

    Returns ``(first, second, nxt)``: the face slots of each edge's first and
    second side (``-1`` on the boundary), edges numbered by their first slot,
    and the slot of the next vertex around each side's polygon.
    """
    off = offsets.astype(np.int64)
    nxt = np.arange(1, faces.size + 1, dtype=np.int64)
    nxt[off[1:] - 1] = off[:-1]
    a = faces.astype(np.int64)
    b = a[nxt]
    key = np.minimum(a, b) * (n_verts + 1) + np.maximum(a, b)
    order = np.argsort(key, kind="stable")
    sorted_key = key[order]
    run_start = np.flatnonzero(np.r_[True, sorted_key[1:] != sorted_key[:-1]])
    first = order[run_start]
    paired = np.diff(np.r_[run_start, order.size]) >= 2
    second = np.full(run_start.size, -1, dtype=np.int64)
    second[paired] = order[run_start[paired] + 1]
    by_first = np.argsort(first)
    return first[by_first], second[by_first], nxt


def _lengths_normals(
    pa: NDArray[np.float64],
    pb: NDArray[np.float64],
    centroid: NDArray[np.float64],
    cell_l: NDArray[np.int32],
    cell_r: NDArray[np.int32],
) -> tuple[NDArray[np.float32], NDArray[np.float32], NDArray[np.float32]]:
    """Length and unit normal of each edge, turned to point from cellL to cellR."""
    dx = pb[:, 0] - pa[:, 0]
    dy = pb[:, 1] - pa[:, 1]
    length = np.sqrt(dx * dx + dy * dy)
    with np.errstate(divide="ignore", invalid="ignore"):
        nx = dy / length
        ny = -dx / length
    degenerate = length < _EDGE_LENGTH_EPS
    nx[degenerate] = 0.0
    ny[degenerate] = 0.0
    inner = np.flatnonzero(cell_r != -1)
    cl = centroid[cell_l[inner]]
    step = centroid[cell_r[inner]] - cl
    nxi, nyi = nx[inner], ny[inner]
    dot = step[:, 0] * nxi + step[:, 1] * nyi
    flip = dot < 0
    tie = np.flatnonzero(dot == 0.0)
    if tie.size:
        mid = 0.5 * (pa[inner[tie]] + pb[inner[tie]])
        side = (mid[:, 0] - cl[tie, 0]) * nxi[tie] + (mid[:, 1] - cl[tie, 1]) * nyi[tie]
        flip[tie] = side < 0
    turned = inner[flip]
    nx[turned] = -nx[turned]
    ny[turned] = -ny[turned]
    return length.astype(np.float32), nx.astype(np.float32), ny.astype(np.float32)


def edge_bed_steps(
    zb: NDArray[np.float32], edge_cellL: NDArray[np.int32], edge_cellR: NDArray[np.int32]
) -> tuple[NDArray[np.float32], NDArray[np.float32]]:
    """Face elevation minus each side's bed, both ``>= 0``, from float64 differences.

    The face sits at the higher of the two beds; a boundary edge mirrors its
    left cell, so both steps are zero (reference geometry.py:241-254).
    """
    z = zb.astype(np.float64)
    z_l = z[edge_cellL]
    z_r = np.where(edge_cellR >= 0, z[np.maximum(edge_cellR, 0)], z_l)
    face = np.maximum(z_l, z_r)
    return (face - z_l).astype(np.float32), (face - z_r).astype(np.float32)


def build_geometry(
    verts: NDArray[np.floating[Any]],
    faces: NDArray[np.int32],
    face_offsets: NDArray[np.int32] | None = None,
    *,
    zb_from_file: NDArray[np.float32],
    manning_n_from_file: NDArray[np.float32] | None = None,
    progress: bool = False,
) -> MeshGeometry:
    """Geometry of a polygon mesh; ``faces`` is ``(N, d)`` or flat with ``face_offsets``."""
    del progress
    world = np.asarray(verts, dtype=np.float64)
    origin = world.min(axis=0)
    xy = world - origin
    faces = np.array(faces, dtype=np.int32, copy=True)
    if faces.ndim == 2:
        n, d = (int(s) for s in faces.shape)
        offsets = np.arange(0, (n + 1) * d, d, dtype=np.int32)
        faces = faces.ravel()
    else:
        if face_offsets is None:
            raise ValueError("face_offsets is required when faces is a 1-D array")
        offsets = np.asarray(face_offsets, dtype=np.int32)
        n = offsets.size - 1
    n_verts = xy.shape[0]
    degrees = np.diff(offsets)
    max_degree = int(degrees.max())

    area, centroid = _cell_area_centroid(xy, faces, offsets)
    slivers = np.flatnonzero(area <= MIN_CELL_AREA)
    if slivers.size:
        raise ValueError(
            f"{slivers.size} cell(s) have area <= {MIN_CELL_AREA} m^2 "
            f"(first: {slivers[:5].tolist()}); merge or remove degenerate cells"
        )
    cell_vertex_ptr = offsets.copy()
    cell_vertices = xy[faces].astype(np.float32)
    starts = cell_vertex_ptr[:-1]
    cell_bbox = np.column_stack(
        [
            np.minimum.reduceat(cell_vertices[:, 0], starts),
            np.maximum.reduceat(cell_vertices[:, 0], starts),
            np.minimum.reduceat(cell_vertices[:, 1], starts),
            np.maximum.reduceat(cell_vertices[:, 1], starts),
        ]
    ).astype(np.float32)

    zb = np.asarray(zb_from_file, dtype=np.float32)
    if zb.shape != (n,):
        raise ValueError(f"zb_from_file has shape {zb.shape}, expected ({n},)")
    if not np.isfinite(zb).all():
        raise ValueError("zb_from_file must contain only finite values")
    manning_n = None
    if manning_n_from_file is not None:
        manning_n = np.asarray(manning_n_from_file, dtype=np.float32).reshape(-1)
        if manning_n.size != n:
            raise ValueError(f"manning_n: expected {n} values, got {manning_n.size}")
        if not np.isfinite(manning_n).all() or not (manning_n > 0.0).all():
            raise ValueError("manning_n must contain finite positive values")

    first, second, nxt = _pair_sides(faces, offsets, n_verts)
    n_edges = first.size
    slot_cell = np.repeat(np.arange(n, dtype=np.int32), degrees)
    slot_side = (np.arange(faces.size) - offsets[slot_cell].astype(np.int64)).astype(np.int32)
    inner = np.flatnonzero(second >= 0)
    cell_l = slot_cell[first]
    cell_r = np.full(n_edges, -1, dtype=np.int32)
    cell_r[inner] = slot_cell[second[inner]]
    side_l = slot_side[first]
    side_r = np.full(n_edges, -1, dtype=np.int32)
    side_r[inner] = slot_side[second[inner]]
    length, nx, ny = _lengths_normals(xy[faces[first]], xy[faces[nxt[first]]], centroid, cell_l, cell_r)
    both = cell_r != -1
    step = centroid[cell_r[both]] - centroid[cell_l[both]]
    if not (step[:, 0] * nx[both] + step[:, 1] * ny[both] >= 0).all():
        raise ValueError("Some interior edge normals point the wrong way!")
    dz_l, dz_r = edge_bed_steps(zb, cell_l, cell_r)

    owner = np.r_[cell_l, cell_r[inner]]
    if owner.size >= 2**31:
        raise ValueError(f"mesh too large for int32 CSR offsets: total_slots={owner.size}")
    sides = np.r_[side_l, side_r[inner]]
    order = np.argsort(owner.astype(np.int64) * max_degree + sides)
    cell_edge_ptr = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(np.bincount(owner, minlength=n), out=cell_edge_ptr[1:])
    cell_edge_idx = np.r_[np.arange(n_edges, dtype=np.int32), inner.astype(np.int32)][order]
    cell_nbr_idx = np.r_[cell_r, cell_l[inner]][order]
    cell_edge_side = np.r_[np.zeros(n_edges, np.int32), np.ones(inner.size, np.int32)][order]
    signed = (cell_edge_idx.astype(np.int32) << 1) | cell_edge_side

    return MeshGeometry(
        origin=origin,
        centroid=centroid.astype(np.float32),
        area=area,
        zb=zb,
        manning_n=manning_n,
        cell_vertices=cell_vertices,
        cell_vertex_ptr=cell_vertex_ptr,
        cell_bbox=cell_bbox,
        edge_len=length,
        edge_nx=nx,
        edge_ny=ny,
        edge_dzL=dz_l,
        edge_dzR=dz_r,
        edge_cellL=cell_l,
        edge_cellR=cell_r,
        edge_sideL=side_l,
        edge_sideR=side_r,
        cell_edge_ptr=cell_edge_ptr,
        cell_edge_idx=cell_edge_idx,
        cell_nbr_idx=cell_nbr_idx,
        cell_edge_side=cell_edge_side,
        cell_edge_idx_signed=signed,
        N=n,
        E=n_edges,
        V=n_verts,
        max_degree=max_degree,
    )


def hilbert_distances(x: NDArray[np.int64], y: NDArray[np.int64], order: int) -> NDArray[np.int64]:
    """Index along the 2-D Hilbert curve of ``order`` bits per axis.

    Skilling's transform ("Programming the Hilbert curve", AIP Conf. Proc. 707,
    2004): undo the excess work of the axes from the top bit down, Gray-decode,
    then interleave the bits with ``x`` as the more significant axis. This is
    the curve the reference orders cells by (geometry.py:505-536).
    """
    px = np.asarray(x, dtype=np.int64).copy()
    py = np.asarray(y, dtype=np.int64).copy()
    top = 1 << (order - 1)
    bit = top
    while bit > 1:
        mask = bit - 1
        px = np.where((px & bit) != 0, px ^ mask, px)
        y_on = (py & bit) != 0
        t = (px ^ py) & mask
        px, py = np.where(y_on, px ^ mask, px ^ t), np.where(y_on, py, py ^ t)
        bit >>= 1
    py ^= px
    flip = np.zeros_like(py)
    bit = top
    while bit > 1:
        flip ^= np.where((py & bit) != 0, bit - 1, 0)
        bit >>= 1
    px ^= flip
    py ^= flip
    index = np.zeros_like(px)
    for b in range(order):
        index |= ((px >> b) & 1) << (2 * b + 1)
        index |= ((py >> b) & 1) << (2 * b)
    return index


def hilbert_permutation(centroid: NDArray[np.float32], hilbert_p: int = 10) -> NDArray[np.int32]:
    """``perm[new] = old``: cells sorted (stably) by the Hilbert index of their centroid."""
    scale = 2**hilbert_p - 1
    cx = centroid[:, 0].astype(np.float64)
    cy = centroid[:, 1].astype(np.float64)
    lo = np.array([cx.min(), cy.min()])
    span = np.array([cx.max() - cx.min(), cy.max() - cy.min()])
    span[span == 0] = 1.0
    ix = ((cx - lo[0]) / span[0] * scale).astype(np.int64)
    iy = ((cy - lo[1]) / span[1] * scale).astype(np.int64)
    return np.argsort(hilbert_distances(ix, iy, hilbert_p), kind="stable").astype(np.int32)


def _permuted_rows(ptr: NDArray[np.int32], perm: NDArray[np.int32]) -> tuple[NDArray[np.int32], NDArray[np.int64]]:
    """Row pointers of a CSR after permuting its rows, and each new slot's old slot."""
    counts = np.diff(ptr)[perm]
    new_ptr = np.zeros(ptr.size, dtype=np.int32)
    np.cumsum(counts, out=new_ptr[1:])
    shift = ptr[perm].astype(np.int64) - new_ptr[:-1]
    return new_ptr, np.repeat(shift, counts) + np.arange(int(new_ptr[-1]))


def hilbert_reorder(
    geom: MeshGeometry, hilbert_p: int = 10, verbose: bool = True
) -> tuple[MeshGeometry, NDArray[np.int32]]:
    """Renumber cells along the Hilbert curve and edges by ``min(cellL, cellR)``.

    Returns the reordered geometry and ``perm`` (``perm[new] = old``).
    """
    del verbose
    n = geom.N
    perm = hilbert_permutation(geom.centroid, hilbert_p=hilbert_p)
    inv = np.empty(n, dtype=np.int32)
    inv[perm] = np.arange(n, dtype=np.int32)

    vptr, vslots = _permuted_rows(geom.cell_vertex_ptr, perm)
    cell_l = inv[geom.edge_cellL].astype(np.int32)
    cell_r = geom.edge_cellR.copy()
    inner = geom.edge_cellR != -1
    cell_r[inner] = inv[geom.edge_cellR[inner]]

    eptr, eslots = _permuted_rows(geom.cell_edge_ptr, perm)
    edge_of_slot = geom.cell_edge_idx[eslots]
    side_of_slot = geom.cell_edge_side[eslots]
    old_nbr = geom.cell_nbr_idx[eslots]
    nbr = np.where(old_nbr == -1, -1, inv[old_nbr])

    centroid = geom.centroid[perm]
    both = cell_r != -1
    step = centroid[cell_r[both]] - centroid[cell_l[both]]
    if not (step[:, 0] * geom.edge_nx[both] + step[:, 1] * geom.edge_ny[both] >= -2.0 * np.spacing(centroid.max())).all():
        raise ValueError("Normal orientation broken after Hilbert reordering!")

    key = np.where(cell_r >= 0, np.minimum(cell_l, cell_r), cell_l)
    eperm = np.argsort(key, kind="stable").astype(np.int32)
    einv = np.empty(geom.E, dtype=np.int32)
    einv[eperm] = np.arange(geom.E, dtype=np.int32)
    new_edge_of_slot = einv[edge_of_slot]

    out = MeshGeometry(
        origin=geom.origin,
        centroid=centroid,
        area=geom.area[perm],
        zb=geom.zb[perm],
        manning_n=None if geom.manning_n is None else geom.manning_n[perm],
        cell_vertices=geom.cell_vertices[vslots],
        cell_vertex_ptr=vptr,
        cell_bbox=geom.cell_bbox[perm],
        edge_len=geom.edge_len[eperm],
        edge_nx=geom.edge_nx[eperm],
        edge_ny=geom.edge_ny[eperm],
        edge_dzL=geom.edge_dzL[eperm],
        edge_dzR=geom.edge_dzR[eperm],
        edge_cellL=cell_l[eperm],
        edge_cellR=cell_r[eperm],
        edge_sideL=geom.edge_sideL[eperm],
        edge_sideR=geom.edge_sideR[eperm],
        cell_edge_ptr=eptr,
        cell_edge_idx=new_edge_of_slot,
        cell_nbr_idx=nbr,
        cell_edge_side=side_of_slot,
        cell_edge_idx_signed=(new_edge_of_slot.astype(np.int32) << 1) | side_of_slot,
        N=n,
        E=geom.E,
        V=geom.V,
        max_degree=geom.max_degree,
    )
    return out, perm


def with_bed(geom: MeshGeometry, zb: NDArray[np.float32]) -> MeshGeometry:
    """The same mesh over another bed: new ``zb`` and recomputed bed steps."""
    zb = np.asarray(zb, dtype=np.float32)
    dz_l, dz_r = edge_bed_steps(zb, geom.edge_cellL, geom.edge_cellR)
    return replace(geom, zb=zb, edge_dzL=dz_l, edge_dzR=dz_r)
