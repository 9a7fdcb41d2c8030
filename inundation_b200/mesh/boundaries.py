"""Open boundary stretches: the wall edges a line selects, and how an inflow splits over them.

A stretch is a polyline in world coordinates; it selects the wall edges (right
cell -1) whose midpoints lie within a tolerance of it (the reference's
``inundation/mesh/boundaries.py:24-58`` selects the same edges). An inflow's
discharge is spread over a stretch's edges by Manning conveyance at the one
water level that carries it, so water enters along the low part of the section
(the reference's ``conveyance_split``, ``boundaries.py:61-100``, splits by the
same rule).

Design: midpoints come from one table of every cell side's midpoint; the
distance to a polyline is one broadcast over all its segments; the water level
is bracketed between sorted bed levels and solved there by Brent's method; the
float32 rounding residual of the split goes to the edge that can absorb it most
finely.
"""

from __future__ import annotations

from collections.abc import Sequence

import numpy as np
from numpy.typing import NDArray
from scipy.optimize import brentq

from .geometry import MeshGeometry

MANNING_EXPONENT = 5.0 / 3.0


def _side_midpoints(geom: MeshGeometry) -> NDArray[np.float64]:
    """Midpoint of every cell side, indexed like ``cell_vertices`` (side k of a cell runs from its vertex k to k+1)."""
    verts = np.asarray(geom.cell_vertices, dtype=np.float64)
    ptr = np.asarray(geom.cell_vertex_ptr, dtype=np.int64)
    following = np.arange(1, verts.shape[0] + 1, dtype=np.int64)
    following[ptr[1:] - 1] = ptr[:-1]  # each ring's last vertex closes back to its first
    return 0.5 * (verts + verts[following])


def boundary_edge_midpoints(geom: MeshGeometry) -> tuple[NDArray[np.int64], NDArray[np.float64]]:
    """Wall edge indices and their midpoints, relative to ``geom.origin``.

    A wall edge is side ``edge_sideL`` of its left cell.
    """
    edges = np.flatnonzero(np.asarray(geom.edge_cellR) == -1)
    slot = np.asarray(geom.cell_vertex_ptr, dtype=np.int64)[np.asarray(geom.edge_cellL)[edges]]
    slot += np.asarray(geom.edge_sideL)[edges].astype(np.int64)
    return edges, _side_midpoints(geom)[slot]


def distance_to_line(points: NDArray[np.float64], line: NDArray[np.float64]) -> NDArray[np.float64]:
    """Euclidean distance from each point to the nearest point of a polyline."""
    p = np.asarray(points, dtype=np.float64)[:, None, :]  # (points, 1, 2)
    line = np.asarray(line, dtype=np.float64)
    a, d = line[:-1][None], np.diff(line, axis=0)[None]  # (1, segments, 2)
    length2 = np.maximum((d * d).sum(axis=-1), 1e-30)
    t = np.clip(((p - a) * d).sum(axis=-1) / length2, 0.0, 1.0)
    gap = p - (a + t[..., None] * d)
    return np.hypot(gap[..., 0], gap[..., 1]).min(axis=1)


def select_boundary_edges(geom: MeshGeometry, line: Sequence[tuple[float, float]], tolerance_m: float) -> NDArray[np.int64]:
    """Wall edges whose midpoints lie within ``tolerance_m`` of a world-coordinate polyline."""
    if len(line) < 2:
        raise ValueError(f"a stretch needs at least 2 points, got {len(line)}")
    local = np.asarray(line, dtype=np.float64) - np.asarray(geom.origin, dtype=np.float64)
    edges, mid = boundary_edge_midpoints(geom)
    if edges.size == 0:
        return edges
    return edges[distance_to_line(mid, local) <= tolerance_m]


def _section_level(discharge: float, rate: NDArray[np.float64], bed: NDArray[np.float64]) -> float:
    """The water level at which sum_e rate_e (level - bed_e)_+^(5/3) equals ``discharge``.

    The sum grows strictly with the level above the lowest bed; its values at
    the sorted bed levels bracket the root between two consecutive beds (or
    above the highest), where Brent's method solves it to float64 precision.
    """

    def excess(level: float) -> float:
        return float((rate * np.maximum(level - bed, 0.0) ** MANNING_EXPONENT).sum()) - discharge

    levels = np.unique(bed)
    below = levels[0]
    for z in levels[1:]:
        if excess(z) >= 0.0:
            return brentq(excess, below, z, xtol=1e-15, rtol=4 * np.finfo(float).eps, maxiter=200)
        below = z
    above = below + 1.0
    while excess(above) < 0.0:
        above = below + 2.0 * (above - below)
    return brentq(excess, below, above, xtol=1e-15, rtol=4 * np.finfo(float).eps, maxiter=200)


def conveyance_split(
    discharge_m3s: float,
    lengths: NDArray[np.float32],
    beds: NDArray[np.float32],
    manning: NDArray[np.float32],
    energy_slope: float,
) -> NDArray[np.float32]:
    """Float32 discharge per unit width on every edge of a section carrying ``discharge_m3s``.

    Edge e at level L carries len_e sqrt(S) / n_e (L - z_e)_+^(5/3); the section's
    level is the one whose total is the discharge, and each edge gets its own
    part. After the cast to float32, the residual of the float64 total goes to
    the wet edge whose float32 step (ulp x length) is finest, so the total over
    the section is the discharge to within half that step.
    """
    length = np.asarray(lengths, dtype=np.float64)
    if discharge_m3s <= 0.0:
        return np.zeros(length.size, dtype=np.float32)
    bed = np.asarray(beds, dtype=np.float64)
    rate = length * np.sqrt(energy_slope) / np.asarray(manning, dtype=np.float64)
    level = _section_level(float(discharge_m3s), rate, bed)
    part = rate * np.maximum(level - bed, 0.0) ** MANNING_EXPONENT
    per_width = (discharge_m3s * (part / part.sum()) / length).astype(np.float32)
    wet = np.flatnonzero(per_width > 0.0)
    fine = wet[np.argmin(np.spacing(per_width[wet]).astype(np.float64) * length[wet])]
    residual = discharge_m3s - float((per_width.astype(np.float64) * length).sum())
    per_width[fine] = np.float32(float(per_width[fine]) + residual / length[fine])
    return per_width


__all__ = ["boundary_edge_midpoints", "conveyance_split", "distance_to_line", "select_boundary_edges"]
