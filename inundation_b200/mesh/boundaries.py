"""Open boundary stretches: which boundary edges a line selects, and how an inflow splits.

The reference's ``inundation/mesh/boundaries.py`` restated. A stretch is a
polyline in world coordinates; it selects the wall edges (right cell -1) whose
midpoints lie within a tolerance of it. An inflow's discharge is spread over a
stretch's edges by Manning conveyance at the common level that carries it, so
water enters along the low part of the section.
"""

from __future__ import annotations

from collections.abc import Sequence

import numpy as np
from numpy.typing import NDArray

from .geometry import MeshGeometry

# Bisections of the conveyance level: enough for a float64 level.
LEVEL_BISECTIONS = 80


def boundary_edge_midpoints(geom: MeshGeometry) -> tuple[NDArray[np.int64], NDArray[np.float64]]:
    """Wall edge indices and their midpoints, relative to ``geom.origin`` (boundaries.py:24-35).

    A wall edge is side ``edge_sideL`` of its left cell, from that ring vertex to the next.
    """
    edges = np.flatnonzero(np.asarray(geom.edge_cellR) == -1)
    cells = np.asarray(geom.edge_cellL)[edges].astype(np.int64)
    side = np.asarray(geom.edge_sideL)[edges].astype(np.int64)
    first = np.asarray(geom.cell_vertex_ptr)[cells].astype(np.int64)
    ring = np.asarray(geom.cell_vertex_ptr)[cells + 1].astype(np.int64) - first
    verts = np.asarray(geom.cell_vertices, dtype=np.float64)
    return edges, 0.5 * (verts[first + side] + verts[first + (side + 1) % ring])


def distance_to_line(points: NDArray[np.float64], line: NDArray[np.float64]) -> NDArray[np.float64]:
    """Distance from each point to a polyline (boundaries.py:38-46)."""
    points = np.asarray(points, dtype=np.float64)
    line = np.asarray(line, dtype=np.float64)
    best = np.full(points.shape[0], np.inf)
    for a, b in zip(line[:-1], line[1:], strict=True):
        ab = b - a
        t = np.clip(((points - a) @ ab) / max(float(ab @ ab), 1e-30), 0.0, 1.0)
        best = np.minimum(best, np.hypot(*(points - (a + t[:, None] * ab)).T))
    return best


def select_boundary_edges(geom: MeshGeometry, line: Sequence[tuple[float, float]], tolerance_m: float) -> NDArray[np.int64]:
    """Wall edges whose midpoints lie within ``tolerance_m`` of a world-coordinate line (boundaries.py:49-58)."""
    if len(line) < 2:
        raise ValueError(f"a stretch needs at least 2 points, got {len(line)}")
    local = np.asarray(line, dtype=np.float64) - np.asarray(geom.origin, dtype=np.float64)
    edges, mid = boundary_edge_midpoints(geom)
    return edges[distance_to_line(mid, local) <= tolerance_m]


def conveyance_split(
    discharge_m3s: float,
    lengths: NDArray[np.float32],
    beds: NDArray[np.float32],
    manning: NDArray[np.float32],
    energy_slope: float,
) -> NDArray[np.float32]:
    """Discharge per unit width on every edge of a section carrying ``discharge_m3s`` (boundaries.py:61-100).

    Edge e at level L carries len_e sqrt(S) / n_e max(L - z_e, 0)^(5/3); the
    level is found by doubling an upper bound from the lowest bed, then
    bisection, and the discharge split in proportion to each edge's share at the
    upper end. Float32 for the kernels; the edge carrying most absorbs the
    rounding of the cast, so the float64 total over the section is the discharge.
    """
    n = np.asarray(lengths).size
    if discharge_m3s <= 0.0:
        return np.zeros(n, dtype=np.float32)
    length = np.asarray(lengths, dtype=np.float64)
    bed = np.asarray(beds, dtype=np.float64)
    rate = length * np.sqrt(energy_slope) / np.asarray(manning, dtype=np.float64)

    def carried(level: float) -> NDArray[np.float64]:
        return rate * np.maximum(level - bed, 0.0) ** (5.0 / 3.0)

    lo = float(bed.min())
    hi = lo + 1.0
    while carried(hi).sum() < discharge_m3s:
        hi = lo + 2.0 * (hi - lo)
    for _ in range(LEVEL_BISECTIONS):
        mid = 0.5 * (lo + hi)
        if carried(mid).sum() < discharge_m3s:
            lo = mid
        else:
            hi = mid
    share = carried(hi)
    q = (discharge_m3s * share / share.sum() / length).astype(np.float32)
    top = int(np.argmax(share))
    q[top] += np.float32((discharge_m3s - float((q.astype(np.float64) * length).sum())) / length[top])
    return q


__all__ = ["LEVEL_BISECTIONS", "boundary_edge_midpoints", "conveyance_split", "distance_to_line", "select_boundary_edges"]
