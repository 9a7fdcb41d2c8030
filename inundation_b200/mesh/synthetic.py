"""Seeded synthetic meshes and terrain for the benchmark and test scenarios.

* ``voronoi_mesh``: the Voronoi diagram of uniform random points in a square,
  bounded by mirroring the points near each side across it, so every cell of
  an original point is a convex polygon clipped to the square.
* ``fractal_dem``: spectral synthesis of a 1/f^beta surface (random phases,
  amplitude k^(-beta/2)), scaled to a relief and sampled at the centroids.
* ``gaussian_bumps``, ``carve_channel``: analytic bed features.
* ``channel_grid``: a straight rectangular channel (the open-boundary cases).

All generators take a seed and are deterministic for it.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from numpy.typing import NDArray


@dataclass(frozen=True)
class PolygonMesh:
    """Vertices ``(V, 2)`` float64 and flat polygon rings with row pointers."""

    verts: NDArray[np.float64]
    faces: NDArray[np.int32]
    offsets: NDArray[np.int32]

    @property
    def n_cells(self) -> int:
        return int(self.offsets.size - 1)


def voronoi_mesh(n_cells: int, side: float, seed: int) -> PolygonMesh:
    """Voronoi cells of ``n_cells`` uniform random points in ``[0, side]^2``."""
    from scipy.spatial import Voronoi

    rng = np.random.default_rng(seed)
    pts = rng.random((n_cells, 2)) * side
    spacing = side / np.sqrt(max(n_cells, 1))
    margin = min(side, 8.0 * spacing)
    ghosts = []
    for axis in (0, 1):
        near_lo = pts[pts[:, axis] < margin].copy()
        near_lo[:, axis] = -near_lo[:, axis]
        near_hi = pts[pts[:, axis] > side - margin].copy()
        near_hi[:, axis] = 2.0 * side - near_hi[:, axis]
        ghosts += [near_lo, near_hi]
    vor = Voronoi(np.concatenate([pts, *ghosts]))
    regions = [vor.regions[r] for r in vor.point_region[:n_cells]]
    degrees = np.fromiter((len(r) for r in regions), dtype=np.int64, count=n_cells)
    flat = np.fromiter((v for r in regions for v in r), dtype=np.int64, count=int(degrees.sum()))
    if (flat < 0).any() or (degrees < 3).any():
        raise ValueError("an original point has an unbounded or degenerate Voronoi cell")
    used, local = np.unique(flat, return_inverse=True)
    verts = np.clip(vor.vertices[used], 0.0, side)
    offsets = np.zeros(n_cells + 1, dtype=np.int32)
    np.cumsum(degrees, out=offsets[1:])
    return PolygonMesh(verts=verts, faces=local.astype(np.int32), offsets=offsets)


def quad_grid(nx: int, ny: int, dx: float) -> PolygonMesh:
    """A structured ``nx`` by ``ny`` grid of square cells of side ``dx``."""
    xs, ys = np.meshgrid(np.arange(nx + 1) * dx, np.arange(ny + 1) * dx)
    verts = np.column_stack([xs.ravel(), ys.ravel()]).astype(np.float64)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    base = (j * (nx + 1) + i).ravel()
    faces = np.column_stack([base, base + 1, base + nx + 2, base + nx + 1]).astype(np.int32)
    return PolygonMesh(verts=verts, faces=faces.ravel(), offsets=np.arange(0, 4 * nx * ny + 1, 4, dtype=np.int32))


def channel_grid(cells: int, across: int, length: float, width: float) -> PolygonMesh:
    """A straight channel of ``cells`` by ``across`` rectangles on [0, length] x [0, width].

    Cell k (original order) is column k % cells, row k // cells, so centres
    along the channel repeat every ``cells`` cells.
    """
    xs, ys = np.meshgrid(np.linspace(0.0, length, cells + 1), np.linspace(0.0, width, across + 1))
    verts = np.column_stack([xs.ravel(), ys.ravel()]).astype(np.float64)
    j, i = np.meshgrid(np.arange(across), np.arange(cells), indexing="ij")
    base = (j * (cells + 1) + i).ravel()
    faces = np.column_stack([base, base + 1, base + cells + 2, base + cells + 1]).astype(np.int32)
    return PolygonMesh(verts=verts, faces=faces.ravel(),
                       offsets=np.arange(0, 4 * cells * across + 1, 4, dtype=np.int32))


def fractal_dem(
    points: NDArray[np.float64], side: float, *, relief: float, beta: float = 2.0, seed: int = 0, grid: int = 512
) -> NDArray[np.float64]:
    """Spectral-synthesis terrain of slope ``beta`` scaled to ``[0, relief]`` at ``points``."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(grid)[:, None]
    ky = np.fft.rfftfreq(grid)[None, :]
    k = np.hypot(kx, ky)
    k[0, 0] = 1.0
    amp = k ** (-beta / 2.0)
    amp[0, 0] = 0.0
    phase = rng.uniform(0.0, 2.0 * np.pi, amp.shape)
    surf = np.fft.irfft2(amp * np.exp(1j * phase), s=(grid, grid))
    surf = (surf - surf.min()) / max(float(np.ptp(surf)), 1e-30) * relief
    u = np.clip(points[:, 0] / side, 0.0, 1.0) * (grid - 1)
    v = np.clip(points[:, 1] / side, 0.0, 1.0) * (grid - 1)
    i0 = np.minimum(np.floor(u).astype(np.int64), grid - 2)
    j0 = np.minimum(np.floor(v).astype(np.int64), grid - 2)
    fu, fv = u - i0, v - j0
    return (
        surf[i0, j0] * (1 - fu) * (1 - fv)
        + surf[i0 + 1, j0] * fu * (1 - fv)
        + surf[i0, j0 + 1] * (1 - fu) * fv
        + surf[i0 + 1, j0 + 1] * fu * fv
    )


def carve_channel(
    points: NDArray[np.float64], bed: NDArray[np.float64], side: float, *, depth: float, width: float, seed: int
) -> NDArray[np.float64]:
    """Lower the bed by ``depth`` along a seeded polyline crossing the square (cosine profile)."""
    rng = np.random.default_rng(seed)
    knots_y = np.linspace(0.0, side, 9)
    knots_x = side * (0.5 + 0.25 * rng.uniform(-1.0, 1.0, knots_y.size))
    line = np.column_stack([knots_x, knots_y])
    dist = np.full(points.shape[0], np.inf)
    for a, b in zip(line[:-1], line[1:], strict=True):
        ab = b - a
        t = np.clip(((points - a) @ ab) / float(ab @ ab), 0.0, 1.0)
        dist = np.minimum(dist, np.hypot(*(points - (a + t[:, None] * ab)).T))
    inside = dist < width
    cut = np.where(inside, depth * 0.5 * (1.0 + np.cos(np.pi * dist / width)), 0.0)
    return bed - cut


def gaussian_bumps(points: NDArray[np.float64], side: float, *, count: int, seed: int) -> NDArray[np.float64]:
    """Sum of ``count`` Gaussian bumps, heights 0.2-0.8 m and sigmas 50-150 m (scaled to ``side``)."""
    rng = np.random.default_rng(seed)
    scale = side / 1000.0
    bed = np.zeros(points.shape[0])
    for _ in range(count):
        cx, cy = rng.uniform(0.0, side, 2)
        height = rng.uniform(0.2, 0.8)
        sigma = rng.uniform(50.0, 150.0) * scale
        bed += height * np.exp(-((points[:, 0] - cx) ** 2 + (points[:, 1] - cy) ** 2) / (2.0 * sigma * sigma))
    return bed
