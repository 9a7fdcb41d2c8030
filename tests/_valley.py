"""Sloped-valley test problem (the reference's ``tests/unit/_valley.py:19-104``).

A Hilbert-ordered 256 x 128 quad grid of 2 m cells (128 active-set blocks)
whose bed falls 0.002 in +x with a shallow valley along the centre line; the
same initial states (dam, sheet, point source) and tolerances of the atomic
path as the reference's fixture.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from inundation_b200.mesh.geometry import MeshGeometry, build_geometry, hilbert_reorder
from inundation_b200.mesh.synthetic import quad_grid

NX, NY, DX = 256, 128, 2.0
MANNING = 0.03
DRY_TOL = 1e-3


def valley_grid(datum: float = 0.0, nx: int = NX, ny: int = NY) -> MeshGeometry:
    q = quad_grid(nx, ny, DX)
    cx = (np.arange(nx * ny) % nx + 0.5) * DX
    cy = (np.arange(nx * ny) // nx + 0.5) * DX
    zb = (datum - 0.002 * cx - 0.3 * np.exp(-(((cy - ny * DX / 2) / (0.2 * ny * DX)) ** 2))).astype(np.float32)
    geom = build_geometry(q.verts.astype(np.float32), q.faces.reshape(-1, 4), zb_from_file=zb)
    return hilbert_reorder(geom, verbose=False)[0]


def cell_near(grid: MeshGeometry, x: float, y: float) -> int:
    d = (grid.centroid[:, 0] - x) ** 2 + (grid.centroid[:, 1] - y) ** 2
    return int(np.argmin(d))


def point_source(grid: MeshGeometry, q: float, x: float, y: float) -> np.ndarray:
    src = np.zeros(grid.N, dtype=np.float32)
    src[cell_near(grid, x, y)] = q
    return src


def dam(grid: MeshGeometry, nx: int = NX, ny: int = NY) -> np.ndarray:
    x, y = grid.centroid[:, 0], grid.centroid[:, 1]
    inside = (x < nx * DX * 0.25) & (np.abs(y - ny * DX / 2) < ny * DX * 0.15)
    return np.where(inside, 1.0, 0.0).astype(np.float32)


def sheet(grid: MeshGeometry, nx: int = NX) -> np.ndarray:
    return np.where(grid.centroid[:, 0] < nx * DX * 0.3, 0.02, 0.0).astype(np.float32)


def run(solver: Any, t_end: float, **kwargs: Any) -> list[np.ndarray]:
    snaps, _ = solver.run(
        t_end=t_end,
        output_interval_s=kwargs.pop("output_interval_s", t_end / 4),
        dt_max=1.0,
        dt_init=0.01,
        cfl_interval=10,
        progress=False,
        **kwargs,
    )
    return snaps


def state(solver: Any) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    return solver.download_h(), solver.download_hu(), solver.download_hv()
