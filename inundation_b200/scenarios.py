"""Seeded synthetic workloads of the benchmark configurations.

Each builder returns a ``Scenario``: a Hilbert-ordered geometry and its
initial state, roughness, sources and run settings. The meshes are Voronoi
diagrams of uniform random points (3 to ~14 sides per cell; the mean is 6);
terrain is spectral-synthesis fractal relief or Gaussian bumps. They stand in
for real meshes and DEMs with the sizes and value ranges the configurations
name.

* ``lake_at_rest``  -- ~8k cells over 1 km, 6 Gaussian bumps, still water at 1 m.
* ``dam_break``     -- 1M cells over 10 km, fractal DEM (beta 2, 20 m relief) with a
  3 m channel, 4 m of water inside 500 m of the centre, n = 0.035, 1 h.
* ``rain_inflow``   -- 4M cells, 40 m relief, n log-uniform in [0.02, 0.08], 50 mm/h rain
  for 30 min and a triangular 200 m^3/s inflow peaking at 20 min, initially dry.
* ``calibration``   -- the adjoint problem: a pond plus an inflow hydrograph of 32 knots,
  200 gauges, a seeded "true" Manning field.
* ``batch_member``  -- one of the batched scenarios: N cells, own DEM, n in
  [0.02, 0.06], triangular inflow of 10-300 m^3/s peaking at 20 min, initially dry.
* ``open_channel``  -- a straight sloped channel of rectangles whose two ends are
  open stretches (``meta["open_edges"]``: upstream, downstream), the layout of
  the reference's open-boundary cases (``inundation/bench/open_boundary.py``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from numpy.typing import NDArray

from .mesh.geometry import MeshGeometry, build_geometry, hilbert_reorder, with_bed
from .mesh.boundaries import select_boundary_edges
from .mesh.synthetic import carve_channel, channel_grid, fractal_dem, gaussian_bumps, voronoi_mesh
from .sources import Hydrograph, triangular_knots
from .tuning import DRY_TOL_DEFAULT


@dataclass
class Scenario:
    name: str
    geom: MeshGeometry
    h0: NDArray[np.float32]
    hu0: NDArray[np.float32]
    hv0: NDArray[np.float32]
    manning: NDArray[np.float32]
    t_end: float
    dt_max: float = 1.0
    dt_init: float = 0.01
    dry_tol: float = DRY_TOL_DEFAULT
    # Piecewise-constant per-cell source rates [m^3/s]: (start time, rate array), the
    # reference's phase form of the sources.
    source_phases: list[tuple[float, NDArray[np.float32]]] = field(default_factory=list)
    # The same sources in the device form: constant per-cell rates [m^3/s] plus hydrographs.
    source_rate: NDArray[np.float32] | None = None
    hydrographs: list[Hydrograph] = field(default_factory=list)
    meta: dict = field(default_factory=dict)

    @property
    def n_cells(self) -> int:
        return int(self.geom.N)


def voronoi_geometry(n_cells: int, side: float, seed: int) -> MeshGeometry:
    """Hilbert-ordered geometry of a seeded Voronoi mesh over ``[0, side]^2`` (flat bed)."""
    mesh = voronoi_mesh(n_cells, side, seed)
    geom = build_geometry(mesh.verts, mesh.faces, mesh.offsets, zb_from_file=np.zeros(mesh.n_cells, np.float32))
    return hilbert_reorder(geom, verbose=False)[0]


def lake_at_rest(n_cells: int = 8000, seed: int = 1, side: float = 1000.0) -> Scenario:
    geom = voronoi_geometry(n_cells, side, seed)
    xy = geom.world_centroid
    zb = gaussian_bumps(xy, side, count=6, seed=seed).astype(np.float32)
    geom = with_bed(geom, zb)
    h0 = np.maximum(1.0 - zb.astype(np.float64), 0.0).astype(np.float32)
    z = np.zeros(geom.N, np.float32)
    return Scenario("lake_at_rest", geom, h0, z, z.copy(), np.full(geom.N, 0.03, np.float32), t_end=600.0,
                    meta={"surface_m": 1.0, "cfl": 0.9})


def fractal_terrain(geom: MeshGeometry, side: float, relief: float, seed: int, channel: float = 3.0) -> NDArray[np.float32]:
    xy = geom.world_centroid
    bed = fractal_dem(xy, side, relief=relief, beta=2.0, seed=seed)
    if channel > 0.0:
        bed = carve_channel(xy, bed, side, depth=channel, width=max(3.0 * side / np.sqrt(geom.N), 10.0), seed=seed + 1)
    return bed.astype(np.float32)


def dam_break(n_cells: int = 1_000_000, seed: int = 2, side: float = 10_000.0) -> Scenario:
    geom = voronoi_geometry(n_cells, side, seed)
    geom = with_bed(geom, fractal_terrain(geom, side, 20.0, seed))
    xy = geom.world_centroid
    r = np.hypot(xy[:, 0] - side / 2, xy[:, 1] - side / 2)
    h0 = np.where(r <= 0.05 * side, 4.0, 0.0).astype(np.float32)
    z = np.zeros(geom.N, np.float32)
    return Scenario("dam_break", geom, h0, z, z.copy(), np.full(geom.N, 0.035, np.float32), t_end=3600.0,
                    meta={"radius_m": 0.05 * side, "depth_m": 4.0, "centre_m": (side / 2, side / 2)})


def triangular_hydrograph(t: NDArray[np.float64] | float, peak: float, t_peak: float, t_end: float):
    """Discharge of a triangle rising from 0 at t=0 to ``peak`` at ``t_peak`` and back to 0 at ``t_end``."""
    t = np.asarray(t, dtype=np.float64)
    up = np.clip(t / t_peak, 0.0, 1.0)
    down = np.clip((t_end - t) / (t_end - t_peak), 0.0, 1.0)
    return peak * np.where(t <= t_peak, up, down)


def rain_inflow(n_cells: int = 4_000_000, seed: int = 3, side: float = 20_000.0, phase_s: float = 60.0) -> Scenario:
    geom = voronoi_geometry(n_cells, side, seed)
    geom = with_bed(geom, fractal_terrain(geom, side, 40.0, seed))
    rng = np.random.default_rng(seed)
    manning = np.exp(rng.uniform(np.log(0.02), np.log(0.08), geom.N)).astype(np.float32)
    z = np.zeros(geom.N, np.float32)
    rain = 0.05 / 3600.0  # 50 mm/h in m/s
    area = geom.area.astype(np.float64)
    inflow_cell = int(np.argmax(geom.zb))  # inflow enters at the highest cell
    phases = []
    for k in range(int(1800.0 / phase_s)):
        t_mid = (k + 0.5) * phase_s
        rate = (rain * area).astype(np.float32)
        rate[inflow_cell] += np.float32(triangular_hydrograph(t_mid, 200.0, 1200.0, 1800.0))
        phases.append((k * phase_s, rate))
    kt, kq = triangular_knots(200.0, 1200.0, 1800.0)
    inflow = Hydrograph(cells=np.array([inflow_cell]), knot_t=kt, knot_q=kq)
    return Scenario("rain_inflow", geom, z.copy(), z.copy(), z.copy(), manning, t_end=1800.0, source_phases=phases,
                    source_rate=(rain * area).astype(np.float32), hydrographs=[inflow],
                    meta={"rain_m_per_s": rain, "inflow_cell": inflow_cell, "peak_m3s": 200.0})


def batch_member(n_cells: int, seed: int, spacing: float = 10.0) -> Scenario:
    side = spacing * np.sqrt(n_cells)
    geom = voronoi_geometry(n_cells, side, seed)
    geom = with_bed(geom, fractal_terrain(geom, side, 20.0, seed))
    rng = np.random.default_rng(seed)
    manning = rng.uniform(0.02, 0.06, geom.N).astype(np.float32)
    peak = float(rng.uniform(10.0, 300.0))
    z = np.zeros(geom.N, np.float32)
    cell = int(np.argmax(geom.zb))
    kt, kq = triangular_knots(peak, 1200.0, 1800.0)
    inflow = Hydrograph(cells=np.array([cell]), knot_t=kt, knot_q=kq)
    return Scenario("batch_member", geom, z.copy(), z.copy(), z.copy(), manning, t_end=1800.0, hydrographs=[inflow],
                    meta={"inflow_cell": cell, "peak_m3s": peak})


def calibration(n_cells: int = 250_000, seed: int = 5, knots: int = 32, gauges: int = 200,
                spacing: float = 10.0) -> Scenario:
    """The adjoint workload: a pond on fractal terrain fed by an inflow hydrograph.

    A Voronoi mesh at ``spacing`` m on a fractal DEM (beta 2, 20 m relief),
    1 m of water within 10 % of the side of a centre point, a triangular
    inflow there (200 m^3/s at 20 min, 0 at 30 min) given by ``knots``
    evenly spaced knots over 30 min, ``gauges`` seeded cells within 20 % of
    the side of that point, and a seeded "true" Manning field uniform in
    [0.02, 0.06]; ``manning`` (the starting guess) is 0.035 everywhere.
    """
    side = spacing * np.sqrt(n_cells)
    geom = voronoi_geometry(n_cells, side, seed)
    geom = with_bed(geom, fractal_terrain(geom, side, 20.0, seed))
    rng = np.random.default_rng(seed)
    xy = geom.world_centroid
    centre = np.array([0.4 * side, 0.5 * side])
    r = np.hypot(xy[:, 0] - centre[0], xy[:, 1] - centre[1])
    h0 = np.where(r <= 0.1 * side, 1.0, 0.0).astype(np.float32)
    inflow_cell = int(np.argmin(r))
    kt = np.linspace(0.0, 1800.0, knots).astype(np.float32)
    kq = np.asarray(triangular_hydrograph(kt.astype(np.float64), 200.0, 1200.0, 1800.0), np.float32)
    inflow = Hydrograph(cells=np.array([inflow_cell]), knot_t=kt, knot_q=kq)
    near = np.flatnonzero(r <= 0.2 * side)
    gauge_cells = np.sort(rng.choice(near, size=min(gauges, near.size), replace=False))
    n_true = rng.uniform(0.02, 0.06, geom.N).astype(np.float32)
    z = np.zeros(geom.N, np.float32)
    return Scenario("calibration", geom, h0, z, z.copy(), np.full(geom.N, 0.035, np.float32), t_end=1800.0,
                    hydrographs=[inflow],
                    meta={"gauges": gauge_cells, "n_true": n_true, "inflow_cell": inflow_cell, "peak_m3s": 200.0})


def batch_sizes(count: int = 64, lo: int = 20_000, hi: int = 500_000, seed: int = 4) -> list[int]:
    rng = np.random.default_rng(seed)
    return [int(v) for v in np.exp(rng.uniform(np.log(lo), np.log(hi), count)).round()]


def open_channel(cells: int = 300, across: int = 20, length: float = 3000.0, width: float = 200.0,
                 slope: float = 1e-3, manning: float = 0.03, depth: float = 0.0, bed_top: float = 10.0) -> Scenario:
    """A channel falling ``slope`` in +x from ``bed_top``, ``depth`` of still water, open at both ends.

    ``meta["open_edges"]`` holds the wall edges at x = 0 and at x = length (the
    reference's ``Channel.end`` stretches, tolerance a quarter cell).
    """
    mesh = channel_grid(cells, across, length, width)
    dx = length / cells
    x = np.tile((np.arange(cells) + 0.5) * dx, across)
    zb = (bed_top - slope * x).astype(np.float32)
    geom = build_geometry(mesh.verts, mesh.faces, mesh.offsets, zb_from_file=zb)
    geom = hilbert_reorder(geom, verbose=False)[0]
    ends = [select_boundary_edges(geom, [(xe, 0.0), (xe, width)], 0.25 * dx) for xe in (0.0, length)]
    h0 = np.full(geom.N, depth, np.float32)
    z = np.zeros(geom.N, np.float32)
    return Scenario("open_channel", geom, h0, z, z.copy(), np.full(geom.N, manning, np.float32), t_end=60.0,
                    dt_max=1.0, dt_init=0.01,
                    meta={"open_edges": ends, "slope": slope, "manning": manning, "dx": dx, "width": width})
