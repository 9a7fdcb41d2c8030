"""Application-facing workflow API, mirroring the reference's ``inundation/workflow.py``.

Same dataclasses, fields, defaults, validation and ``SWEWorkflow.prepare() /
run(phases) -> WorkflowResult`` flow as the reference (``workflow.py:60-256,
635-969``), with one more backend name in the registry: ``b200_resident``,
the CUDA backend of this package (and the default here). The reference's
Vulkan backends (``baseline``, ``fixed_dt_batch_barrier``,
``gpu_resident_batch``) are accepted by the config, as in the reference, and
refused by ``prepare()``: this package has no Vulkan path.

Open boundaries work as in the reference (``workflow.py:361-445, 789-806,
859-867, 947-953``): each ``OpenBoundary`` line selects its stretch of wall
edges at ``prepare()``, every phase names a condition for every stretch, and
``WorkflowResult.boundary_volumes_m3`` holds each stretch's cumulative volume
out of and into the mesh at every snapshot.

Not carried over: the GIS mesh readers (meshes come from a geometry-cache
artifact, an ``.obj`` or an ``.npz`` file, or a ``MeshGeometry`` passed in).
"""

from __future__ import annotations

import os
import sys
import time
from collections.abc import Mapping, Sequence
from dataclasses import dataclass, field
from pathlib import Path
from dataclasses import astuple
from typing import Any, Literal

import numpy as np
from numpy.typing import NDArray

from .mesh.boundaries import conveyance_split, select_boundary_edges
from .mesh.cache import geometry_cache_key, load_geometry_cache, load_geometry_cache_artifact, save_geometry_cache
from .mesh.geometry import MeshGeometry, build_geometry, hilbert_reorder
from .mesh.loader import load_mesh_file
from .tuning import (
    B200_BACKEND,
    DRY_TOL_DEFAULT,
    GRAVITY_G,
    MOMENTUM_SNAPSHOT_BACKENDS,
    OPEN_BOUNDARY_BACKENDS,
    OPEN_FREE,
    OPEN_INFLOW,
    OPEN_NORMAL,
    OPEN_STAGE,
    OPEN_WALL,
    SOLVER_IMPLS,
)

INITIAL_STATE_METADATA_KEYS = frozenset({"saved_order", "mesh_source", "t_end_s", "dt_max", "cfl_interval"})


@dataclass(frozen=True)
class PointSource:
    """Volumetric source over a circular area: total discharge [m^3/s], centre (mesh coordinates), radius [m]."""

    discharge_m3s: float
    center_xy: tuple[float, float]
    radius_m: float


@dataclass(frozen=True)
class OpenBoundary:
    name: str
    line: Sequence[tuple[float, float]]
    tolerance_m: float


@dataclass(frozen=True)
class Wall:
    """The stretch stays closed for this phase."""


@dataclass(frozen=True)
class FreeOutflow:
    """Zero-gradient outflow."""


@dataclass(frozen=True)
class NormalDepth:
    energy_slope: float


@dataclass(frozen=True)
class Stage:
    elevation_m: float


@dataclass(frozen=True)
class Inflow:
    discharge_m3s: float
    energy_slope: float


BoundaryCondition = Wall | FreeOutflow | NormalDepth | Stage | Inflow


@dataclass(frozen=True)
class SimulationPhase:
    """One phase of a hydrograph schedule."""

    duration_s: float
    sources: Sequence[PointSource]
    boundaries: Mapping[str, BoundaryCondition] = field(default_factory=dict)


@dataclass(frozen=True)
class WorkflowConfig:
    """Runtime configuration of ``SWEWorkflow`` (the reference's fields and checks)."""

    mesh_source: str | None
    manning_n: float
    output_interval_s: float
    dt_max: float
    cfl_interval: int
    gravity: float = GRAVITY_G
    dry_tol: float = DRY_TOL_DEFAULT
    cfl: float | None = None
    workgroup_size: int = 256
    dt_init: float = 1e-2
    use_hilbert_reorder: bool = True
    progress: bool = True
    area_tol: float = 1e-6
    initial_state_source: dict[str, object] | str | os.PathLike[str] | None = None
    initial_state_order: str = "solver"
    initial_state_id_col: str = "cell_id"
    track_clamp_mass: bool = False
    geometry_cache_dir: str | os.PathLike[str] | None = None
    geometry_cache_source: str | os.PathLike[str] | None = None
    capture_momentum_snapshots: bool = False
    open_boundaries: Sequence[OpenBoundary] = ()
    steps_per_graph: int | None = None
    deterministic: bool | None = None
    compensated: bool | None = None
    output_every_steps: int | None = None
    solver_impl: Literal["baseline", "fixed_dt_batch_barrier", "gpu_resident_batch", "b200_resident"] = B200_BACKEND

    def __post_init__(self) -> None:
        if self.mesh_source is None and self.geometry_cache_source is None:
            raise ValueError(
                "mesh_source is required unless geometry_cache_source points at a prebuilt geometry-cache artifact"
            )
        if self.manning_n <= 0:
            raise ValueError(f"manning_n must be positive, got {self.manning_n}")
        if self.output_interval_s <= 0:
            raise ValueError(f"output_interval_s must be positive, got {self.output_interval_s}")
        if self.dt_max <= 0:
            raise ValueError(f"dt_max must be positive, got {self.dt_max}")
        if self.cfl_interval <= 0:
            raise ValueError(f"cfl_interval must be positive, got {self.cfl_interval}")
        if self.steps_per_graph is not None and self.steps_per_graph <= 0:
            raise ValueError(f"steps_per_graph must be positive, got {self.steps_per_graph}")
        if self.output_every_steps is not None and self.output_every_steps <= 0:
            raise ValueError(f"output_every_steps must be positive, got {self.output_every_steps}")
        if self.solver_impl not in SOLVER_IMPLS:
            raise ValueError(f"unsupported solver_impl: {self.solver_impl}")
        if self.capture_momentum_snapshots and self.solver_impl not in MOMENTUM_SNAPSHOT_BACKENDS:
            raise ValueError(
                f"capture_momentum_snapshots is not supported by solver_impl {self.solver_impl!r}; "
                f"use one of {sorted(MOMENTUM_SNAPSHOT_BACKENDS)}"
            )
        if self.open_boundaries:
            if self.solver_impl not in OPEN_BOUNDARY_BACKENDS:
                raise ValueError(
                    f"open_boundaries is not supported by solver_impl {self.solver_impl!r}; "
                    f"use one of {sorted(OPEN_BOUNDARY_BACKENDS)}"
                )
            if self.deterministic is False:
                raise ValueError("open_boundaries need deterministic accumulation")
            names = [b.name for b in self.open_boundaries]
            if len(set(names)) != len(names):
                raise ValueError(f"open boundary names repeat: {sorted(names)}")


@dataclass
class WorkflowResult:
    snapshots: list[NDArray[np.float32]]
    snap_times: list[float]
    h_final: NDArray[np.float32]
    volume_final_m3: float
    volume_injected_m3: float
    wall_seconds: float
    steps_total: int
    hu_final: NDArray[np.float32] | None = None
    hv_final: NDArray[np.float32] | None = None
    hu_snapshots: list[NDArray[np.float32]] | None = None
    hv_snapshots: list[NDArray[np.float32]] | None = None
    clamp_mass_m3: float | None = None
    boundary_volumes_m3: dict[str, NDArray[np.float64]] = field(default_factory=dict)


def _point_in_polygon(point: NDArray[np.float64], polygon: NDArray[np.float64]) -> bool:
    """Inside or on the boundary of a polygon (the reference's ``workflow.py:294-314``)."""
    x, y = float(point[0]), float(point[1])
    tol = 1e-10 * max(1.0, float(np.abs(polygon).max()), abs(x), abs(y))
    inside = False
    for a, b in zip(polygon, np.roll(polygon, -1, axis=0), strict=True):
        ax, ay, bx, by = float(a[0]), float(a[1]), float(b[0]), float(b[1])
        cross = (x - ax) * (by - ay) - (y - ay) * (bx - ax)
        if abs(cross) <= tol and min(ax, bx) - tol <= x <= max(ax, bx) + tol and min(ay, by) - tol <= y <= max(ay, by) + tol:
            return True
        if (ay > y) != (by > y) and x < ax + (y - ay) * (bx - ax) / (by - ay):
            inside = not inside
    return inside


def select_cells_within_radius(
    centroid: NDArray[np.float32],
    center_xy: tuple[float, float],
    radius_m: float,
    valid_mask: NDArray[np.bool_] | None = None,
    cell_vertices: NDArray[np.float32] | None = None,
    cell_vertex_ptr: NDArray[np.int32] | None = None,
    cell_bbox: NDArray[np.float32] | None = None,
) -> NDArray[np.bool_]:
    """Cells whose centroid is within the radius, plus the cell containing the centre."""
    center = np.asarray(center_xy, dtype=np.float64)
    if radius_m < 0.0:
        return np.zeros(centroid.shape[0], dtype=bool)
    mask = np.hypot(centroid[:, 0] - center[0], centroid[:, 1] - center[1]) <= float(radius_m)
    if valid_mask is not None:
        mask &= valid_mask
    if cell_vertices is None or cell_vertex_ptr is None or cell_bbox is None or not centroid.shape[0]:
        return mask
    bbox = np.asarray(cell_bbox, dtype=np.float64)
    cand = (bbox[:, 0] <= center[0]) & (bbox[:, 1] >= center[0]) & (bbox[:, 2] <= center[1]) & (bbox[:, 3] >= center[1])
    if valid_mask is not None:
        cand &= valid_mask
    for c in np.flatnonzero(cand):
        ring = np.asarray(cell_vertices[int(cell_vertex_ptr[c]): int(cell_vertex_ptr[c + 1])], dtype=np.float64)
        if _point_in_polygon(center, ring):
            mask[c] = True
    return mask


def build_phase_source_rate(geom: MeshGeometry, phase: SimulationPhase, valid_cell: NDArray[np.bool_]) -> NDArray[np.float32]:
    """Per-cell source [m^3/s] of a phase: each source's discharge split by area (``workflow.py:599-625``)."""
    src = np.zeros(geom.N, dtype=np.float32)
    ox, oy = geom.origin.tolist()
    for source in phase.sources:
        cx, cy = source.center_xy
        mask = select_cells_within_radius(
            geom.centroid, (cx - ox, cy - oy), source.radius_m, valid_mask=valid_cell,
            cell_vertices=geom.cell_vertices, cell_vertex_ptr=geom.cell_vertex_ptr, cell_bbox=geom.cell_bbox,
        )
        if not mask.any():
            continue
        a = geom.area[mask]
        total = float(a.sum())
        if total <= 0.0:
            continue
        src[mask] += np.float32(source.discharge_m3s) * (a / total)
    return src


def _as_f32(name: str, values: object, n: int) -> NDArray[np.float32]:
    arr = np.asarray(values, dtype=np.float32).reshape(-1)
    if arr.size != n:
        raise ValueError(f"{name}: expected {n} values, got {arr.size}")
    if not np.isfinite(arr).all():
        raise ValueError(f"{name}: contains non-finite values")
    return arr


def load_initial_state(source, n_cells: int, zb: NDArray[np.float32], *, order: str, id_col: str,
                       perm: NDArray[np.int32], dry_tol: float):
    """Optional per-cell initial state ``(h, hu, hv, n or None)`` (the reference's ``workflow.py:450-596``)."""
    if source is None:
        return None
    if isinstance(source, dict):
        state = {k: np.asarray(v) for k, v in source.items()}
    else:
        path = Path(os.fspath(source))
        if not path.exists():
            raise FileNotFoundError(f"Initial state file not found: {path}")
        suffix = path.suffix.lower()
        if suffix == ".npz":
            with np.load(path) as npz:
                state = {k: npz[k] for k in npz.files}
        elif suffix == ".npy":
            arr = np.load(path)
            if arr.ndim != 2 or arr.shape[1] not in (3, 4):
                raise ValueError("For .npy input, expected shape (N,3)=[h,hu,hv] or (N,4)=[h,hu,hv,n_mann]")
            state = {"h": arr[:, 0], "hu": arr[:, 1], "hv": arr[:, 2]}
            if arr.shape[1] == 4:
                state["n_mann"] = arr[:, 3]
        elif suffix in (".csv", ".parquet"):
            import pandas as pd

            df = pd.read_csv(path) if suffix == ".csv" else pd.read_parquet(path)
            state = {c: df[c].to_numpy() for c in df.columns}
        else:
            raise ValueError(f"Unsupported initial state format: {suffix}. Use .npz, .npy, .csv, or .parquet")
    valid = {"h", "wse", "hu", "hv", "u", "v", "n_mann", id_col}
    state = {k: v for k, v in state.items() if k not in INITIAL_STATE_METADATA_KEYS}
    bad = sorted(k for k in state if k not in valid)
    if bad:
        raise ValueError(f"initial state contains unsupported fields: {bad}. Supported fields: {sorted(valid)}")
    if id_col in state:
        raw = np.asarray(state[id_col]).reshape(-1)
        try:
            ids_f = raw.astype(np.float64)
        except (TypeError, ValueError) as exc:
            raise ValueError(f"{id_col}: values must be numeric integers") from exc
        if not np.isfinite(ids_f).all():
            raise ValueError(f"{id_col}: values must be finite numeric integers")
        if not np.equal(ids_f, np.floor(ids_f)).all():
            raise ValueError(f"{id_col}: values must be integers")
        ids = ids_f.astype(np.int64)
        if ids.size != n_cells:
            raise ValueError(f"{id_col}: expected {n_cells} rows, got {ids.size}")
        if np.unique(ids).size != n_cells:
            raise ValueError(f"{id_col}: values must be unique")
        if ids.min() < 0 or ids.max() >= n_cells:
            raise ValueError(f"{id_col}: values must be in [0, {n_cells - 1}]")
        aligned = {}
        for key, values in state.items():
            if key == id_col:
                continue
            src = np.asarray(values).reshape(-1)
            if src.size != n_cells:
                raise ValueError(f"{key}: expected {n_cells} rows, got {src.size}")
            dst = np.empty(n_cells, dtype=src.dtype)
            dst[ids] = src
            aligned[key] = dst
        state = aligned
    if "h" in state:
        h = _as_f32("h", state["h"], n_cells)
    elif "wse" in state:
        h = _as_f32("wse", state["wse"], n_cells) - zb.astype(np.float32)
    else:
        raise ValueError("Initial state must provide 'h' or 'wse'")
    if "hu" in state and "hv" in state:
        hu, hv = _as_f32("hu", state["hu"], n_cells), _as_f32("hv", state["hv"], n_cells)
    elif "u" in state and "v" in state:
        hu, hv = h * _as_f32("u", state["u"], n_cells), h * _as_f32("v", state["v"], n_cells)
    else:
        raise ValueError("Initial state must provide (hu,hv) or (u,v)")
    n_mann = _as_f32("n_mann", state["n_mann"], n_cells) if "n_mann" in state else None
    if order not in ("solver", "original"):
        raise ValueError("initial_state_order must be 'solver' or 'original'")
    if order == "original":
        h, hu, hv = h[perm], hu[perm], hv[perm]
        if n_mann is not None:
            n_mann = n_mann[perm]
    h = np.maximum(h, 0.0).astype(np.float32)
    wet = h > np.float32(dry_tol)
    hu = np.where(wet, hu, 0.0).astype(np.float32)
    hv = np.where(wet, hv, 0.0).astype(np.float32)
    if n_mann is not None:
        n_mann = np.maximum(n_mann.astype(np.float32), np.float32(1e-4))
    return h, hu, hv, n_mann


def open_stretch_edges(geom: MeshGeometry, boundaries: Sequence[OpenBoundary]) -> list[NDArray[np.int64]]:
    """Each stretch's wall edges (``workflow.py:361-377``); a stretch selecting none, or an edge twice, raises."""
    stretches = [select_boundary_edges(geom, b.line, b.tolerance_m) for b in boundaries]
    for b, edges in zip(boundaries, stretches, strict=True):
        if not edges.size:
            raise ValueError(f"open boundary {b.name!r} selects no boundary edges within {b.tolerance_m} m of its line")
    every = np.concatenate(stretches) if stretches else np.empty(0, dtype=np.int64)
    if np.unique(every).size != every.size:
        raise ValueError("open boundaries select the same edge twice")
    return stretches


def open_conditions(geom: MeshGeometry, manning: NDArray[np.float32], boundary: OpenBoundary,
                    condition: BoundaryCondition, edges: NDArray[np.int64]) -> tuple[int, NDArray[np.float32]]:
    """Condition code and per-edge value of one stretch (``workflow.py:380-412``).

    Normal depth: sqrt(S) / n of the cell inside; stage: the level's depth over
    that cell's bed (0 below it); inflow: discharge per unit width by conveyance.
    """
    cells = geom.edge_cellL[edges]
    if not np.isfinite(astuple(condition)).all():
        raise ValueError(f"open boundary {boundary.name!r} has a non-finite value: {condition}")
    if isinstance(condition, Wall):
        return OPEN_WALL, np.zeros(edges.size, dtype=np.float32)
    if isinstance(condition, FreeOutflow):
        return OPEN_FREE, np.zeros(edges.size, dtype=np.float32)
    if isinstance(condition, NormalDepth):
        if condition.energy_slope <= 0.0:
            raise ValueError(f"open boundary {boundary.name!r} needs a positive energy slope")
        return OPEN_NORMAL, (np.sqrt(condition.energy_slope) / manning[cells]).astype(np.float32)
    if isinstance(condition, Stage):
        depth = condition.elevation_m - geom.zb[cells].astype(np.float64)
        return OPEN_STAGE, np.maximum(depth, 0.0).astype(np.float32)
    if condition.energy_slope <= 0.0:
        raise ValueError(f"open boundary {boundary.name!r} needs a positive energy slope")
    if condition.discharge_m3s < 0.0:
        raise ValueError(f"open boundary {boundary.name!r} has a negative inflow")
    return OPEN_INFLOW, conveyance_split(condition.discharge_m3s, geom.edge_len[edges], geom.zb[cells],
                                         manning[cells], condition.energy_slope)


def build_phase_open_conditions(geom: MeshGeometry, manning: NDArray[np.float32], boundaries: Sequence[OpenBoundary],
                                stretches: Sequence[NDArray[np.int64]],
                                phase: SimulationPhase) -> tuple[NDArray[np.uint32], NDArray[np.float32]]:
    """Per-edge condition codes and values of one phase, in stretch order (``workflow.py:415-437``)."""
    names = {b.name for b in boundaries}
    if set(phase.boundaries) != names:
        raise ValueError(f"phase boundaries {sorted(phase.boundaries)} must name every open boundary: {sorted(names)}")
    kinds, values = [], []
    for b, edges in zip(boundaries, stretches, strict=True):
        kind, value = open_conditions(geom, manning, b, phase.boundaries[b.name], edges)
        kinds.append(np.full(edges.size, kind, dtype=np.uint32))
        values.append(value)
    return np.concatenate(kinds), np.concatenate(values)


def _backend_class(name: str):
    if name == B200_BACKEND:
        from .backend import SWESolverB200Resident

        return SWESolverB200Resident
    raise RuntimeError(
        f"solver_impl {name!r} is a Vulkan/Kompute backend of the reference, which inundation_b200 does not "
        f"include; use solver_impl={B200_BACKEND!r}"
    )


class SWEWorkflow:
    """``prepare()`` once (geometry, initial state, device buffers), then ``run(phases)`` per request."""

    def __init__(self, config: WorkflowConfig, geometry: MeshGeometry | None = None) -> None:
        self.config = config
        self.geom: MeshGeometry | None = None
        self.perm: NDArray[np.int32] | None = None
        self.solver: Any = None
        self._geometry = geometry
        self._open_stretches: list[NDArray[np.int64]] = []
        self._manning: NDArray[np.float32] | None = None

    def _log(self, msg: str) -> None:
        if self.config.progress:
            sys.stdout.write(f"[prepare] {msg}\n")
            sys.stdout.flush()

    def _load_geometry(self) -> tuple[MeshGeometry, NDArray[np.int32]]:
        cfg = self.config
        if self._geometry is not None:
            return self._geometry, np.arange(self._geometry.N, dtype=np.int32)
        if cfg.geometry_cache_source is not None:
            geom, perm, meta = load_geometry_cache_artifact(cfg.geometry_cache_source)
            if meta.use_hilbert_reorder != cfg.use_hilbert_reorder:
                raise ValueError(
                    f"geometry cache artifact {cfg.geometry_cache_source} was built with use_hilbert_reorder="
                    f"{meta.use_hilbert_reorder}, but WorkflowConfig.use_hilbert_reorder is {cfg.use_hilbert_reorder}"
                )
            self._log(f"geometry cache artifact loaded ({cfg.geometry_cache_source})")
            return geom, perm
        if cfg.mesh_source is None:
            raise RuntimeError("mesh_source is None without a geometry cache source")
        key = ""
        if cfg.geometry_cache_dir is not None:
            key = geometry_cache_key(cfg.mesh_source, use_hilbert_reorder=cfg.use_hilbert_reorder)
            cached = load_geometry_cache(cfg.geometry_cache_dir, key)
            if cached is not None:
                self._log("geometry cache hit")
                return cached
        verts, faces, offsets, zb, manning = load_mesh_file(cfg.mesh_source)
        geom = build_geometry(verts, faces, offsets, zb_from_file=zb, manning_n_from_file=manning)
        perm = np.arange(geom.N, dtype=np.int32)
        if cfg.use_hilbert_reorder:
            geom, perm = hilbert_reorder(geom, verbose=False)
        if cfg.geometry_cache_dir is not None:
            save_geometry_cache(cfg.geometry_cache_dir, key, geom, perm)
        return geom, perm

    def prepare(self) -> None:
        cfg = self.config
        cls = _backend_class(cfg.solver_impl)
        geom, perm = self._load_geometry()
        h0 = np.zeros(geom.N, dtype=np.float32)
        hu0 = np.zeros(geom.N, dtype=np.float32)
        hv0 = np.zeros(geom.N, dtype=np.float32)
        n0 = geom.manning_n if geom.manning_n is not None else np.full(geom.N, cfg.manning_n, dtype=np.float32)
        loaded = load_initial_state(
            cfg.initial_state_source, geom.N, geom.zb, order=cfg.initial_state_order,
            id_col=cfg.initial_state_id_col, perm=perm, dry_tol=cfg.dry_tol,
        )
        if loaded is not None:
            h0, hu0, hv0, n_loaded = loaded
            if n_loaded is not None:
                n0 = n_loaded
        self._open_stretches = open_stretch_edges(geom, cfg.open_boundaries)
        self._manning = np.asarray(n0, dtype=np.float32)
        open_args: dict[str, Any] = {"open_edges": self._open_stretches} if self._open_stretches else {}
        solver = cls(geom, None, h0, hu0, hv0, n0, g=cfg.gravity, dry_tol=cfg.dry_tol, cfl=cfg.cfl,
                     workgroup_size=cfg.workgroup_size, **open_args)
        if cfg.track_clamp_mass:
            solver.track_clamp = True
        if cfg.steps_per_graph is not None:
            solver.steps_per_graph = cfg.steps_per_graph
        if cfg.deterministic is not None:
            solver.deterministic = cfg.deterministic
        if cfg.compensated is not None:
            solver.compensated = cfg.compensated
        self.geom, self.perm, self.solver = geom, perm, solver

    def run(self, phases: Sequence[SimulationPhase]) -> WorkflowResult:
        """Run the phases back to back (``workflow.py:828-969``)."""
        if self.geom is None or self.solver is None:
            raise RuntimeError("Workflow not prepared. Call prepare() first.")
        if not phases:
            raise ValueError("At least one phase is required.")
        cfg = self.config
        area = self.geom.area
        valid = area > cfg.area_tol
        snaps: list[NDArray[np.float32]] = []
        times: list[float] = []
        hu_s: list[NDArray[np.float32]] | None = [] if cfg.capture_momentum_snapshots else None
        hv_s: list[NDArray[np.float32]] | None = [] if cfg.capture_momentum_snapshots else None
        t = 0.0
        wall0 = time.perf_counter()
        for k, phase in enumerate(phases):
            if phase.duration_s <= 0.0:
                raise ValueError(f"Phase {k} has non-positive duration.")
            t_end = t + phase.duration_s
            if self._open_stretches:
                self.solver.set_open_conditions(*build_phase_open_conditions(
                    self.geom, self._manning, cfg.open_boundaries, self._open_stretches, phase))
            out = self.solver.run(
                t_end=t_end, output_interval_s=cfg.output_interval_s, dt_max=cfg.dt_max, dt_init=cfg.dt_init,
                progress=cfg.progress, source_rate=build_phase_source_rate(self.geom, phase, valid), resume=k > 0,
                t_start=t, cfl_interval=cfg.cfl_interval, output_every_steps=None,
                capture_momentum_snapshots=cfg.capture_momentum_snapshots,
            )
            if cfg.capture_momentum_snapshots:
                ph_s, ph_t, ph_hu, ph_hv = out
                hu_s.extend(ph_hu)
                hv_s.extend(ph_hv)
            else:
                ph_s, ph_t = out
            snaps.extend(ph_s)
            times.extend(ph_t)
            t = t_end
        wall = time.perf_counter() - wall0
        h_final = self.solver.download_h()
        volume = float((self.solver.download_h_precise() * area.astype(np.float64)).sum())
        injected = float(sum(p.duration_s * sum(s.discharge_m3s for s in p.sources) for p in phases))
        clamp = None
        if cfg.track_clamp_mass:
            clamp = float(np.asarray(self.solver.download_clamp_mass(), dtype=np.float64).sum())
        volumes: dict[str, NDArray[np.float64]] = {}
        if self._open_stretches:
            stacked = np.stack(self.solver.open_volume_snapshots)
            volumes = {b.name: stacked[:, k] for k, b in enumerate(cfg.open_boundaries)}
        return WorkflowResult(
            snapshots=snaps, snap_times=times, h_final=h_final, volume_final_m3=volume,
            volume_injected_m3=injected, wall_seconds=wall, steps_total=int(self.solver.steps_total),
            hu_final=self.solver.download_hu(), hv_final=self.solver.download_hv(), hu_snapshots=hu_s,
            hv_snapshots=hv_s, clamp_mass_m3=clamp, boundary_volumes_m3=volumes,
        )


def inflow_phases(upstream: WorkflowResult, outlet: str, into: str, energy_slope: float,
                  other_boundaries: Mapping[str, BoundaryCondition] | None = None,
                  sources: Sequence[PointSource] = ()) -> list[SimulationPhase]:
    """Phases passing an upstream stretch's outflow into the next basin (``workflow.py:258-291``)."""
    times = np.asarray(upstream.snap_times, dtype=np.float64)
    volumes = upstream.boundary_volumes_m3[outlet][:, 0]
    ends = np.flatnonzero(np.diff(times) > 0.0) + 1
    starts = np.r_[0, ends[:-1]]
    return [
        SimulationPhase(
            float(times[e] - times[s]), sources,
            {**(other_boundaries or {}), into: Inflow(float((volumes[e] - volumes[s]) / (times[e] - times[s])), energy_slope)},
        )
        for s, e in zip(starts.tolist(), ends.tolist(), strict=True)
    ]


__all__ = [
    "BoundaryCondition", "FreeOutflow", "Inflow", "NormalDepth", "OpenBoundary", "PointSource", "SWEWorkflow",
    "SimulationPhase", "Stage", "Wall", "WorkflowConfig", "WorkflowResult", "build_phase_open_conditions",
    "build_phase_source_rate", "inflow_phases", "load_initial_state", "open_conditions", "open_stretch_edges",
    "select_cells_within_radius",
]
