"""``b200_resident``: the reference's GPU-resident backend protocol on B200 kernels.

Same constructor, ``run`` signature and semantics, ``download_*`` methods and
attributes as the reference's ``SWESolverGpuResidentBatch``
(``inundation/vulkan/gpu_resident_batch.py:140-762``, base class
``inundation/vulkan/solver.py:118-497``): every step picks its own dt on the
device from the CFL bound of its corrector fluxes, simulated time is a uint64
count of 2^-20 s ticks, each output window runs whole submits of
``steps_per_graph`` steps (no-op steps past the window's stop do nothing) and
the host reads the 48-byte control block after each submit.

Open boundaries (``open_edges``, ``set_open_conditions``,
``download_open_volumes``, ``open_volume_snapshots``) follow the reference's
base solver and resident backend (``solver.py:140-165, 236-243, 427-440``,
``gpu_resident_batch.py:447-466``): open edge ``k`` (stretch order) has right
cell ``-2 - k``, every other boundary edge stays a wall, and the volume through
each edge is kept as exact float pairs on the device and summed per stretch in
float64 on the host.

B200 specifics: a submit is one replay of a CUDA graph of ``steps_per_graph``
steps; torch CUDA tensors own all device memory; the C ABI kernels borrow
their pointers. There is no CPU fallback: without a GPU and the built
library, construction raises.
"""

from __future__ import annotations

import dataclasses
import math
import sys
import time as _time
from collections.abc import Callable, Sequence

import numpy as np
import torch
from numpy.typing import NDArray

from .engine import KERNELS, RESIDENT_CTRL_DTYPE, ResidentEngine
from .layout import build_tile_layout
from .mesh.geometry import MeshGeometry
from .tuning import (
    ACTIVE_BLOCK_CELLS,
    B200_BACKEND,
    DRY_TOL_DEFAULT,
    GRAVITY_G,
    dt_to_ticks,
    output_window_stops,
    seconds_to_ticks,
    ticks_to_seconds,
)

STEPS_PER_GRAPH_DEFAULT = 200
KERNEL_NAMES = {v: k for k, v in KERNELS.items()}


@dataclasses.dataclass(frozen=True)
class SubmitRecord:
    """One submit of a run: the clock after it, the steps it ran, the kernel that ran them and the
    active blocks the dilation left for the next submit (what ``stage_kernel = "auto"`` reads)."""

    now_ticks: int
    steps: int
    kernel: str
    active_blocks: int
    computed_cells: int  # cells of computed tiles over the run so far
    wall_s: float  # host monotonic clock when the submit's control block was read


class SWESolverB200Resident(ResidentEngine):
    """GPU-resident Heun steps with an integer clock, on one B200."""

    name = B200_BACKEND
    steps_per_graph: int = STEPS_PER_GRAPH_DEFAULT
    # Fixed-order gathers are the only accumulation: repeat runs are bit-identical.
    deterministic: bool = True
    # A list to have run() append one SubmitRecord per submit (None: no record is kept).
    submit_log: list[SubmitRecord] | None = None

    def __init__(
        self,
        geom: MeshGeometry,
        spv: object | None,
        h0: NDArray[np.float32],
        hu0: NDArray[np.float32],
        hv0: NDArray[np.float32],
        n0: NDArray[np.float32],
        *,
        g: float = GRAVITY_G,
        dry_tol: float = DRY_TOL_DEFAULT,
        cfl: float | None = None,
        workgroup_size: int = 256,
        open_edges: Sequence[NDArray[np.int64]] = (),
        device: int | str | torch.device | None = None,
    ) -> None:
        del spv  # no shader binaries: the kernels are in the CUDA library
        if workgroup_size != ACTIVE_BLOCK_CELLS:
            raise ValueError(f"{B200_BACKEND} needs workgroup_size={ACTIVE_BLOCK_CELLS}, got {workgroup_size}")
        self.geom = geom
        self.N, self.E = int(geom.N), int(geom.E)
        self.steps_total = 0
        self._pinned: dict[str, torch.Tensor] = {}
        self._open_stretches = [np.asarray(edges, dtype=np.int64).ravel() for edges in open_edges]
        # (stretches, 2) volume out of and into the mesh at every snapshot of a run.
        self.open_volume_snapshots: list[NDArray[np.float64]] = []
        open_ids = np.concatenate([np.empty(0, dtype=np.int64), *self._open_stretches])
        if open_ids.size:
            if open_ids.min() < 0 or open_ids.max() >= self.E:
                raise ValueError(f"open edges must index the mesh's {self.E} edges")
            if np.unique(open_ids).size != open_ids.size:
                raise ValueError("an edge is open more than once")
            if (geom.edge_cellR[open_ids] != -1).any():
                raise ValueError("open edges must be boundary edges (right cell -1)")
        self._open_cells = geom.edge_cellL[open_ids].astype(np.int64)
        self._h0 = np.asarray(h0, np.float32).ravel().copy()
        self._hu0 = np.asarray(hu0, np.float32).ravel().copy()
        self._hv0 = np.asarray(hv0, np.float32).ravel().copy()
        for name, arr in (("h0", self._h0), ("hu0", self._hu0), ("hv0", self._hv0)):
            if arr.size != self.N:
                raise ValueError(f"{name} has {arr.size} values for {self.N} cells")
        n0 = np.asarray(n0, np.float32).ravel()
        if n0.size != self.N:
            raise ValueError(f"n0 has {n0.size} values for {self.N} cells")
        cell_r = np.asarray(geom.edge_cellR).copy()
        cell_r[open_ids] = -2 - np.arange(open_ids.size, dtype=cell_r.dtype)
        layout = build_tile_layout(dataclasses.replace(geom, edge_cellR=cell_r) if open_ids.size else geom)
        n_pad = np.concatenate([n0, np.full(layout.n_padded_cells - self.N, 0.03, np.float32)])
        self._init_engine(layout, n_pad, g=g, dry_tol=dry_tol, cfl=cfl, device=device)
        self.reset(self._h0, self._hu0, self._hv0)

    # -- public state access (reference solver.py:390-497) --------------------------------------
    def _staging(self, name: str) -> torch.Tensor:
        """A page-locked host array of N floats, one per purpose, kept for the solver's life."""
        buf = self._pinned.get(name)
        if buf is None:
            buf = torch.empty(self.N, dtype=torch.float32).pin_memory()
            self._pinned[name] = buf
        return buf

    def _download(self, name: str) -> NDArray[np.float32]:
        # straight into a new host array: one copy (measured faster than a page-locked
        # staging buffer followed by a host copy into the array the caller keeps)
        out = np.empty(self.N, np.float32)
        with torch.cuda.stream(self._stream):
            torch.from_numpy(out).copy_(self._t[name][: self.N])
        return out

    def download_h(self) -> NDArray[np.float32]:
        return self._download("h")

    def download_hu(self) -> NDArray[np.float32]:
        return self._download("hu")

    def download_hv(self) -> NDArray[np.float32]:
        return self._download("hv")

    def download_h_residual(self) -> NDArray[np.float32]:
        return self._download("h_lo")

    def download_h_precise(self) -> NDArray[np.float64]:
        return self.download_h().astype(np.float64) + self.download_h_residual().astype(np.float64)

    def download_clamp_mass(self) -> NDArray[np.float32]:
        return self._download("clamp_mass")

    def reset_clamp_mass(self) -> None:
        with torch.cuda.stream(self._stream):
            self._t["clamp_mass"].zero_()

    def upload(self, name: str, values: NDArray[np.float32]) -> None:
        """Overwrite one state array (``h``, ``hu``, ``hv``, ``h1``, ...) on the device."""
        src = torch.from_numpy(np.ascontiguousarray(values, np.float32).ravel())
        with torch.cuda.stream(self._stream):
            self._t[name][: self.N].copy_(src)
        self._stream.synchronize()

    def reset(self, h0: NDArray[np.float32], hu0: NDArray[np.float32], hv0: NDArray[np.float32]) -> None:
        """Upload initial conditions; the compensated low words start at zero.

        The initial state is kept in page-locked host arrays of the solver (one per
        array), from which this and every later reset copy it asynchronously.
        """
        kept = []
        with torch.cuda.stream(self._stream):
            for name, values in (("h", h0), ("hu", hu0), ("hv", hv0)):
                buf = self._staging("initial_" + name)
                host = buf.numpy()
                src = np.asarray(values, np.float32).ravel()
                if src.ctypes.data != host.ctypes.data:  # a reset to the kept state copies nothing on the host
                    host[:] = src
                self._t[name][: self.N].copy_(buf, non_blocking=True)
                kept.append(host)
            self._t["h_lo"].zero_()
            self._t["h1_lo"].zero_()
            self._open_vol.zero_()
        self._stream.synchronize()
        self._h0, self._hu0, self._hv0 = kept

    def _reset_to_initial(self) -> None:
        self.reset(self._h0, self._hu0, self._hv0)

    def set_open_conditions(self, kinds: NDArray[np.uint32], values: NDArray[np.float32]) -> None:
        """Set every open edge's condition (``OPEN_*``), in stretch order, before a run or a phase.

        A block with an edge that can bring water in from outside stays active
        for as long as these conditions hold.
        """
        kinds, values = np.asarray(kinds), np.asarray(values)
        if kinds.size != self.n_open or values.size != self.n_open:
            raise ValueError(
                f"expected {self.n_open} open edges, got {kinds.size} kinds and {values.size} values"
            )
        self.set_open_edge_conditions(kinds, values)

    def download_open_volumes(self) -> NDArray[np.float64]:
        """``(stretches, 2)`` volume [m^3] out of and into the mesh since the start."""
        per_edge = self.download_open_edge_volumes()
        out = np.zeros((len(self._open_stretches), 2), dtype=np.float64)
        first = 0
        for s, edges in enumerate(self._open_stretches):
            out[s] = per_edge[first : first + edges.size].sum(axis=0)
            first += edges.size
        return out

    def _set_sources(self, source_rate: NDArray[np.float32] | None) -> None:
        """The reference's ``_set_sources`` (gpu_resident_batch.py:529-560): nonzero cells as (cell, rate / area)."""
        self.set_sources([source_rate])

    # -- the run loop (reference gpu_resident_batch.py:609-762) -----------------------------------
    def run(
        self,
        t_end: float,
        output_interval_s: float,
        dt_max: float,
        dt_init: float,
        cfl_interval: int,
        progress: bool = True,
        source_rate: NDArray[np.float32] | None = None,
        source_fn: Callable[[float], NDArray[np.float32]] | None = None,
        resume: bool = False,
        t_start: float = 0.0,
        capture_momentum_snapshots: bool = False,
        output_every_steps: int | None = None,
    ):
        """Advance to ``t_end``; snapshot every ``output_interval_s`` from the run's start.

        ``cfl_interval`` and ``output_every_steps`` are accepted for interface
        compatibility and ignored: the CFL bound is recomputed every step.
        """
        del cfl_interval, output_every_steps
        if source_fn is not None:
            raise ValueError(f"{B200_BACKEND} takes a constant source_rate per run, not source_fn")
        if self.steps_per_graph < 1:
            raise ValueError(f"steps_per_graph must be positive, got {self.steps_per_graph}")
        if not self.deterministic:
            raise ValueError(f"{B200_BACKEND} sums fluxes in a fixed order only; deterministic must stay True")
        dt_max_ticks = dt_to_ticks(dt_max)
        dry_dt_ticks = dt_to_ticks(min(dt_init, dt_max))
        start_ticks = seconds_to_ticks(t_start if resume else 0.0)
        end_ticks = seconds_to_ticks(t_end)
        interval_ticks = seconds_to_ticks(output_interval_s)
        if not resume:
            self._reset_to_initial()
            self.open_volume_snapshots = []
        # The open-edge volume tally is a two-sum too (gpu_resident_batch.py:659-660).
        if self.compensated or self.n_open:
            self._check_error_free_arithmetic()
        self._set_sources(source_rate)

        snapshots = [self.download_h() if resume else self._h0.copy()]
        snap_times = [ticks_to_seconds(start_ticks)]
        hu_snaps: list[NDArray[np.float32]] = []
        hv_snaps: list[NDArray[np.float32]] = []

        def capture() -> None:
            if capture_momentum_snapshots:
                hu_snaps.append(self.download_hu())
                hv_snaps.append(self.download_hv())
            if self.n_open:
                self.open_volume_snapshots.append(self.download_open_volumes())

        capture()
        ctrl = self._ctrl
        ctrl["error"] = 0
        ctrl["now_ticks"] = start_ticks
        ctrl["steps"] = 0
        ctrl["dt_ticks"] = 0
        ctrl["dt_max_ticks"] = dt_max_ticks
        ctrl["dry_dt_ticks"] = dry_dt_ticks
        ctrl["cfl_safety"] = self.cfl_safety
        self._graph()  # capture before the first window
        planned = False
        wall0 = _time.monotonic()
        last_log = wall0
        finite = True
        h_snap, snap_ticks = None, None  # the last window's depth and the clock it was read at
        for stop in output_window_stops(start_ticks, end_ticks, interval_ticks):
            ctrl["stop_ticks"] = stop
            self._sync_ctrl_to_device()
            if planned:
                self._enqueue_retarget()
            else:
                self._enqueue_prologue()
                planned = True
            self._read_ctrl()
            while int(ctrl["now_ticks"][0]) < stop:
                before = int(ctrl["now_ticks"][0])
                steps_before = int(ctrl["steps"][0])
                kernel = self._kernel  # per submit: "auto" may change kernel with the active fraction
                graph = self._graph()
                with torch.cuda.stream(self._stream):
                    graph.replay()
                self._read_ctrl()
                now_ticks = int(ctrl["now_ticks"][0])
                if self.submit_log is not None:
                    self.submit_log.append(SubmitRecord(now_ticks, int(ctrl["steps"][0]) - steps_before,
                                                        KERNEL_NAMES[kernel], self._active_blocks,
                                                        self._computed_cells_read(), _time.monotonic()))
                if now_ticks == before:
                    raise RuntimeError(
                        f"GPU-resident run made no time progress at t={ticks_to_seconds(now_ticks):.6f}s "
                        "(CFL bound below one tick)"
                    )
                now = _time.monotonic()
                if progress and now - last_log >= 10.0:
                    self._log_progress(now - wall0, now_ticks, start_ticks, end_ticks)
                    last_log = now
            h_snap, snap_ticks = self.download_h(), int(ctrl["now_ticks"][0])
            if not np.isfinite(h_snap).all():
                snapshots.append(np.nan_to_num(h_snap, nan=0.0, posinf=0.0))
                snap_times.append(ticks_to_seconds(stop))
                capture()
                finite = False
                break
            if (stop - start_ticks) % interval_ticks == 0:
                if progress:
                    sys.stdout.write(
                        f"[solver] snapshot {len(snapshots)} captured at t={ticks_to_seconds(stop):.2f}s "
                        f"(wall={_time.monotonic() - wall0:.1f}s)\n"
                    )
                    sys.stdout.flush()
                snapshots.append(h_snap)
                snap_times.append(ticks_to_seconds(stop))
                capture()
        self.steps_total += int(ctrl["steps"][0])
        if finite:
            # the state has not moved since the last window's read when the clock has not
            same = h_snap is not None and snap_ticks == int(ctrl["now_ticks"][0])
            h_final = h_snap if same else self.download_h()
            if not (np.array_equal(snapshots[-1], h_final) or np.allclose(snapshots[-1], h_final)):
                snapshots.append(h_final)
                snap_times.append(ticks_to_seconds(int(ctrl["now_ticks"][0])))
                capture()
        if capture_momentum_snapshots:
            return snapshots, snap_times, hu_snaps, hv_snaps
        return snapshots, snap_times

    def _log_progress(self, wall: float, now_ticks: int, start_ticks: int, end_ticks: int) -> None:
        t_sim, t_end = ticks_to_seconds(now_ticks), ticks_to_seconds(end_ticks)
        done = now_ticks - start_ticks
        eta = wall / done * (end_ticks - now_ticks) if done > 0 else math.inf
        pct = t_sim / t_end * 100.0 if t_end > 0 else 0.0
        sys.stdout.write(
            f"[solver][{B200_BACKEND} {int(self._ctrl['steps'][0])}] sim={t_sim:.2f}/{t_end:.2f}s ({pct:.1f}%) "
            f"eta~{eta:.1f}s\n"
        )
        sys.stdout.flush()


__all__ = ["RESIDENT_CTRL_DTYPE", "STEPS_PER_GRAPH_DEFAULT", "SWESolverB200Resident", "SubmitRecord"]
