"""Batches of independent scenarios in one resident launch sequence.

Every instance (its own mesh, bed, roughness, initial state and sources)
takes whole 256-cell blocks of one concatenated layout
(``layout.build_batch_layout``) and keeps its own integer clock, dt and CFL
bound on the device. One step of the batch is one launch of each kernel over
the active tiles of all instances together, so many small meshes fill the
GPU that one alone would leave mostly idle; a CUDA graph holds
``steps_per_graph`` such steps. An instance whose window is done runs no-op
steps until the others finish.

Each instance's results are bit-identical to a run of that scenario alone
(same tiles, same gather order, its own dt), which the tests check.
No counterpart in the reference, which runs one scenario per solver.
"""

from __future__ import annotations

import math
import sys
import time as _time
from collections.abc import Sequence
from dataclasses import dataclass, field

import numpy as np
import torch
from numpy.typing import NDArray

from .engine import ResidentEngine
from .layout import build_batch_layout
from .mesh.geometry import MeshGeometry
from .sources import Hydrograph
from .tuning import DRY_TOL_DEFAULT, GRAVITY_G, dt_to_ticks, seconds_to_ticks, ticks_to_seconds

_FOREVER_TICKS = 1 << 62  # a stop no run reaches: fixed-step runs


@dataclass
class BatchMember:
    """One scenario of a batch."""

    geom: MeshGeometry
    h0: NDArray[np.float32]
    hu0: NDArray[np.float32]
    hv0: NDArray[np.float32]
    n0: NDArray[np.float32]
    source_rate: NDArray[np.float32] | None = None  # m^3/s per cell, constant
    hydrographs: list[Hydrograph] = field(default_factory=list)


@dataclass
class BatchRun:
    """Outcome of ``BatchedSolver.run``: per instance, its steps and its depth at every window end."""

    steps: NDArray[np.int64]
    times: list[float]
    snapshots: list[list[NDArray[np.float32]]]


class BatchedSolver(ResidentEngine):
    """Resident Heun steps of many scenarios at once, one clock per scenario."""

    def __init__(
        self,
        members: Sequence[BatchMember],
        *,
        g: float = GRAVITY_G,
        dry_tol: float = DRY_TOL_DEFAULT,
        cfl: float | None = None,
        device: int | str | torch.device | None = None,
    ) -> None:
        if not members:
            raise ValueError("a batch needs at least one scenario")
        self.members = list(members)
        for i, m in enumerate(self.members):
            n = int(m.geom.N)
            for name in ("h0", "hu0", "hv0", "n0"):
                if np.asarray(getattr(m, name)).size != n:
                    raise ValueError(f"instance {i}: {name} has {np.asarray(getattr(m, name)).size} values for {n} cells")
        layout = build_batch_layout([m.geom for m in self.members])
        n_pad = np.full(layout.n_padded_cells, 0.03, np.float32)
        for i, m in enumerate(self.members):
            off = int(layout.inst_cell_offset[i])
            n_pad[off : off + int(m.geom.N)] = np.asarray(m.n0, np.float32).ravel()
        self._init_engine(layout, n_pad, g=g, dry_tol=dry_tol, cfl=cfl, device=device)
        self.set_sources([m.source_rate for m in self.members], [list(m.hydrographs) for m in self.members])
        self.reset()

    @property
    def cells(self) -> NDArray[np.int64]:
        return self.layout.inst_cells.copy()

    def reset(self) -> None:
        """Initial states of every instance; the compensated low words start at zero."""
        for name in ("h", "hu", "hv", "h_lo", "h1_lo", "h1", "hu1", "hv1"):
            with torch.cuda.stream(self._stream):
                self._t[name].zero_()
        for i, m in enumerate(self.members):
            for name, values in (("h", m.h0), ("hu", m.hu0), ("hv", m.hv0)):
                self.upload_state(name, values, i)

    def download_h(self, inst: int) -> NDArray[np.float32]:
        return self.download_state("h", inst)

    def download_hu(self, inst: int) -> NDArray[np.float32]:
        return self.download_state("hu", inst)

    def download_hv(self, inst: int) -> NDArray[np.float32]:
        return self.download_state("hv", inst)

    def download_h_residual(self, inst: int) -> NDArray[np.float32]:
        return self.download_state("h_lo", inst)

    @property
    def steps(self) -> NDArray[np.int64]:
        """Real steps of every instance since the last ``start``."""
        self._read_ctrl()
        return self._ctrl["steps"].astype(np.int64)

    @property
    def sim_time(self) -> NDArray[np.float64]:
        self._read_ctrl()
        return self._ctrl["now_ticks"].astype(np.float64) / float(1 << 20)

    # -- runs ------------------------------------------------------------------------------------
    def start(self, dt_max: float, dt_init: float, stop_s: float | Sequence[float] | None = None) -> None:
        """Reset every clock to 0 and run the prologue (marks, CFL bound, first dt).

        ``stop_s``: each instance's first stop in seconds, or in ticks as a
        uint64 array (None: no stop, for fixed-step runs).
        """
        if self.compensated:
            self._check_error_free_arithmetic()
        c = self._ctrl
        c["error"] = 0
        c["now_ticks"] = 0
        c["steps"] = 0
        c["dt_ticks"] = 0
        c["dt_max_ticks"] = dt_to_ticks(dt_max)
        c["dry_dt_ticks"] = dt_to_ticks(min(dt_init, dt_max))
        c["cfl_safety"] = self.cfl_safety
        c["stop_ticks"] = stop_s if isinstance(stop_s, np.ndarray) and stop_s.dtype == np.uint64 else self._stops(stop_s)
        self._sync_ctrl_to_device()
        self._enqueue_prologue()
        self._read_ctrl()

    def _stops(self, stop_s: float | Sequence[float] | None) -> NDArray[np.uint64]:
        if stop_s is None:
            return np.full(self.n_inst, _FOREVER_TICKS, np.uint64)
        if np.isscalar(stop_s):
            return np.full(self.n_inst, seconds_to_ticks(float(stop_s)), np.uint64)
        stops = [seconds_to_ticks(float(t)) for t in stop_s]
        if len(stops) != self.n_inst:
            raise ValueError(f"need {self.n_inst} stop times, got {len(stops)}")
        return np.asarray(stops, np.uint64)

    def retarget(self, stop_s: float | Sequence[float] | None) -> None:
        """Move every instance's stop (RETARGET): their clocks resume from where they are."""
        self._read_ctrl()
        self._ctrl["stop_ticks"] = self._stops(stop_s)
        self._sync_ctrl_to_device()
        self._enqueue_retarget()

    def run_steps(self, n_steps: int) -> None:
        """``n_steps`` batched steps (whole graphs of ``steps_per_graph`` plus one remainder graph), no host sync."""
        full, rest = divmod(int(n_steps), self.steps_per_graph)
        if full:
            graph = self._graph()
            with torch.cuda.stream(self._stream):
                for _ in range(full):
                    graph.replay()
        if rest:
            graph = self._graph(rest)
            with torch.cuda.stream(self._stream):
                graph.replay()

    def run(
        self,
        t_end: float | Sequence[float],
        dt_max: float,
        dt_init: float,
        output_interval_s: float | None = None,
        progress: bool = False,
    ) -> BatchRun:
        """Advance every instance to its ``t_end``; snapshot depths at every window end.

        Windows end every ``output_interval_s`` (the same grid for all
        instances, each capped at its own end) and at the ends themselves.
        Like the single solver, a window that makes no progress raises.
        """
        ends = self._stops(t_end)
        interval = seconds_to_ticks(output_interval_s) if output_interval_s else int(ends.max())
        stops = list(range(interval, int(ends.max()), interval)) + [int(ends.max())]
        self.reset()
        snaps: list[list[NDArray[np.float32]]] = [[self.download_h(i)] for i in range(self.n_inst)]
        times = [0.0]
        wall0 = last_log = _time.monotonic()
        for k, stop in enumerate(stops):
            window = np.minimum(ends, np.uint64(stop))
            if k == 0:
                self.start(dt_max, dt_init, window)
            else:
                self._ctrl["stop_ticks"] = window
                self._sync_ctrl_to_device()
                self._enqueue_retarget()
                self._read_ctrl()
            while (self._ctrl["now_ticks"] < window).any():
                before = self._ctrl["now_ticks"].copy()
                self.step_graph()
                self._read_ctrl()
                stuck = (self._ctrl["now_ticks"] == before) & (before < window)
                if stuck.any():
                    i = int(np.flatnonzero(stuck)[0])
                    raise RuntimeError(
                        f"batched run: instance {i} made no time progress at "
                        f"t={ticks_to_seconds(int(before[i])):.6f}s (CFL bound below one tick)"
                    )
                now = _time.monotonic()
                if progress and now - last_log >= 10.0:
                    done = float(self._ctrl["now_ticks"].min()) / float(1 << 20)
                    sys.stdout.write(f"[batch] slowest instance at {done:.2f}s, wall {now - wall0:.1f}s\n")
                    sys.stdout.flush()
                    last_log = now
            for i in range(self.n_inst):
                snaps[i].append(self.download_h(i))
            times.append(ticks_to_seconds(stop))
        return BatchRun(steps=self._ctrl["steps"].astype(np.int64), times=times, snapshots=snaps)


# -- autotuner ---------------------------------------------------------------------------------
_TUNED: dict[tuple, dict] = {}


def _signature(solver: ResidentEngine) -> tuple:
    L = solver.layout
    return (L.n_blocks, L.n_inst, L.blocks.max_edges, L.subs.max_edges, L.subs.max_slots,
            bool(solver.active_set), bool(solver.compensated))


def autotune(
    solver: BatchedSolver,
    dt_max: float,
    dt_init: float,
    steps: int = 40,
    candidates: Sequence[tuple[str, int | None]] | None = None,
    rounds: int = 2,
) -> dict:
    """Pick the stage kernel (64-cell tiles or 256-cell blocks) and the CTAs per SM.

    Each candidate runs ``steps`` batched steps from the solver's initial
    state, timed with CUDA events on the solver's stream (best of
    ``rounds``); the fastest is set on the solver. The state is reset to the
    initial state afterwards. Results are remembered per layout signature.
    Persistent candidates whose grid cannot hold every tile of a step are
    skipped.
    """
    key = _signature(solver)
    if key in _TUNED:
        best = _TUNED[key]
        solver.stage_kernel, solver.ctas_per_sm = best["stage_kernel"], best["ctas_per_sm"]
        return best
    if candidates is None:
        candidates = [(k, c) for k in ("tiled", "plain", "staged", "persistent") for c in (None, 4, 2)]
    saved_spg = solver.steps_per_graph
    results = []
    for kernel, per_sm in candidates:
        solver.stage_kernel, solver.ctas_per_sm = kernel, per_sm
        if kernel == "persistent" and not solver._persistent_fits:
            continue  # its grid cannot hold every tile of a step
        solver.steps_per_graph = steps
        best_ms = math.inf
        for _ in range(rounds):
            solver.reset()
            solver.start(dt_max, dt_init)
            graph = solver._graph()
            with torch.cuda.stream(solver._stream):
                graph.replay()  # warm-up of this candidate
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(solver._stream):
                ev0.record(solver._stream)
                graph.replay()
                ev1.record(solver._stream)
            ev1.synchronize()
            best_ms = min(best_ms, ev0.elapsed_time(ev1) / steps)
        results.append({"stage_kernel": kernel, "ctas_per_sm": per_sm, "grid": solver.grid(), "ms_per_step": best_ms})
    solver.steps_per_graph = saved_spg
    solver._graphs = {}
    best = min(results, key=lambda r: r["ms_per_step"])
    choice = {"stage_kernel": best["stage_kernel"], "ctas_per_sm": best["ctas_per_sm"], "results": results}
    solver.stage_kernel, solver.ctas_per_sm = best["stage_kernel"], best["ctas_per_sm"]
    solver.reset()
    _TUNED[key] = choice
    return choice


__all__ = ["BatchMember", "BatchRun", "BatchedSolver", "autotune"]
