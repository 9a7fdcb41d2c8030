"""Gradients of a gauge misfit through the resident step: a hand-written adjoint on the GPU.

``GaugeCalibration`` runs a fixed number of resident steps of one mesh and
sums the squared misfit of the depth (h + h_lo) at gauge cells against
observations after every step. Its gradient with respect to Manning's n and
the bed elevation of every cell and to the discharge knots of the inflow
hydrographs comes from the CUDA adjoint kernels (``swe_adjoint.cu``), with
every step's dt frozen at its forward value:

* the forward run keeps a checkpoint of the whole device state every
  ``checkpoint_every`` steps;
* the backward pass restores each checkpoint, last first, runs its segment
  again while taping each step's start state, stage sums, dt, clock and
  active list (``swe_tape_record`` + ``swe_stage_taped``; the taped run is
  bit-identical to the forward), then reverses the segment step by step
  (``swe_adjoint_segment``).

Device memory is the state, the checkpoints (16 B per cell each) and one
segment's tape (about 40 B per cell and step). ``MisfitFunction`` wraps it
as a ``torch.autograd.Function``. No counterpart in the reference.
"""

from __future__ import annotations

import ctypes
import math
from collections.abc import Sequence

import numpy as np
import torch
from numpy.typing import NDArray

from . import native
from .engine import ResidentEngine, START
from .layout import build_tile_layout
from .mesh.geometry import MeshGeometry
from .sources import Hydrograph
from .tuning import B200_BACKEND, DRY_TOL_DEFAULT, GRAVITY_G, dt_to_ticks

_FOREVER_TICKS = 1 << 62
_SNAPSHOT = ("h", "hu", "hv", "h_lo")


def _as_tensor(x, device, dtype=torch.float32) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.detach().to(device=device, dtype=dtype).reshape(-1)
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=device).reshape(-1)


class GaugeCalibration(ResidentEngine):
    """Misfit of ``steps`` resident steps at gauge cells, and its adjoint gradient.

    ``cut_depth`` (metres, 0 by default): no derivative flows through a cell
    depth or a face depth below it. 0 gives the exact derivative of the
    discrete step. Over long runs with wetting fronts that derivative is
    dominated by cells near the dry threshold (film drag, the desingularised
    velocity and the dry-bed wave-speed blend change steeply there) and can
    grow without bound; a cut at the film depth (4 dry_tol) keeps the
    derivatives of the wet flow only.
    """

    cut_depth: float = 0.0
    # the segment graphs capture one swe_step per step: a per-step stage kernel
    stage_kernel: str = "tiled"
    # reverse each segment in one cooperative launch (grid barriers between phases) instead of one
    # launch per phase and step; the arithmetic is the same. Off by default: at 250k cells the
    # per-phase launches fill more SMs and measured faster (121 against 135 ms for 2000 steps).
    persistent_reverse: bool = False

    def __init__(
        self,
        geom: MeshGeometry,
        h0: NDArray[np.float32],
        hu0: NDArray[np.float32],
        hv0: NDArray[np.float32],
        *,
        gauges: NDArray[np.int64],
        steps: int,
        hydrographs: Sequence[Hydrograph] = (),
        source_rate: NDArray[np.float32] | None = None,
        checkpoint_every: int = 50,
        dt_max: float = 1.0,
        dt_init: float = 0.01,
        g: float = GRAVITY_G,
        dry_tol: float = DRY_TOL_DEFAULT,
        cfl: float | None = None,
        device: int | str | torch.device | None = None,
    ) -> None:
        self.N = int(geom.N)
        self.geom = geom
        self.steps = int(steps)
        self.K = int(checkpoint_every)
        if self.steps < 1 or self.K < 1:
            raise ValueError("steps and checkpoint_every must be positive")
        gauges = np.asarray(gauges, np.int64).ravel()
        if gauges.size == 0 or np.unique(gauges).size != gauges.size or gauges.min() < 0 or gauges.max() >= self.N:
            raise ValueError(f"gauges must be distinct cells in [0, {self.N})")
        layout = build_tile_layout(geom)
        self._init_engine(layout, np.full(layout.n_padded_cells, 0.03, np.float32), g=g, dry_tol=dry_tol, cfl=cfl,
                          device=device)
        self.set_sources([source_rate], [list(hydrographs)])
        self.n_knots = int(sum(np.asarray(h.knot_q).size for h in hydrographs))
        self._h0 = np.asarray(h0, np.float32).ravel().copy()
        self._hu0 = np.asarray(hu0, np.float32).ravel().copy()
        self._hv0 = np.asarray(hv0, np.float32).ravel().copy()
        self.dt_max, self.dt_init = float(dt_max), float(dt_init)
        n, nb, dev = layout.n_padded_cells, layout.n_blocks, self.device
        f32 = lambda *shape: torch.zeros(*shape, dtype=torch.float32, device=dev)  # noqa: E731

        self._gcells = self._dev(gauges.astype(np.int32))
        self._obs = f32(self.steps * gauges.size)
        self._loss = torch.zeros(1, dtype=torch.float64, device=dev)
        self.gauges = gauges
        gg = native.SweGauges(cells=self._gcells.data_ptr(), obs=self._obs.data_ptr(), loss=self._loss.data_ptr(),
                              count=gauges.size, steps=self.steps)
        self._gauges = gg

        K = self.K
        self._tape_t = {name: f32((K + 1) * n) for name in _SNAPSHOT}
        self._tape_t["s0"] = f32(K * 3 * n)
        self._tape_t["s1"] = f32(K * 3 * n)
        self._tape_t["dt"] = torch.zeros(K, dtype=torch.int32, device=dev)
        self._tape_t["t"] = f32(K)
        self._tape_t["list"] = torch.zeros(K * nb, dtype=torch.int32, device=dev)
        self._tape_t["count"] = torch.zeros(K, dtype=torch.int32, device=dev)
        tape = native.SweTape(capacity=K)
        for name, tensor in self._tape_t.items():
            setattr(tape, name, tensor.data_ptr())
        self._tape = tape

        self._adj_t = {name: f32(n) for name in ("lh", "lhu", "lhv", "lsh", "lshu", "lshv", "uh", "ulo", "uhu", "uhv",
                                                 "gn", "gz")}
        self._adj_t["ls"] = f32(3 * n)
        self._adj_t["mark"] = torch.zeros(nb, dtype=torch.int32, device=dev)
        self._adj_t["gq"] = torch.zeros(max(self.n_knots, 1), dtype=torch.float64, device=dev)
        adj = native.SweAdjoint()
        for name, tensor in self._adj_t.items():
            setattr(adj, name, tensor.data_ptr())
        if self.n_knots == 0:
            adj.gq = None
        self._adj_sync = torch.zeros(64, dtype=torch.int32, device=dev)  # grid barrier of the reverse launch
        self._adj = adj

        self._checkpoints: list[dict[str, torch.Tensor]] = []
        self._segment_graphs: dict[tuple, torch.cuda.CUDAGraph] = {}
        self._has_forward = False

    # -- parameters ---------------------------------------------------------------------------------
    def set_parameters(self, n=None, z=None, q=None) -> None:
        """Manning's n and bed of every cell, and the knot discharges (concatenated in hydrograph order)."""
        with torch.cuda.stream(self._stream):
            if n is not None:
                self._mesh_t["n_mann"][: self.N].copy_(_as_tensor(n, self.device))
            if z is not None:
                zpad = torch.zeros(self.layout.n_padded_cells, dtype=torch.float32, device=self.device)
                zpad[: self.N].copy_(_as_tensor(z, self.device))
                self._zpad = zpad
                t = self._mesh_t
                native.check(
                    self._lib.swe_bed_steps(
                        ctypes.byref(self._mesh), zpad.data_ptr(), t["tile_dzl"].data_ptr(), t["tile_dzr"].data_ptr(),
                        t["tile_dzl"].numel(), t["sub_dzl"].data_ptr(), t["sub_dzr"].data_ptr(), t["sub_dzl"].numel(),
                        self._cuda_stream,
                    ),
                    "swe_bed_steps",
                )
            if q is not None:
                if self._src_hydro is None or self.n_knots == 0:
                    raise ValueError("this problem has no hydrograph knots")
                self._src_hydro["knot_q"].copy_(_as_tensor(q, self.device))
        self._stream.synchronize()

    # -- device-state snapshots ----------------------------------------------------------------------
    def _state_tensors(self) -> dict[str, torch.Tensor]:
        d = {name: self._t[name] for name in _SNAPSHOT}
        d.update(blk=self._blk, active_list=self._active_list, items=self._items, sched=self._sched,
                 dt_buf=self._dt_buf, ctrl=self._ctrl_dev)
        return d

    def _snapshot_into(self, idx: int) -> None:
        with torch.cuda.stream(self._stream):
            if idx >= len(self._checkpoints):
                self._checkpoints.append({k: v.clone() for k, v in self._state_tensors().items()})
            else:
                for k, v in self._state_tensors().items():
                    self._checkpoints[idx][k].copy_(v)

    def _restore(self, idx: int) -> None:
        with torch.cuda.stream(self._stream):
            for k, v in self._state_tensors().items():
                v.copy_(self._checkpoints[idx][k])

    # -- forward ----------------------------------------------------------------------------------------
    def _start(self) -> None:
        with torch.cuda.stream(self._stream):
            for name in ("h", "hu", "hv", "h_lo", "h1", "hu1", "hv1", "h1_lo"):
                self._t[name].zero_()
            self._t["h"][: self.N].copy_(torch.from_numpy(self._h0))
            self._t["hu"][: self.N].copy_(torch.from_numpy(self._hu0))
            self._t["hv"][: self.N].copy_(torch.from_numpy(self._hv0))
            self._loss.zero_()
        self._check_error_free_arithmetic()
        c = self._ctrl
        c[...] = 0
        c["stop_ticks"] = _FOREVER_TICKS
        c["dt_max_ticks"] = dt_to_ticks(self.dt_max)
        c["dry_dt_ticks"] = dt_to_ticks(min(self.dt_init, self.dt_max))
        c["cfl_safety"] = self.cfl_safety
        self._sync_ctrl_to_device()
        self._enqueue_prologue()

    def _segment_graph(self, n_steps: int, record: int) -> torch.cuda.CUDAGraph:
        key = ("fwd", n_steps, record, self._kernel, self.grid(), self._src_version)
        graph = self._segment_graphs.get(key)
        if graph is None:
            params, sources = self._params(), self._sources()
            mesh, state = ctypes.byref(self._mesh), ctypes.byref(self._state)
            graph = torch.cuda.CUDAGraph()
            self._stream.synchronize()
            with torch.cuda.graph(graph, stream=self._stream):
                st = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
                for _ in range(n_steps):
                    native.check(self._lib.swe_step(mesh, state, ctypes.byref(params), ctypes.byref(sources), st),
                                 "swe_step")
                    native.check(self._lib.swe_gauge_misfit(state, ctypes.byref(self._gauges), record, st),
                                 "swe_gauge_misfit")
            self._segment_graphs[key] = graph
        return graph

    def _taped_graph(self, n_steps: int) -> torch.cuda.CUDAGraph:
        key = ("tape", n_steps, self._src_version)
        graph = self._segment_graphs.get(key)
        if graph is None:
            params, sources = self._params(), self._sources()
            params.kernel = 0  # 64-cell tiles, recording the gathered sums
            mesh, state, tape = ctypes.byref(self._mesh), ctypes.byref(self._state), ctypes.byref(self._tape)
            n = self.layout.n_padded_cells
            s0, s1 = self._tape_t["s0"], self._tape_t["s1"]
            graph = torch.cuda.CUDAGraph()
            self._stream.synchronize()
            with torch.cuda.graph(graph, stream=self._stream):
                st = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
                pp, sp = ctypes.byref(params), ctypes.byref(sources)
                for j in range(n_steps):
                    lib = self._lib
                    native.check(lib.swe_tape_record(mesh, state, tape, j, st), "swe_tape_record")
                    native.check(lib.swe_stage_taped(mesh, state, pp, 0, s0[3 * n * j:].data_ptr(), st), "stage 0")
                    native.check(lib.swe_stage_taped(mesh, state, pp, 1, s1[3 * n * j:].data_ptr(), st), "stage 1")
                    if sources.count:
                        native.check(lib.swe_apply_sources(mesh, state, pp, sp, st), "swe_apply_sources")
                    native.check(lib.swe_block_dilate_compact(mesh, state, pp, 0, 1, st), "swe_block_dilate_compact")
                # the end state of the segment goes into the slot after its last step
                native.check(lib.swe_tape_record(mesh, state, tape, n_steps, st), "swe_tape_record")
            self._segment_graphs[key] = graph
        return graph

    def _run(self, record: int, checkpoints: bool) -> None:
        if not self.compensated:
            raise ValueError("the adjoint differentiates the compensated step; keep compensated=True")
        self._start()
        done = 0
        seg = 0
        while done < self.steps:
            n = min(self.K, self.steps - done)
            if checkpoints:
                self._snapshot_into(seg)
            graph = self._segment_graph(n, record)
            with torch.cuda.stream(self._stream):
                graph.replay()
            done += n
            seg += 1
        self._read_ctrl()
        if int(self._ctrl["steps"][0]) != self.steps:
            raise RuntimeError(
                f"{B200_BACKEND}: the run made {int(self._ctrl['steps'][0])} real steps of {self.steps} (the clock stalled)"
            )

    def observe(self, n=None, z=None, q=None) -> NDArray[np.float32]:
        """Run with these parameters and keep its gauge depths as the observations; returns them."""
        self.set_parameters(n, z, q)
        self._run(record=1, checkpoints=False)
        self._has_forward = False
        with torch.cuda.stream(self._stream):
            out = self._obs.cpu().numpy()
        return out.reshape(self.steps, self.gauges.size).copy()

    def set_observations(self, obs: NDArray[np.float32]) -> None:
        obs = np.ascontiguousarray(obs, np.float32).reshape(-1)
        if obs.size != self._obs.numel():
            raise ValueError(f"need {self.steps} x {self.gauges.size} observations")
        with torch.cuda.stream(self._stream):
            self._obs.copy_(torch.from_numpy(obs))
        self._stream.synchronize()

    def loss(self, n=None, z=None, q=None, *, checkpoints: bool = True) -> float:
        """The misfit with these parameters (checkpoints kept for ``gradient``)."""
        self.set_parameters(n, z, q)
        self._run(record=0, checkpoints=checkpoints)
        self._has_forward = checkpoints
        with torch.cuda.stream(self._stream):
            out = float(self._loss.cpu().item())
        return out

    def clock(self) -> tuple[NDArray[np.float64], NDArray[np.float64]]:
        """dt and hydrograph time (seconds) of every step of a run at the current parameters."""
        self._start()
        dts, ts = [], []
        done = 0
        while done < self.steps:
            n = min(self.K, self.steps - done)
            graph = self._taped_graph(n)
            with torch.cuda.stream(self._stream):
                graph.replay()
                dt = self._tape_t["dt"][:n].cpu().numpy().view(np.float32).astype(np.float64)
                t = self._tape_t["t"][:n].cpu().numpy().astype(np.float64)
            dts.append(dt)
            ts.append(t)
            done += n
        return np.concatenate(dts), np.concatenate(ts)

    # -- backward -----------------------------------------------------------------------------------------
    def gradient(self) -> tuple[NDArray[np.float32], NDArray[np.float32], NDArray[np.float64]]:
        """d loss / d (n, z, knots) at the parameters of the last ``loss`` call."""
        self.backward()
        self._stream.synchronize()
        self._check_reverse()
        with torch.cuda.stream(self._stream):
            gn = self._adj_t["gn"][: self.N].cpu().numpy().copy()
            gz = self._adj_t["gz"][: self.N].cpu().numpy().copy()
            gq = self._adj_t["gq"][: self.n_knots].cpu().numpy().copy()
        return gn, gz, gq

    def backward(self) -> None:
        """Enqueue the adjoint pass (results stay on the device in the gradient buffers)."""
        if not self._has_forward:
            raise RuntimeError("call loss(...) with checkpoints before the gradient")
        params, sources = self._params(), self._sources()
        params.grid = 0 if self.persistent_reverse else min(self.n_blocks, 4 * self._sms)
        self._adj.cut_depth = float(self.cut_depth)
        self._adj.sync = self._adj_sync.data_ptr() if self.persistent_reverse else None
        with torch.cuda.stream(self._stream):
            for t in self._adj_t.values():
                t.zero_()
            self._adj_sync.zero_()
        segments = math.ceil(self.steps / self.K)
        for seg in range(segments - 1, -1, -1):
            first = seg * self.K
            n = min(self.K, self.steps - first)
            self._restore(seg)
            graph = self._taped_graph(n)
            with torch.cuda.stream(self._stream):
                graph.replay()
                native.check(
                    self._lib.swe_adjoint_segment(
                        ctypes.byref(self._mesh), ctypes.byref(params), ctypes.byref(self._tape),
                        ctypes.byref(self._adj), ctypes.byref(sources), ctypes.byref(self._gauges), n, first, first,
                        self._cuda_stream,
                    ),
                    "swe_adjoint_segment",
                )

    def _check_reverse(self) -> None:
        if self.persistent_reverse and int(self._adj_sync[40].item()):
            raise RuntimeError(f"{B200_BACKEND}: a grid barrier wait of the reverse pass timed out")

    def gradient_tensors(self) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """The gradient buffers as device tensors (valid after ``backward``)."""
        self._stream.synchronize()
        self._check_reverse()
        return self._adj_t["gn"][: self.N], self._adj_t["gz"][: self.N], self._adj_t["gq"][: self.n_knots]


class MisfitFunction(torch.autograd.Function):
    """loss = MisfitFunction.apply(n, z, q, problem): the gauge misfit, differentiable in n, z and q."""

    @staticmethod
    def forward(ctx, n: torch.Tensor, z: torch.Tensor, q: torch.Tensor, problem: GaugeCalibration) -> torch.Tensor:
        value = problem.loss(n, z, q if problem.n_knots else None, checkpoints=True)
        ctx.problem = problem
        return torch.tensor(value, dtype=torch.float64, device=n.device)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        problem: GaugeCalibration = ctx.problem
        problem.backward()
        gn, gz, gq = problem.gradient_tensors()
        s = grad_out.to(torch.float64)
        return (gn.double() * s).to(torch.float32), (gz.double() * s).to(torch.float32), (gq * s).to(torch.float32), None


__all__ = ["GaugeCalibration", "MisfitFunction", "START"]
