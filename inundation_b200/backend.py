"""``b200_resident``: the reference's GPU-resident backend protocol on B200 kernels.

Same constructor, ``run`` signature and semantics, ``download_*`` methods and
attributes as the reference's ``SWESolverGpuResidentBatch``
(``inundation/vulkan/gpu_resident_batch.py:140-762``, base class
``inundation/vulkan/solver.py:118-497``): every step picks its own dt on the
device from the CFL bound of its corrector fluxes, simulated time is a uint64
count of 2^-20 s ticks, each output window runs whole submits of
``steps_per_graph`` steps (no-op steps past the window's stop do nothing) and
the host reads the 48-byte control block after each submit.

B200 specifics: a submit is one replay of a CUDA graph of ``steps_per_graph``
steps; torch CUDA tensors own all device memory; the C ABI kernels borrow
their pointers. There is no CPU fallback: without a GPU and the built
library, construction raises.
"""

from __future__ import annotations

import ctypes
import math
import sys
import time as _time
from collections.abc import Callable, Sequence

import numpy as np
import torch
from numpy.typing import NDArray

from . import native
from .layout import TileLayout, build_tile_layout
from .mesh.geometry import MeshGeometry
from .tuning import (
    ACTIVE_BLOCK_CELLS,
    B200_BACKEND,
    CFL_DEFAULT,
    DRY_TOL_DEFAULT,
    GRAVITY_G,
    dt_to_ticks,
    output_window_stops,
    seconds_to_ticks,
    ticks_to_seconds,
)

STEPS_PER_GRAPH_DEFAULT = 200

# Host mirror of swe_ctrl_t (the reference's RESIDENT_CTRL_DTYPE, 48 bytes).
RESIDENT_CTRL_DTYPE = np.dtype(
    [
        ("now_ticks", "<u8"),
        ("stop_ticks", "<u8"),
        ("steps", "<u8"),
        ("dt_ticks", "<u4"),
        ("dt_max_ticks", "<u4"),
        ("dry_dt_ticks", "<u4"),
        ("last_raw", "<f4"),
        ("cfl_safety", "<f4"),
        ("error", "<u4"),
    ]
)

START, STEP, RETARGET = 0, 1, 2
_SENTINEL_BITS = 0x7149F2CA  # float32 1e30


def _i32(a: NDArray) -> NDArray[np.int32]:
    return np.ascontiguousarray(a).view(np.int32)


class SWESolverB200Resident:
    """GPU-resident Heun steps with an integer clock, on one B200."""

    name = B200_BACKEND
    default_cfl: float = CFL_DEFAULT
    steps_per_graph: int = STEPS_PER_GRAPH_DEFAULT
    active_set: bool = True
    # Fixed-order gathers are the only accumulation: repeat runs are bit-identical.
    deterministic: bool = True
    compensated: bool = True
    cfl_safety: float = 1.0
    # Stage kernel: "tiled" (64-cell tiles from the dilation's work items, staged by bulk copies)
    # or "plain" (256-cell blocks, direct loads).
    stage_kernel: str = "tiled"

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
        if any(np.asarray(e).size for e in open_edges):
            raise ValueError(f"{B200_BACKEND} does not support open boundaries yet")
        if not torch.cuda.is_available():
            raise RuntimeError(f"{B200_BACKEND} needs a CUDA device; none is visible")
        self._lib = native.load()
        self.geom = geom
        self.N, self.E = int(geom.N), int(geom.E)
        self._g = float(g)
        self._dry_tol = float(dry_tol)
        self._cfl = float(self.default_cfl if cfl is None else cfl)
        self.track_clamp = False
        self.steps_total = 0
        self.open_volume_snapshots: list[NDArray[np.float64]] = []
        self.n_open = 0
        self._h0 = np.asarray(h0, np.float32).ravel().copy()
        self._hu0 = np.asarray(hu0, np.float32).ravel().copy()
        self._hv0 = np.asarray(hv0, np.float32).ravel().copy()
        self._area = np.asarray(geom.area, np.float32)
        for name, arr in (("h0", self._h0), ("hu0", self._hu0), ("hv0", self._hv0)):
            if arr.size != self.N:
                raise ValueError(f"{name} has {arr.size} values for {self.N} cells")
        n0 = np.asarray(n0, np.float32).ravel()
        if n0.size != self.N:
            raise ValueError(f"n0 has {n0.size} values for {self.N} cells")

        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self._stream = torch.cuda.Stream(device=self.device)
        self.layout: TileLayout = build_tile_layout(geom)
        self.n_blocks = self.layout.n_blocks
        self._upload_mesh(self.layout, n0)
        self._alloc_state()
        self._graphs: dict[tuple, torch.cuda.CUDAGraph] = {}
        self._eft_checked = False
        self._src_cells = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._src_rate = torch.zeros(1, dtype=torch.float32, device=self.device)
        self._src_count = 0
        self.reset(self._h0, self._hu0, self._hv0)

    # -- device memory ------------------------------------------------------------------
    def _dev(self, a: NDArray) -> torch.Tensor:
        return torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

    def _upload_mesh(self, L: TileLayout, n0: NDArray[np.float32]) -> None:
        B, S = L.blocks, L.subs
        t = {"cptr": self._dev(_i32(L.cptr)), "area": self._dev(L.area),
             "n_mann": self._dev(np.concatenate([n0, np.full(L.n_padded_cells - L.n_cells, 0.03, np.float32)])),
             "ring_ptr": self._dev(_i32(L.ring_ptr)), "ring_idx": self._dev(_i32(L.ring_idx))}
        for prefix, T in (("tile_", B), ("sub_", S)):
            for name in ("cl", "cr", "nx", "ny", "len", "dzl", "dzr"):
                t[prefix + name] = self._dev(getattr(T, name))
            t[prefix + "ptr"] = self._dev(_i32(T.ptr))
            t[prefix + "count"] = self._dev(_i32(T.count))
        t["lcsr"] = self._dev(B.lcsr.view(np.int16))
        t["block_inst"] = self._dev(np.zeros(L.n_blocks, np.int32))
        t["block_cells"] = self._dev(_i32(L.block_cells))
        t["sub_lcsr"] = self._dev(S.lcsr_blk.view(np.int16))
        t["sub_lcsr_ptr"] = self._dev(_i32(S.lcsr_ptr))
        self._mesh_t = t
        m = native.SweMesh()
        m.n_cells = L.n_cells
        m.n_blocks = L.n_blocks
        m.max_tile_edges = B.max_edges
        m.n_inst = 1
        m.max_sub_edges = S.max_edges
        m.max_sub_slots = S.max_slots
        for name, tensor in t.items():
            setattr(m, name, tensor.data_ptr())
        self._mesh = m
        self._sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        self._grids: dict[int, int] = {}
        for kernel in (0, 1):
            per_sm = ctypes.c_int(0)
            with torch.cuda.device(self.device):
                native.check(self._lib.swe_configure(ctypes.byref(m), kernel, ctypes.byref(per_sm)), "swe_configure")
            units = 4 * L.n_blocks if kernel == 0 else L.n_blocks  # the tiled kernel works on 64-cell tiles
            self._grids[kernel] = max(1, min(units, per_sm.value * self._sms))

    _KERNELS = {"tiled": 0, "plain": 1}

    @property
    def _kernel(self) -> int:
        if self.stage_kernel not in self._KERNELS:
            raise ValueError(f"stage_kernel must be one of {sorted(self._KERNELS)}, got {self.stage_kernel!r}")
        return self._KERNELS[self.stage_kernel]

    def _alloc_state(self) -> None:
        n, nb, dev = self.layout.n_padded_cells, self.n_blocks, self.device
        z = lambda: torch.zeros(n, dtype=torch.float32, device=dev)  # noqa: E731
        self._t = {name: z() for name in ("h", "hu", "hv", "h_lo", "h1", "hu1", "hv1", "h1_lo", "clamp_mass")}
        self._blk = torch.zeros(3 * nb, dtype=torch.int32, device=dev)
        self._active_list = torch.zeros(nb, dtype=torch.int32, device=dev)
        self._items = torch.zeros(16 * nb, dtype=torch.int32, device=dev)  # 4 tiles x 4 words per block
        self._sched = torch.zeros(8, dtype=torch.int64, device=dev)  # 16 uint32 words
        self._dt_buf = torch.tensor([0, _SENTINEL_BITS, 0, 0], dtype=torch.int64, device=dev).to(torch.int32)
        self._ctrl_dev = torch.zeros(6, dtype=torch.int64, device=dev)
        self._ctrl_pinned = torch.zeros(6, dtype=torch.int64).pin_memory()
        self._ctrl = self._ctrl_pinned.numpy().view(RESIDENT_CTRL_DTYPE)
        self._partials = torch.zeros(int(self._lib.swe_volume_partials(n)), dtype=torch.float64, device=dev)
        self._volume = torch.zeros(1, dtype=torch.float64, device=dev)
        s = native.SweState()
        for name, tensor in self._t.items():
            setattr(s, name, tensor.data_ptr())
        s.blk = self._blk.data_ptr()
        s.active_list = self._active_list.data_ptr()
        s.items = self._items.data_ptr()
        s.sched = self._sched.data_ptr()
        s.dt_buf = self._dt_buf.data_ptr()
        s.ctrl = self._ctrl_dev.data_ptr()
        self._state = s

    def _params(self) -> native.SweParams:
        return native.SweParams(
            g=self._g,
            dry_tol=self._dry_tol,
            cfl=self._cfl,
            compensated=int(bool(self.compensated)),
            track_clamp=int(bool(self.track_clamp)),
            active_set=int(bool(self.active_set)),
            grid=self._grids[self._kernel],
            kernel=self._kernel,
        )

    def _sources(self) -> native.SweSources:
        return native.SweSources(
            cells=self._src_cells.data_ptr(), rate=self._src_rate.data_ptr(), count=self._src_count
        )

    @property
    def _cuda_stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(self._stream.cuda_stream)

    # -- public state access (reference solver.py:390-497) --------------------------------------
    def _download(self, tensor: torch.Tensor) -> NDArray[np.float32]:
        with torch.cuda.stream(self._stream):
            out = tensor[: self.N].cpu().numpy()
        return out.copy()

    def download_h(self) -> NDArray[np.float32]:
        return self._download(self._t["h"])

    def download_hu(self) -> NDArray[np.float32]:
        return self._download(self._t["hu"])

    def download_hv(self) -> NDArray[np.float32]:
        return self._download(self._t["hv"])

    def download_h_residual(self) -> NDArray[np.float32]:
        return self._download(self._t["h_lo"])

    def download_h_precise(self) -> NDArray[np.float64]:
        return self.download_h().astype(np.float64) + self.download_h_residual().astype(np.float64)

    def download_clamp_mass(self) -> NDArray[np.float32]:
        return self._download(self._t["clamp_mass"])

    def download_block_flags(self) -> NDArray[np.uint32]:
        """``(n_blocks, 3)`` flags: wet, active, forced."""
        with torch.cuda.stream(self._stream):
            words = self._blk.cpu().numpy()
        return words.view(np.uint32).reshape(self.n_blocks, 3).copy()

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
        """Upload initial conditions; the compensated low words start at zero."""
        self._h0 = np.asarray(h0, np.float32).ravel().copy()
        self._hu0 = np.asarray(hu0, np.float32).ravel().copy()
        self._hv0 = np.asarray(hv0, np.float32).ravel().copy()
        with torch.cuda.stream(self._stream):
            self._t["h"][: self.N].copy_(torch.from_numpy(self._h0))
            self._t["hu"][: self.N].copy_(torch.from_numpy(self._hu0))
            self._t["hv"][: self.N].copy_(torch.from_numpy(self._hv0))
            self._t["h_lo"].zero_()
            self._t["h1_lo"].zero_()
        self._stream.synchronize()

    def _reset_to_initial(self) -> None:
        self.reset(self._h0, self._hu0, self._hv0)

    def set_open_conditions(self, kinds: NDArray[np.uint32], values: NDArray[np.float32]) -> None:
        raise ValueError(f"{B200_BACKEND} does not support open boundaries yet")

    def download_open_volumes(self) -> NDArray[np.float64]:
        return np.zeros((0, 2), dtype=np.float64)

    def volume_fp64(self) -> float:
        """Sum of (h + h_lo) * area in float64 on the device, in a fixed order."""
        with torch.cuda.stream(self._stream):
            native.check(
                self._lib.swe_volume_fp64(
                    self._t["h"].data_ptr(), self._t["h_lo"].data_ptr(), self._mesh_t["area"].data_ptr(), self.N,
                    self._partials.data_ptr(), self._volume.data_ptr(), self._cuda_stream,
                ),
                "swe_volume_fp64",
            )
            out = float(self._volume.cpu().item())
        return out

    @property
    def computed_cells(self) -> int:
        """Cells in computed blocks summed over all real steps (the roofline's cell-step count)."""
        self._stream.synchronize()
        return int(self._sched.cpu().numpy().view(np.uint64)[3])

    # -- kernels ----------------------------------------------------------------------------------
    def _check_error_free_arithmetic(self) -> None:
        if self._eft_checked:
            return
        v = torch.tensor([1.0, 1e-9, 0.0], dtype=torch.float32, device=self.device)
        with torch.cuda.stream(self._stream):
            native.check(self._lib.swe_eft_probe(v.data_ptr(), self._cuda_stream), "swe_eft_probe")
            got = v.cpu().numpy()
        if float(got[2]) != float(np.float32(1e-9)):
            raise RuntimeError("error-free arithmetic is broken on this device, so compensated depth would leak mass")
        self._eft_checked = True

    def _set_sources(self, source_rate: NDArray[np.float32] | None) -> None:
        if source_rate is None:
            self._src_count = 0
            return
        per_sec = np.asarray(source_rate, dtype=np.float32).ravel() * (1.0 / self._area).astype(np.float32)
        cells = np.flatnonzero(per_sec)
        self._src_count = int(cells.size)
        if cells.size:
            self._src_cells = self._dev(cells.astype(np.int32))
            self._src_rate = self._dev(per_sec[cells].astype(np.float32))

    def _sync_ctrl_to_device(self) -> None:
        with torch.cuda.stream(self._stream):
            self._ctrl_dev.copy_(self._ctrl_pinned, non_blocking=True)

    def _read_ctrl(self) -> None:
        with torch.cuda.stream(self._stream):
            self._ctrl_pinned.copy_(self._ctrl_dev, non_blocking=True)
        self._stream.synchronize()
        if int(self._ctrl["error"][0]):
            raise RuntimeError(
                f"{B200_BACKEND}: a bounded device wait for staged data timed out (error {int(self._ctrl['error'][0])})"
            )

    def _enqueue_prologue(self) -> None:
        p = self._params()
        with torch.cuda.stream(self._stream):
            self._sched[:3].zero_()  # list counters; words 6-7 keep the computed-cells total
            self._sched[4:].zero_()
            native.check(
                self._lib.swe_prologue(
                    ctypes.byref(self._mesh), ctypes.byref(self._state), ctypes.byref(p), self._cuda_stream
                ),
                "swe_prologue",
            )

    def _enqueue_retarget(self) -> None:
        """RETARGET the clock to a new stop, rebuilding the active lists first.

        A no-op step leaves its instance out of the lists, so the lists are
        rebuilt by a forced dilation (the flags come out the same: they were
        dilated from the same wet marks after the last real step).
        """
        p = self._params()
        with torch.cuda.stream(self._stream):
            native.check(
                self._lib.swe_block_dilate_compact(
                    ctypes.byref(self._mesh), ctypes.byref(self._state), ctypes.byref(p), 1, RETARGET,
                    self._cuda_stream,
                ),
                "swe_block_dilate_compact",
            )

    def _enqueue_steps(self, n_steps: int, params: native.SweParams, sources: native.SweSources) -> None:
        mesh, state = ctypes.byref(self._mesh), ctypes.byref(self._state)
        pp, sp = ctypes.byref(params), ctypes.byref(sources)
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        for _ in range(n_steps):
            native.check(self._lib.swe_step(mesh, state, pp, sp, stream), "swe_step")

    def _graph(self) -> torch.cuda.CUDAGraph:
        key = (
            self.steps_per_graph,
            bool(self.compensated),
            bool(self.track_clamp),
            bool(self.active_set),
            self._kernel,
            self._src_count,
            self._src_cells.data_ptr(),
            self._src_rate.data_ptr(),
        )
        graph = self._graphs.get(key)
        if graph is None:
            params, sources = self._params(), self._sources()
            graph = torch.cuda.CUDAGraph()
            self._stream.synchronize()
            with torch.cuda.graph(graph, stream=self._stream):
                self._enqueue_steps(self.steps_per_graph, params, sources)
            self._graphs = {key: graph}  # one live graph per solver
        return graph

    def step_graph(self) -> None:
        """Replay one submit of ``steps_per_graph`` steps (no host sync)."""
        graph = self._graph()
        with torch.cuda.stream(self._stream):
            graph.replay()

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
        if self.compensated:
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

        capture()
        ctrl = self._ctrl
        ctrl["error"] = 0
        ctrl["now_ticks"] = start_ticks
        ctrl["steps"] = 0
        ctrl["dt_ticks"] = 0
        ctrl["dt_max_ticks"] = dt_max_ticks
        ctrl["dry_dt_ticks"] = dry_dt_ticks
        ctrl["cfl_safety"] = self.cfl_safety
        graph = self._graph()
        planned = False
        wall0 = _time.monotonic()
        last_log = wall0
        finite = True
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
                with torch.cuda.stream(self._stream):
                    graph.replay()
                self._read_ctrl()
                now_ticks = int(ctrl["now_ticks"][0])
                if now_ticks == before:
                    raise RuntimeError(
                        f"GPU-resident run made no time progress at t={ticks_to_seconds(now_ticks):.6f}s "
                        "(CFL bound below one tick)"
                    )
                now = _time.monotonic()
                if progress and now - last_log >= 10.0:
                    self._log_progress(now - wall0, now_ticks, start_ticks, end_ticks)
                    last_log = now
            h_snap = self.download_h()
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
            h_final = self.download_h()
            if not np.allclose(snapshots[-1], h_final):
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


__all__ = ["RESIDENT_CTRL_DTYPE", "STEPS_PER_GRAPH_DEFAULT", "SWESolverB200Resident"]
