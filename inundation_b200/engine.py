"""Device state of the resident shallow-water step: one or more meshes on one B200.

``ResidentEngine`` owns every device buffer (torch CUDA tensors), fills the
C-ABI structs with their pointers and enqueues the library's kernels on its
own stream: prologue, RETARGET, steps captured in CUDA graphs, the float64
volume. It is the machinery under both host APIs, the reference's solver
protocol (``backend.SWESolverB200Resident``, one mesh) and batches of
independent meshes (``batch.BatchedSolver``). A batch is laid out by
``layout.build_batch_layout``: every instance on whole 256-cell blocks, with
its own clock (48-byte control block), dt words and CFL bound.

There is no CPU fallback: without a CUDA device and the built library,
construction raises.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch
from numpy.typing import NDArray

from . import native
from .layout import TileLayout
from .sources import NO_HYDROGRAPH, Hydrograph
from .tuning import ACTIVE_BLOCK_CELLS, B200_BACKEND, CFL_DEFAULT, DRY_TOL_DEFAULT, GRAVITY_G, OPEN_INFLOW, OPEN_STAGE

# Host mirror of swe_ctrl_t (the reference's RESIDENT_CTRL_DTYPE, 48 bytes;
# the reference's padding word carries the device error flag).
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
STATE_ARRAYS = ("h", "hu", "hv", "h_lo", "h1", "hu1", "hv1", "h1_lo", "clamp_mass")
KERNELS = {"tiled": 0, "plain": 1, "persistent": 2, "staged": 3}
# "auto": the persistent kernel while few blocks are active (its phases are latency-bound), the
# staged 256-cell block kernel once more than this fraction of blocks is active (work for the
# whole GPU), unless every active tile still has a CTA of the persistent grid to itself (a small mesh).
AUTO_DENSE_FRACTION = 0.25
PERSISTENT_EXTRA_TILES = 512  # kExtraCap of the persistent kernel


def _i32(a: NDArray) -> NDArray[np.int32]:
    return np.ascontiguousarray(a).view(np.int32)


# The two-sum probe's input: its third word comes back as the error term of 1 + 1e-9.
EFT_PROBE_WORDS = (1.0, 1e-9, 0.0)


def check_eft_probe(words: NDArray[np.float32]) -> None:
    """Raise if the probe lost two-sum's error term, which must be 1e-9 exactly in float32.

    The reference refuses to run then (``inundation/vulkan/solver.py:461-466``):
    compensated depth and the open-edge tallies would leak mass.
    """
    got = np.asarray(words, np.float32).ravel()
    if got.size != 3 or float(got[2]) != float(np.float32(EFT_PROBE_WORDS[1])):
        raise RuntimeError(
            "error-free arithmetic is broken on this device, so compensated depth would leak mass: "
            "rebuild the library without fast math, or set compensated = False"
        )


class ResidentEngine:
    """Device buffers and kernel launches of a batch of meshes (a single mesh is a batch of one)."""

    default_cfl: float = CFL_DEFAULT
    steps_per_graph: int = 200
    active_set: bool = True
    compensated: bool = True
    track_clamp: bool = False
    cfl_safety: float = 1.0
    # Stage kernel: "tiled" (64-cell tiles from the dilation's work items, staged by bulk copies),
    # "plain" (256-cell blocks, direct loads), "staged" (256-cell blocks staged by bulk copies),
    # "persistent" (the tiled stages and the rest of the
    # step in one cooperative launch per submit, phases separated by grid barriers) or "auto"
    # (persistent or staged by the active fraction read after every submit). All give the same bits.
    stage_kernel: str = "auto"

    def _init_engine(
        self,
        layout: TileLayout,
        n_mann: NDArray[np.float32],
        *,
        g: float = GRAVITY_G,
        dry_tol: float = DRY_TOL_DEFAULT,
        cfl: float | None = None,
        device: int | str | torch.device | None = None,
    ) -> None:
        if not torch.cuda.is_available():
            raise RuntimeError(f"{B200_BACKEND} needs a CUDA device; none is visible")
        self._lib = native.load()
        self.layout = layout
        self.n_blocks = layout.n_blocks
        self.n_inst = layout.n_inst
        self._g = float(g)
        self._dry_tol = float(dry_tol)
        self._cfl = float(self.default_cfl if cfl is None else cfl)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self._stream = torch.cuda.Stream(device=self.device)
        self._upload_mesh(layout, n_mann)
        self._alloc_state()
        self._graphs: dict[tuple, torch.cuda.CUDAGraph] = {}
        self._eft_checked = False
        self._src_version = 0
        self.clear_sources()

    # -- device memory ------------------------------------------------------------------
    def _dev(self, a: NDArray) -> torch.Tensor:
        return torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

    def _upload_mesh(self, L: TileLayout, n_mann: NDArray[np.float32]) -> None:
        B, S = L.blocks, L.subs
        if n_mann.size != L.n_padded_cells:
            raise ValueError(f"n_mann has {n_mann.size} values for {L.n_padded_cells} padded cells")
        t = {"cptr": self._dev(_i32(L.cptr)), "area": self._dev(L.area),
             "n_mann": self._dev(np.asarray(n_mann, np.float32)),
             "ring_ptr": self._dev(_i32(L.ring_ptr)), "ring_idx": self._dev(_i32(L.ring_idx)),
             "block_inst": self._dev(_i32(L.block_inst)), "block_cells": self._dev(_i32(L.block_cells))}
        for prefix, T in (("tile_", B), ("sub_", S)):
            for name in ("cl", "cr", "nx", "ny", "len", "dzl", "dzr"):
                t[prefix + name] = self._dev(getattr(T, name))
            t[prefix + "ptr"] = self._dev(_i32(T.ptr))
            t[prefix + "count"] = self._dev(_i32(T.count))
        t["lcsr"] = self._dev(B.lcsr.view(np.int16))
        t["sub_lcsr"] = self._dev(S.lcsr_blk.view(np.int16))
        t["sub_lcsr_ptr"] = self._dev(_i32(S.lcsr_ptr))
        t["blk_lcsr"] = self._dev(B.lcsr_blk.view(np.int16))
        t["blk_lcsr_ptr"] = self._dev(_i32(B.lcsr_ptr))
        self.n_open = L.n_open
        if L.n_open:  # conditions start as walls; the pointer stays fixed, so graphs see every update
            t["open_cond"] = torch.zeros(2 * L.n_open, dtype=torch.int32, device=self.device)
        self._mesh_t = t
        m = native.SweMesh()
        m.n_cells = L.n_padded_cells
        m.n_blocks = L.n_blocks
        m.max_tile_edges = B.max_edges
        m.n_inst = L.n_inst
        m.max_sub_edges = S.max_edges
        m.max_sub_slots = S.max_slots
        m.max_blk_slots = B.max_slots
        for name, tensor in t.items():
            setattr(m, name, tensor.data_ptr())
        m.n_open = L.n_open
        self._mesh = m
        self._sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        self._per_sm: dict[int, int] = {}
        for kernel in KERNELS.values():
            per_sm = ctypes.c_int(0)
            with torch.cuda.device(self.device):
                native.check(self._lib.swe_configure(ctypes.byref(m), kernel, ctypes.byref(per_sm)), "swe_configure")
            self._per_sm[kernel] = max(1, per_sm.value)
            if kernel == KERNELS["staged"]:  # 0: the mesh's largest block does not fit its shared memory
                self._staged_fits = per_sm.value > 0
        self.ctas_per_sm: int | None = None  # None: as many as fit
        self.max_grid: int | None = None  # an upper bound on the persistent CTAs (None: none)

    def grid(self, kernel: int | None = None) -> int:
        """Persistent CTAs of a stage kernel: CTAs per SM x SMs, at most one per work unit."""
        kernel = self._kernel if kernel is None else kernel
        per_sm = self._per_sm[kernel] if self.ctas_per_sm is None else min(self.ctas_per_sm, self._per_sm[kernel])
        units = self.n_blocks if kernel in (1, 3) else 4 * self.n_blocks  # 256-cell blocks, or 64-cell tiles
        grid = min(units, per_sm * self._sms)
        if self.max_grid is not None:
            grid = min(grid, self.max_grid)
        return max(1, grid)

    @property
    def _kernel(self) -> int:
        if self.stage_kernel == "auto":
            dense = self._active_blocks > AUTO_DENSE_FRACTION * self.n_blocks
            seated = 4 * self._active_blocks <= self.grid(KERNELS["persistent"])
            if self._persistent_fits and (seated or not dense):
                return KERNELS["persistent"]
            return KERNELS["staged"] if self._staged_fits else KERNELS["plain"]
        if self.stage_kernel not in KERNELS:
            raise ValueError(f"stage_kernel must be one of {sorted(KERNELS)} or 'auto', got {self.stage_kernel!r}")
        return KERNELS[self.stage_kernel]

    @property
    def _persistent_fits(self) -> bool:
        """The persistent kernel gives every CTA one seat and up to PERSISTENT_EXTRA_TILES other tiles a step."""
        return 4 * self.n_blocks <= self.grid(KERNELS["persistent"]) * (1 + PERSISTENT_EXTRA_TILES)

    def _alloc_state(self) -> None:
        n, nb, ni, dev = self.layout.n_padded_cells, self.n_blocks, self.n_inst, self.device
        self._t = {name: torch.zeros(n, dtype=torch.float32, device=dev) for name in STATE_ARRAYS}
        self._blk = torch.zeros(3 * nb, dtype=torch.int32, device=dev)
        self._active_list = torch.zeros(2 * nb, dtype=torch.int32, device=dev)  # two halves
        self._items = torch.zeros(32 * nb, dtype=torch.int32, device=dev)  # two halves of 4 tiles x 4 words per block
        self._marks = torch.zeros(2 * nb, dtype=torch.int32, device=dev)  # listed / spread epochs
        self._sched = torch.zeros(8, dtype=torch.int64, device=dev)  # 16 uint32 words
        dt = np.zeros(4 * ni, np.uint32)
        dt[1::4] = np.float32(1e30).view(np.uint32)
        self._dt_buf = self._dev(dt.view(np.int32))
        self._ctrl_dev = torch.zeros(6 * ni, dtype=torch.int64, device=dev)
        self._sync = torch.zeros(64, dtype=torch.int32, device=dev)  # grid barrier words of the persistent kernel
        self._open_vol = torch.zeros(4 * max(self.n_open, 1), dtype=torch.float32, device=dev)  # out, in pairs
        self._ctrl_pinned = torch.zeros(6 * ni, dtype=torch.int64).pin_memory()
        self._ctrl = self._ctrl_pinned.numpy().view(RESIDENT_CTRL_DTYPE)
        self._sched_pinned = torch.zeros(8, dtype=torch.int64).pin_memory()
        self._active_blocks = 0  # blocks in the current active list, as of the last control-block read
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
        s.sync = self._sync.data_ptr()
        s.marks = self._marks.data_ptr()
        s.open_vol = self._open_vol.data_ptr() if self.n_open else None
        self._state = s

    def _params(self) -> native.SweParams:
        return native.SweParams(
            g=self._g,
            dry_tol=self._dry_tol,
            cfl=self._cfl,
            compensated=int(bool(self.compensated)),
            track_clamp=int(bool(self.track_clamp)),
            active_set=int(bool(self.active_set)),
            grid=self.grid(),
            kernel=self._kernel,
        )

    @property
    def _cuda_stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(self._stream.cuda_stream)

    # -- sources ----------------------------------------------------------------------
    def clear_sources(self) -> None:
        self._set_source_arrays(np.zeros(0, np.int64), np.zeros(0, np.float32), None, None, [])

    def set_sources(
        self,
        rates: list[NDArray[np.float32] | None],
        hydrographs: list[list[Hydrograph]] | None = None,
    ) -> None:
        """Per-instance sources: ``rates[i]`` in m^3/s per cell (the reference's
        ``source_rate``, divided by the cell area on the way in) and inflow
        hydrographs. One source entry per cell: a cell with both adds both.
        """
        L = self.layout
        hydrographs = hydrographs or [[] for _ in range(self.n_inst)]
        if len(rates) != self.n_inst or len(hydrographs) != self.n_inst:
            raise ValueError(f"need sources for {self.n_inst} instances")
        cells_all, rate_all, hidx_all, hscale_all = [], [], [], []
        knots: list[tuple[NDArray, NDArray]] = []
        any_hydro = False
        for i in range(self.n_inst):
            if rates[i] is None and not hydrographs[i]:
                continue  # no sources on this instance
            off, n = int(L.inst_cell_offset[i]), int(L.inst_cells[i])
            area = L.area[off : off + n]
            rate = np.zeros(n, np.float32)
            if rates[i] is not None:
                r = np.asarray(rates[i], np.float32).ravel()
                if r.size != n:
                    raise ValueError(f"source_rate of instance {i} has {r.size} values for {n} cells")
                rate = r * (1.0 / area).astype(np.float32)
            hidx = np.full(n, NO_HYDROGRAPH, np.uint32)
            hscale = np.zeros(n, np.float32)
            for hg in hydrographs[i]:
                hg.validate(n)
                cells = np.asarray(hg.cells, np.int64).ravel()
                if (hidx[cells] != NO_HYDROGRAPH).any():
                    raise ValueError("two hydrographs share a cell")
                hidx[cells] = len(knots)
                hscale[cells] = hg.shares() * (1.0 / area[cells]).astype(np.float32)
                knots.append((np.asarray(hg.knot_t, np.float32).ravel(), np.asarray(hg.knot_q, np.float32).ravel()))
                any_hydro = True
            live = np.flatnonzero((rate != 0) | (hidx != NO_HYDROGRAPH))
            cells_all.append(live + off)
            rate_all.append(rate[live])
            hidx_all.append(hidx[live])
            hscale_all.append(hscale[live])
        self._set_source_arrays(
            np.concatenate([np.zeros(0, np.int64), *cells_all]),
            np.concatenate([np.zeros(0, np.float32), *rate_all]),
            np.concatenate(hidx_all) if any_hydro else None,
            np.concatenate(hscale_all) if any_hydro else None,
            knots,
        )

    def _set_source_arrays(self, cells, rate, hidx, hscale, knots) -> None:
        # The same sources again (every run() passes its own): keep the device arrays and the captured graphs.
        host = [np.asarray(cells, np.int64), np.asarray(rate, np.float32),
                None if hidx is None else np.asarray(hidx), None if hscale is None else np.asarray(hscale),
                [(np.asarray(t, np.float32), np.asarray(q, np.float32)) for t, q in knots]]
        if getattr(self, "_src_host", None) is not None and _same_sources(self._src_host, host):
            return
        self._src_host = host
        dev = self._dev
        self._src_count = int(cells.size)
        self._src_cells = dev(cells.astype(np.int32) if cells.size else np.zeros(1, np.int32))
        self._src_rate = dev(rate.astype(np.float32) if cells.size else np.zeros(1, np.float32))
        self._src_hydro = None
        if hidx is not None and knots:
            ptr = np.zeros(len(knots) + 1, np.int64)
            np.cumsum([t.size for t, _ in knots], out=ptr[1:])
            self._src_hydro = {
                "hydro": dev(hidx.view(np.int32)),
                "hscale": dev(hscale.astype(np.float32)),
                "knot_ptr": dev(ptr.astype(np.int32)),
                "knot_t": dev(np.concatenate([t for t, _ in knots])),
                "knot_q": dev(np.concatenate([q for _, q in knots])),
                "n": len(knots),
            }
        self._src_version += 1

    def _sources(self) -> native.SweSources:
        s = native.SweSources(cells=self._src_cells.data_ptr(), rate=self._src_rate.data_ptr(), count=self._src_count)
        if self._src_hydro is not None:
            h = self._src_hydro
            for name in ("hydro", "hscale", "knot_ptr", "knot_t", "knot_q"):
                setattr(s, name, h[name].data_ptr())
            s.n_hydro = h["n"]
        return s

    # -- state access ---------------------------------------------------------------------
    def _inst_range(self, inst: int) -> slice:
        off = int(self.layout.inst_cell_offset[inst])
        return slice(off, off + int(self.layout.inst_cells[inst]))

    def download_state(self, name: str, inst: int = 0) -> NDArray[np.float32]:
        with torch.cuda.stream(self._stream):  # a new host array, written by the copy itself
            return self._t[name][self._inst_range(inst)].cpu().numpy()

    def upload_state(self, name: str, values: NDArray[np.float32], inst: int = 0) -> None:
        src = torch.from_numpy(np.ascontiguousarray(values, np.float32).ravel())
        with torch.cuda.stream(self._stream):
            self._t[name][self._inst_range(inst)].copy_(src)
        self._stream.synchronize()

    # -- open boundaries ----------------------------------------------------------------
    def set_open_edge_conditions(self, kinds: NDArray[np.uint32], values: NDArray[np.float32]) -> None:
        """Every open edge's condition, by open index, and the blocks it forces.

        A block with an open edge that can bring water in (an inflow or a stage
        with a positive value) is forced: it and its two-ring stay active while
        the condition holds (``inundation/vulkan/gpu_resident_batch.py:447-458``).
        Takes effect at the next start of a run (its prologue rebuilds the lists).
        """
        kinds = np.asarray(kinds, np.uint32).ravel()
        values = np.asarray(values, np.float32).ravel()
        if kinds.size != self.n_open or values.size != self.n_open:
            raise ValueError(f"expected {self.n_open} open edges, got {kinds.size} kinds and {values.size} values")
        if not self.n_open:
            return
        words = np.empty(2 * self.n_open, np.uint32)
        words[0::2] = kinds
        words[1::2] = values.view(np.uint32)
        forced = np.zeros(self.n_blocks, np.int32)
        brings_water = np.isin(kinds, (OPEN_INFLOW, OPEN_STAGE)) & (values > 0.0)
        forced[self.layout.open_cells[brings_water] // ACTIVE_BLOCK_CELLS] = 1
        with torch.cuda.stream(self._stream):
            self._mesh_t["open_cond"].copy_(torch.from_numpy(words.view(np.int32)))
            self._blk.view(self.n_blocks, 3)[:, 2].copy_(torch.from_numpy(forced))
        self._stream.synchronize()

    def download_open_edge_volumes(self) -> NDArray[np.float64]:
        """``(n_open, 2)`` volume out of and into the mesh through every open edge, float64."""
        if not self.n_open:
            return np.zeros((0, 2), np.float64)
        with torch.cuda.stream(self._stream):
            words = self._open_vol.cpu().numpy().astype(np.float64)
        pairs = words[: 4 * self.n_open].reshape(-1, 4)
        return np.column_stack([pairs[:, 0] + pairs[:, 1], pairs[:, 2] + pairs[:, 3]])

    def reset_open_volumes(self) -> None:
        with torch.cuda.stream(self._stream):
            self._open_vol.zero_()

    def download_block_flags(self) -> NDArray[np.uint32]:
        """``(n_blocks, 3)`` flags: wet, active, forced."""
        with torch.cuda.stream(self._stream):
            words = self._blk.cpu().numpy()
        return words.view(np.uint32).reshape(self.n_blocks, 3).copy()

    def volume_fp64(self, inst: int = 0) -> float:
        """Sum of (h + h_lo) * area of one instance in float64 on the device, in a fixed order."""
        r = self._inst_range(inst)
        off, n = r.start, r.stop - r.start
        with torch.cuda.stream(self._stream):
            native.check(
                self._lib.swe_volume_fp64(
                    self._t["h"][off:].data_ptr(), self._t["h_lo"][off:].data_ptr(),
                    self._mesh_t["area"][off:].data_ptr(), n, self._partials.data_ptr(), self._volume.data_ptr(),
                    self._cuda_stream,
                ),
                "swe_volume_fp64",
            )
            out = float(self._volume.cpu().item())
        return out

    @property
    def computed_cells(self) -> int:
        """Cells in computed tiles summed over all real steps (the roofline's cell-step count)."""
        self._stream.synchronize()
        return int(self._sched.cpu().numpy().view(np.uint64)[3])

    # -- kernels ----------------------------------------------------------------------------------
    def _eft_probe(self) -> NDArray[np.float32]:
        """The device's two-sum of 1 and 1e-9: words (1, 1e-9, error term)."""
        v = torch.tensor(EFT_PROBE_WORDS, dtype=torch.float32, device=self.device)
        with torch.cuda.stream(self._stream):
            native.check(self._lib.swe_eft_probe(v.data_ptr(), self._cuda_stream), "swe_eft_probe")
            return v.cpu().numpy()

    def _check_error_free_arithmetic(self) -> None:
        """Refuse to run once if the device loses two-sum's error term (solver.py:449-467)."""
        if self._eft_checked:
            return
        check_eft_probe(self._eft_probe())
        self._eft_checked = True

    def _sync_ctrl_to_device(self) -> None:
        with torch.cuda.stream(self._stream):
            self._ctrl_dev.copy_(self._ctrl_pinned, non_blocking=True)

    def _read_ctrl(self) -> None:
        with torch.cuda.stream(self._stream):
            self._ctrl_pinned.copy_(self._ctrl_dev, non_blocking=True)
            self._sched_pinned.copy_(self._sched, non_blocking=True)
        self._stream.synchronize()
        self._active_blocks = int(self._sched_pinned.numpy().view(np.uint32)[0])
        err = int(self._ctrl["error"].max())
        if err:
            what = " and ".join(w for bit, w in ((1, "for staged data"), (2, "at a grid barrier"),
                                                   (4, "for a step's dt")) if err & bit)
            raise RuntimeError(f"{B200_BACKEND}: a bounded device wait {what} timed out (error {err})")

    def _computed_cells_read(self) -> int:
        """The computed-cells total as of the last control-block read (no device access)."""
        return int(self._sched_pinned.numpy().view(np.uint64)[3])

    def _enqueue_prologue(self) -> None:
        p = self._params()
        with torch.cuda.stream(self._stream):
            self._sched[:3].zero_()  # list counters and epoch; words 6-7 keep the computed-cells total
            self._sched[4:].zero_()
            self._marks.zero_()
            self._sync.zero_()  # barrier counters: consistent again even after a launch that stopped on a timeout
            native.check(
                self._lib.swe_prologue(
                    ctypes.byref(self._mesh), ctypes.byref(self._state), ctypes.byref(p), self._cuda_stream
                ),
                "swe_prologue",
            )

    def _enqueue_retarget(self) -> None:
        """RETARGET every clock to its new stop, rebuilding the active lists first.

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
        native.check(self._lib.swe_steps(mesh, state, pp, sp, n_steps, stream), "swe_steps")

    def _graph(self, steps: int | None = None):
        """A replayable submit of ``steps`` steps: a CUDA graph, or for the persistent kernel its one launch."""
        steps = self.steps_per_graph if steps is None else steps
        if self._kernel == KERNELS["persistent"]:
            return _PersistentSubmit(self, steps)
        key = (
            steps,
            bool(self.compensated),
            bool(self.track_clamp),
            bool(self.active_set),
            self._kernel,
            self.grid(),
            self._src_version,
        )
        graph = self._graphs.get(key)
        if graph is None:
            params, sources = self._params(), self._sources()
            graph = torch.cuda.CUDAGraph()
            self._stream.synchronize()
            with torch.cuda.graph(graph, stream=self._stream):
                self._enqueue_steps(steps, params, sources)
            while len(self._graphs) >= 4:  # keep the few most recent graphs alive
                self._graphs.pop(next(iter(self._graphs)))
            self._graphs[key] = graph
        return graph

    def step_graph(self) -> None:
        """Replay one submit of ``steps_per_graph`` steps (no host sync)."""
        graph = self._graph()
        with torch.cuda.stream(self._stream):
            graph.replay()


def _same_sources(a: list, b: list) -> bool:
    for x, y in zip(a[:4], b[:4], strict=True):
        if (x is None) != (y is None) or (x is not None and not np.array_equal(x, y)):
            return False
    return len(a[4]) == len(b[4]) and all(
        np.array_equal(t0, t1) and np.array_equal(q0, q1) for (t0, q0), (t1, q1) in zip(a[4], b[4], strict=True)
    )


class _PersistentSubmit:
    """One cooperative launch of the persistent kernel per replay (its own grid barriers replace the graph)."""

    def __init__(self, engine: ResidentEngine, steps: int) -> None:
        self.engine, self.steps = engine, steps
        self.params, self.sources = engine._params(), engine._sources()

    def replay(self) -> None:
        e = self.engine
        native.check(
            e._lib.swe_steps(ctypes.byref(e._mesh), ctypes.byref(e._state), ctypes.byref(self.params),
                             ctypes.byref(self.sources), self.steps, e._cuda_stream),
            "swe_steps",
        )


__all__ = ["KERNELS", "NO_HYDROGRAPH", "RESIDENT_CTRL_DTYPE", "Hydrograph", "ResidentEngine", "START", "STEP", "RETARGET"]
