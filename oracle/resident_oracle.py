"""Host loop of the FP32 resident oracle (TEST INFRASTRUCTURE ONLY).

The checker, never the product: only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline arm may use it. It drives the C kernels of
``fp32_resident.c`` the way the reference's ``SWESolverGpuResidentBatch``
drives its shaders:

* data layout of ``_build_tensors`` (``inundation/vulkan/gpu_resident_batch.py:160-282``):
  edges sorted by the block of their left cell, remapped signed CSR,
  per-workgroup block ranges, block two-ring, ``(dzL, dzR)`` pairs;
* ``_set_sources`` (``:529-560``): nonzero cells as (cell, rate / area);
* ``_record_prologue`` (``:567-591``), ``_record_step`` (``:489-513``) and the
  window loop of ``run`` (``:609-762``), with ``steps_per_graph`` steps per
  submit and the control block read back after each;
* open boundaries as ``SWESolver`` numbers them (``inundation/vulkan/solver.py:236-243``,
  open edge k has right cell ``-2 - k`` in stretch order), their conditions and
  forced blocks (``gpu_resident_batch.py:447-458``) and the volume through each
  stretch (``solver.py:432-440``).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from inundation_b200.mesh.blocks import (
    block_adjacency,
    block_two_ring,
    edge_order_by_block,
    edge_workgroup_block_ranges,
    remap_cell_edges,
)
from inundation_b200.tuning import (
    ACTIVE_BLOCK_CELLS,
    CFL_DEFAULT,
    DRY_TOL_DEFAULT,
    GRAVITY_G,
    dt_to_ticks,
    num_blocks,
    output_window_stops,
    seconds_to_ticks,
    ticks_to_seconds,
)

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle_fp32.so"
SOURCE = HERE / "fp32_resident.c"

CTRL_DTYPE = np.dtype(
    [
        ("now_ticks", "<u8"),
        ("stop_ticks", "<u8"),
        ("steps", "<u8"),
        ("dt_ticks", "<u4"),
        ("dt_max_ticks", "<u4"),
        ("dry_dt_ticks", "<u4"),
        ("last_raw", "<f4"),
        ("cfl_safety", "<f4"),
        ("_pad", "<u4"),
    ]
)


def build(force: bool = False) -> Path:
    """Compile the C oracle (no FMA contraction, no fast math) into ``_build/``."""
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= SOURCE.stat().st_mtime:
        return LIB_PATH
    LIB_PATH.parent.mkdir(parents=True, exist_ok=True)
    tmp = LIB_PATH.with_suffix(f".{os.getpid()}.tmp")
    subprocess.run(
        ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", str(tmp), str(SOURCE), "-lm"],
        check=True,
    )
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_LIB: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(str(build()))
        _LIB.oracle_inv_pow43.restype = ctypes.c_float
        _LIB.oracle_inv_pow43.argtypes = [ctypes.c_float]
        _LIB.oracle_sizeof.restype = ctypes.c_size_t
        _LIB.oracle_ctrl_sizeof.restype = ctypes.c_size_t
    return _LIB


class _Oracle(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_uint32),
        ("E", ctypes.c_uint32),
        ("n_blocks", ctypes.c_uint32),
        ("g", ctypes.c_float),
        ("dry_tol", ctypes.c_float),
        ("cfl", ctypes.c_float),
        *[(name, ctypes.c_void_p) for name in (
            "ecL", "ecR", "enx", "eny", "elen", "edz", "area", "n_mann", "cptr", "cidx", "erange", "bptr", "bidx",
            "h", "hu", "hv", "h1", "hu1", "hv1", "h_lo", "h1_lo", "ef", "touched", "blk", "dt_buf", "clamp_mass", "ctrl",
            "src_hydro", "src_hscale", "knot_ptr", "knot_t", "knot_q", "open_cond", "open_vol",
        )],
    ]


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


@dataclass
class ResidentOracle:
    """FP32 restatement of one resident solver (same constructor arguments as the reference's)."""

    geom: object
    h0: np.ndarray
    hu0: np.ndarray
    hv0: np.ndarray
    n0: np.ndarray
    g: float = GRAVITY_G
    dry_tol: float = DRY_TOL_DEFAULT
    cfl: float | None = None
    steps_per_graph: int = 200
    active_set: bool = True
    compensated: bool = True
    track_clamp: bool = False
    cfl_safety: float = 1.0
    steps_total: int = 0
    open_edges: tuple = ()
    arrays: dict = field(default_factory=dict)

    def __post_init__(self) -> None:
        geom = self.geom
        self.N, self.E = int(geom.N), int(geom.E)
        self.cfl = float(CFL_DEFAULT if self.cfl is None else self.cfl)
        order = edge_order_by_block(geom.edge_cellL, ACTIVE_BLOCK_CELLS)
        self.edge_order = order
        self._open_stretches = [np.asarray(e, np.int64).ravel() for e in self.open_edges]
        open_ids = np.concatenate([np.empty(0, np.int64), *self._open_stretches])
        self.n_open = int(open_ids.size)
        self._open_cells = geom.edge_cellL[open_ids].astype(np.int64)
        cell_r = geom.edge_cellR.astype(np.int32).copy()
        cell_r[open_ids] = -2 - np.arange(self.n_open, dtype=np.int32)
        self.open_volume_snapshots: list[np.ndarray] = []
        ecl = geom.edge_cellL[order].astype(np.int32)
        ecr = cell_r[order]
        self.n_blocks = num_blocks(self.N)
        bptr, bidx = block_two_ring(*block_adjacency(ecl, ecr, self.N, ACTIVE_BLOCK_CELLS))
        f32 = np.float32
        a = self.arrays
        a["ecL"], a["ecR"] = ecl, ecr
        a["enx"] = geom.edge_nx[order].astype(f32)
        a["eny"] = geom.edge_ny[order].astype(f32)
        a["elen"] = geom.edge_len[order].astype(f32)
        a["edz"] = np.column_stack([geom.edge_dzL[order], geom.edge_dzR[order]]).astype(f32).ravel()
        a["area"] = geom.area.astype(f32)
        a["n_mann"] = np.asarray(self.n0, f32).copy()
        a["cptr"] = geom.cell_edge_ptr.astype(np.uint32)
        a["cidx"] = remap_cell_edges(geom.cell_edge_idx_signed, order)
        a["erange"] = edge_workgroup_block_ranges(ecl, 256, ACTIVE_BLOCK_CELLS).ravel().astype(np.uint32)
        a["bptr"] = bptr.astype(np.uint32)
        a["bidx"] = bidx.astype(np.uint32) if bidx.size else np.zeros(1, np.uint32)
        for name in ("h1", "hu1", "hv1", "h_lo", "h1_lo", "clamp_mass"):
            a[name] = np.zeros(self.N, f32)
        a["h"] = np.asarray(self.h0, f32).copy()
        a["hu"] = np.asarray(self.hu0, f32).copy()
        a["hv"] = np.asarray(self.hv0, f32).copy()
        a["ef"] = np.zeros(6 * max(self.E, 1), f32)
        a["touched"] = np.zeros(self.N, np.uint32)
        a["blk"] = np.zeros(3 * max(self.n_blocks, 1), np.uint32)
        a["dt_buf"] = np.array([0, 0x7149F2CA, 0, 0], np.uint32)
        a["open_cond"] = np.zeros(2 * max(self.n_open, 1), np.uint32)
        a["open_vol"] = np.zeros(4 * max(self.n_open, 1), np.float32)
        self.ctrl = np.zeros(1, CTRL_DTYPE)
        self._struct = _Oracle(self.N, self.E, self.n_blocks, self.g, self.dry_tol, self.cfl)
        for name, arr in a.items():
            setattr(self._struct, name, _ptr(arr))
        if not self.n_open:
            self._struct.open_cond = None
            self._struct.open_vol = None
        self._struct.ctrl = _ptr(self.ctrl)
        self._sp = ctypes.byref(self._struct)
        self._src_cells = np.zeros(1, np.uint32)
        self._src_rate = np.zeros(1, np.float32)
        self._n_src = 0

    # -- state access ---------------------------------------------------------------
    def download_h(self) -> np.ndarray:
        return self.arrays["h"].copy()

    def download_hu(self) -> np.ndarray:
        return self.arrays["hu"].copy()

    def download_hv(self) -> np.ndarray:
        return self.arrays["hv"].copy()

    def download_h_residual(self) -> np.ndarray:
        return self.arrays["h_lo"].copy()

    def download_h_precise(self) -> np.ndarray:
        return self.arrays["h"].astype(np.float64) + self.arrays["h_lo"].astype(np.float64)

    def download_clamp_mass(self) -> np.ndarray:
        return self.arrays["clamp_mass"].copy()

    def download_block_flags(self) -> np.ndarray:
        return self.arrays["blk"][: 3 * self.n_blocks].reshape(self.n_blocks, 3).copy()

    def reset(self) -> None:
        a = self.arrays
        a["h"][:] = self.h0
        a["hu"][:] = self.hu0
        a["hv"][:] = self.hv0
        a["h_lo"][:] = 0.0
        a["h1_lo"][:] = 0.0
        a["open_vol"][:] = 0.0

    # -- open boundaries ---------------------------------------------------------------
    def set_open_conditions(self, kinds: np.ndarray, values: np.ndarray) -> None:
        """Every open edge's condition in stretch order; blocks an inflow or stage can wet stay forced."""
        kinds = np.asarray(kinds, np.uint32).ravel()
        values = np.asarray(values, np.float32).ravel()
        if kinds.size != self.n_open or values.size != self.n_open:
            raise ValueError(f"expected {self.n_open} open edges, got {kinds.size} kinds and {values.size} values")
        words = self.arrays["open_cond"]
        words[0 : 2 * self.n_open : 2] = kinds
        words[1 : 2 * self.n_open : 2] = values.view(np.uint32)
        blk = self.arrays["blk"]
        blk[2::3] = 0
        brings_water = np.isin(kinds, (3, 4)) & (values > 0.0)
        blk[3 * (self._open_cells[brings_water] // ACTIVE_BLOCK_CELLS) + 2] = 1

    def download_open_volumes(self) -> np.ndarray:
        """``(stretches, 2)`` volume out of and into the mesh since the start, float64."""
        if not self._open_stretches:
            return np.zeros((0, 2), np.float64)
        pairs = self.arrays["open_vol"][: 4 * self.n_open].astype(np.float64).reshape(-1, 4)
        per_edge = np.column_stack([pairs[:, 0] + pairs[:, 1], pairs[:, 2] + pairs[:, 3]])
        sizes = [e.size for e in self._open_stretches]
        out = np.zeros((len(sizes), 2), np.float64)
        o = 0
        for s, n in enumerate(sizes):
            out[s] = per_edge[o : o + n].sum(axis=0)
            o += n
        return out

    # -- kernels --------------------------------------------------------------------
    def set_sources(self, source_rate: np.ndarray | None, hydrographs: list | None = None) -> None:
        """Constant rates (m^3/s per cell) and inflow hydrographs, one entry per cell.

        A hydrograph has ``cells``, ``knot_t``, ``knot_q`` and optional ``share``
        (equal parts by default): cell k gains ``share[k] * q(t) / area`` m/s.
        """
        area = self.arrays["area"]
        rate = np.zeros(self.N, np.float32)
        if source_rate is not None:
            rate = np.asarray(source_rate, np.float32) * (1.0 / area).astype(np.float32)
        hidx = np.full(self.N, 0xFFFFFFFF, np.uint32)
        hscale = np.zeros(self.N, np.float32)
        knots_t, knots_q, ptr = [], [], [0]
        for j, hg in enumerate(hydrographs or []):
            cells = np.asarray(hg.cells, np.int64).ravel()
            share = (np.full(cells.size, 1.0 / cells.size, np.float32) if getattr(hg, "share", None) is None
                     else np.asarray(hg.share, np.float32).ravel())
            hidx[cells] = j
            hscale[cells] = share * (1.0 / area[cells]).astype(np.float32)
            knots_t.append(np.asarray(hg.knot_t, np.float32).ravel())
            knots_q.append(np.asarray(hg.knot_q, np.float32).ravel())
            ptr.append(ptr[-1] + knots_t[-1].size)
        cells = np.flatnonzero((rate != 0) | (hidx != 0xFFFFFFFF)).astype(np.uint32)
        self._src_cells = cells if cells.size else np.zeros(1, np.uint32)
        self._src_rate = rate[cells].astype(np.float32) if cells.size else np.zeros(1, np.float32)
        self._n_src = int(cells.size)
        self._hydro = None
        if knots_t and cells.size:
            self._hydro = {
                "src_hydro": np.ascontiguousarray(hidx[cells]),
                "src_hscale": np.ascontiguousarray(hscale[cells]),
                "knot_ptr": np.asarray(ptr, np.uint32),
                "knot_t": np.concatenate(knots_t),
                "knot_q": np.concatenate(knots_q),
            }
        for name in ("src_hydro", "src_hscale", "knot_ptr", "knot_t", "knot_q"):
            setattr(self._struct, name, _ptr(self._hydro[name]) if self._hydro else None)

    def prologue(self) -> None:
        L = lib()
        L.oracle_block_mark(self._sp, ctypes.c_int(0 if self.active_set else 1))
        if self.active_set:
            L.oracle_block_dilate(self._sp, ctypes.c_int(1))
        L.oracle_cfl_prologue(self._sp)
        L.oracle_step_control(ctypes.c_void_p(_ptr(self.ctrl)), ctypes.c_void_p(_ptr(self.arrays["dt_buf"])), ctypes.c_int(0))

    def retarget(self) -> None:
        lib().oracle_step_control(
            ctypes.c_void_p(_ptr(self.ctrl)), ctypes.c_void_p(_ptr(self.arrays["dt_buf"])), ctypes.c_int(2)
        )

    def step(self) -> None:
        lib().oracle_step(
            self._sp,
            ctypes.c_void_p(_ptr(self._src_cells)),
            ctypes.c_void_p(_ptr(self._src_rate)),
            ctypes.c_uint32(self._n_src),
            ctypes.c_int(int(self.compensated)),
            ctypes.c_int(int(self.track_clamp)),
            ctypes.c_int(int(self.active_set)),
        )

    def run(
        self,
        t_end: float,
        output_interval_s: float,
        dt_max: float,
        dt_init: float,
        cfl_interval: int = 1,
        progress: bool = False,
        source_rate: np.ndarray | None = None,
        resume: bool = False,
        t_start: float = 0.0,
        hydrographs: list | None = None,
    ) -> tuple[list[np.ndarray], list[float]]:
        """The reference's window loop (gpu_resident_batch.py:648-762), on the C kernels.

        ``cfl_interval`` and ``progress`` are accepted like the reference's and ignored.
        """
        del cfl_interval, progress
        dt_max_ticks = dt_to_ticks(dt_max)
        dry_dt_ticks = dt_to_ticks(min(dt_init, dt_max))
        start = seconds_to_ticks(t_start if resume else 0.0)
        end = seconds_to_ticks(t_end)
        interval = seconds_to_ticks(output_interval_s)
        if not resume:
            self.reset()
            self.open_volume_snapshots = []
        self.set_sources(source_rate, hydrographs)
        snaps = [self.download_h()]
        times = [ticks_to_seconds(start)]
        self._capture_open()
        c = self.ctrl
        c["now_ticks"] = start
        c["steps"] = 0
        c["dt_ticks"] = 0
        c["dt_max_ticks"] = dt_max_ticks
        c["dry_dt_ticks"] = dry_dt_ticks
        c["cfl_safety"] = self.cfl_safety
        planned = False
        finite = True
        for stop in output_window_stops(start, end, interval):
            c["stop_ticks"] = stop
            if planned:
                self.retarget()
            else:
                self.prologue()
                planned = True
            while int(c["now_ticks"][0]) < stop:
                before = int(c["now_ticks"][0])
                for _ in range(self.steps_per_graph):
                    self.step()
                if int(c["now_ticks"][0]) == before:
                    raise RuntimeError("oracle run made no time progress (CFL bound below one tick)")
            h = self.download_h()
            if not np.isfinite(h).all():
                snaps.append(np.nan_to_num(h, nan=0.0, posinf=0.0))
                times.append(ticks_to_seconds(stop))
                self._capture_open()
                finite = False
                break
            if (stop - start) % interval == 0:
                snaps.append(h)
                times.append(ticks_to_seconds(stop))
                self._capture_open()
        self.steps_total += int(c["steps"][0])
        if finite:
            h = self.download_h()
            if not np.allclose(snaps[-1], h):
                snaps.append(h)
                times.append(ticks_to_seconds(int(c["now_ticks"][0])))
                self._capture_open()
        return snaps, times

    def _capture_open(self) -> None:
        if self.n_open:
            self.open_volume_snapshots.append(self.download_open_volumes())


def inv_pow43(x: float) -> float:
    """x^(-4/3) as the kernels evaluate it (the friction slope's depth power)."""
    return float(lib().oracle_inv_pow43(ctypes.c_float(x)))


def step_control(ctrl: np.ndarray, dt_buf: np.ndarray, mode: int) -> None:
    """Run the restated ``step_control`` on a host control block and dt words in place."""
    lib().oracle_step_control(ctypes.c_void_p(_ptr(ctrl)), ctypes.c_void_p(_ptr(dt_buf)), ctypes.c_int(mode))


def hllc_f32(g: float, dry_tol: float, states: np.ndarray) -> np.ndarray:
    """Rows of (hL, hqnL, hqtL, hR, hqnR, hqtR) -> rows of (Fh, Fhn, Fht, Smax) in float32."""
    states = np.ascontiguousarray(states, np.float32)
    out = np.zeros((states.shape[0], 4), np.float32)
    for k in range(states.shape[0]):
        lib().oracle_hllc(
            ctypes.c_float(g), ctypes.c_float(dry_tol), ctypes.c_void_p(_ptr(states[k])), ctypes.c_void_p(_ptr(out[k]))
        )
    return out


def hllc_speeds_f32(g: float, dry_tol: float, rows: np.ndarray) -> np.ndarray:
    rows = np.ascontiguousarray(rows, np.float32)
    out = np.zeros((rows.shape[0], 2), np.float32)
    for k in range(rows.shape[0]):
        lib().oracle_hllc_speeds(
            ctypes.c_float(g), ctypes.c_float(dry_tol), ctypes.c_void_p(_ptr(rows[k])), ctypes.c_void_p(_ptr(out[k]))
        )
    return out


def math_ok() -> bool:
    """The compiled two-sum keeps its error term (the reference's EFT guard, solver.py:449-467)."""
    se = np.zeros(2, np.float32)
    lib().oracle_two_sum(ctypes.c_float(1.0), ctypes.c_float(1e-9), ctypes.c_void_p(_ptr(se)))
    return float(se[1]) == float(np.float32(1e-9))



def open_ghost_f32(g: float, dry_tol: float, cases: np.ndarray, kinds: np.ndarray, values: np.ndarray) -> np.ndarray:
    """Rows of (h, hu, hv, nx, ny, HLLC mass flux) under open conditions -> rows of the
    ghost (h, hu, hv) and the boundary mass flux, in float32 (the probe of the
    reference's ``tests/unit/test_gpu_open_ghost.py``)."""
    cases = np.ascontiguousarray(cases, np.float32).reshape(-1, 6)
    cond = np.zeros((cases.shape[0], 2), np.uint32)
    cond[:, 0] = np.asarray(kinds, np.uint32).ravel()
    cond[:, 1] = np.asarray(values, np.float32).ravel().view(np.uint32)
    out = np.zeros((cases.shape[0], 4), np.float32)
    lib().oracle_open_ghost(ctypes.c_float(g), ctypes.c_float(dry_tol), ctypes.c_void_p(_ptr(cases)),
                            ctypes.c_void_p(_ptr(cond)), ctypes.c_void_p(_ptr(out)), ctypes.c_uint32(cases.shape[0]))
    return out
