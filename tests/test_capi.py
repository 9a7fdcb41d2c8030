"""The C ABI library loads and exports every function ``include/*.h`` declares (no GPU needed).

Also the host-side layout the kernels index: every CSR slot of a cell must
name, through its tile position, the edge the reference's remapped CSR names
(``inundation/mesh/blocks.py:33-44``), with the cell on the stated side, and
the kernels' launch arguments must refuse null pointers.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from inundation_b200 import native
from inundation_b200.build import LIB_PATH, build
from inundation_b200.layout import TILE_ALIGN, build_tile_layout
from inundation_b200.mesh.blocks import edge_order_by_block, remap_cell_edges
from inundation_b200.mesh.geometry import build_geometry, hilbert_reorder

HEADERS = sorted((Path(__file__).resolve().parent.parent / "include").glob("*.h"))
GEO = np.load(Path(__file__).parent / "golden" / "geometry.npz")


def declared_functions() -> list[str]:
    names: list[str] = []
    for header in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(swe_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib() -> ctypes.CDLL:
    build()
    return native.load()


def test_library_is_built_in_tree() -> None:
    build()
    assert LIB_PATH.exists() and LIB_PATH.is_relative_to(Path(native.__file__).resolve().parent)


def test_every_declared_function_is_exported(lib: ctypes.CDLL) -> None:
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert set(names) == set(native.exported_symbols())


def test_status_strings_and_argument_checks(lib: ctypes.CDLL) -> None:
    assert lib.swe_status_string(0) == b"ok"
    assert b"argument" in lib.swe_status_string(1)
    # Null structs are refused before anything touches a device.
    assert lib.swe_stage(None, None, None, 0, None) == 1
    assert lib.swe_step(None, None, None, None, None) == 1
    assert lib.swe_prologue(None, None, None, None) == 1
    assert lib.swe_step_control(None, None, 1, 0, None) == 1
    assert lib.swe_volume_fp64(None, None, None, 0, None, None, None) == 1
    assert lib.swe_workspace_bytes(3907, 1) >= 3907 * 4 * 36 + 64 + 256 + 16 + 48
    assert lib.swe_workspace_bytes(3907, 64) == lib.swe_workspace_bytes(3907, 1) + 63 * (16 + 48)
    assert lib.swe_configure(None, 0, None) == 1


def test_stage_refuses_kernel_2_and_a_staged_kernel_without_its_csr(lib: ctypes.CDLL) -> None:
    """swe_stage runs kernels 0, 1 and 3; kernel 3 also needs the regrouped block CSR.

    Placeholder addresses again: both refusals come from host-side checks before any device call.
    """
    mesh = native.SweMesh(n_cells=256, n_blocks=1, max_tile_edges=64, n_inst=1, max_sub_edges=64, max_sub_slots=64)
    for name, kind in native.SweMesh._fields_:
        if kind is native._P and name not in ("open_cond", "blk_lcsr", "blk_lcsr_ptr"):
            setattr(mesh, name, 0x10000)
    state = native.SweState(**{name: 0x20000 for name, _ in native.SweState._fields_})
    for kernel in (2, 3, 4):
        params = native.SweParams(g=9.81, dry_tol=1e-4, cfl=0.8, compensated=1, active_set=1, kernel=kernel)
        for stage in (0, 1):
            assert lib.swe_stage(ctypes.byref(mesh), ctypes.byref(state), ctypes.byref(params), stage, None) == 1


def test_whole_steps_refuse_a_misaligned_dt_buffer(lib: ctypes.CDLL) -> None:
    """Kernel 2 publishes each dt as a 64-bit pair in dt words 2..3: dt_buf must be 16-byte aligned.

    The structs carry placeholder addresses that nothing dereferences: the argument
    checks run on the host before any device call.
    """
    mesh = native.SweMesh(n_cells=256, n_blocks=1, max_tile_edges=64, n_inst=1, max_sub_edges=64, max_sub_slots=64)
    for name, kind in native.SweMesh._fields_:
        if kind is native._P and name != "open_cond":
            setattr(mesh, name, 0x10000)
    state = native.SweState(**{name: 0x20000 for name, _ in native.SweState._fields_})
    params = native.SweParams(g=9.81, dry_tol=1e-4, cfl=0.8, compensated=1, active_set=1, kernel=2)
    sources = native.SweSources()
    state.dt_buf = 0x20008
    assert lib.swe_steps(ctypes.byref(mesh), ctypes.byref(state), ctypes.byref(params), ctypes.byref(sources), 1,
                         None) == 1
    import torch

    if not torch.cuda.is_available():  # with a device, an aligned buffer would launch on the placeholders
        state.dt_buf = 0x20010
        assert lib.swe_steps(ctypes.byref(mesh), ctypes.byref(state), ctypes.byref(params), ctypes.byref(sources),
                             1, None) == 2  # past the argument checks: the CUDA runtime finds no device


def test_ctypes_structs_match_the_header_layout() -> None:
    # ... n_open (padded), open_cond, max_blk_slots (padded), blk_lcsr, blk_lcsr_ptr
    assert ctypes.sizeof(native.SweMesh) == 16 + 17 * 8 + 8 + 11 * 8 + 8 + 8 + 8 + 8 + 8
    assert native.SweMesh.n_open.offset == 248 and native.SweMesh.open_cond.offset == 256
    assert native.SweMesh.max_blk_slots.offset == 264 and native.SweMesh.blk_lcsr_ptr.offset == 280
    assert ctypes.sizeof(native.SweState) == 18 * 8
    assert ctypes.sizeof(native.SweParams) == 32
    assert ctypes.sizeof(native.SweSources) == 7 * 8 + 8


@pytest.mark.parametrize("name", ["voronoi", "valley", "mixed"])
def test_tile_segments_put_the_records_that_read_other_tiles_last(name: str) -> None:
    """Per segment: edges with both cells in the tile (or a wall), then the tile's edges to other
    tiles, then the edges whose left cell is outside; each group in resident order."""
    offsets = GEO[f"{name}_in_offsets"]
    raw = build_geometry(GEO[f"{name}_in_verts"], GEO[f"{name}_in_faces"], offsets if offsets.size else None,
                         zb_from_file=GEO[f"{name}_in_zb"])
    layout = build_tile_layout(hilbert_reorder(raw, verbose=False)[0])
    for T in (layout.blocks, layout.subs):
        for t in range(T.n_tiles):
            r = slice(int(T.ptr[t]), int(T.ptr[t]) + int(T.count[t]))
            left_in = T.cl[r] // T.tile_cells == t
            right_in = (T.cr[r] < 0) | (T.cr[r] // T.tile_cells == t)
            group = np.where(left_in & right_in, 0, np.where(left_in, 1, 2))
            assert (np.diff(group) >= 0).all()
            edge = T.edge[r]
            for k in range(3):
                assert (np.diff(edge[group == k]) > 0).all()  # resident order within each group


@pytest.mark.parametrize("name", ["voronoi", "valley", "mixed"])
def test_tile_layout_resolves_every_csr_slot(name: str) -> None:
    offsets = GEO[f"{name}_in_offsets"]
    raw = build_geometry(GEO[f"{name}_in_verts"], GEO[f"{name}_in_faces"], offsets if offsets.size else None,
                         zb_from_file=GEO[f"{name}_in_zb"])
    g = hilbert_reorder(raw, verbose=False)[0]
    layout = build_tile_layout(g)
    order = edge_order_by_block(g.edge_cellL, 256)
    signed = remap_cell_edges(g.cell_edge_idx_signed, order).astype(np.int64)
    cell = np.repeat(np.arange(g.N), np.diff(g.cell_edge_ptr))
    for T in (layout.blocks, layout.subs):
        tile = cell // T.tile_cells
        local, side = T.lcsr.astype(np.int64) >> 1, T.lcsr.astype(np.int64) & 1
        rec = T.ptr[tile].astype(np.int64) + local
        assert (local < T.count[tile]).all()
        np.testing.assert_array_equal(T.edge[rec], signed >> 1)
        np.testing.assert_array_equal(side, signed & 1)
        np.testing.assert_array_equal(np.where(side == 1, T.cr[rec], T.cl[rec]), cell)
        assert (T.ptr % TILE_ALIGN == 0).all() and (T.lcsr_ptr % 8 == 0).all()
        # every edge is in the tile of its left cell exactly once, and in its right cell's tile if that differs
        assert np.bincount(T.edge[T.edge >= 0], minlength=g.E).min() >= 1
        assert T.max_edges == int(T.count.max())
        for t in range(T.n_tiles):
            s0 = g.cell_edge_ptr[min(t * T.tile_cells, g.N)]
            s1 = g.cell_edge_ptr[min((t + 1) * T.tile_cells, g.N)]
            np.testing.assert_array_equal(T.lcsr_blk[T.lcsr_ptr[t]: T.lcsr_ptr[t] + s1 - s0], T.lcsr[s0:s1])


def test_the_dt_wait_probe_refuses_a_misaligned_or_missing_buffer(lib: ctypes.CDLL) -> None:
    state = native.SweState()
    assert lib.swe_dt_wait_probe(ctypes.byref(state), 1, ctypes.c_void_p(16), None) == 1  # no dt words
    state.dt_buf, state.ctrl = 0x20008, 0x30000
    assert lib.swe_dt_wait_probe(ctypes.byref(state), 1, ctypes.c_void_p(16), None) == 1  # not 16-byte aligned
