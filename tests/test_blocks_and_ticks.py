"""Active-set block topology and the integer clock, against the reference.

Golden values come from the reference's ``inundation/mesh/blocks.py`` and
``inundation/tuning.py`` (``tests/golden/blocks.npz``, ``ticks.npz``); the
property tests restate the reference's ``tests/unit/test_mesh_blocks.py`` and
``tests/unit/test_sim_ticks.py``.
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from inundation_b200.mesh import blocks as B
from inundation_b200.mesh.geometry import build_geometry, hilbert_reorder
from inundation_b200.mesh.synthetic import quad_grid
from inundation_b200.tuning import (
    ACTIVE_BLOCK_CELLS,
    SIM_DT_MAX_TICKS,
    SIM_TICKS_PER_SECOND,
    dt_to_ticks,
    num_blocks,
    output_window_stops,
    seconds_to_ticks,
    ticks_to_seconds,
)

GOLD = Path(__file__).parent / "golden"
BLK = np.load(GOLD / "blocks.npz")
TCK = np.load(GOLD / "ticks.npz")
GEO = np.load(GOLD / "geometry.npz")


@pytest.fixture(scope="module")
def voronoi():
    raw = build_geometry(GEO["voronoi_in_verts"], GEO["voronoi_in_faces"], GEO["voronoi_in_offsets"], zb_from_file=GEO["voronoi_in_zb"])
    return hilbert_reorder(raw, verbose=False)[0]


@pytest.fixture(scope="module")
def grid():
    q = quad_grid(64, 48, 1.0)
    g = build_geometry(q.verts, q.faces.reshape(-1, 4), zb_from_file=np.zeros(64 * 48, np.float32))
    return hilbert_reorder(g, verbose=False)[0]


@pytest.mark.parametrize("bc", [256, 16])
def test_block_topology_matches_the_reference(voronoi, bc: int) -> None:
    order = B.edge_order_by_block(voronoi.edge_cellL, bc)
    np.testing.assert_array_equal(order, BLK[f"b{bc}_order"])
    np.testing.assert_array_equal(B.remap_cell_edges(voronoi.cell_edge_idx_signed, order), BLK[f"b{bc}_remap"])
    ecl, ecr = voronoi.edge_cellL[order], voronoi.edge_cellR[order]
    np.testing.assert_array_equal(B.edge_workgroup_block_ranges(ecl, 256, bc), BLK[f"b{bc}_ranges"])
    ptr, idx = B.block_adjacency(ecl, ecr, voronoi.N, bc)
    np.testing.assert_array_equal(ptr, BLK[f"b{bc}_adj_ptr"])
    np.testing.assert_array_equal(idx, BLK[f"b{bc}_adj_idx"])
    p2, i2 = B.block_two_ring(ptr, idx)
    np.testing.assert_array_equal(p2, BLK[f"b{bc}_ring_ptr"])
    np.testing.assert_array_equal(i2, BLK[f"b{bc}_ring_idx"])
    np.testing.assert_array_equal(B.dilate_blocks(BLK[f"b{bc}_flags"], p2, i2), BLK[f"b{bc}_dilated"])


@pytest.mark.parametrize(("cells", "expected"), [(0, 0), (1, 1), (256, 1), (257, 2), (512, 2)])
def test_num_blocks_rounds_up(cells: int, expected: int) -> None:
    assert num_blocks(cells, 256) == expected


def test_num_blocks_rejects_non_positive_size() -> None:
    with pytest.raises(ValueError, match="block_cells"):
        num_blocks(10, 0)


def test_edge_order_is_stable_by_left_block() -> None:
    cell_l = np.array([5, 1, 9, 0, 6, 2], dtype=np.int32)
    order = B.edge_order_by_block(cell_l, 4)
    assert (cell_l[order] // 4).tolist() == [0, 0, 0, 1, 1, 2]
    assert cell_l[order][:3].tolist() == [1, 0, 2]


def test_remap_follows_the_permutation_and_keeps_the_side_bit() -> None:
    order = np.array([1, 2, 0], dtype=np.int64)
    signed = np.array([0 << 1 | 1, 1 << 1, 2 << 1 | 1], dtype=np.int32)
    assert B.remap_cell_edges(signed, order).tolist() == [2 << 1 | 1, 0 << 1, 1 << 1 | 1]


def test_workgroup_ranges_and_unsorted_edges() -> None:
    r = B.edge_workgroup_block_ranges(np.array([0, 1, 4, 5, 5, 9, 12], np.int32), workgroup=3, block_cells=4)
    assert r.tolist() == [[0, 1], [1, 2], [3, 3]]
    with pytest.raises(ValueError, match="sorted"):
        B.edge_workgroup_block_ranges(np.array([8, 0], np.int32), 2, 4)


def test_chain_adjacency_and_two_ring() -> None:
    ptr, idx = B.block_adjacency(np.array([0, 1, 2, 3, 4, 5, 6, 0], np.int32), np.array([1, 2, 3, 4, 5, 6, 7, -1], np.int32), 8, 2)
    assert [idx[ptr[b]: ptr[b + 1]].tolist() for b in range(4)] == [[1], [0, 2], [1, 3], [2]]
    p2, i2 = B.block_two_ring(ptr, idx)
    assert [i2[p2[b]: p2[b + 1]].tolist() for b in range(4)] == [[1, 2], [0, 2, 3], [0, 1, 3], [1, 2]]


def test_single_block_has_no_neighbours() -> None:
    ptr, idx = B.block_adjacency(np.array([0, 0], np.int32), np.array([1, -1], np.int32), 2, 256)
    assert ptr.tolist() == [0, 0] and idx.size == 0


def _cell_dilate(wet: np.ndarray, geom) -> np.ndarray:
    out = wet.copy()
    inner = geom.edge_cellR >= 0
    left, right = geom.edge_cellL[inner], geom.edge_cellR[inner]
    out[left] |= wet[right]
    out[right] |= wet[left]
    return out


def test_one_dilation_over_the_two_ring_equals_two(grid) -> None:
    ptr, idx = B.block_adjacency(grid.edge_cellL, grid.edge_cellR, grid.N, ACTIVE_BLOCK_CELLS)
    p2, i2 = B.block_two_ring(ptr, idx)
    rng = np.random.default_rng(7)
    for _ in range(20):
        flags = rng.random(ptr.size - 1) < 0.05
        np.testing.assert_array_equal(B.dilate_blocks(flags, p2, i2), B.dilate_blocks(B.dilate_blocks(flags, ptr, idx), ptr, idx))


def test_two_cell_rings_stay_inside_the_block_two_ring(voronoi) -> None:
    p2, i2 = B.block_two_ring(*B.block_adjacency(voronoi.edge_cellL, voronoi.edge_cellR, voronoi.N, ACTIVE_BLOCK_CELLS))
    cell_block = np.arange(voronoi.N) // ACTIVE_BLOCK_CELLS
    rng = np.random.default_rng(3)
    for frac in (0.0005, 0.005, 0.05):
        wet = rng.random(voronoi.N) < frac
        marked = np.zeros(p2.size - 1, dtype=bool)
        marked[cell_block[wet]] = True
        active = B.dilate_blocks(marked, p2, i2)
        reach = _cell_dilate(_cell_dilate(wet, voronoi), voronoi)
        assert active[cell_block[reach]].all()


# -- ticks ------------------------------------------------------------------------------------------
def test_ticks_match_the_reference() -> None:
    assert [seconds_to_ticks(float(s)) for s in TCK["seconds"]] == TCK["seconds_ticks"].tolist()
    assert [dt_to_ticks(float(d)) for d in TCK["dts"]] == TCK["dt_ticks"].tolist()
    assert list(output_window_stops(0, 1000, 600)) == TCK["windows_a"].tolist()
    assert list(output_window_stops(7200 << 20, (7200 + 3600) << 20, 1800 << 20)) == TCK["windows_b"].tolist()


@pytest.mark.parametrize("seconds", [0.0, 0.5, 1.0, 600.0, 1800.0, 7200.0, 86400.0])
def test_binary_fraction_times_are_exact(seconds: float) -> None:
    t = seconds_to_ticks(seconds)
    assert t == int(seconds * SIM_TICKS_PER_SECOND)
    assert ticks_to_seconds(t) == seconds


def test_summed_phases_land_on_the_total() -> None:
    assert sum(seconds_to_ticks(d) for d in [600.0] * 12 + [79_200.0]) == seconds_to_ticks(86_400.0)


@pytest.mark.parametrize("bad", [-1.0, math.nan, math.inf, -math.inf])
def test_rejects_bad_times(bad: float) -> None:
    with pytest.raises(ValueError, match="simulated time"):
        seconds_to_ticks(bad)


def test_dt_rounds_down_and_is_bounded() -> None:
    t = dt_to_ticks(0.0314)
    assert ticks_to_seconds(t) <= 0.0314 < ticks_to_seconds(t + 1)
    assert dt_to_ticks(16.0) == SIM_DT_MAX_TICKS
    for bad in (16.5, 0.0, -0.1, math.nan, math.inf, 0.5 / SIM_TICKS_PER_SECOND):
        with pytest.raises(ValueError, match="dt"):
            dt_to_ticks(bad)


def test_every_tick_count_is_exact_in_float32() -> None:
    ticks = np.arange(1, SIM_DT_MAX_TICKS + 1, dtype=np.int64)
    as_f32 = ticks.astype(np.float32) * np.float32(1.0 / SIM_TICKS_PER_SECOND)
    assert np.array_equal(as_f32.astype(np.float64), ticks / SIM_TICKS_PER_SECOND)


def test_window_edge_cases() -> None:
    assert list(output_window_stops(0, 500, 600)) == [500]
    assert list(output_window_stops(1000, 1000, 600)) == []
    with pytest.raises(ValueError, match="interval"):
        list(output_window_stops(0, 1000, 0))
