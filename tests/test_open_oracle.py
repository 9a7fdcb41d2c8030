"""Open boundaries on the CPU: the oracle's ghost states against the reference's
known answers, the host-side stretch selection and inflow split, the layout of
open edges, and run-level properties of the oracle.

The ghost cases are those of the reference's ``tests/unit/test_gpu_open_ghost.py``
(formulas of ``inundation/vulkan/shaders/flux.py:187-281``), here pinning the C
restatement that the device kernels are then compared with bit for bit.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from inundation_b200.layout import build_tile_layout
from inundation_b200.mesh.boundaries import conveyance_split, select_boundary_edges
from inundation_b200.scenarios import open_channel
from inundation_b200.tuning import GRAVITY_G, OPEN_FREE, OPEN_INFLOW, OPEN_NORMAL, OPEN_STAGE, OPEN_WALL
from oracle.resident_oracle import ResidentOracle, open_ghost_f32

DRY_TOL = 1e-4


def ghost(h, hu, hv, kind, value=0.0, *, normal=(1.0, 0.0), hllc_flux=0.0):
    out = open_ghost_f32(GRAVITY_G, DRY_TOL, np.array([[h, hu, hv, normal[0], normal[1], hllc_flux]]), [kind], [value])
    return tuple(float(v) for v in out[0])


def root(q: float, riemann: float) -> float:
    """``hG`` solving ``-q/hG + 2 sqrt(g hG) = riemann`` by bisection on sqrt(hG)."""
    rg = math.sqrt(GRAVITY_G)
    lo, hi = 1e-9, 100.0
    for _ in range(200):
        s = 0.5 * (lo + hi)
        if 2.0 * rg * s - q / (s * s) < riemann:
            lo = s
        else:
            hi = s
    return hi * hi


def test_free_outflow_copies_the_interior() -> None:
    assert ghost(1.0, 0.5, 0.2, OPEN_FREE, hllc_flux=0.5) == pytest.approx((1.0, 0.5, 0.2, 0.5), rel=1e-6)


def test_free_outflow_mirrors_flow_running_inward() -> None:
    assert ghost(1.0, -0.5, 0.2, OPEN_FREE, hllc_flux=-0.5) == pytest.approx((1.0, 0.5, 0.2, 0.0), rel=1e-6)


@pytest.mark.parametrize("kind", [OPEN_FREE, OPEN_NORMAL])
def test_outflow_conditions_never_take_a_negative_flux(kind: int) -> None:
    assert ghost(1.0, 0.0, 0.0, kind, 1.0, hllc_flux=-0.25)[3] == 0.0


def test_normal_depth_uses_the_manning_velocity() -> None:
    value = math.sqrt(1e-3) / 0.03
    h = 0.8
    un = value * h ** (2.0 / 3.0)
    assert ghost(h, 0.1, 0.05, OPEN_NORMAL, value) == pytest.approx((h, h * un, 0.05, 0.0), rel=1e-5)


def test_a_stage_keeps_the_outgoing_characteristic() -> None:
    h, u, depth = 1.0, 0.5, 2.0
    un = u + 2.0 * (math.sqrt(GRAVITY_G * h) - math.sqrt(GRAVITY_G * depth))
    assert ghost(h, h * u, 0.0, OPEN_STAGE, depth, hllc_flux=-0.7) == pytest.approx((depth, depth * un, 0.0, -0.7),
                                                                                    rel=1e-5)


def test_a_stage_cannot_reach_a_supercritical_outflow() -> None:
    h, u = 0.1, 3.0
    assert ghost(h, h * u, 0.0, OPEN_STAGE, 2.0)[:3] == pytest.approx((h, h * u, 0.0), rel=1e-5)


def test_a_stage_over_a_dry_cell_enters_as_a_dam_break() -> None:
    depth = 0.5
    un = -2.0 * math.sqrt(GRAVITY_G * depth)
    assert ghost(0.0, 0.0, 0.0, OPEN_STAGE, depth)[:2] == pytest.approx((depth, depth * un), rel=1e-5)


def test_a_wall_kind_mirrors_and_passes_nothing() -> None:
    assert ghost(1.0, 0.5, 0.2, OPEN_WALL, hllc_flux=0.3) == pytest.approx((1.0, -0.5, 0.2, 0.0), rel=1e-6)


@pytest.mark.parametrize(("h", "u", "q"), [(0.0, 0.0, 0.25), (0.05, 0.0, 2.0), (1.0, -0.2, 0.25), (3.0, 0.5, 5.0),
                                           (0.2, 0.0, 17.0)])
def test_inflow_solves_the_outgoing_characteristic(h: float, u: float, q: float) -> None:
    riemann = u + 2.0 * math.sqrt(GRAVITY_G * h)
    depth = root(q, riemann)
    assert ghost(h, h * u, 0.7 * h, OPEN_INFLOW, q, hllc_flux=9.0) == pytest.approx((depth, -q, 0.0, -q), rel=1e-4,
                                                                                    abs=1e-6)


def test_ghosts_follow_the_edge_normal() -> None:
    nx, ny = 0.6, 0.8
    h, q = 1.0, 0.5
    depth = root(q, 2.0 * math.sqrt(GRAVITY_G * h))
    assert ghost(h, 0.0, 0.0, OPEN_INFLOW, q, normal=(nx, ny))[:3] == pytest.approx((depth, -q * nx, -q * ny), rel=1e-4)


def test_an_inflow_of_nothing_is_a_wall() -> None:
    assert ghost(1.0, 0.5, 0.2, OPEN_INFLOW, 0.0, hllc_flux=0.3) == pytest.approx((1.0, -0.5, 0.2, -0.0), rel=1e-6)


# -- host side ---------------------------------------------------------------------------------------
def test_a_line_selects_the_end_of_a_channel() -> None:
    sc = open_channel(cells=30, across=4, length=300.0, width=40.0)
    g = sc.geom
    up, down = sc.meta["open_edges"]
    assert up.size == down.size == 4
    assert (g.edge_cellR[up] == -1).all() and (g.edge_cellR[down] == -1).all()
    np.testing.assert_allclose(g.edge_len[up], 10.0)
    assert (g.centroid[g.edge_cellL[up], 0] == 5.0).all()
    assert (g.centroid[g.edge_cellL[down], 0] == 295.0).all()
    assert select_boundary_edges(g, [(150.0, 10.0), (150.0, 30.0)], 1.0).size == 0  # interior line: no walls


def test_conveyance_split_carries_the_discharge_along_the_low_part() -> None:
    lengths = np.full(5, 10.0, np.float32)
    beds = np.array([1.0, 0.5, 0.0, 0.5, 1.0], np.float32)
    n = np.full(5, 0.03, np.float32)
    q = conveyance_split(20.0, lengths, beds, n, 1e-3)
    assert q.dtype == np.float32
    assert float((q.astype(np.float64) * 10.0).sum()) == pytest.approx(20.0, rel=1e-7)  # one float32 rounding
    assert q[2] > q[1] == pytest.approx(q[3]) and q[1] >= q[0]
    assert not conveyance_split(0.0, lengths, beds, n, 1e-3).any()


def test_open_edges_sit_in_the_tile_of_their_cell() -> None:
    import dataclasses

    sc = open_channel(cells=60, across=8, length=600.0, width=80.0)
    g = sc.geom
    ids = np.concatenate(sc.meta["open_edges"])
    cell_r = g.edge_cellR.copy()
    cell_r[ids] = -2 - np.arange(ids.size)
    layout = build_tile_layout(dataclasses.replace(g, edge_cellR=cell_r))
    assert layout.n_open == ids.size
    np.testing.assert_array_equal(layout.open_cells, g.edge_cellL[ids])
    for T in (layout.blocks, layout.subs):
        rec = T.edge >= 0
        open_rec = rec & (T.cr < -1)
        assert open_rec.sum() == ids.size  # once each, in the tile of the left cell
        tile = np.searchsorted(T.ptr, np.flatnonzero(open_rec), side="right") - 1
        np.testing.assert_array_equal(T.cl[open_rec] // T.tile_cells, tile)


# -- the oracle over whole runs ---------------------------------------------------------------------
def oracle_channel(depth: float = 0.0, open_ends: bool = True, **kw):
    sc = open_channel(cells=60, across=4, length=600.0, width=40.0, depth=depth, **kw)
    o = ResidentOracle(sc.geom, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=DRY_TOL, steps_per_graph=20,
                       open_edges=tuple(sc.meta["open_edges"]) if open_ends else ())
    return sc, o


def conditions(sc, up: tuple[int, float], down: tuple[int, float]):
    a, b = sc.meta["open_edges"]
    kinds = np.concatenate([np.full(a.size, up[0]), np.full(b.size, down[0])]).astype(np.uint32)
    values = np.concatenate([np.full(a.size, up[1]), np.full(b.size, down[1])]).astype(np.float32)
    return kinds, values


def test_a_wall_stretch_behaves_like_no_stretch() -> None:
    sc, closed = oracle_channel(depth=0.5)
    closed.set_open_conditions(*conditions(sc, (OPEN_WALL, 0.0), (OPEN_WALL, 0.0)))
    _, plain = oracle_channel(depth=0.5, open_ends=False)
    a, _ = closed.run(t_end=20.0, output_interval_s=10.0, dt_max=1.0, dt_init=0.01)
    b, _ = plain.run(t_end=20.0, output_interval_s=10.0, dt_max=1.0, dt_init=0.01)
    assert closed.steps_total == plain.steps_total
    # the wall-kind ghost mirrors through film-safe velocities: equal up to rounding
    np.testing.assert_allclose(a[-1], b[-1], atol=1e-5)
    assert not closed.download_open_volumes().any()


def test_the_balance_closes_while_water_enters_and_leaves() -> None:
    sc, o = oracle_channel(depth=0.5)
    q = np.float32(0.25)  # per unit width: 10 m^3/s over the 40 m section
    o.set_open_conditions(*conditions(sc, (OPEN_INFLOW, q), (OPEN_NORMAL, math.sqrt(1e-3) / 0.03)))
    area = sc.geom.area.astype(np.float64)
    v0 = float((sc.h0.astype(np.float64) * area).sum())
    o.run(t_end=60.0, output_interval_s=20.0, dt_max=1.0, dt_init=0.01)
    vol = o.download_open_volumes()
    went_in, went_out = vol[0, 1], vol[1, 0]
    assert went_in == pytest.approx(float(q) * 40.0 * 60.0, rel=1e-6)
    assert went_out > 0.0 and vol[0, 0] == 0.0 and vol[1, 1] == 0.0
    v1 = float((o.download_h_precise() * area).sum())
    assert abs(v0 + went_in - went_out - v1) / v0 < 1e-7
    assert len(o.open_volume_snapshots) == 4  # the start and every 20 s


@pytest.mark.parametrize("kind", [OPEN_FREE, OPEN_NORMAL])
def test_outflow_conditions_never_draw_water_in(kind: int) -> None:
    sc, o = oracle_channel(depth=0.5)
    hu = np.full(sc.geom.N, -0.25, np.float32)  # water running away from the outlet
    o.hu0 = hu
    o.set_open_conditions(*conditions(sc, (OPEN_WALL, 0.0), (kind, math.sqrt(1e-3) / 0.03)))
    o.run(t_end=10.0, output_interval_s=10.0, dt_max=1.0, dt_init=0.01)
    assert o.download_open_volumes()[1, 1] == 0.0


def test_a_trickle_too_thin_to_wet_a_cell_still_arrives() -> None:
    sc, o = oracle_channel()
    q = np.float32(1e-3 / 40.0)
    o.set_open_conditions(*conditions(sc, (OPEN_INFLOW, q), (OPEN_WALL, 0.0)))
    assert o.download_block_flags()[:, 2].sum() > 0  # the inflow forces its blocks
    o.run(t_end=30.0, output_interval_s=30.0, dt_max=1.0, dt_init=0.01)
    assert float(o.download_h().max()) < DRY_TOL
    assert o.download_open_volumes()[0, 1] == pytest.approx(float(q) * 40.0 * 30.0, rel=1e-6)
    v = float((o.download_h_precise() * sc.geom.area.astype(np.float64)).sum())
    assert v == pytest.approx(float(q) * 40.0 * 30.0, rel=1e-6)
