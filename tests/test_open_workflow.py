"""Open boundaries at the workflow level, on the CPU: which edges a stretch
selects, how an inflow splits, what the configuration refuses, and the
per-edge conditions a phase hands to the solver (the cases of the reference's
``tests/unit/test_open_boundaries.py``)."""

from __future__ import annotations

from typing import Any

import numpy as np
import pytest

from inundation_b200.mesh.boundaries import (
    boundary_edge_midpoints,
    conveyance_split,
    distance_to_line,
    select_boundary_edges,
)
from inundation_b200.mesh.geometry import build_geometry, hilbert_reorder
from inundation_b200.workflow import (
    FreeOutflow,
    Inflow,
    NormalDepth,
    OpenBoundary,
    PointSource,
    SimulationPhase,
    Stage,
    Wall,
    WorkflowConfig,
    WorkflowResult,
    build_phase_open_conditions,
    inflow_phases,
    open_stretch_edges,
)

UTM = (512_345.5, 5_512_345.25)
NX, NY, DX = 6, 4, 2.0


def grid(offset=UTM):
    x, y = np.meshgrid(np.arange(NX + 1.0), np.arange(NY + 1.0))
    verts = DX * np.column_stack([x.ravel(), y.ravel()]) + offset
    a = (np.arange(NY)[:, None] * (NX + 1) + np.arange(NX)).ravel()
    faces = np.column_stack([a, a + 1, a + NX + 2, a + NX + 1]).astype(np.int32)
    zb = np.arange(NX * NY, dtype=np.float32) * 0.1
    return hilbert_reorder(build_geometry(verts, faces, zb_from_file=zb), verbose=False)[0]


def east_line():
    x = UTM[0] + NX * DX
    return [(x, UTM[1]), (x, UTM[1] + NY * DX)]


def config(**overrides: Any) -> WorkflowConfig:
    base: dict[str, Any] = {"mesh_source": "unused.obj", "manning_n": 0.03, "output_interval_s": 1.0, "dt_max": 0.1,
                            "cfl_interval": 1}
    return WorkflowConfig(**{**base, **overrides})


def test_a_line_in_world_coordinates_selects_its_edges() -> None:
    g = grid()
    edges = select_boundary_edges(g, east_line(), 0.5)
    assert edges.size == NY
    assert (g.edge_cellR[edges] == -1).all()
    assert (g.edge_len[edges] == DX).all()
    east = g.centroid[g.edge_cellL[edges], 0]
    assert (east == east.max()).all()


def test_a_line_follows_each_of_its_segments() -> None:
    g = grid()
    x, y = UTM[0] + NX * DX, UTM[1] + NY * DX
    assert select_boundary_edges(g, [(x, UTM[1]), (x, y), (UTM[0], y)], 0.5).size == NX + NY


def test_a_line_away_from_the_rim_selects_nothing() -> None:
    x = UTM[0] + 0.5 * NX * DX
    assert select_boundary_edges(grid(), [(x, UTM[1] + 1.0), (x, UTM[1] + 3.0)], 0.5).size == 0


def test_a_stretch_needs_two_points() -> None:
    with pytest.raises(ValueError, match="at least 2 points"):
        select_boundary_edges(grid(), [(0.0, 0.0)], 1.0)


def test_boundary_normals_point_out_of_the_mesh() -> None:
    g = grid()
    edges, mid = boundary_edge_midpoints(g)
    out = mid - g.centroid[g.edge_cellL[edges]].astype(np.float64)
    assert (out[:, 0] * g.edge_nx[edges] + out[:, 1] * g.edge_ny[edges] > 0.0).all()


def test_distance_to_line_stops_at_the_segment_end() -> None:
    line = np.array([[0.0, 0.0], [10.0, 0.0]])
    pts = np.array([[5.0, 3.0], [14.0, 3.0], [-3.0, -4.0]])
    np.testing.assert_allclose(distance_to_line(pts, line), [3.0, 5.0, 5.0])


def section():
    return (np.array([5.0, 4.0, 6.0, 3.0], np.float32), np.array([12.0, 10.0, 10.5, 30.0], np.float32),
            np.array([0.03, 0.04, 0.03, 0.03], np.float32))


def test_inflow_splits_to_exactly_the_discharge() -> None:
    lengths, beds, n = section()
    q = conveyance_split(7.3, lengths, beds, n, 1e-3)
    assert float((q.astype(np.float64) * lengths.astype(np.float64)).sum()) == pytest.approx(7.3, rel=2e-7)


def test_inflow_enters_along_the_low_part_of_the_section() -> None:
    q = conveyance_split(7.3, *section(), 1e-3)
    assert q[3] == 0.0 and q[1] > 0.0 and q[2] > 0.0


def test_inflow_follows_manning_on_a_flat_section() -> None:
    q = conveyance_split(6.0, np.full(3, 2.0, np.float32), np.full(3, 5.0, np.float32),
                         np.array([0.02, 0.04, 0.08], np.float32), 1e-3).astype(np.float64)
    np.testing.assert_allclose(q[0] / q, [1.0, 2.0, 4.0], rtol=1e-5)


def test_no_inflow_splits_to_zero() -> None:
    assert not conveyance_split(0.0, *section(), 1e-3).any()


@pytest.mark.parametrize("backend", ["fixed_dt_batch_barrier"])
def test_other_backends_refuse_open_boundaries(backend: str) -> None:
    with pytest.raises(ValueError, match=rf"open_boundaries.*{backend}"):
        config(solver_impl=backend, open_boundaries=[OpenBoundary("a", east_line(), 1.0)])


def test_the_b200_backend_takes_open_boundaries() -> None:
    config(open_boundaries=[OpenBoundary("a", east_line(), 1.0)])


def test_open_boundaries_need_deterministic_accumulation() -> None:
    with pytest.raises(ValueError, match="deterministic"):
        config(deterministic=False, open_boundaries=[OpenBoundary("a", east_line(), 1.0)])


def test_stretch_names_must_differ() -> None:
    with pytest.raises(ValueError, match="names repeat"):
        config(open_boundaries=[OpenBoundary("a", east_line(), 1.0), OpenBoundary("a", east_line(), 1.0)])


def test_a_stretch_selecting_nothing_raises() -> None:
    with pytest.raises(ValueError, match="'lost' selects no boundary edges"):
        open_stretch_edges(grid(), [OpenBoundary("lost", [(0.0, 0.0), (1.0, 0.0)], 1.0)])


def test_an_edge_selected_twice_raises() -> None:
    with pytest.raises(ValueError, match="same edge twice"):
        open_stretch_edges(grid(), [OpenBoundary("a", east_line(), 1.0), OpenBoundary("b", east_line(), 1.0)])


def conditions(**boundaries: Any):
    g = grid()
    stretch = OpenBoundary("a", east_line(), 1.0)
    edges = open_stretch_edges(g, [stretch])
    return build_phase_open_conditions(g, np.full(g.N, 0.04, np.float32), [stretch], edges,
                                       SimulationPhase(1.0, [], boundaries))


def test_a_phase_must_set_every_stretch() -> None:
    with pytest.raises(ValueError, match="must name every open boundary"):
        conditions()


def test_a_phase_must_not_name_an_unknown_stretch() -> None:
    with pytest.raises(ValueError, match="must name every open boundary"):
        conditions(a=Wall(), b=Wall())


@pytest.mark.parametrize("condition", [NormalDepth(0.0), Inflow(1.0, 0.0), Inflow(-1.0, 1e-3), Stage(float("nan")),
                                       NormalDepth(float("inf")), Inflow(float("nan"), 1e-3)])
def test_bad_condition_values_raise(condition: Any) -> None:
    with pytest.raises(ValueError, match="open boundary 'a'"):
        conditions(a=condition)


def test_condition_values_reach_the_kernels() -> None:
    kinds, values = conditions(a=NormalDepth(1e-2))
    assert (kinds == 2).all()
    np.testing.assert_allclose(values, 0.1 / 0.04)
    assert (conditions(a=FreeOutflow())[0] == 1).all()
    assert (conditions(a=Wall())[0] == 0).all()
    kinds, values = conditions(a=Inflow(3.0, 1e-3))
    assert (kinds == 4).all() and float((values.astype(np.float64) * DX).sum()) == pytest.approx(3.0, rel=2e-7)


def test_a_stage_gives_depth_over_each_cell_bed_and_never_below_it() -> None:
    g = grid()
    cells = g.edge_cellL[select_boundary_edges(g, east_line(), 1.0)]
    level = float(g.zb[cells].mean())
    values = conditions(a=Stage(level))[1]
    np.testing.assert_allclose(values, np.maximum(level - g.zb[cells].astype(np.float64), 0.0), atol=1e-6)
    assert (values == 0.0).any()


def upstream() -> WorkflowResult:
    times = [0.0, 5.0, 10.0, 10.0, 15.0, 20.0, 20.0, 25.0, 30.0]  # three 10 s phases, each repeating its start
    volumes = np.zeros((len(times), 2))
    volumes[:, 0] = [0.0, 10.0, 30.0, 30.0, 30.0, 40.0, 40.0, 40.0, 100.0]
    empty = np.zeros(1, np.float32)
    return WorkflowResult(snapshots=[], snap_times=times, h_final=empty, volume_final_m3=0.0, volume_injected_m3=0.0,
                          wall_seconds=0.0, steps_total=0, boundary_volumes_m3={"outlet": volumes})


def test_inflow_phases_pass_the_volume_of_every_window() -> None:
    phases = inflow_phases(upstream(), "outlet", "from_a", 1e-3)
    assert [p.duration_s for p in phases] == [5.0] * 6
    rates = [p.boundaries["from_a"].discharge_m3s for p in phases]
    assert rates == [2.0, 4.0, 0.0, 2.0, 0.0, 12.0]
    assert sum(q * p.duration_s for q, p in zip(rates, phases, strict=True)) == 100.0


def test_inflow_phases_carry_the_rest_of_the_downstream_run() -> None:
    source = PointSource(1.0, (0.0, 0.0), 1.0)
    phases = inflow_phases(upstream(), "outlet", "from_a", 1e-3, {"down": FreeOutflow()}, [source])
    assert set(phases[0].boundaries) == {"from_a", "down"}
    assert phases[0].sources == [source]
