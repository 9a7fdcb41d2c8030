"""Open boundaries through the workflow on the device: the reference's
behaviour tests of ``tests/unit/test_gpu_open_boundaries.py`` on its channel
(3 km by 200 m, 300 x 20 cells, bed falling 1e-3 from 10 m, open at both ends),
with the tolerances of its resident backend (bit-identical where it asks for
atol 0)."""

from __future__ import annotations

from typing import Any

import numpy as np
import pytest

from inundation_b200.scenarios import open_channel
from inundation_b200.workflow import (
    FreeOutflow,
    Inflow,
    NormalDepth,
    OpenBoundary,
    SimulationPhase,
    Stage,
    SWEWorkflow,
    Wall,
    WorkflowConfig,
    WorkflowResult,
)

pytestmark = pytest.mark.gpu

LENGTH_M, WIDTH_M, CELLS, ACROSS = 3000.0, 200.0, 300, 20
SLOPE, MANNING, END_S = 1e-3, 0.03, 60.0
DX = LENGTH_M / CELLS


def workflow(*, open_boundaries: bool = True, initial_depth: float | np.ndarray | None = None,
             initial_velocity: float = 0.0, **config: Any) -> SWEWorkflow:
    sc = open_channel(CELLS, ACROSS, LENGTH_M, WIDTH_M, SLOPE, MANNING)
    state = None
    if initial_depth is not None:
        depth = np.broadcast_to(np.asarray(initial_depth, np.float32), (sc.geom.N,)).astype(np.float32)
        state = {"h": depth, "hu": initial_velocity * depth, "hv": np.zeros_like(depth)}
    ends = [OpenBoundary("up", [(0.0, 0.0), (0.0, WIDTH_M)], 0.25 * DX),
            OpenBoundary("down", [(LENGTH_M, 0.0), (LENGTH_M, WIDTH_M)], 0.25 * DX)]
    wf = SWEWorkflow(WorkflowConfig(mesh_source="channel", manning_n=MANNING, output_interval_s=5.0, dt_max=1.0,
                                    cfl_interval=1, progress=False, track_clamp_mass=True, initial_state_source=state,
                                    open_boundaries=ends if open_boundaries else (), **config), geometry=sc.geom)
    wf.prepare()
    return wf


def phase(up: Any, down: Any, duration_s: float = END_S) -> SimulationPhase:
    return SimulationPhase(duration_s, [], {"up": up, "down": down})


def bits(r: WorkflowResult) -> bytes:
    return r.h_final.tobytes() + b"".join(v.tobytes() for v in r.boundary_volumes_m3.values())


def channel_x(wf: SWEWorkflow) -> np.ndarray:
    return wf.geom.world_centroid[:, 0]


def test_volumes_line_up_with_the_snapshots() -> None:
    r = workflow().run([phase(Inflow(50.0, SLOPE), Wall(), 12.0), phase(Inflow(20.0, SLOPE), Wall(), 8.0)])
    v = r.boundary_volumes_m3["up"]
    assert v.shape == (len(r.snap_times), 2)
    assert (np.diff(v[:, 1]) >= 0.0).all()
    t = np.asarray(r.snap_times)
    for k in np.flatnonzero(t == 12.0):
        assert v[k, 1] == pytest.approx(50.0 * 12.0, rel=1e-6)
    assert v[-1, 1] == pytest.approx(50.0 * 12.0 + 20.0 * 8.0, rel=1e-6)


def test_a_trickle_too_thin_to_wet_a_cell_still_arrives() -> None:
    r = workflow().run([phase(Inflow(1e-3, SLOPE), Wall())])
    assert float(r.h_final.max()) < 1e-4
    assert r.boundary_volumes_m3["up"][-1, 1] == pytest.approx(1e-3 * END_S, rel=1e-6)
    assert r.volume_final_m3 == pytest.approx(1e-3 * END_S, rel=1e-6)


def test_balance_closes_while_water_enters_and_leaves() -> None:
    initial = 0.5 * LENGTH_M * WIDTH_M
    r = workflow(initial_depth=0.5).run([phase(Inflow(50.0, SLOPE), NormalDepth(SLOPE), 120.0)])
    went_in, went_out = r.boundary_volumes_m3["up"][-1, 1], r.boundary_volumes_m3["down"][-1, 0]
    assert went_out > 0.0
    assert abs(initial + went_in - went_out - r.volume_final_m3) / initial < 1e-7


@pytest.mark.parametrize("down", [FreeOutflow(), NormalDepth(SLOPE)], ids=["free", "normal"])
def test_outflow_conditions_never_draw_water_in(down: Any) -> None:
    r = workflow(initial_depth=0.5).run([phase(Wall(), down)])
    assert r.boundary_volumes_m3["down"][-1, 1] == 0.0


@pytest.mark.parametrize("down", [FreeOutflow(), NormalDepth(SLOPE)], ids=["free", "normal"])
def test_flow_running_away_from_an_outlet_draws_nothing_in(down: Any) -> None:
    r = workflow(initial_depth=0.5, initial_velocity=-0.5).run([phase(Wall(), down, 5.0)])
    assert r.boundary_volumes_m3["down"][-1, 1] == 0.0


def test_an_outlet_that_draws_nothing_in_acts_as_a_wall() -> None:
    # Water running away from the outlet faster than the normal-depth ghost leaves: the
    # edge is redone as a wall at every stage, momentum included.
    def run(down: Any) -> WorkflowResult:
        return workflow(initial_depth=0.5, initial_velocity=-2.0).run([phase(Wall(), down, 1.0)])

    closed, outlet = run(Wall()), run(NormalDepth(1e-5))
    np.testing.assert_array_equal(outlet.h_final, closed.h_final)
    np.testing.assert_array_equal(outlet.hu_final, closed.hu_final)


def test_a_dry_outflow_passes_nothing() -> None:
    r = workflow().run([phase(Wall(), FreeOutflow())])
    assert not r.boundary_volumes_m3["down"].any()
    assert not r.h_final.any()


def test_the_tally_stops_when_an_outlet_runs_dry() -> None:
    wf = workflow(initial_depth=0.0)
    depth = np.where(channel_x(wf) > LENGTH_M - DX, 1.003e-4, 0.0).astype(np.float32)
    wf = workflow(initial_depth=depth)
    initial = float(depth.astype(np.float64).sum()) * DX * WIDTH_M / ACROSS
    r = wf.run([phase(Wall(), NormalDepth(1.0), 800.0)])
    assert float(r.h_final.max()) < 1e-4
    went_out = r.boundary_volumes_m3["down"][-1, 0]
    assert went_out > 0.0
    assert abs(initial - went_out - r.volume_final_m3) / initial < 1e-5


def test_the_first_step_sees_the_water_waiting_beyond_a_stage() -> None:
    r = workflow(initial_depth=0.01).run([phase(Stage(30.0), Wall(), 1.0)])
    assert r.steps_total >= 3


def test_closing_a_stretch_releases_its_blocks() -> None:
    wf = workflow()
    wf.run([phase(Inflow(50.0, SLOPE), Wall(), 5.0)])
    assert wf.solver.download_block_flags()[:, 2].sum() > 0
    wf.run([phase(Wall(), Wall(), 5.0)])
    assert wf.solver.download_block_flags()[:, 2].sum() == 0


def test_water_entering_a_dry_mesh_is_the_same_with_skipping_off() -> None:
    on_wf = workflow()
    on = on_wf.run([phase(Stage(10.4), NormalDepth(SLOPE))])
    assert int((on_wf.solver.download_block_flags()[:, 1] == 0).sum()) > 0
    off_wf = workflow()
    off_wf.solver.active_set = False
    off = off_wf.run([phase(Stage(10.4), NormalDepth(SLOPE))])
    assert bits(on) == bits(off) and on.steps_total == off.steps_total


def test_repeat_runs_are_bit_identical() -> None:
    phases = [phase(Inflow(50.0, SLOPE), Stage(7.3))]
    assert bits(workflow().run(phases)) == bits(workflow().run(phases))


def test_a_wall_stretch_behaves_like_no_stretch() -> None:
    closed = workflow(initial_depth=0.5).run([phase(Wall(), Wall())])
    plain = workflow(open_boundaries=False, initial_depth=0.5).run([SimulationPhase(END_S, [])])
    # A wall-kind ghost mirrors through the film-safe velocities, a plain wall mirrors the momentum
    # itself: the same state up to rounding (the reference's own bound).
    np.testing.assert_allclose(closed.h_final, plain.h_final, atol=1e-5)
    assert closed.steps_total == plain.steps_total


def test_inflow_carries_momentum_into_the_mesh() -> None:
    wf = workflow(initial_depth=0.5)
    r = wf.run([phase(Inflow(200.0, SLOPE), Wall())])
    inlet = channel_x(wf) < 2.0 * LENGTH_M / CELLS
    assert float(r.hu_final[inlet].mean()) > 0.05
