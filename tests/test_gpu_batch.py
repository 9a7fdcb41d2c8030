"""Batched scenarios: every instance of a batch must reproduce its own run bit for bit.

Instances of different sizes, beds, roughness, initial states and sources
(constant rates, device-evaluated inflow hydrographs, both on one cell) run
together with their own clocks; each is checked against the FP32 oracle of
that scenario alone, and against the single-mesh solver where the reference
API can express its sources.
"""

from __future__ import annotations

import numpy as np
import pytest

from inundation_b200.scenarios import batch_member, voronoi_geometry
from inundation_b200.mesh.geometry import with_bed
from inundation_b200.sources import Hydrograph, triangular_knots
from inundation_b200.tuning import dt_to_ticks
from oracle.resident_oracle import ResidentOracle

from ._valley import DRY_TOL, DX, MANNING, cell_near, dam, point_source, sheet, valley_grid

pytestmark = pytest.mark.gpu


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def members():
    from inundation_b200.batch import BatchMember

    out = []
    g0 = valley_grid(nx=48, ny=21)  # 1008 cells: a partial last block
    z0 = np.zeros(g0.N, np.float32)
    out.append((BatchMember(g0, dam(g0, 48, 21), z0, z0, np.full(g0.N, MANNING, np.float32)), 40.0))
    g1 = valley_grid(nx=64, ny=32)
    z1 = np.zeros(g1.N, np.float32)
    kt, kq = triangular_knots(0.6, 20.0, 45.0)
    inflow = Hydrograph(cells=np.array([cell_near(g1, 64 * DX * 0.5, 32 * DX * 0.5), cell_near(g1, 10.0, 10.0)]),
                        knot_t=kt, knot_q=kq, share=np.array([0.75, 0.25], np.float32))
    rain = np.where(np.arange(g1.N) % 7 == 0, 0.004, 0.0).astype(np.float32)
    rain[inflow.cells[0]] = 0.01  # a cell with both a constant rate and a hydrograph
    out.append((BatchMember(g1, sheet(g1, 64), z1, z1, np.full(g1.N, 0.02, np.float32), source_rate=rain,
                            hydrographs=[inflow]), 60.0))
    g2 = voronoi_geometry(3000, 300.0, 5)
    zb = (0.01 * g2.world_centroid[:, 0]).astype(np.float32)
    g2 = with_bed(g2, zb)
    rng = np.random.default_rng(5)
    n2 = rng.uniform(0.02, 0.06, g2.N).astype(np.float32)
    z2 = np.zeros(g2.N, np.float32)
    out.append((BatchMember(g2, np.where(g2.world_centroid[:, 0] < 80.0, 0.5, 0.0).astype(np.float32), z2, z2, n2,
                            source_rate=point_source(g2, 0.2, 150.0, 150.0)), 25.0))
    return out


def oracle_of(m, t_end: float, interval: float):
    o = ResidentOracle(m.geom, m.h0, m.hu0, m.hv0, m.n0, dry_tol=DRY_TOL, steps_per_graph=50)
    snaps, times = o.run(t_end=t_end, output_interval_s=interval, dt_max=1.0, dt_init=0.01,
                         source_rate=m.source_rate, hydrographs=m.hydrographs)
    return o, snaps, times


@pytest.fixture(scope="module")
def batch_case():
    from inundation_b200.batch import BatchedSolver

    ms = members()
    solver = BatchedSolver([m for m, _ in ms], dry_tol=DRY_TOL)
    solver.steps_per_graph = 50
    return solver, ms


@pytest.mark.parametrize("kernel", ["tiled", "plain", "staged", "persistent"])
def test_every_instance_matches_its_own_oracle_run(kernel: str, batch_case) -> None:
    solver, ms = batch_case
    solver.stage_kernel = kernel
    interval = 10.0
    ends = [t for _, t in ms]
    res = solver.run(ends, dt_max=1.0, dt_init=0.01, output_interval_s=interval)
    for i, (m, t_end) in enumerate(ms):
        o, snaps, times = oracle_of(m, t_end, interval)
        assert int(res.steps[i]) == o.steps_total > 10
        k = len(times) - 1
        for w in range(1, k + 1):
            np.testing.assert_array_equal(bits(res.snapshots[i][w]), bits(snaps[w]), err_msg=f"instance {i} window {w}")
        np.testing.assert_array_equal(bits(solver.download_h(i)), bits(o.download_h()))
        np.testing.assert_array_equal(bits(solver.download_hu(i)), bits(o.download_hu()))
        np.testing.assert_array_equal(bits(solver.download_hv(i)), bits(o.download_hv()))
        np.testing.assert_array_equal(bits(solver.download_h_residual(i)), bits(o.download_h_residual()))
        assert float(solver.sim_time[i]) == t_end


def test_batch_instance_matches_the_single_mesh_solver(batch_case) -> None:
    from inundation_b200.backend import SWESolverB200Resident

    solver, ms = batch_case
    solver.stage_kernel = "tiled"
    ends = [t for _, t in ms]
    solver.run(ends, dt_max=1.0, dt_init=0.01, output_interval_s=10.0)
    for i in (0, 2):  # sources the reference API can express
        m, t_end = ms[i]
        single = SWESolverB200Resident(m.geom, None, m.h0, m.hu0, m.hv0, m.n0, dry_tol=DRY_TOL)
        single.steps_per_graph = 50
        single.run(t_end=t_end, output_interval_s=10.0, dt_max=1.0, dt_init=0.01, cfl_interval=1, progress=False,
                   source_rate=m.source_rate)
        assert single.steps_total == int(solver.steps[i])
        np.testing.assert_array_equal(bits(single.download_h()), bits(solver.download_h(i)))
        np.testing.assert_array_equal(bits(single.download_hu()), bits(solver.download_hu(i)))


def test_hydrograph_volume_is_the_integral_of_its_discharge() -> None:
    """A walled flat basin fed by one hydrograph: the FP64 volume equals sum(dt * q(t_step))."""
    from inundation_b200.batch import BatchedSolver, BatchMember

    g = valley_grid(nx=32, ny=32)
    g = with_bed(g, np.zeros(g.N, np.float32))
    z = np.zeros(g.N, np.float32)
    kt = np.array([0.0, 5.0, 12.0, 20.0], np.float32)
    kq = np.array([0.0, 0.4, 0.1, 0.3], np.float32)
    cell = cell_near(g, 32.0, 32.0)
    hg = Hydrograph(cells=np.array([cell]), knot_t=kt, knot_q=kq)
    solver = BatchedSolver([BatchMember(g, np.full(g.N, 0.05, np.float32), z, z, np.full(g.N, MANNING, np.float32),
                                        hydrographs=[hg])], dry_tol=DRY_TOL)
    v0 = solver.volume_fp64(0)
    solver.run(25.0, dt_max=0.25, dt_init=0.01)
    gained = solver.volume_fp64(0) - v0
    exact = float(np.trapezoid(np.append(kq, kq[-1]), np.append(kt, 25.0)))
    # left-point sampling of a piecewise-linear discharge over steps <= 0.25 s
    assert gained == pytest.approx(exact, rel=0.02)
    o = ResidentOracle(g, solver.members[0].h0, z, z, solver.members[0].n0, dry_tol=DRY_TOL)
    o.run(t_end=25.0, output_interval_s=25.0, dt_max=0.25, dt_init=0.01, hydrographs=[hg])
    np.testing.assert_array_equal(bits(solver.download_h(0)), bits(o.download_h()))


def test_fixed_step_runs_and_autotuner_keep_results() -> None:
    from inundation_b200.batch import BatchedSolver, BatchMember, autotune

    scs = [batch_member(n, seed) for n, seed in ((6000, 21), (2500, 22), (9000, 23))]
    ms = [BatchMember(s.geom, s.h0, s.hu0, s.hv0, s.manning, hydrographs=s.hydrographs) for s in scs]
    for m in ms:  # start with some water so the active sets are not trivial
        m.h0 = np.where(np.arange(m.geom.N) < m.geom.N // 5, 0.3, 0.0).astype(np.float32)
    solver = BatchedSolver(ms)
    choice = autotune(solver, dt_max=1.0, dt_init=0.01, steps=20)
    assert {r["stage_kernel"] for r in choice["results"]} == {"tiled", "plain", "staged", "persistent"}
    assert solver.stage_kernel == choice["stage_kernel"]
    outs = []
    for kernel in ("tiled", "plain", "staged", "persistent"):
        solver.stage_kernel = kernel
        solver.reset()
        solver.start(dt_max=1.0, dt_init=0.01)
        solver.steps_per_graph = 40
        solver.run_steps(100)
        assert (solver.steps == 100).all()
        outs.append([solver.download_h(i) for i in range(3)])
    for other in outs[1:]:
        for a, b in zip(outs[0], other, strict=True):
            np.testing.assert_array_equal(bits(a), bits(b))
    for i, s in enumerate(scs):
        o = ResidentOracle(s.geom, ms[i].h0, s.hu0, s.hv0, s.manning, steps_per_graph=100)
        o.set_sources(None, s.hydrographs)
        o.ctrl["stop_ticks"] = 1 << 62
        o.ctrl["dt_max_ticks"] = 1 << 20
        o.ctrl["dry_dt_ticks"] = dt_to_ticks(0.01)
        o.ctrl["cfl_safety"] = 1.0
        o.prologue()
        for _ in range(100):
            o.step()
        np.testing.assert_array_equal(bits(outs[0][i]), bits(o.download_h()))
