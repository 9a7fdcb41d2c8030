"""Behaviour of the B200 resident backend, restating the reference's GPU tests.

* determinism and stale-state poisoning (``tests/unit/test_gpu_deterministic.py``),
* active set on vs off and its flags (``tests/unit/test_gpu_active_set.py``),
* compensated depth: closed-domain volume, sub-ulp sources, walls, film drag,
  pair invariants (``tests/unit/test_gpu_compensated.py``),
* integer clock, injected volume, output times, submit size
  (``tests/unit/test_gpu_resident_clock.py:217-372``),
* a long adaptive run with sources, bit for bit against the FP32 oracle,
* the workflow API end to end.
"""

from __future__ import annotations

import numpy as np
import pytest

from inundation_b200.mesh.geometry import build_geometry
from inundation_b200.mesh.synthetic import quad_grid
from oracle.resident_oracle import ResidentOracle

from ._valley import DRY_TOL, DX, MANNING, NX, NY, dam, point_source, run, sheet, state, valley_grid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grid():
    return valley_grid()


def make(grid, h0, hu0=None, hv0=None, *, dry_tol=None, n=MANNING, **attrs):
    from inundation_b200.backend import SWESolverB200Resident

    z = np.zeros(grid.N, np.float32)
    kw = {} if dry_tol is None else {"dry_tol": dry_tol}
    solver = SWESolverB200Resident(
        grid, None, h0, z if hu0 is None else hu0, z if hv0 is None else hv0, np.full(grid.N, n, np.float32), **kw
    )
    for k, v in attrs.items():
        setattr(solver, k, v)
    return solver


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def assert_identical(a, b, snaps_a, snaps_b) -> None:
    assert a.steps_total == b.steps_total
    for x, y in zip([*snaps_a, *state(a)], [*snaps_b, *state(b)], strict=True):
        np.testing.assert_array_equal(bits(x), bits(y))


def cases(grid):
    dry = np.zeros(grid.N, np.float32)
    return {
        "wetting": (dry, point_source(grid, 1.0, NX * DX * 0.2, NY * DX / 2), 200.0),
        "dam_break": (dam(grid), None, 60.0),
        "draining": (sheet(grid), None, 300.0),
    }


# -- determinism ---------------------------------------------------------------------------------
@pytest.mark.parametrize("case", ["wetting", "dam_break", "draining"])
def test_repeat_runs_are_bit_identical(case: str, grid) -> None:
    h0, src, t_end = cases(grid)[case]
    a, b = make(grid, h0), make(grid, h0)
    assert_identical(a, b, run(a, t_end, source_rate=src), run(b, t_end, source_rate=src))


@pytest.mark.parametrize("kernel", ["tiled", "plain", "staged", "persistent"])
@pytest.mark.parametrize("fill", [0.5, float("nan")], ids=["wet", "nan"])
def test_stale_predictor_state_is_never_read(kernel: str, fill: float, grid) -> None:
    h0 = dam(grid)
    clean, poisoned = make(grid, h0, stage_kernel=kernel), make(grid, h0, stage_kernel=kernel)
    garbage = np.full(grid.N, fill, np.float32)  # wet garbage, or NaN that any read would carry into the state
    for name in ("h1", "hu1", "hv1"):
        poisoned.upload(name, garbage)
    assert_identical(clean, poisoned, run(clean, 30.0), run(poisoned, 30.0))


@pytest.mark.parametrize("other", ["plain", "staged", "persistent"])
def test_stage_kernels_agree_bit_for_bit(other: str, grid) -> None:
    h0, src, t_end = cases(grid)["wetting"]
    a, b = make(grid, h0, stage_kernel="tiled"), make(grid, h0, stage_kernel=other)
    assert_identical(a, b, run(a, t_end, source_rate=src), run(b, t_end, source_rate=src))


@pytest.mark.parametrize("case", ["wetting", "dam_break", "draining"])
@pytest.mark.parametrize("ctas", [3, 5])
def test_persistent_kernel_on_a_few_ctas_agrees_bit_for_bit(case: str, ctas: int, grid) -> None:
    """The 32 tiles of the valley on 3 or 5 CTAs: each CTA computes its seat, keeps one other tile
    from step to step and takes the rest from the queue, while tiles wet, dry and change hands."""
    h0, src, t_end = cases(grid)[case]
    a = make(grid, h0, stage_kernel="tiled")
    b = make(grid, h0, stage_kernel="persistent", max_grid=ctas)
    assert b.grid(2) == ctas
    assert_identical(a, b, run(a, t_end, source_rate=src), run(b, t_end, source_rate=src))


# -- active set ---------------------------------------------------------------------------------------
def same_on_off(on, off, snaps_on, snaps_off) -> None:
    assert on.steps_total == off.steps_total and len(snaps_on) == len(snaps_off)
    for x, y in zip([*snaps_on, *state(on)], [*snaps_off, *state(off)], strict=True):
        np.testing.assert_array_equal(x, y)  # exact; -0.0 and +0.0 compare equal


def active_fraction(solver) -> float:
    return float(solver.download_block_flags()[:, 1].mean())


@pytest.mark.parametrize("case", ["wetting", "dam_break", "draining"])
def test_active_set_on_and_off_agree_exactly(case: str, grid) -> None:
    h0, src, t_end = cases(grid)[case]
    on, off = make(grid, h0, active_set=True), make(grid, h0, active_set=False)
    same_on_off(on, off, run(on, t_end, source_rate=src), run(off, t_end, source_rate=src))
    if case == "wetting":
        assert active_fraction(on) < 0.6 and active_fraction(off) == 1.0


def test_chained_runs_with_changing_sources(grid) -> None:
    z = np.zeros(grid.N, np.float32)
    near = point_source(grid, 0.5, NX * DX * 0.2, NY * DX / 2)
    far = point_source(grid, 0.3, NX * DX * 0.9, NY * DX * 0.8) + near
    solvers = [make(grid, z, active_set=True), make(grid, z, active_set=False)]
    for solver in solvers:
        t = 0.0
        for t_end, src in ((100.0, near), (200.0, far), (260.0, np.zeros(grid.N, np.float32))):
            solver.run(t_end=t_end, output_interval_s=50.0, dt_max=1.0, dt_init=0.01, cfl_interval=10, progress=False,
                       source_rate=src, resume=t > 0.0, t_start=t)
            t = t_end
    same_on_off(*solvers, [], [])


def test_dry_cells_with_momentum_are_cleared_not_frozen(grid) -> None:
    far = grid.centroid[:, 0] > NX * DX * 0.8
    hu0 = np.where(far, 0.1, 0.0).astype(np.float32)
    on = make(grid, dam(grid), hu0, -hu0, active_set=True)
    off = make(grid, dam(grid), hu0, -hu0, active_set=False)
    run(on, 2.0)
    run(off, 2.0)
    assert on.steps_total > 3
    same_on_off(on, off, [], [])
    assert float(np.abs(on.download_hu()[far]).max()) == 0.0


def test_flags_follow_the_water(grid) -> None:
    solver = make(grid, dam(grid), active_set=True)
    run(solver, 30.0)
    h, hu, hv = state(solver)
    live = (h >= DRY_TOL) | (hu != 0.0) | (hv != 0.0)
    flags = solver.download_block_flags()
    assert flags[np.unique(np.flatnonzero(live) // 256), 1].all()
    assert flags[:, 1].sum() < flags.shape[0]
    z = np.zeros(grid.N, np.float32)
    hu0 = np.where(grid.centroid[:, 0] > NX * DX * 0.8, 0.1, 0.0).astype(np.float32)
    moving = make(grid, z, hu0, z)
    run(moving, 3.0)
    assert moving.steps_total > 200 and float(np.abs(moving.download_hu()).max()) == 0.0
    assert active_fraction(moving) == 0.0
    dry = make(grid, z)
    run(dry, 5.0)
    assert active_fraction(dry) == 0.0 and float(dry.download_h().max()) == 0.0


def test_source_in_a_dry_inactive_region_injects_its_volume(grid) -> None:
    solver = make(grid, np.zeros(grid.N, np.float32), active_set=True)
    run(solver, 50.0, source_rate=point_source(grid, 0.2, NX * DX * 0.9, NY * DX * 0.1))
    assert solver.volume_fp64() == pytest.approx(0.2 * 50.0, rel=1e-4)


def test_rejects_bad_arguments(grid) -> None:
    with pytest.raises(ValueError, match="workgroup_size"):
        from inundation_b200.backend import SWESolverB200Resident

        z = np.zeros(grid.N, np.float32)
        SWESolverB200Resident(grid, None, z, z, z, z + 0.03, workgroup_size=128)
    solver = make(grid, np.zeros(grid.N, np.float32))
    with pytest.raises(ValueError, match="source_fn"):
        run(solver, 1.0, source_fn=lambda _t: None)
    with pytest.raises(ValueError, match="dt"):
        solver.run(t_end=1.0, output_interval_s=1.0, dt_max=32.0, dt_init=0.01, cfl_interval=1, progress=False)
    solver.deterministic = False
    with pytest.raises(ValueError, match="deterministic"):
        run(solver, 1.0)


# -- compensated depth ------------------------------------------------------------------------------------
def volume_error(solver, grid, h0, src, t_end) -> float:
    area = grid.area.astype(np.float64)
    v0 = float((h0.astype(np.float64) * area).sum())
    v1 = float((solver.download_h_precise() * area).sum())
    clamp = float(solver.download_clamp_mass().astype(np.float64).sum())
    injected = 0.0 if src is None else float(src.astype(np.float64).sum()) * t_end
    return (v1 - v0 - injected - clamp) / v1


def comp_cases(grid):
    return {
        "dam_break": (dam(grid), None, 600.0),
        "draining": (sheet(grid), None, 600.0),
        "wetting": (np.zeros(grid.N, np.float32), point_source(grid, 1.0, NX * DX * 0.2, NY * DX / 2), 600.0),
    }


@pytest.mark.parametrize("case", ["dam_break", "draining", "wetting"])
def test_volume_change_is_exactly_the_clamp_and_the_sources(case: str, grid) -> None:
    h0, src, t_end = comp_cases(grid)[case]
    solver = make(grid, h0, dry_tol=DRY_TOL, compensated=True, track_clamp=True)
    run(solver, t_end, source_rate=src)
    assert solver.steps_total > 1000
    assert abs(volume_error(solver, grid, h0, src, t_end)) < 3e-9


@pytest.mark.parametrize("case", ["dam_break", "wetting"])
def test_the_plain_update_drifts(case: str, grid) -> None:
    h0, src, t_end = comp_cases(grid)[case]
    solver = make(grid, h0, dry_tol=DRY_TOL, compensated=False, track_clamp=True)
    run(solver, t_end, source_rate=src)
    assert abs(volume_error(solver, grid, h0, src, t_end)) > 3e-8


def basin(n: int = 24):
    q = quad_grid(n, n, 1.0)
    return build_geometry(q.verts, q.faces.reshape(-1, 4), zb_from_file=np.zeros(n * n, np.float32))


def test_a_source_below_half_an_ulp_is_kept_in_the_low_word() -> None:
    g = basin()
    src = np.zeros(g.N, np.float32)
    src[g.N // 2 + 12] = 1e-7
    solver = make(g, np.ones(g.N, np.float32))
    solver.run(t_end=0.5, output_interval_s=0.5, dt_max=0.05, dt_init=0.05, cfl_interval=1, progress=False,
               source_rate=src)
    np.testing.assert_array_equal(solver.download_h(), np.ones(g.N, np.float32))
    gained = float(((solver.download_h_precise() - 1.0) * g.area.astype(np.float64)).sum())
    assert gained == pytest.approx(1e-7 * 0.5, rel=1e-3)


def triangle():
    verts = np.array([[0.0, 0.0], [7.3, 1.1], [2.9, 6.7]], dtype=np.float32)
    return build_geometry(verts, np.array([[0, 1, 2]], np.int32), zb_from_file=np.zeros(1, np.float32))


def test_a_closed_cell_keeps_its_depth_bit_for_bit() -> None:
    g = triangle()
    h0 = np.array([0.3137], np.float32)
    solver = make(g, h0, np.array([0.0917], np.float32), np.array([-0.0531], np.float32))
    solver.run(t_end=2.0, output_interval_s=2.0, dt_max=0.01, dt_init=0.01, cfl_interval=1, progress=False)
    assert solver.steps_total > 100
    np.testing.assert_array_equal(solver.download_h_precise(), h0.astype(np.float64))


def test_film_damping_does_not_depend_on_the_tick_size() -> None:
    def decayed(dt: float) -> float:
        g = triangle()
        solver = make(g, np.array([2e-4], np.float32), np.array([2e-5], np.float32), np.zeros(1, np.float32), n=1e-4)
        solver.run(t_end=2.0**-8, output_interval_s=2.0**-8, dt_max=dt, dt_init=dt, cfl_interval=1, progress=False)
        return float(solver.download_hu()[0])

    coarse, fine = decayed(2.0**-10), decayed(2.0**-12)
    assert 0.0 < fine < 2e-5 and coarse == pytest.approx(fine, rel=0.15)


def test_pair_invariants_and_reset(grid) -> None:
    solver = make(grid, dam(grid), dry_tol=DRY_TOL, compensated=True)
    run(solver, 60.0)
    h, lo = solver.download_h(), solver.download_h_residual()
    assert (np.abs(lo) <= np.spacing(np.abs(h)) / 2).all() and np.count_nonzero(lo) > 0
    np.testing.assert_array_equal((h.astype(np.float64) + lo).astype(np.float32), h)
    solver._reset_to_initial()
    assert np.count_nonzero(solver.download_h_residual()) == 0
    drained = make(grid, sheet(grid), dry_tol=DRY_TOL)
    run(drained, 300.0)
    h, lo = drained.download_h(), drained.download_h_residual()
    assert (lo[h == 0.0] == 0.0).all() and (h.astype(np.float64) + lo >= 0.0).all()
    plain = make(grid, dam(grid), compensated=False)
    run(plain, 20.0, source_rate=point_source(grid, 1.0, NX * DX * 0.2, NY * DX / 2))
    assert np.count_nonzero(plain.download_h_residual()) == 0


def test_point_source_into_a_dry_cell_creates_no_clamp_mass(grid) -> None:
    solver = make(grid, np.zeros(grid.N, np.float32), dry_tol=DRY_TOL, track_clamp=True)
    solver.run(t_end=20.0, output_interval_s=20.0, dt_max=1.0, dt_init=0.01, cfl_interval=1, progress=False,
               source_rate=point_source(grid, 2.0, NX * DX * 0.2, NY * DX / 2))
    assert float(solver.download_clamp_mass().astype(np.float64).sum()) == 0.0


# -- clock ----------------------------------------------------------------------------------------------------
def hump(g):
    cx, cy = g.centroid[:, 0], g.centroid[:, 1]
    return (0.5 + 0.2 * np.exp(-((cx - 12.0) ** 2 + (cy - 12.0) ** 2) / 10.0)).astype(np.float32)


def crun(solver, **kw):
    base = {"output_interval_s": 10.0, "dt_max": 1.0, "dt_init": 0.01, "cfl_interval": 10, "progress": False}
    return solver.run(**{**base, **kw})


@pytest.mark.parametrize("t0", [0.0, 70_000.0])
def test_injected_volume_matches_the_schedule_at_any_start_time(t0: float) -> None:
    g = basin()
    src = np.zeros(g.N, np.float32)
    src[g.N // 2 + 12] = 1.0
    solver = make(g, np.full(g.N, 0.05, np.float32))
    v0 = solver.volume_fp64()
    crun(solver, t_end=t0 + 30.0, source_rate=src, resume=True, t_start=t0)
    assert solver.volume_fp64() - v0 == pytest.approx(30.0, rel=1e-4)


def test_chained_phases_and_dry_start() -> None:
    g = basin()
    src = np.zeros(g.N, np.float32)
    src[g.N // 2 + 12] = 1.0
    solver = make(g, np.full(g.N, 0.05, np.float32))
    v0 = solver.volume_fp64()
    crun(solver, t_end=20.0, source_rate=0.5 * src)
    crun(solver, t_end=50.0, source_rate=1.5 * src, resume=True, t_start=20.0)
    assert solver.volume_fp64() - v0 == pytest.approx(0.5 * 20.0 + 1.5 * 30.0, rel=1e-4)
    dry = make(g, np.zeros(g.N, np.float32))
    crun(dry, t_end=10.0, source_rate=0.2 * src)
    assert dry.volume_fp64() == pytest.approx(2.0, rel=1e-4)


def test_outputs_land_exactly_on_their_times() -> None:
    g = basin()
    _, times = crun(make(g, hump(g)), t_end=10.0, output_interval_s=2.5)
    assert times == [0.0, 2.5, 5.0, 7.5, 10.0]
    solver = make(g, hump(g))
    crun(solver, t_end=3.0)
    _, times = crun(solver, t_end=8.0, output_interval_s=2.0, resume=True, t_start=3.0)
    assert times == [3.0, 5.0, 7.0, 8.0]


@pytest.mark.parametrize("steps_per_graph", [1, 7, 500])
def test_submit_size_changes_nothing(steps_per_graph: int) -> None:
    g = basin()
    ref, cand = make(g, hump(g)), make(g, hump(g), steps_per_graph=steps_per_graph)
    crun(ref, t_end=5.0, output_interval_s=1.0)
    crun(cand, t_end=5.0, output_interval_s=1.0)
    assert ref.steps_total == cand.steps_total > 0
    np.testing.assert_array_equal(bits(ref.download_h()), bits(cand.download_h()))


def test_closed_basin_conserves_volume() -> None:
    g = basin()
    solver = make(g, hump(g))
    v0 = solver.volume_fp64()
    crun(solver, t_end=20.0)
    assert solver.volume_fp64() == pytest.approx(v0, rel=1e-6)
    host = float((solver.download_h_precise() * g.area.astype(np.float64)).sum())
    assert solver.volume_fp64() == pytest.approx(host, rel=1e-12)


# -- long adaptive run against the FP32 oracle ---------------------------------------------------------------
@pytest.mark.parametrize("kernel", ["tiled", "plain", "staged", "persistent"])
def test_adaptive_run_with_sources_matches_the_fp32_oracle(kernel: str) -> None:
    g = valley_grid(nx=64, ny=32)
    h0 = sheet(g, nx=64)
    src = point_source(g, 0.4, 64 * DX * 0.6, 32 * DX / 2) + point_source(g, 0.1, 64 * DX * 0.9, 32 * DX * 0.2)
    solver = make(g, h0, dry_tol=DRY_TOL, stage_kernel=kernel, steps_per_graph=37)
    oracle = ResidentOracle(g, h0, np.zeros(g.N, np.float32), np.zeros(g.N, np.float32),
                            np.full(g.N, MANNING, np.float32), dry_tol=DRY_TOL, steps_per_graph=37)
    kw = {"t_end": 60.0, "output_interval_s": 15.0, "dt_max": 1.0, "dt_init": 0.01, "cfl_interval": 1,
          "source_rate": src}
    snaps_s, times_s = solver.run(progress=False, **kw)
    snaps_o, times_o = oracle.run(**kw)
    assert solver.steps_total == oracle.steps_total > 100
    assert times_s == times_o
    for a, b in zip(snaps_s, snaps_o, strict=True):
        np.testing.assert_array_equal(bits(a), bits(b))
    for a, b in zip((solver.download_hu(), solver.download_hv(), solver.download_h_residual()),
                    (oracle.download_hu(), oracle.download_hv(), oracle.download_h_residual()), strict=True):
        np.testing.assert_array_equal(bits(a), bits(b))
    np.testing.assert_array_equal(solver.download_block_flags(), oracle.download_block_flags())


# -- workflow ------------------------------------------------------------------------------------------------
def test_workflow_runs_phases_end_to_end() -> None:
    """Two phases through the public API, bit for bit against the FP32 oracle run through the same phases."""
    from inundation_b200.workflow import PointSource, SimulationPhase, SWEWorkflow, WorkflowConfig, build_phase_source_rate

    g = valley_grid(nx=64, ny=32)
    cfg = WorkflowConfig(mesh_source=None, geometry_cache_source="unused.npz", manning_n=MANNING, output_interval_s=20.0,
                         dt_max=1.0, cfl_interval=1, dry_tol=DRY_TOL, progress=False, capture_momentum_snapshots=True,
                         track_clamp_mass=True)
    wf = SWEWorkflow(cfg, geometry=g)
    wf.prepare()
    x0, y0 = g.origin
    phases = [SimulationPhase(30.0, [PointSource(0.5, (x0 + 40.0, y0 + 32.0), 3.0)]),
              SimulationPhase(30.0, [PointSource(1.0, (x0 + 40.0, y0 + 32.0), 3.0)])]
    res = wf.run(phases)
    assert res.volume_injected_m3 == pytest.approx(45.0)
    # positivity clamps add their mass to what the sources put in (reference workflow.py:913-945)
    assert res.clamp_mass_m3 is not None and res.clamp_mass_m3 >= 0.0
    assert res.volume_final_m3 == pytest.approx(res.volume_injected_m3 + res.clamp_mass_m3, rel=1e-6)
    assert res.snap_times[0] == 0.0 and res.snap_times[-1] == 60.0
    assert len(res.hu_snapshots) == len(res.snapshots) == len(res.snap_times)
    assert res.steps_total > 0 and res.h_final.shape == (g.N,)

    # the same phases on the FP32 oracle: every snapshot and the final state bit for bit
    geom = wf.geom
    zero = np.zeros(geom.N, np.float32)
    oracle = ResidentOracle(geom, wf.solver._h0, zero, zero, np.full(geom.N, MANNING, np.float32), dry_tol=DRY_TOL,
                            steps_per_graph=wf.solver.steps_per_graph)
    oracle.track_clamp = True
    valid = geom.area > cfg.area_tol
    snaps, times, t = [], [], 0.0
    for k, phase in enumerate(phases):
        s, ts = oracle.run(t_end=t + phase.duration_s, output_interval_s=cfg.output_interval_s, dt_max=cfg.dt_max,
                           dt_init=cfg.dt_init, source_rate=build_phase_source_rate(geom, phase, valid),
                           resume=k > 0, t_start=t)
        snaps += s
        times += ts
        t += phase.duration_s
    assert res.steps_total == oracle.steps_total
    assert res.snap_times == times
    for a, b in zip(res.snapshots, snaps, strict=True):
        np.testing.assert_array_equal(bits(a), bits(b))
    for a, b in ((res.h_final, oracle.download_h()), (res.hu_final, oracle.download_hu()),
                 (res.hv_final, oracle.download_hv()), (wf.solver.download_h_residual(), oracle.download_h_residual()),
                 (wf.solver.download_clamp_mass(), oracle.download_clamp_mass())):
        np.testing.assert_array_equal(bits(a), bits(b))


# -- the run loop's failure branches (reference gpu_resident_batch.py:715-736) --------------------------------
def test_a_bound_below_one_tick_stops_the_run_with_no_progress(grid) -> None:
    """A CFL bound under 2^-20 s rounds to zero ticks: the run raises instead of stalling."""
    h0 = np.ones(grid.N, np.float32)
    hu0 = np.zeros(grid.N, np.float32)
    hu0[grid.N // 2] = 1e9  # a velocity of 1e9 m/s on 2 m cells: a bound of ~1e-9 s
    solver = make(grid, h0, hu0)
    with pytest.raises(RuntimeError, match=r"made no time progress at t=0\.000000s \(CFL bound below one tick\)"):
        run(solver, 1.0)
    oracle = ResidentOracle(grid, h0, hu0, np.zeros(grid.N, np.float32), np.full(grid.N, MANNING, np.float32))
    with pytest.raises(RuntimeError, match="no time progress"):
        oracle.run(t_end=1.0, output_interval_s=0.25, dt_max=1.0, dt_init=0.01)


def test_a_non_finite_depth_ends_the_run_with_a_cleaned_snapshot(grid) -> None:
    """NaN in the state: the window's snapshot is nan_to_num'd, it is the last one, and run() returns."""
    h0 = dam(grid)
    h0[0] = np.nan
    solver = make(grid, h0)
    snaps, times = solver.run(t_end=40.0, output_interval_s=10.0, dt_max=1.0, dt_init=0.01, cfl_interval=1,
                              progress=False)
    assert times == [0.0, 10.0]  # stopped after the first window
    assert len(snaps) == 2 and np.isnan(snaps[0][0])  # the initial state as given
    assert np.isfinite(snaps[1]).all()
    h_dev = solver.download_h()
    assert not np.isfinite(h_dev).all()
    bad = ~np.isfinite(h_dev)
    assert (snaps[1][bad] == 0.0).all()
    np.testing.assert_array_equal(bits(snaps[1][~bad]), bits(h_dev[~bad]))
    assert 0 < solver.steps_total
    oracle = ResidentOracle(grid, h0, np.zeros(grid.N, np.float32), np.zeros(grid.N, np.float32),
                            np.full(grid.N, MANNING, np.float32))
    o_snaps, o_times = oracle.run(t_end=40.0, output_interval_s=10.0, dt_max=1.0, dt_init=0.01)
    assert o_times == times and oracle.steps_total == solver.steps_total
    np.testing.assert_array_equal(bits(o_snaps[1]), bits(snaps[1]))


def test_a_device_that_loses_the_two_sum_error_is_refused(grid, monkeypatch) -> None:
    """The guard's refusing branch: a probe whose error term comes back lost stops run() before any step."""
    solver = make(grid, dam(grid))
    monkeypatch.setattr(solver, "_eft_probe", lambda: np.array([1.0, 1e-9, 0.0], np.float32))
    with pytest.raises(RuntimeError, match="error-free arithmetic is broken"):
        run(solver, 1.0)
    assert solver.steps_total == 0
    solver.compensated = False  # a closed mesh without the compensated pair needs no check
    run(solver, 1.0)
    assert solver.steps_total > 0
