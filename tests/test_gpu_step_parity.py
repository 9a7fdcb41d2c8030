"""CUDA step against the FP64 oracle and, bit for bit, the FP32 oracle.

Follows the reference's ``tests/unit/test_gpu_step_parity.py``: a few
fixed-dt Heun steps (dt = 2^-10 s, exact in ticks and in float32) on the
valley must match the float64 step within |dh| <= 2e-6 m and |dq| <= 2e-5
(8 steps), and at a 300 m bed datum within 5e-6 / 6e-7 (64 steps); dry cells
carry exactly zero momentum; the prologue CFL bound matches the float64
bound to 1e-4 relative. On top of the reference's checks, every result must
equal the FP32 restatement of the reference's kernels bit for bit.
"""

from __future__ import annotations

from collections.abc import Callable

import numpy as np
import pytest

from inundation_b200.tuning import CFL_DEFAULT, GRAVITY_G
from oracle import fp64_step
from oracle.resident_oracle import ResidentOracle

from ._valley import DRY_TOL, DX, MANNING, NX, dam, sheet, valley_grid

pytestmark = pytest.mark.gpu

DT = 2.0**-10
STEPS = 8
ATOL_H = 2e-6
ATOL_Q = 2e-5
LONG_STEPS = 64
LONG_ATOL_H = 5e-6
LONG_ATOL_Q = 6e-7


@pytest.fixture(scope="module")
def grid():
    return valley_grid()


@pytest.fixture(scope="module")
def high_grid():
    return valley_grid(datum=300.0)


def wet_lake(grid) -> fp64_step.State:
    x = grid.centroid[:, 0].astype(np.float64)
    h = float(grid.zb.max()) + 0.5 - grid.zb.astype(np.float64)
    assert (h > 10 * DRY_TOL).all()
    hu = 0.1 * np.sin(2 * np.pi * x / (NX * DX)) * h
    return fp64_step.State(h, hu, np.zeros_like(h))


def dam_break(grid) -> fp64_step.State:
    h = dam(grid).astype(np.float64)
    return fp64_step.State(h, np.zeros_like(h), np.zeros_like(h))


def draining(grid) -> fp64_step.State:
    h = sheet(grid).astype(np.float64)
    return fp64_step.State(h, np.where(h > 0.0, 0.05, 0.0), np.zeros_like(h))


def dry_momentum(grid) -> fp64_step.State:
    h = dam(grid).astype(np.float64)
    far = grid.centroid[:, 0] > NX * DX * 0.8
    hu = np.where(far, 0.1, 0.0)
    return fp64_step.State(h, hu, -hu)


CASES: dict[str, Callable] = {
    "wet_lake": wet_lake,
    "dam_break": dam_break,
    "draining": draining,
    "dry_momentum": dry_momentum,
}


def make_solver(grid, s: fp64_step.State, kernel: str = "tiled", grid_limit: int | None = None):
    from inundation_b200.backend import SWESolverB200Resident

    f32 = [a.astype(np.float32) for a in (s.h, s.hu, s.hv)]
    solver = SWESolverB200Resident(grid, None, *f32, np.full(grid.N, MANNING, np.float32), dry_tol=DRY_TOL)
    solver.stage_kernel = kernel
    if grid_limit is not None:
        # Few persistent CTAs: each loops over many tiles, so the tiled kernel's
        # prefetch of the next work item overlaps the current one.
        solver.max_grid = grid_limit
    return solver


def make_oracle(grid, s: fp64_step.State) -> ResidentOracle:
    f32 = [a.astype(np.float32) for a in (s.h, s.hu, s.hv)]
    return ResidentOracle(grid, *f32, np.full(grid.N, MANNING, np.float32), dry_tol=DRY_TOL)


def step(solver, steps: int) -> fp64_step.State:
    solver.run(t_end=steps * DT, output_interval_s=steps * DT, dt_max=DT, dt_init=DT, cfl_interval=steps, progress=False)
    assert solver.steps_total == steps
    return fp64_step.State(*(a.astype(np.float64) for a in (solver.download_h(), solver.download_hu(), solver.download_hv())))


def assert_close(got: fp64_step.State, want: fp64_step.State, atol_h: float, atol_q: float) -> None:
    for name, a, b, atol in (("h", got.h, want.h, atol_h), ("hu", got.hu, want.hu, atol_q), ("hv", got.hv, want.hv, atol_q)):
        worst = float(np.abs(a - b).max())
        assert worst <= atol, f"{name}: max |gpu - fp64| = {worst:.3e} > {atol:.1e}"


def assert_same_bits(a: np.ndarray, b: np.ndarray, what: str) -> None:
    a32, b32 = np.ascontiguousarray(a, np.float32).view(np.uint32), np.ascontiguousarray(b, np.float32).view(np.uint32)
    bad = np.flatnonzero(a32 != b32)
    assert bad.size == 0, f"{what}: {bad.size} cells differ from the FP32 oracle (first {bad[:5].tolist()})"


@pytest.mark.parametrize("kernel,grid_limit", [("tiled", None), ("plain", None), ("staged", None), ("persistent", None),
                                                ("tiled", 3), ("plain", 5), ("staged", 5), ("persistent", 3)],
                         ids=["tiled", "plain", "staged", "persistent", "tiled-3ctas", "plain-5ctas", "staged-5ctas",
                              "persistent-3ctas"])
@pytest.mark.parametrize("case", list(CASES))
def test_steps_match_fp64_and_fp32_oracles(case: str, kernel: str, grid_limit, grid) -> None:
    s0 = CASES[case](grid)
    n = np.full(grid.N, MANNING, np.float32)
    want = fp64_step.run_steps(
        grid, s0.h.astype(np.float32), s0.hu.astype(np.float32), s0.hv.astype(np.float32), n, DT, STEPS,
        g=GRAVITY_G, dry_tol=DRY_TOL,
    )
    solver = make_solver(grid, s0, kernel, grid_limit)
    got = step(solver, STEPS)
    assert_close(got, want, ATOL_H, ATOL_Q)
    oracle = make_oracle(grid, s0)
    step(oracle, STEPS)
    assert_same_bits(solver.download_h(), oracle.download_h(), "h")
    assert_same_bits(solver.download_hu(), oracle.download_hu(), "hu")
    assert_same_bits(solver.download_hv(), oracle.download_hv(), "hv")
    assert_same_bits(solver.download_h_residual(), oracle.download_h_residual(), "h_lo")
    np.testing.assert_array_equal(solver.download_block_flags(), oracle.download_block_flags())


@pytest.mark.parametrize("case", ["dam_break", "draining"])
def test_steps_on_high_terrain_match_fp64(case: str, high_grid) -> None:
    s0 = CASES[case](high_grid)
    n = np.full(high_grid.N, MANNING, np.float32)
    want = fp64_step.run_steps(
        high_grid, s0.h.astype(np.float32), s0.hu.astype(np.float32), s0.hv.astype(np.float32), n, DT, LONG_STEPS,
        g=GRAVITY_G, dry_tol=DRY_TOL,
    )
    got = step(make_solver(high_grid, s0), LONG_STEPS)
    assert_close(got, want, LONG_ATOL_H, LONG_ATOL_Q)


@pytest.mark.parametrize("case", list(CASES))
def test_dry_cells_carry_no_momentum(case: str, grid) -> None:
    got = step(make_solver(grid, CASES[case](grid)), STEPS)
    dry = got.h < DRY_TOL
    assert float(np.abs(got.hu[dry]).max(initial=0.0)) == 0.0
    assert float(np.abs(got.hv[dry]).max(initial=0.0)) == 0.0


def prologue_bound(solver) -> float:
    solver._ctrl[...] = 0
    solver._sync_ctrl_to_device()
    solver._enqueue_prologue()
    solver._read_ctrl()
    return float(solver._ctrl["last_raw"][0])


@pytest.mark.parametrize("case", list(CASES))
def test_cfl_bound_matches_fp64_and_fp32(case: str, grid) -> None:
    s0 = CASES[case](grid)
    s32 = fp64_step.State(*(a.astype(np.float32).astype(np.float64) for a in (s0.h, s0.hu, s0.hv)))
    want = fp64_step.cfl_dt(grid, s32, g=GRAVITY_G, dry_tol=DRY_TOL, cfl=CFL_DEFAULT)
    got = prologue_bound(make_solver(grid, s0))
    assert got == pytest.approx(want, rel=1e-4)
    oracle = make_oracle(grid, s0)
    oracle.prologue()
    assert np.float32(got) == oracle.ctrl["last_raw"][0]
