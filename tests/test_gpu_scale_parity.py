"""Bit-for-bit parity with the FP32 oracle at benchmark scale.

The dam break of the 1M-cell workload at a quarter of its area: 262,144
Voronoi cells over 5 km (the same ~10 m spacing, fractal DEM with a carved
channel, 4 m inside 5 % of the side), 60 simulated seconds of adaptive steps
(about 2,000). On the persistent kernel the front keeps activating blocks,
whose tiles reach CTAs through the tile queue, and tiles that dry out give
their seats up. Every output window's
depth, the final h, hu, hv, h_lo and the active-set flags must equal the C
oracle's bit for bit, for every stage kernel.

A fully wet variant (every cell at least 0.5 m deep, 200+ steps) keeps all
4,096 tiles active: the persistent kernel runs it on its full grid, and on a
grid of 8 CTAs, where each CTA takes 512 tiles a step, the most its extra-tile
capacity allows besides its seat; the staged block kernel runs it on its full
grid and on 7 CTAs, each restaging its shared memory for about 146 blocks.
"""

from __future__ import annotations

import numpy as np
import pytest

from inundation_b200.scenarios import dam_break
from oracle.resident_oracle import ResidentOracle

pytestmark = pytest.mark.gpu

CELLS, SIDE = 262_144, 5000.0


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def run_kw(t_end: float, interval: float, sc) -> dict:
    return {"t_end": t_end, "output_interval_s": interval, "dt_max": sc.dt_max, "dt_init": sc.dt_init}


@pytest.fixture(scope="module")
def scenario():
    return dam_break(n_cells=CELLS, seed=2, side=SIDE)


def oracle_run(sc, h0: np.ndarray, t_end: float, interval: float):
    o = ResidentOracle(sc.geom, h0, sc.hu0, sc.hv0, sc.manning, dry_tol=sc.dry_tol, steps_per_graph=200)
    snaps, times = o.run(**run_kw(t_end, interval, sc))
    return o, snaps, times


@pytest.fixture(scope="module")
def dam_oracle(scenario):
    return oracle_run(scenario, scenario.h0, 60.0, 20.0)


def wet_start(sc) -> np.ndarray:
    return np.maximum(sc.h0, np.float32(0.5)).astype(np.float32)


@pytest.fixture(scope="module")
def wet_oracle(scenario):
    return oracle_run(scenario, wet_start(scenario), 7.5, 2.5)


def solver_run(sc, h0, kernel: str, t_end: float, interval: float, max_grid: int | None = None):
    from inundation_b200.backend import SWESolverB200Resident

    s = SWESolverB200Resident(sc.geom, None, h0, sc.hu0, sc.hv0, sc.manning, dry_tol=sc.dry_tol)
    s.stage_kernel = kernel
    s.max_grid = max_grid
    snaps, times = s.run(cfl_interval=1, progress=False, **run_kw(t_end, interval, sc))
    return s, snaps, times


def assert_same(s, snaps, times, oracle) -> None:
    o, o_snaps, o_times = oracle
    assert s.steps_total == o.steps_total
    assert times == o_times
    for a, b in zip(snaps, o_snaps, strict=True):
        np.testing.assert_array_equal(bits(a), bits(b))
    for a, b in ((s.download_hu(), o.download_hu()), (s.download_hv(), o.download_hv()),
                 (s.download_h_residual(), o.download_h_residual())):
        np.testing.assert_array_equal(bits(a), bits(b))
    np.testing.assert_array_equal(s.download_block_flags(), o.download_block_flags())


@pytest.mark.parametrize("kernel", ["persistent", "plain", "staged", "tiled", "auto"])
def test_dam_break_262k_over_2000_steps(scenario, dam_oracle, kernel: str) -> None:
    s, snaps, times = solver_run(scenario, scenario.h0, kernel, 60.0, 20.0)
    assert s.steps_total >= 1000
    assert_same(s, snaps, times, dam_oracle)
    flags = s.download_block_flags()
    # the front has spread: far more blocks are active than the dam's own
    assert int(flags[:, 1].sum()) > 2 * int((scenario.h0.reshape(-1, 256) > 0).any(axis=1).sum())


@pytest.mark.parametrize("kernel, max_grid", [("persistent", None), ("persistent", 8), ("plain", None), ("staged", None),
                                             ("staged", 7), ("auto", None)])
def test_all_wet_262k_over_200_steps(scenario, wet_oracle, kernel: str, max_grid: int | None) -> None:
    s, snaps, times = solver_run(scenario, wet_start(scenario), kernel, 7.5, 2.5, max_grid)
    assert s.steps_total >= 200
    if kernel == "persistent" and max_grid is not None:
        assert s.grid(2) == max_grid and 4 * s.n_blocks == 4096 <= max_grid * 513
    if kernel == "staged" and max_grid is not None:
        assert s.grid(3) == max_grid  # each CTA stages its blocks one after another
    assert_same(s, snaps, times, wet_oracle)
    assert s.download_block_flags()[:, 1].all()
