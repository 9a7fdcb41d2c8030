"""The smaller benchmark configurations as behaviour tests.

* Lake at rest (config 1): 8k Voronoi cells over 1 km, six Gaussian bumps
  breaking a 1 m surface, CFL 0.9; the reference's own gate
  (``inundation/bench/lake_at_rest.py:197-204``: max |u| over cells deeper
  than 10 dry_tol, volume drift) with round-off bounds instead of its 0.01 m/s
  escalation threshold.
* Rain plus point inflow (config 3, scaled down): uniform 50 mm/h rain on
  every cell and a triangular inflow hydrograph on a dry fractal terrain in a
  walled box; bit for bit against the FP32 oracle, and the float64 volume
  equals the rain plus the inflow delivered.
"""

from __future__ import annotations

import numpy as np
import pytest

from inundation_b200.scenarios import lake_at_rest, rain_inflow
from oracle.resident_oracle import ResidentOracle

pytestmark = pytest.mark.gpu


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("kernel", ["tiled", "persistent"])
def test_lake_at_rest_stays_at_rest(kernel: str) -> None:
    from inundation_b200.backend import SWESolverB200Resident

    sc = lake_at_rest(8000, seed=1)
    solver = SWESolverB200Resident(sc.geom, None, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=sc.dry_tol,
                                   cfl=sc.meta["cfl"])
    solver.stage_kernel = kernel
    v0 = solver.volume_fp64()
    solver.run(t_end=600.0, output_interval_s=600.0, dt_max=1.0, dt_init=0.01, cfl_interval=10, progress=False)
    assert solver.steps_total >= 1000
    h, hu, hv = solver.download_h(), solver.download_hu(), solver.download_hv()
    wet = h > 10 * sc.dry_tol
    max_u = float(max((np.abs(hu[wet]) / h[wet]).max(), (np.abs(hv[wet]) / h[wet]).max()))
    drift = abs(solver.volume_fp64() - v0) / v0
    assert max_u < 1e-5, max_u
    assert drift < 1e-9, drift
    np.testing.assert_allclose(h[wet], sc.h0[wet], atol=1e-5)


def test_rain_and_inflow_match_the_oracle_and_the_delivered_volume() -> None:
    from inundation_b200.batch import BatchedSolver, BatchMember

    sc = rain_inflow(12_000, seed=3, side=1_100.0)
    t_end = 300.0
    solver = BatchedSolver([BatchMember(sc.geom, sc.h0, sc.hu0, sc.hv0, sc.manning, source_rate=sc.source_rate,
                                        hydrographs=sc.hydrographs)], dry_tol=sc.dry_tol)
    v0 = solver.volume_fp64(0)
    res = solver.run(t_end, dt_max=sc.dt_max, dt_init=sc.dt_init, output_interval_s=100.0)
    oracle = ResidentOracle(sc.geom, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=sc.dry_tol)
    snaps, _ = oracle.run(t_end=t_end, output_interval_s=100.0, dt_max=sc.dt_max, dt_init=sc.dt_init,
                          source_rate=sc.source_rate, hydrographs=sc.hydrographs)
    assert int(res.steps[0]) == oracle.steps_total
    for a, b in zip(res.snapshots[0][1:], snaps[1:], strict=False):
        np.testing.assert_array_equal(bits(a), bits(b))
    np.testing.assert_array_equal(bits(solver.download_hu(0)), bits(oracle.download_hu()))
    # walled box: every drop of rain and inflow stays
    rain = float(sc.source_rate.astype(np.float64).sum()) * t_end
    hg = sc.hydrographs[0]
    kt = np.append(hg.knot_t.astype(np.float64), t_end)
    kq = np.append(hg.knot_q.astype(np.float64), np.interp(t_end, hg.knot_t, hg.knot_q))
    inflow = float(np.trapezoid(kq[kt <= t_end], kt[kt <= t_end]))
    gained = solver.volume_fp64(0) - v0
    assert gained == pytest.approx(rain + inflow, rel=5e-3)
    assert (solver.download_h(0) >= sc.dry_tol).mean() > 0.5  # the rain has wetted most of the box
