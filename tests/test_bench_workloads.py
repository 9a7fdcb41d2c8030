"""The bench's workloads build at small sizes and describe themselves correctly (no GPU).

``bench.py --workload W`` names the configuration it measures in its JSON line's
``config``; these checks keep those descriptions tied to the scenarios actually
built (cells, CFL, the L2 statement, the sources of the rain).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def args_for(workload: str, *extra: str):
    argv = sys.argv
    try:
        sys.argv = ["bench.py", "--workload", workload, *extra]
        return bench.parse_args()
    finally:
        sys.argv = argv


def test_every_workload_has_defaults() -> None:
    assert set(bench.WORKLOADS) == {"dam_break", "full_wet", "one_cell", "lake_at_rest", "rain_inflow"}
    assert args_for("dam_break").cells == 1_000_000 and args_for("dam_break").seed == 2
    assert args_for("lake_at_rest").cells == 8_000 and args_for("lake_at_rest").seed == 1
    assert args_for("rain_inflow").cells == 4_000_000 and args_for("rain_inflow").spin_up == 60.0
    assert args_for("rain_inflow", "--cells", "5000", "--seed", "9").cells == 5000


@pytest.mark.parametrize("workload", sorted(bench.WORKLOADS))
def test_small_workloads_and_their_config(workload: str) -> None:
    args = args_for(workload, "--cells", "3000")
    sc = bench.build_scenario(workload, args.cells, args.seed)
    cfl = float(sc.meta.get("cfl", 0.8))
    cfg = bench.workload_config(sc, args, cfl)
    assert cfg["workload"] == f"{workload}_3k_voronoi" and cfg["cells"] == sc.geom.N
    assert cfg["cfl"] == (0.9 if workload == "lake_at_rest" else 0.8)
    assert "water" in cfg and "terrain" in cfg
    assert cfg["l2"].startswith("inputs fit in L2")  # 3k cells: about 1 MiB a step
    wet = sc.h0 >= sc.dry_tol
    if workload == "one_cell":
        assert wet.sum() == 1
    elif workload == "full_wet":
        assert wet.all()
    elif workload == "rain_inflow":
        assert not wet.any() and sc.source_rate is not None and len(sc.hydrographs) == 1
        np.testing.assert_allclose(sc.source_rate, sc.meta["rain_m_per_s"] * sc.geom.area, rtol=1e-6)
    else:
        assert wet.any()



def test_reference_arm_states_the_cuda_arms_config(capsys: pytest.CaptureFixture[str]) -> None:
    """Both arms print the same ``config`` for the same workload, so their lines compare directly."""
    import json

    args = args_for("dam_break", "--impl", "reference", "--cells", "3000", "--steps", "1", "--warmup", "1")
    bench.run_reference(args, world=1, rank=0)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    sc = bench.build_scenario("dam_break", args.cells, args.seed)
    assert line["config"] == json.loads(json.dumps(bench.workload_config(sc, args, 0.8)))
    assert line["impl"] == "reference" and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["value"] > 0
