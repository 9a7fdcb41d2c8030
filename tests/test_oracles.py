"""The oracles themselves, pinned to the reference before they check the CUDA path.

* The FP64 oracle (``oracle/fp64_step.py``) must reproduce the reference's
  ``tests/unit/_cpu_step.py`` outputs stored in ``tests/golden/cpu_step.npz``.
* The FP32 oracle (``oracle/fp32_resident.c``) must stay within the
  reference's GPU-vs-FP64 tolerances (``tests/unit/test_gpu_step_parity.py:31-34,
  158-163``) of those outputs, pass the reference's ``step_control`` known-answer
  tests (``tests/unit/test_gpu_resident_clock.py:118-214``) and its HLLC speed
  continuity tests (``tests/unit/test_hllc_speeds.py``).
"""

from __future__ import annotations

import struct
from pathlib import Path

import numpy as np
import pytest

from inundation_b200.mesh.geometry import build_geometry, hilbert_reorder
from inundation_b200.tuning import SIM_TICKS_PER_SECOND
from oracle import fp64_step
from oracle.resident_oracle import CTRL_DTYPE, ResidentOracle, hllc_f32, hllc_speeds_f32, inv_pow43, math_ok, step_control

GOLD = Path(__file__).parent / "golden"
STEP = np.load(GOLD / "cpu_step.npz")
GEO = np.load(GOLD / "geometry.npz")
G, DRY, MANNING, DT = 9.81, 1e-3, 0.03, 2.0**-10
CASES = ["wet_lake", "dam_break", "draining", "dry_momentum"]


def golden_grid(name: str):
    offsets = GEO[f"{name}_in_offsets"]
    raw = build_geometry(GEO[f"{name}_in_verts"], GEO[f"{name}_in_faces"], offsets if offsets.size else None,
                         zb_from_file=GEO[f"{name}_in_zb"])
    return hilbert_reorder(raw, verbose=False)[0]


@pytest.fixture(scope="module")
def valley():
    return golden_grid("valley")


@pytest.fixture(scope="module")
def valley300():
    return golden_grid("valley300")


@pytest.fixture(scope="module")
def voronoi():
    return golden_grid("voronoi")


def _inputs(key: str):
    return STEP[f"{key}_h0"], STEP[f"{key}_hu0"], STEP[f"{key}_hv0"]


@pytest.mark.parametrize("case", CASES)
def test_fp64_oracle_reproduces_the_reference_step(case: str, valley, valley300) -> None:
    for grid, name, steps in ((valley, "valley", 8), (valley300, "valley300", 64)):
        key = f"{name}_{case}"
        h, hu, hv = _inputs(key)
        s = fp64_step.run_steps(grid, h, hu, hv, np.full(grid.N, MANNING, np.float32), DT, steps, g=G, dry_tol=DRY)
        np.testing.assert_allclose(s.h, STEP[f"{key}_h"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(s.hu, STEP[f"{key}_hu"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(s.hv, STEP[f"{key}_hv"], rtol=0, atol=1e-12)
        s0 = fp64_step.State(*(a.astype(np.float64) for a in (h, hu, hv)))
        assert fp64_step.cfl_dt(grid, s0, g=G, dry_tol=DRY, cfl=0.8) == pytest.approx(float(STEP[f"{key}_cfl"]), rel=1e-14)


def test_fp64_oracle_on_a_voronoi_mesh(voronoi) -> None:
    z = np.zeros(voronoi.N, np.float32)
    s = fp64_step.run_steps(voronoi, STEP["voronoi_h0"], z, z, STEP["voronoi_n"], 0.05, 8, g=G, dry_tol=1e-4)
    for name in ("h", "hu", "hv"):
        np.testing.assert_allclose(getattr(s, name), STEP[f"voronoi_{name}"], rtol=0, atol=1e-12)


def test_fp64_hllc_and_speeds_match_the_reference() -> None:
    st = STEP["hllc_in"]
    out = np.column_stack(fp64_step.hllc(*(st[:, k] for k in range(6)), g=G, dry_tol=DRY))
    np.testing.assert_allclose(out, STEP["hllc_out"], rtol=1e-14, atol=1e-14)
    sp = STEP["speeds_in"]
    out = np.column_stack(fp64_step.hllc_speeds(sp[:, 0], sp[:, 1], sp[:, 2], sp[:, 3], g=G, dry_tol=DRY))
    np.testing.assert_allclose(out, STEP["speeds_out"], rtol=1e-14, atol=1e-14)


def test_fp32_hllc_is_float32_close_to_the_reference() -> None:
    st = STEP["hllc_in"]
    got = hllc_f32(G, DRY, st).astype(np.float64)
    want = STEP["hllc_out"]
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=2e-5)


@pytest.mark.parametrize("case", CASES)
def test_fp32_oracle_is_within_the_reference_gpu_tolerance(case: str, valley, valley300) -> None:
    for grid, name, steps, atol_h, atol_q in ((valley, "valley", 8, 2e-6, 2e-5), (valley300, "valley300", 64, 5e-6, 6e-7)):
        if name == "valley300" and case not in ("dam_break", "draining"):
            continue
        key = f"{name}_{case}"
        o = ResidentOracle(grid, *_inputs(key), np.full(grid.N, MANNING, np.float32), dry_tol=DRY)
        o.run(t_end=steps * DT, output_interval_s=steps * DT, dt_max=DT, dt_init=DT)
        assert o.steps_total == steps
        assert float(np.abs(o.download_h().astype(np.float64) - STEP[f"{key}_h"]).max()) <= atol_h
        assert float(np.abs(o.download_hu().astype(np.float64) - STEP[f"{key}_hu"]).max()) <= atol_q
        assert float(np.abs(o.download_hv().astype(np.float64) - STEP[f"{key}_hv"]).max()) <= atol_q


# -- step_control known answers (reference test_gpu_resident_clock.py:118-214) ----------------------
def _bits(v: float) -> int:
    return struct.unpack("<I", struct.pack("<f", v))[0]


def _run_control(mode: int, slot0: float = 0.0, slot1: float = 1e30, **fields):
    c = np.zeros(1, CTRL_DTYPE)
    c["dt_max_ticks"] = SIM_TICKS_PER_SECOND
    c["dry_dt_ticks"] = SIM_TICKS_PER_SECOND // 100
    c["cfl_safety"] = 0.8
    c["stop_ticks"] = 10**9
    for k, v in fields.items():
        c[k] = v
    dt = np.array([_bits(slot0), _bits(slot1), 0, 0], np.uint32)
    step_control(c, dt, mode)
    return c[0], dt


def _ticks(raw: float, safety: float = 0.8) -> int:
    return int(np.float32(raw) * np.float32(safety) * np.float32(SIM_TICKS_PER_SECOND))


def test_start_takes_the_prologue_bound_with_safety() -> None:
    c, dt = _run_control(0, slot0=0.05, now_ticks=123)
    assert c["dt_ticks"] == _ticks(0.05) and c["now_ticks"] == 123 and c["steps"] == 0
    assert dt[0] == _bits(_ticks(0.05) / SIM_TICKS_PER_SECOND) and dt[1] == _bits(1e30)


def test_dt_is_exactly_the_tick_count() -> None:
    c, dt = _run_control(0, slot0=0.0314)
    assert struct.unpack("<f", struct.pack("<I", int(dt[0])))[0] * SIM_TICKS_PER_SECOND == int(c["dt_ticks"])


def test_step_advances_counts_and_replans() -> None:
    c, _ = _run_control(1, slot1=0.02, now_ticks=1000, dt_ticks=777, steps=5)
    assert c["now_ticks"] == 1777 and c["steps"] == 6 and c["dt_ticks"] == _ticks(0.02)
    assert c["last_raw"] == np.float32(0.02)


def test_noop_step_keeps_clock_count_and_bound() -> None:
    c, _ = _run_control(1, now_ticks=1000, dt_ticks=0, steps=5, last_raw=0.03)
    assert c["now_ticks"] == 1000 and c["steps"] == 5 and c["dt_ticks"] == _ticks(0.03)


def test_retarget_replans_from_the_last_bound() -> None:
    c, _ = _run_control(2, slot1=0.5, now_ticks=1000, dt_ticks=0, last_raw=0.03)
    assert c["now_ticks"] == 1000 and c["dt_ticks"] == _ticks(0.03)


def test_caps_window_stop_dry_fallback_and_stall() -> None:
    assert _run_control(0, slot0=50.0, dt_max_ticks=4096)[0]["dt_ticks"] == 4096
    assert _run_control(0, slot0=0.05, now_ticks=10_000, stop_ticks=10_005)[0]["dt_ticks"] == 5
    c, dt = _run_control(1, slot1=0.05, now_ticks=9_000, dt_ticks=1_000, stop_ticks=10_000)
    assert c["now_ticks"] == 10_000 and c["dt_ticks"] == 0 and dt[0] == 0
    assert _run_control(0, slot0=1e30, dry_dt_ticks=2048)[0]["dt_ticks"] == 2048
    assert _run_control(0, slot0=1e-12)[0]["dt_ticks"] == 0


def test_clock_carries_past_32_bits() -> None:
    start = 2**32 - 3
    c, _ = _run_control(1, slot1=0.05, now_ticks=start, dt_ticks=10, stop_ticks=2**40)
    assert c["now_ticks"] == start + 10


# -- HLLC speeds (reference test_hllc_speeds.py) ---------------------------------------------------
def _speeds(h_l: float, u_l: float, h_r: float, u_r: float, f32: bool) -> tuple[float, float]:
    if f32:
        out = hllc_speeds_f32(G, DRY, np.array([[h_l, u_l, h_r, u_r]]))[0]
        return float(out[0]), float(out[1])
    sl, sr = fp64_step.hllc_speeds(np.array([h_l]), np.array([u_l]), np.array([h_r]), np.array([u_r]), g=G, dry_tol=DRY)
    return float(sl[0]), float(sr[0])


@pytest.mark.parametrize("f32", [False, True], ids=["fp64", "fp32"])
@pytest.mark.parametrize("edge", [DRY, 2.0 * DRY])
@pytest.mark.parametrize("wet", [(0.05, 0.3), (0.5, -0.4), (0.01, 0.0)])
def test_speeds_are_continuous_as_a_side_dries(f32: bool, edge: float, wet: tuple[float, float]) -> None:
    h, u = wet
    eps = 1e-9 if not f32 else 1e-5
    atol = 1e-5 if not f32 else 2e-3
    assert _speeds(h, u, edge * (1 - eps), 0.0, f32) == pytest.approx(_speeds(h, u, edge * (1 + eps), 0.0, f32), abs=atol)
    assert _speeds(edge * (1 - eps), 0.0, h, u, f32) == pytest.approx(_speeds(edge * (1 + eps), 0.0, h, u, f32), abs=atol)


@pytest.mark.parametrize("f32", [False, True], ids=["fp64", "fp32"])
def test_dry_bed_and_roe_speeds(f32: bool) -> None:
    h, u = 0.5, 0.3
    c = float(np.sqrt(G * h))
    assert _speeds(h, u, 0.0, 0.0, f32) == pytest.approx((u - c, u + 2.0 * c), rel=1e-6)
    assert _speeds(0.0, 0.0, h, -u, f32) == pytest.approx((-u - 2.0 * c, -u + c), rel=1e-6)
    s_l, s_r = _speeds(0.5, 0.0, 0.2, 0.0, f32)
    c_roe = float(np.sqrt(G * 0.35))
    assert s_l == pytest.approx(min(-float(np.sqrt(G * 0.5)), -c_roe), rel=1e-6)
    assert s_r == pytest.approx(max(float(np.sqrt(G * 0.2)), c_roe), rel=1e-6)


# -- arithmetic ------------------------------------------------------------------------------------
def test_friction_depth_power_is_within_six_ulp() -> None:
    """h^(-4/3) by the division-free Newton sequence, against the float64 power (GLSL's pow has no
    fixed rounding; six ulp of the power is a relative error below 4e-7)."""
    xs = np.concatenate([np.geomspace(1e-12, 1e6, 20000),
                         np.array([1.0, 8.0, 0.001, 2.0, 27.0, 1e-4, 4e-4])]).astype(np.float32)
    got = np.array([inv_pow43(float(x)) for x in xs], dtype=np.float32)
    exact = xs.astype(np.float64) ** (-4.0 / 3.0)
    ulp = np.spacing(exact.astype(np.float32)).astype(np.float64)
    assert float((np.abs(got.astype(np.float64) - exact) / ulp).max()) <= 6.0


def test_two_sum_keeps_its_error_term() -> None:
    assert math_ok()


def test_closed_basin_conserves_volume_with_compensation() -> None:
    from inundation_b200.mesh.synthetic import quad_grid

    q = quad_grid(24, 24, 1.0)
    g = build_geometry(q.verts, q.faces.reshape(-1, 4), zb_from_file=np.zeros(576, np.float32))
    cx, cy = g.centroid[:, 0], g.centroid[:, 1]
    h0 = (0.5 + 0.2 * np.exp(-((cx - 12) ** 2 + (cy - 12) ** 2) / 10.0)).astype(np.float32)
    z = np.zeros(576, np.float32)
    o = ResidentOracle(g, h0, z, z, np.full(576, 0.03, np.float32))
    v0 = float((h0.astype(np.float64) * g.area).sum())
    o.run(t_end=20.0, output_interval_s=10.0, dt_max=1.0, dt_init=0.01)
    assert o.steps_total > 50
    assert float((o.download_h_precise() * g.area).sum()) == pytest.approx(v0, rel=1e-6)


def test_a_region_steps_like_the_whole_mesh_while_its_rim_stays_dry() -> None:
    """``fp64_step.restrict``: the float64 step over a region equals the whole mesh's there, bit for bit."""
    from tests._valley import dam, valley_grid

    g = valley_grid(nx=64, ny=32)
    h0 = dam(g, 64, 32).astype(np.float64)
    cells = np.flatnonzero(g.centroid[:, 0] < 64 * 2.0 * 0.6)
    region = fp64_step.restrict(g, cells)
    assert region.N == cells.size and region.rim.size > 0
    n = np.full(g.N, 0.03)
    whole = fp64_step.State(h0, 0 * h0, 0 * h0)
    part = fp64_step.State(h0[cells], 0 * h0[cells], 0 * h0[cells])
    for _ in range(40):
        whole = fp64_step.heun_step(g, whole, n, 2.0**-6, g=9.81, dry_tol=1e-3)
        part = fp64_step.heun_step(region, part, n[cells], 2.0**-6, g=9.81, dry_tol=1e-3)
    assert part.h[region.rim].max() == 0.0 and whole.h[np.setdiff1d(np.arange(g.N), cells)].max() == 0.0
    for a, b in ((whole.h, part.h), (whole.hu, part.hu), (whole.hv, part.hv)):
        np.testing.assert_array_equal(a[cells], b)
