"""Open boundaries on the device against the FP32 oracle, bit for bit.

* The ghost state and boundary mass flux of every condition (the device half
  of the reference's ghost probe, ``tests/unit/test_gpu_open_ghost.py``).
* Whole runs of a 300 x 20 channel open at both ends (the layout of the
  reference's ``tests/unit/test_gpu_open_boundaries.py``) under each
  condition, on every stage kernel: depths, momenta, low words, step counts and
  the per-stretch volume snapshots equal the oracle's.
* The reference's behaviour tests of that file: skipping on and off give the
  same bits, the balance closes, only flowing inflows force blocks, the first
  step sees the water beyond a stage.
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from inundation_b200.scenarios import open_channel
from inundation_b200.tuning import GRAVITY_G, OPEN_FREE, OPEN_INFLOW, OPEN_NORMAL, OPEN_STAGE, OPEN_WALL
from oracle.resident_oracle import ResidentOracle, open_ghost_f32

pytestmark = pytest.mark.gpu

DRY_TOL = 1e-4
SLOPE = 1e-3
MANNING = 0.03
NORMAL = math.sqrt(SLOPE) / MANNING


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_device_ghosts_match_the_oracle_bit_for_bit() -> None:
    from inundation_b200 import native

    rng = np.random.default_rng(11)
    n = 4096
    h = rng.uniform(0.0, 3.0, n) * (rng.random(n) > 0.15)
    h[:64] = rng.uniform(0.0, 4.0 * DRY_TOL, 64)  # films and near-dry cells
    theta = rng.uniform(0.0, 2.0 * np.pi, n)
    cases = np.column_stack([h, rng.uniform(-3, 3, n) * h, rng.uniform(-3, 3, n) * h, np.cos(theta), np.sin(theta),
                             rng.uniform(-5, 5, n)]).astype(np.float32)
    kinds = rng.integers(0, 5, n).astype(np.uint32)
    values = np.where(rng.random(n) < 0.1, 0.0, rng.uniform(0.0, 20.0, n)).astype(np.float32)
    want = open_ghost_f32(GRAVITY_G, DRY_TOL, cases, kinds, values)
    lib = native.load()
    cond = np.column_stack([kinds, values.view(np.uint32)]).ravel()
    dev = torch.device("cuda", 0)
    c = torch.from_numpy(cases).to(dev)
    w = torch.from_numpy(cond.view(np.int32)).to(dev)
    out = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    native.check(lib.swe_open_ghost_probe(c.data_ptr(), w.data_ptr(), out.data_ptr(), n, GRAVITY_G, DRY_TOL, None),
                 "swe_open_ghost_probe")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(bits(out.cpu().numpy()), bits(want))


# name: (initial depth, initial x-velocity, upstream condition, downstream condition, end time)
CASES = {
    "inflow_normal": (0.5, 0.0, (OPEN_INFLOW, 0.25), (OPEN_NORMAL, NORMAL), 40.0),
    "inflow_dry": (0.0, 0.0, (OPEN_INFLOW, 0.25), (OPEN_WALL, 0.0), 40.0),
    "stage_free": (0.01, 0.0, (OPEN_STAGE, 0.6), (OPEN_FREE, 0.0), 30.0),
    "stage_dry": (0.0, 0.0, (OPEN_STAGE, 0.6), (OPEN_WALL, 0.0), 30.0),
    "draining": (0.3, 0.4, (OPEN_WALL, 0.0), (OPEN_FREE, 0.0), 30.0),
    "backflow": (0.5, -0.5, (OPEN_WALL, 0.0), (OPEN_NORMAL, NORMAL), 10.0),
}


def channel(case: str):
    depth, u, up, down, t_end = CASES[case]
    sc = open_channel(depth=depth)
    sc.hu0 = (sc.h0 * np.float32(u)).astype(np.float32)
    a, b = sc.meta["open_edges"]
    kinds = np.concatenate([np.full(a.size, up[0]), np.full(b.size, down[0])]).astype(np.uint32)
    values = np.concatenate([np.full(a.size, up[1]), np.full(b.size, down[1])]).astype(np.float32)
    return sc, kinds, values, t_end


def solver_of(sc, kinds, values, kernel: str = "tiled"):
    from inundation_b200.backend import SWESolverB200Resident

    s = SWESolverB200Resident(sc.geom, None, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=DRY_TOL,
                              open_edges=sc.meta["open_edges"])
    if kernel == "persistent-3ctas":  # 94 tiles on 3 CTAs: seats, kept tiles and the queue
        kernel, s.max_grid = "persistent", 3
    s.stage_kernel = kernel
    s.steps_per_graph = 20
    s.set_open_conditions(kinds, values)
    return s


def run(s, t_end: float):
    return s.run(t_end=t_end, output_interval_s=10.0, dt_max=0.25, dt_init=0.01, cfl_interval=1, progress=False)


def oracle_run(sc, kinds, values, t_end: float):
    o = ResidentOracle(sc.geom, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=DRY_TOL, steps_per_graph=20,
                       open_edges=tuple(sc.meta["open_edges"]))
    o.set_open_conditions(kinds, values)
    snaps, times = o.run(t_end=t_end, output_interval_s=10.0, dt_max=0.25, dt_init=0.01)
    return o, snaps, times


@pytest.fixture(scope="module")
def oracles():
    out = {}
    for case in CASES:
        sc, kinds, values, t_end = channel(case)
        out[case] = oracle_run(sc, kinds, values, t_end)
    return out


@pytest.mark.parametrize("kernel", ["tiled", "plain", "staged", "persistent", "persistent-3ctas"])
@pytest.mark.parametrize("case", list(CASES))
def test_runs_match_the_oracle_bit_for_bit(case: str, kernel: str, oracles) -> None:
    sc, kinds, values, t_end = channel(case)
    s = solver_of(sc, kinds, values, kernel)
    snaps, times = run(s, t_end)
    o, osnaps, otimes = oracles[case]
    assert s.steps_total == o.steps_total > 10
    assert times == otimes
    for a, b in zip(snaps, osnaps, strict=True):
        np.testing.assert_array_equal(bits(a), bits(b))
    np.testing.assert_array_equal(bits(s.download_hu()), bits(o.download_hu()))
    np.testing.assert_array_equal(bits(s.download_hv()), bits(o.download_hv()))
    np.testing.assert_array_equal(bits(s.download_h_residual()), bits(o.download_h_residual()))
    assert len(s.open_volume_snapshots) == len(o.open_volume_snapshots) == len(times)
    for a, b in zip(s.open_volume_snapshots, o.open_volume_snapshots, strict=True):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("case", ["inflow_dry", "stage_dry"])
def test_water_entering_a_dry_mesh_is_the_same_with_skipping_off(case: str) -> None:
    sc, kinds, values, t_end = channel(case)
    on = solver_of(sc, kinds, values)
    a, _ = run(on, t_end)
    assert int((on.download_block_flags()[:, 1] == 0).sum()) > 0, "the active set must skip something"
    off = solver_of(sc, kinds, values)
    off.active_set = False
    b, _ = run(off, t_end)
    assert on.steps_total == off.steps_total
    np.testing.assert_array_equal(bits(a[-1]), bits(b[-1]))
    np.testing.assert_array_equal(on.download_open_volumes(), off.download_open_volumes())


def test_the_balance_closes_while_water_enters_and_leaves() -> None:
    sc, kinds, values, _ = channel("inflow_normal")
    s = solver_of(sc, kinds, values, "persistent")
    v0 = s.volume_fp64()
    run(s, 120.0)
    vol = s.download_open_volumes()
    went_in, went_out = vol[0, 1], vol[1, 0]
    assert went_in == pytest.approx(0.25 * 200.0 * 120.0, rel=1e-6)
    assert went_out > 0.0
    assert abs(v0 + went_in - went_out - s.volume_fp64()) / v0 < 1e-7
    # the run continues as a phase: conditions change, volumes keep accumulating
    s.set_open_conditions(kinds, np.where(kinds == OPEN_INFLOW, 0.1, values).astype(np.float32))
    s.run(t_end=150.0, output_interval_s=10.0, dt_max=0.25, dt_init=0.01, cfl_interval=1, progress=False, resume=True,
          t_start=120.0)
    assert s.download_open_volumes()[0, 1] == pytest.approx(0.25 * 200.0 * 120.0 + 0.1 * 200.0 * 30.0, rel=1e-6)


def test_inflow_only_forces_blocks_while_it_flows() -> None:
    sc, kinds, values, _ = channel("inflow_dry")
    s = solver_of(sc, kinds, np.zeros_like(values))
    assert s.download_block_flags()[:, 2].sum() == 0
    s.set_open_conditions(kinds, values)
    assert s.download_block_flags()[:, 2].sum() > 0
    s.set_open_conditions(np.zeros_like(kinds), np.zeros_like(values))
    assert s.download_block_flags()[:, 2].sum() == 0


def test_the_first_step_sees_the_water_waiting_beyond_a_stage() -> None:
    sc, kinds, values, _ = channel("stage_free")
    s = solver_of(sc, kinds, np.where(kinds == OPEN_STAGE, 20.0, 0.0).astype(np.float32))
    s.run(t_end=1.0, output_interval_s=1.0, dt_max=1.0, dt_init=0.01, cfl_interval=1, progress=False)
    assert s.steps_total >= 3


def test_repeat_runs_are_bit_identical() -> None:
    sc, kinds, values, t_end = channel("stage_free")
    s = solver_of(sc, kinds, values, "persistent")
    a, _ = run(s, t_end)
    va = s.download_open_volumes()
    b, _ = run(s, t_end)
    np.testing.assert_array_equal(bits(a[-1]), bits(b[-1]))
    np.testing.assert_array_equal(va, s.download_open_volumes())


def test_an_open_mesh_checks_the_two_sum_even_uncompensated(monkeypatch) -> None:
    """The open-edge tallies are two-sums: the guard runs for an open mesh with compensated off
    (the reference's ``compensated or n_open``, gpu_resident_batch.py:659-660)."""
    sc, kinds, values, t_end = channel("draining")
    s = solver_of(sc, kinds, values)
    s.compensated = False
    probes = []

    def lost():
        probes.append(1)
        return np.array([1.0, 1e-9, 0.0], np.float32)

    monkeypatch.setattr(s, "_eft_probe", lost)
    with pytest.raises(RuntimeError, match="error-free arithmetic is broken"):
        run(s, 1.0)
    assert probes and s.steps_total == 0
