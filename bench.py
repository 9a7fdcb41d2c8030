#!/usr/bin/env python
"""Benchmark of the B200 shallow-water step (one JSON line on rank 0).

Workload (default): the 1M-cell forward run -- a seeded Voronoi mesh over a
10 km square on fractal terrain (beta 2, 20 m relief, 3 m channel), a 4 m
circular dam of 500 m radius, n = 0.035, float32 state, CFL 0.8 per step.
A step is one Heun step of the whole mesh (blocks outside the two-ring of
wet blocks are skipped, as in the reference's resident backend).

* ``value``: cells x steps / device time of exactly ``--steps`` steps after
  ``--warmup`` steps, inputs resident in HBM, steps replayed as CUDA graphs.
* ``computed_cell_steps_per_s``: the same over the cells actually computed.
* ``roofline``: the fused stage kernel's algorithmic bytes over its mean
  launch time (CUDA events recorded inside the graphs), against the measured
  HBM copy bandwidth.
* ``e2e``: the same metric through the public ``run()`` call with host
  arrays: upload of the initial state, the run, control-block reads after
  every submit, download of the final state.
* ``cpu_baseline``: the float64 oracle step timed on one host core on the
  same mesh; its result also gives the stated float64 error of the CUDA step.

Other workloads (``--workload``): ``full_wet`` and ``one_cell`` on the same
mesh (every block active; a single wet cell), ``lake_at_rest`` (8k cells over
1 km, six Gaussian bumps under a 1 m surface, CFL 0.9) and ``rain_inflow``
(4M cells over 20 km, 40 m relief, n log-uniform in [0.02, 0.08], 50 mm/h
rain on every cell plus a triangular inflow of 200 m^3/s peak; timed after a
spin-up in which the rain wets the mesh).

``--impl reference`` times the reference's CPU step (its float64 NumPy
restatement) on all host cores instead; under torchrun only rank 0 works.
With N GPUs every rank runs an independent replica (the single-mesh path
does not shard): ``value`` is the sum of the replicas' cell-steps over the
slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-steps/s fwd and fwd+adjoint, plain vs batched, at stated FP64-oracle error"
UNIT = "cell-steps/s"
L2_BYTES = 126 * 2**20
SENTINEL_STOP = 1 << 62
# workload: default cells and seed
WORKLOADS = {
    "dam_break": (1_000_000, 2),
    "full_wet": (1_000_000, 2),
    "one_cell": (1_000_000, 2),
    "lake_at_rest": (8_000, 1),
    "rain_inflow": (4_000_000, 3),
}


def parse_args() -> argparse.Namespace:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="dam_break")
    ap.add_argument("--cells", type=int, default=None, help="mesh cells (default: the workload's)")
    ap.add_argument("--seed", type=int, default=None, help="mesh and terrain seed (default: the workload's)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--chunk", type=int, default=500, help="steps per captured graph in the timed region")
    ap.add_argument("--kernel", choices=["auto", "tiled", "plain", "staged", "persistent"], default="auto",
                    help="stage kernel variant (auto: by the active fraction after the prologue)")
    ap.add_argument("--ctas-per-sm", type=int, default=None, help="persistent CTAs per SM of the stage kernel")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-scenarios measurement")
    ap.add_argument("--batch-count", type=int, default=64, help="scenarios in the batched measurement")
    ap.add_argument("--batch-steps", type=int, default=2000, help="steps of every scenario in the batched measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the forward+adjoint measurement")
    ap.add_argument("--adjoint-cells", type=int, default=250_000)
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    ap.add_argument("--spin-up", type=float, default=60.0,
                    help="rain_inflow: simulated seconds run before the timed steps")
    ap.add_argument("--start-at", type=float, default=0.0,
                    help="forward workloads: simulated seconds run through run() first; the timed steps then go on "
                         "from that state with a fresh clock (no e2e)")
    ap.add_argument("--no-hour", action="store_true", help="skip the whole simulated hour of the dam break")
    ap.add_argument("--no-horizon", action="store_true", help="skip the float64 error at 8, 64 and 512 steps")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the lake-at-rest and rain-plus-inflow configurations of the default line")
    ap.add_argument("--adjoint-fd", action="store_true",
                    help="only check the adjoint at 250k cells against float64 central differences and print that")
    ap.add_argument("--fd-steps", type=int, default=200, help="--adjoint-fd: steps of the checked run")
    ap.add_argument("--fd-directions", type=int, default=20, help="--adjoint-fd: random directions")
    ap.add_argument("--fd-eps", default="1e-2,3e-3",
                    help="--adjoint-fd: the two step sizes of the central differences (a direction counts as smooth "
                         "where they agree)")
    args = ap.parse_args()
    cells, seed = WORKLOADS[args.workload]
    args.cells = cells if args.cells is None else args.cells
    args.seed = seed if args.seed is None else args.seed
    return args


# -- workload ----------------------------------------------------------------------------------
def build_scenario(name: str, cells: int, seed: int):
    from inundation_b200 import scenarios

    if name == "lake_at_rest":
        return scenarios.lake_at_rest(cells, seed=seed, side=1000.0 * np.sqrt(cells / 8000))
    if name == "rain_inflow":
        return scenarios.rain_inflow(cells, seed=seed, side=20_000.0 * np.sqrt(cells / 4_000_000))
    side = 10_000.0 * np.sqrt(cells / 1_000_000)
    sc = scenarios.dam_break(cells, seed=seed, side=side)
    if name == "full_wet":
        # Every block active for the whole run: still water 1 m over the highest bed plus a current.
        zb = sc.geom.zb.astype(np.float64)
        h = (float(zb.max()) + 1.0 - zb).astype(np.float32)
        x = sc.geom.world_centroid[:, 0]
        sc.h0 = h
        sc.hu0 = (0.2 * np.sin(2 * np.pi * x / side) * h).astype(np.float32)
        sc.name = "full_wet"
    elif name == "one_cell":
        # A single wet cell: the launch latency of a step with a handful of active blocks.
        h = np.zeros(sc.geom.N, np.float32)
        h[sc.geom.N // 2] = 1.0
        sc.h0 = h
        sc.name = "one_cell"
    return sc


WORKLOAD_TEXT = {
    "dam_break": {"terrain": "fractal beta 2, 20 m relief, 3 m channel",
                  "water": "4 m depth within 500 m of the centre, dry outside", "manning_n": 0.035},
    "full_wet": {"terrain": "fractal beta 2, 20 m relief, 3 m channel", "water": "still water + current, all wet",
                 "manning_n": 0.035},
    "one_cell": {"terrain": "fractal beta 2, 20 m relief, 3 m channel", "water": "one wet cell (1 m), dry elsewhere",
                 "manning_n": 0.035},
    "lake_at_rest": {"terrain": "six Gaussian bumps (0.2-0.8 m, sigma 50-150 m) on a flat bed",
                     "water": "still surface at 1 m, zero momentum", "manning_n": 0.03},
    "rain_inflow": {"terrain": "fractal beta 2, 40 m relief, 3 m channel",
                    "water": "initially dry; 50 mm/h rain on every cell, triangular inflow (200 m^3/s at 20 min) "
                             "at the highest cell", "manning_n": "log-uniform in [0.02, 0.08]"},
}


def workload_config(sc, args, cfl: float = 0.8) -> dict:
    g = sc.geom
    from inundation_b200.layout import algorithmic_bytes_per_cell_step

    per_step = algorithmic_bytes_per_cell_step(g) * g.N
    l2 = (f"inputs larger than L2: {per_step / 2**20:.0f} MiB algorithmic traffic per full step, "
          f"{L2_BYTES // 2**20} MiB L2; no flush") if per_step > L2_BYTES else (
          f"inputs fit in L2 ({per_step / 2**20:.1f} MiB algorithmic traffic per full step, "
          f"{L2_BYTES // 2**20} MiB L2): latency-bound steps, no flush")
    return {
        "workload": f"{sc.name}_{g.N // 1000}k_voronoi",
        "cells": int(g.N),
        "edges": int(g.E),
        "csr_slots": int(g.cell_edge_ptr[-1]),
        "max_degree": int(g.max_degree),
        **WORKLOAD_TEXT.get(sc.name, {}),
        "cfl": cfl,
        "active_set": True,
        "compensated": True,
        "seed": args.seed,
        "l2": l2,
        "parallelism": f"replicas{args.gpus}" if args.gpus > 1 else "single",
    }


# -- clocks ------------------------------------------------------------------------------------
class ClockSampler:
    """``nvidia-smi`` clock and throttle samples every 200 ms while running."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
        "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
        "clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index: int) -> None:
        self.index = index
        self.proc: subprocess.Popen | None = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL,
            )
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.file.flush()
        rows = [r.split(", ") for r in Path(self.file.name).read_text().strip().splitlines() if r.count(",") >= 8]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        load = sorted(sm)[len(sm) // 2:] if sm else []
        return {
            "sm_mhz": float(np.median(load)) if load else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": reasons,
            "samples": len(rows),
        }


# -- distributed plumbing ---------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    return world, rank, local


def reduce_max(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"  # gloo (the CPU tests) reduces host tensors
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def peaks() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# -- CUDA arm ------------------------------------------------------------------------------------
def plan(solver, sc) -> None:
    from inundation_b200.tuning import dt_to_ticks

    c = solver._ctrl
    c[...] = 0
    c["stop_ticks"] = SENTINEL_STOP
    c["dt_max_ticks"] = dt_to_ticks(sc.dt_max)
    c["dry_dt_ticks"] = dt_to_ticks(min(sc.dt_init, sc.dt_max))
    c["cfl_safety"] = solver.cfl_safety
    solver._sync_ctrl_to_device()
    solver._enqueue_prologue()
    solver._read_ctrl()


def capture_chunks(solver, steps: int, chunk: int, timed: bool):
    """Graphs covering exactly ``steps`` steps; with ``timed``, events around every stage launch."""
    import ctypes

    import torch

    from inundation_b200 import native

    graphs, events = [], []
    if solver.stage_kernel == "persistent":
        # one cooperative launch per chunk; its phases are not separate launches to time
        left = steps
        while left > 0:
            n = min(chunk, left)
            left -= n
            graphs.append(solver._graph(n))
        return graphs, events
    params, sources = solver._params(), solver._sources()
    mesh, state = ctypes.byref(solver._mesh), ctypes.byref(solver._state)
    left = steps
    while left > 0:
        n = min(chunk, left)
        left -= n
        g = torch.cuda.CUDAGraph()
        ev = [torch.cuda.Event(enable_timing=True, external=True) for _ in range(3 * n + 1)] if timed else []
        solver._stream.synchronize()
        with torch.cuda.graph(g, stream=solver._stream):
            st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            for k in range(n):
                if timed:
                    ev[3 * k].record()
                native.check(solver._lib.swe_stage(mesh, state, ctypes.byref(params), 0, st), "stage 0")
                if timed:
                    ev[3 * k + 1].record()
                native.check(solver._lib.swe_stage(mesh, state, ctypes.byref(params), 1, st), "stage 1")
                if timed:
                    ev[3 * k + 2].record()
                if sources.count:
                    native.check(solver._lib.swe_apply_sources(mesh, state, ctypes.byref(params), ctypes.byref(sources), st), "sources")
                native.check(solver._lib.swe_block_dilate_compact(mesh, state, ctypes.byref(params), 0, 1, st), "dilate")
            if timed:
                ev[3 * n].record()
        graphs.append(g)
        events.append(ev)
    return graphs, events


def cpu_baseline_and_error(sc, solver_cls, device: str) -> tuple[dict, dict]:
    """FP64 oracle steps on one core (timed) and the CUDA step's error against them."""
    import torch

    from oracle import fp64_step

    g = sc.geom
    s0 = fp64_step.State(*(a.astype(np.float64) for a in (sc.h0, sc.hu0, sc.hv0)))
    dt_cfl = fp64_step.cfl_dt(g, s0, g=9.81, dry_tol=sc.dry_tol, cfl=0.8)
    dt = 2.0 ** np.floor(np.log2(min(dt_cfl, 1.0)))
    steps = 3  # the stated error is after 3 steps; the timed sample runs on to about 10 s of CPU work
    n64 = sc.manning.astype(np.float64)
    t0 = time.perf_counter()
    fp64_step.heun_step(g, s0, n64, dt, g=9.81, dry_tol=sc.dry_tol)  # warm caches
    timed = int(np.clip(np.ceil(10.0 / max(time.perf_counter() - t0, 1e-6)), steps, 30))
    t0 = time.perf_counter()
    s = s0
    for k in range(timed):
        s = fp64_step.heun_step(g, s, n64, dt, g=9.81, dry_tol=sc.dry_tol)
        if k + 1 == steps:
            s_err = s
    wall = time.perf_counter() - t0
    solver = solver_cls(g, None, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=sc.dry_tol, device=device)
    solver.run(t_end=steps * dt, output_interval_s=steps * dt, dt_max=dt, dt_init=dt, cfl_interval=1, progress=False)
    h, hu, hv = solver.download_h_precise(), solver.download_hu(), solver.download_hv()
    del solver
    torch.cuda.empty_cache()
    cpu = {
        "value": g.N * timed / wall,
        "unit": UNIT,
        "cores": 1,
        "kind": "port",
        "source": "oracle/fp64_step.py: the reference's float64 CPU step tests/unit/_cpu_step.py restated, "
        "pinned to that file's outputs to 1e-12 by tests/golden/cpu_step.npz",
        "sample": f"{timed} float64 Heun steps (dt={dt:g} s) of the full {g.N}-cell mesh, single process, "
        f"{wall:.1f} s",
    }
    err = {
        "steps": steps,
        "dt_s": dt,
        "h_max_abs_m": float(np.abs(h - s_err.h).max()),
        "hu_max_abs": float(np.abs(hu - s_err.hu).max()),
        "hv_max_abs": float(np.abs(hv - s_err.hv).max()),
        "tolerance_h_m": 1e-5,
    }
    return cpu, err


def forward_line(args, sc, world: int, local: int):
    """Exactly ``args.steps`` steps of ``sc`` after ``args.warmup``, timed on the device: the line's
    measured keys, and the solver with the simulated seconds of the timed steps."""
    import torch

    from inundation_b200.backend import SWESolverB200Resident
    from inundation_b200.layout import algorithmic_bytes_per_cell_step

    device = f"cuda:{local}"
    g = sc.geom
    cfl = float(sc.meta.get("cfl", 0.8))
    solver = SWESolverB200Resident(g, None, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=sc.dry_tol, cfl=cfl,
                                   device=device)
    solver.stage_kernel = args.kernel
    solver.ctas_per_sm = args.ctas_per_sm
    v0 = solver.volume_fp64() if sc.name == "lake_at_rest" else None
    if args.start_at > 0.0:  # the state of a later moment of the run; the clock restarts below
        spg = solver.steps_per_graph
        solver.steps_per_graph = 500
        solver.run(t_end=args.start_at, output_interval_s=args.start_at, dt_max=sc.dt_max, dt_init=sc.dt_init,
                   cfl_interval=1, progress=False)
        solver.steps_per_graph = spg
    plan(solver, sc)
    if args.kernel == "auto":  # the choice "auto" makes for this state, fixed for the timed region
        from inundation_b200.engine import KERNELS

        args.kernel = {v: k for k, v in KERNELS.items()}[solver._kernel]
        solver.stage_kernel = args.kernel
    warm, _ = capture_chunks(solver, args.warmup, args.chunk, timed=False)
    graphs, events = capture_chunks(solver, args.steps, args.chunk, timed=True)
    for gr in warm:
        gr.replay()
    solver._stream.synchronize()
    computed0 = solver.computed_cells
    solver._read_ctrl()
    steps0, t0_ticks = int(solver._ctrl["steps"][0]), int(solver._ctrl["now_ticks"][0])

    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(solver._stream):
        start.record()
        for gr in graphs:
            gr.replay()
        end.record()
    torch.cuda.synchronize()
    clock = clocks.stop()
    barrier(world)
    ms = start.elapsed_time(end)
    ms_max = reduce_max(ms, world)

    solver._read_ctrl()
    done = int(solver._ctrl["steps"][0]) - steps0
    if done != args.steps:
        raise RuntimeError(f"timed region ran {done} real steps, expected {args.steps} (the clock stalled)")
    t_sim = (int(solver._ctrl["now_ticks"][0]) - t0_ticks) / 2**20
    computed = solver.computed_cells - computed0
    stage_ms = 0.0
    dilate_ms = 0.0
    if not events:  # the persistent kernel: whole steps in one launch
        stage_ms = ms
    for ev in events:
        n = (len(ev) - 1) // 3
        for k in range(n):
            stage_ms += ev[3 * k].elapsed_time(ev[3 * k + 1]) + ev[3 * k + 1].elapsed_time(ev[3 * k + 2])
            dilate_ms += ev[3 * k + 2].elapsed_time(ev[3 * k + 3])
    launches = 2 * args.steps if events else len(graphs)
    bpc = algorithmic_bytes_per_cell_step(g)
    alg_bytes = computed * bpc  # over all stage launches of the timed region
    achieved = alg_bytes / (stage_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    traffic = None
    tfile = ROOT / "profiles" / "stage_kernel_traffic.json"
    if tfile.exists():  # ncu DRAM bytes per computed cell-step of this kernel, scaled to a launch
        per_cell = json.loads(tfile.read_text()).get(args.kernel, {}).get("dram_bytes_per_computed_cell_step")
        if per_cell:
            traffic = per_cell * computed / launches
    value = world * g.N * args.steps / (ms_max * 1e-3)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic: seeded Voronoi mesh, fractal DEM (no real DEM or mesh files)",
        "config": {**workload_config(sc, args, cfl), **({"start_at_s": args.start_at} if args.start_at > 0.0 else {})},
        "mode": "forward, plain (one mesh per GPU)",
        "computed_cell_steps_per_s": world * computed / (ms_max * 1e-3),
        "active_fraction": computed / (g.N * args.steps),
        "simulated_s": t_sim,
        "gpu_launches": 3 * args.steps if events else len(graphs),
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "kernel": f"stage kernel, {args.kernel} (fused edge flux + gather + Heun update), both stages"
            if events else "persistent step kernel (whole steps: both stages, dilation, step control; grid barriers)",
            "algorithmic_bytes_per_cell_step": bpc,
            "launches": launches,
            "mean_launch_us": stage_ms * 1e3 / launches,
            "peak_kind": f"{peak_kind} HBM copy bandwidth",
            "stage_share_of_step": stage_ms / (stage_ms + dilate_ms),
        },
        "clocks": clock,
    }
    if v0 is not None:  # the reference's gate: |u| over cells deeper than 10 dry_tol, float64 volume drift
        h, hu, hv = solver.download_h(), solver.download_hu(), solver.download_hv()
        wet = h > 10 * sc.dry_tol
        line["lake_at_rest_check"] = {
            "steps_before_check": args.warmup + args.steps,
            "max_abs_u_mps": float(max((np.abs(hu[wet]) / h[wet]).max(), (np.abs(hv[wet]) / h[wet]).max())),
            "volume_drift_rel": abs(solver.volume_fp64() - v0) / v0,
        }
    del graphs, warm
    return line, solver, t_sim


def run_b200(args, world: int, rank: int, local: int) -> None:
    import torch

    from inundation_b200.backend import SWESolverB200Resident

    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    if args.workload == "rain_inflow":
        line = run_sources_workload(args, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    # The default line (the 1M-cell dam break on one GPU) also carries the other configurations;
    # the meshes of the 4M-cell one and the float64 error's oracle run in other processes meanwhile.
    full = args.workload == "dam_break" and world == 1 and not args.no_configs
    helpers = None
    if full or (args.workload == "dam_break" and world == 1 and not args.no_horizon):
        import concurrent.futures as cf
        import multiprocessing as mp

        helpers = cf.ProcessPoolExecutor(max_workers=2, mp_context=mp.get_context("spawn"))
    rain_future = helpers.submit(_build_timed, "rain_inflow", WORKLOADS["rain_inflow"][0],
                                 WORKLOADS["rain_inflow"][1]) if full else None
    sc = build_scenario(args.workload, args.cells, args.seed)
    line, solver, t_sim = forward_line(args, sc, world, local)
    g = sc.geom
    if not args.no_e2e and args.start_at <= 0.0:  # every replica, over the slowest rank's wall time
        e2e = e2e_run(solver, sc, t_sim, args)
        if world > 1:
            e2e["wall_s"] = reduce_max(e2e["wall_s"], world)
            e2e["value"] = world * g.N * e2e["steps"] / e2e["wall_s"]
        line["e2e"] = e2e
    del solver
    torch.cuda.empty_cache()
    horizon_job = None
    if helpers is not None and not args.no_horizon:
        horizon_job = start_error_by_horizon(sc, device, helpers)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        cpu, err = cpu_baseline_and_error(sc, SWESolverB200Resident, device)
        line["cpu_baseline"] = cpu
        line["fp64_oracle_error"] = err
    # the whole-run, batched, forward+adjoint and other-configuration figures are single-GPU
    # measurements: with N replicas the line reports the replicas' forward only
    if args.workload == "dam_break" and world == 1 and not args.no_hour:
        line["whole_run"] = run_whole_hour(sc, args, device)
    if not args.no_batch and world == 1:
        line["batched"] = run_batch(args, world, local)
    if not args.no_adjoint and world == 1:
        line["adjoint"] = run_adjoint(args, world, local)
    if full:
        line["configs"] = {
            "lake_at_rest": config_lake_at_rest(args, world, local),
            "rain_inflow": config_rain_inflow(args, world, rank, local, rain_future.result()),
        }
    if horizon_job is not None:
        line["fp64_error_by_horizon"] = finish_error_by_horizon(*horizon_job)
    if helpers is not None:
        helpers.shutdown()
    if rank == 0:
        print(json.dumps(line), flush=True)


def sub_args(args, **overrides) -> argparse.Namespace:
    """A copy of the command line for another configuration of the same run."""
    return argparse.Namespace(**{**vars(args), **overrides})


def _build_timed(name: str, cells: int, seed: int):
    """A scenario and the seconds its build took (run in a helper process)."""
    os.environ.setdefault("OMP_NUM_THREADS", "4")
    t0 = time.perf_counter()
    sc = build_scenario(name, cells, seed)
    return sc, time.perf_counter() - t0


def config_lake_at_rest(args, world: int, local: int) -> dict:
    """Configuration 1: ~8k cells over 1 km, six Gaussian bumps under a still 1 m surface, CFL 0.9,
    2000 timed steps (after the warm-up), then the reference's lake gate (max |u| over cells deeper
    than 10 dry_tol) and the float64 volume drift."""
    import torch

    cells, seed = WORKLOADS["lake_at_rest"]
    a = sub_args(args, workload="lake_at_rest", cells=cells, seed=seed, steps=2000, kernel="auto")
    sc = build_scenario("lake_at_rest", cells, seed)
    line, solver, t_sim = forward_line(a, sc, world, local)
    line["e2e"] = e2e_run(solver, sc, t_sim, a)
    del solver
    torch.cuda.empty_cache()
    keep = ("value", "ms_per_step", "steps", "warmup", "computed_cell_steps_per_s", "active_fraction",
            "simulated_s", "gpu_launches", "roofline", "lake_at_rest_check", "e2e", "config", "clocks")
    return {k: line[k] for k in keep if k in line}


def config_rain_inflow(args, world: int, rank: int, local: int, built) -> dict:
    """Configuration 3: 4M cells over 20 km, 40 m relief, rain 50 mm/h on every cell plus a
    triangular 200 m^3/s inflow, timed over 200 steps after the ``--spin-up`` seconds in which
    the rain wets the mesh (the mesh was built in a helper process meanwhile)."""
    cells, seed = WORKLOADS["rain_inflow"]
    a = sub_args(args, workload="rain_inflow", cells=cells, seed=seed, steps=max(args.steps, 200), kernel="auto")
    line = run_sources_workload(a, world, rank, local, built=built)
    drop = ("metric", "unit", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "dtype", "data")
    return {k: v for k, v in line.items() if k not in drop}


def run_whole_hour(sc, args, device: str) -> dict:
    """Configuration 2 as it is defined: the dam break over one simulated hour through ``run()``
    (output every 5 min, the kernel picked by ``stage_kernel = "auto"`` after every submit).

    The reference's whole-run convention: cells x steps over the run's wall time
    (``inundation/bench/flood_propagation.py:646``). The trajectory gives, per output
    window, the steps, the wall time, the computed (active) fraction and the steps
    each kernel ran; the switches list when "auto" changed kernel.
    """
    import torch

    from inundation_b200.backend import SWESolverB200Resident
    from inundation_b200.tuning import SIM_TICKS_PER_SECOND

    g = sc.geom
    t_end, interval = 3600.0, 300.0
    solver = SWESolverB200Resident(g, None, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=sc.dry_tol, cfl=0.8,
                                   device=device)
    solver.steps_per_graph = 500
    solver.run(t_end=1.0, output_interval_s=1.0, dt_max=sc.dt_max, dt_init=sc.dt_init, cfl_interval=1,
               progress=False)  # the two-sum probe and the first kernel's set-up, outside the timing
    solver.submit_log = log = []
    computed0 = solver.computed_cells
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    t0 = time.perf_counter()
    w0 = time.monotonic()
    snaps, times = solver.run(t_end=t_end, output_interval_s=interval, dt_max=sc.dt_max, dt_init=sc.dt_init,
                              cfl_interval=1, progress=False)
    wall = time.perf_counter() - t0
    clock = clocks.stop()
    steps = sum(r.steps for r in log)
    computed = log[-1].computed_cells - computed0 if log else 0
    per_tick = float(SIM_TICKS_PER_SECOND)
    windows = []
    prev_wall, prev_computed = w0, computed0
    for k in range(int(round(t_end / interval))):
        lo, hi = k * interval * per_tick, (k + 1) * interval * per_tick
        recs = [r for r in log if lo < r.now_ticks <= hi]
        if not recs:
            continue
        n = sum(r.steps for r in recs)
        kernels: dict[str, int] = {}
        for r in recs:
            kernels[r.kernel] = kernels.get(r.kernel, 0) + r.steps
        c = recs[-1].computed_cells - prev_computed
        windows.append({
            "t_end_s": (k + 1) * interval,
            "steps": n,
            "wall_s": recs[-1].wall_s - prev_wall,
            "active_fraction": c / (g.N * n) if n else 0.0,
            "active_blocks_max": max(r.active_blocks for r in recs if r.steps) / solver.n_blocks
            if any(r.steps for r in recs) else 0.0,
            "kernel_steps": kernels,
        })
        prev_wall, prev_computed = recs[-1].wall_s, recs[-1].computed_cells
    switches = []
    for a, b in zip(log[:-1], log[1:]):
        if a.kernel != b.kernel:
            switches.append({"t_s": a.now_ticks / per_tick, "from": a.kernel, "to": b.kernel,
                             "active_blocks": a.active_blocks / solver.n_blocks})
    volume = solver.volume_fp64()
    del solver
    torch.cuda.empty_cache()
    return {
        "workload": f"dam_break_{g.N // 1000}k_voronoi, one simulated hour",
        "simulated_s": t_end,
        "output_interval_s": interval,
        "steps": steps,
        "wall_s": wall,
        "value": g.N * steps / wall,
        "unit": UNIT,
        "ms_per_step": wall * 1e3 / steps,
        "computed_cell_steps_per_s": computed / wall,
        "mean_active_fraction": computed / (g.N * steps),
        "snapshots": len(snaps),
        "volume_final_m3": volume,
        "volume_initial_m3": float((sc.h0.astype(np.float64) * g.area.astype(np.float64)).sum()),
        "trajectory": windows,
        "kernel_switches": switches,
        "clocks": clock,
        "note": "host wall time of SWESolverB200Resident.run(t_end=3600) with the state resident: control-block "
        "reads after every 500-step submit and the 12 snapshot downloads included (the reference's whole-run "
        "convention)",
    }


# -- float64 error by horizon ---------------------------------------------------------------------
HORIZONS = (8, 64, 512)


def _fp64_region_run(region, h0, hu0, hv0, n, dts, horizons, dry_tol: float) -> dict:
    """The float64 oracle over a region of the mesh with a given dt per step (run in a helper process):
    the state at every horizon, and the deepest water on the region's rim by then."""
    sys.path.insert(0, str(ROOT))
    from oracle import fp64_step

    s = fp64_step.State(np.asarray(h0, np.float64), np.asarray(hu0, np.float64), np.asarray(hv0, np.float64))
    n64 = np.asarray(n, np.float64)
    out, rim = {}, 0.0
    t0 = time.perf_counter()
    for k, dt in enumerate(dts, start=1):
        s = fp64_step.heun_step(region, s, n64, float(dt), g=9.81, dry_tol=dry_tol)
        rim = max(rim, float(s.h[region.rim].max()) if region.rim.size else 0.0)
        if k in horizons:
            out[k] = (s.h.copy(), s.hu.copy(), s.hv.copy(), rim)
    return {"states": out, "cpu_s": time.perf_counter() - t0}


def start_error_by_horizon(sc, device: str, pool, horizons=HORIZONS):
    """The CUDA run of the dam break for max(horizons) adaptive steps, one step per submit (each step's
    dt read from the control block), and the float64 oracle's run with those dt in a helper process.

    The oracle runs over the region the water can reach by the last horizon (every cell within the
    dam's radius plus 25 m/s times the simulated time plus 100 m); cells outside it stay dry in
    both runs, which the result checks: the region's rim must stay dry in the oracle, every cell
    outside it in the CUDA run.
    """
    import torch

    from oracle import fp64_step
    from inundation_b200.backend import SWESolverB200Resident

    g = sc.geom
    solver = SWESolverB200Resident(g, None, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=sc.dry_tol, cfl=0.8,
                                   device=device)
    plan(solver, sc)
    before = int(solver._ctrl["now_ticks"][0])
    dts, states = [], {}
    for k in range(1, max(horizons) + 1):
        sub = solver._graph(1)  # "auto" may change kernel between steps; every kernel gives the same bits
        with torch.cuda.stream(solver._stream):
            sub.replay()
        solver._read_ctrl()
        now = int(solver._ctrl["now_ticks"][0])
        if now == before:
            raise RuntimeError("the error-by-horizon run made no progress")
        dts.append((now - before) / 2**20)
        before = now
        if k in horizons:
            states[k] = (solver.download_h_precise(), solver.download_hu().astype(np.float64),
                         solver.download_hv().astype(np.float64))
    del solver
    torch.cuda.empty_cache()
    xy = g.world_centroid
    centre = np.asarray(sc.meta["centre_m"], np.float64)
    reach = float(sc.meta["radius_m"]) + 25.0 * float(sum(dts)) + 100.0
    cells = np.flatnonzero(np.hypot(xy[:, 0] - centre[0], xy[:, 1] - centre[1]) <= reach)
    region = fp64_step.restrict(g, cells)
    fut = pool.submit(_fp64_region_run, region, sc.h0[cells], sc.hu0[cells], sc.hv0[cells], sc.manning[cells],
                      dts, tuple(horizons), sc.dry_tol)
    return fut, region, states, dts, reach


def finish_error_by_horizon(fut, region, states, dts, reach) -> dict:
    got = fut.result()
    outside = np.ones(states[max(states)][0].size, bool)
    outside[region.cells] = False
    rows = []
    for k, (h, hu, hv) in sorted(states.items()):
        h64, hu64, hv64, rim = got["states"][k]
        rows.append({
            "steps": k,
            "simulated_s": float(sum(dts[:k])),
            "h_max_abs_m": float(np.abs(h[region.cells] - h64).max()),
            "hu_max_abs": float(np.abs(hu[region.cells] - hu64).max()),
            "hv_max_abs": float(np.abs(hv[region.cells] - hv64).max()),
            "h_rms_wet_m": float(np.sqrt(np.mean((h[region.cells] - h64)[h64 > 0] ** 2))) if (h64 > 0).any() else 0.0,
            "h_p999_abs_m": float(np.quantile(np.abs(h[region.cells] - h64)[h64 > 0], 0.999)) if (h64 > 0).any() else 0.0,
            "cells_over_tolerance": int((np.abs(h[region.cells] - h64) > 1e-5).sum()),
            "wet_cells": int((h64 > 0).sum()),
            "oracle_rim_max_h_m": rim,
            "cuda_max_h_outside_m": float(np.abs(h[outside]).max()) if outside.any() else 0.0,
        })
    held = all(r["oracle_rim_max_h_m"] == 0.0 and r["cuda_max_h_outside_m"] == 0.0 for r in rows)
    return {
        "protocol": "CUDA float32 run of the dam break with its own adaptive dt; the float64 oracle "
        "(oracle/fp64_step.py, the reference's _cpu_step restated) from the same float32 initial state "
        "with the same dt per step; depth is h + h_lo",
        "mesh_cells": int(states[max(states)][0].size),
        "oracle_region_cells": int(region.N),
        "oracle_region_radius_m": reach,
        "region_held": held,  # no water reached the oracle region's rim, none left it in the CUDA run
        "oracle_cpu_s": got["cpu_s"],
        "tolerance_h_m": 1e-5,
        "horizons": rows,
    }


def e2e_run(solver, sc, t_sim: float, args) -> dict:
    """The public reset() + run() + download_*() calls with host arrays, timed on the host clock."""
    from inundation_b200.tuning import seconds_to_ticks

    t_end = max(seconds_to_ticks(t_sim) / 2**20, 1.0 / 2**20)
    solver.run(t_end=min(t_end, 1.0), output_interval_s=t_end, dt_max=sc.dt_max, dt_init=sc.dt_init, cfl_interval=1,
               progress=False)  # capture the submit graph outside the timed region
    before = solver.steps_total
    t0 = time.perf_counter()
    solver.reset(sc.h0, sc.hu0, sc.hv0)
    solver.run(t_end=t_end, output_interval_s=t_end, dt_max=sc.dt_max, dt_init=sc.dt_init, cfl_interval=1,
               progress=False, resume=True, t_start=0.0)
    solver.download_h(), solver.download_hu(), solver.download_hv()
    wall = time.perf_counter() - t0
    steps = solver.steps_total - before
    submits = -(-steps // solver.steps_per_graph)
    n = sc.geom.N
    # H2D: h, hu, hv and one control block; D2H: the run's initial, window-end and final depth,
    # the three final arrays, and a control block after the prologue and after every submit.
    return {
        "value": n * steps / wall,
        "unit": UNIT,
        "steps": steps,
        "wall_s": wall,
        "h2d_bytes_per_step": (12 * n + 48) / steps,
        "d2h_bytes_per_step": (24 * n + 48 * (submits + 1)) / steps,
        "path": "SWESolverB200Resident.reset(host h, hu, hv) + run(t_end) + download_h/hu/hv",
    }


def run_sources_workload(args, world: int, rank: int, local: int, built=None) -> dict:
    """Rain on every cell plus an inflow hydrograph: the sparse-sources path, timed after a spin-up.

    One ``BatchedSolver`` instance (the solver that takes hydrographs). The mesh
    starts dry; the timed steps begin once ``--spin-up`` simulated seconds have
    run, by when the rain has wetted it. The end-to-end run uploads that state
    from host arrays, restarts the clock and runs the same number of steps.
    ``built``: the scenario and its build seconds, when built beforehand.
    """
    import torch

    from inundation_b200.batch import BatchedSolver, BatchMember
    from inundation_b200.engine import KERNELS
    from inundation_b200.layout import algorithmic_bytes_per_cell_step

    device = f"cuda:{local}"
    if built is None:
        t_build = time.perf_counter()
        sc = build_scenario(args.workload, args.cells, args.seed)
        t_build = time.perf_counter() - t_build
    else:
        sc, t_build = built
    g = sc.geom
    member = BatchMember(g, sc.h0, sc.hu0, sc.hv0, sc.manning, source_rate=sc.source_rate,
                         hydrographs=sc.hydrographs)
    solver = BatchedSolver([member], dry_tol=sc.dry_tol, device=device)
    solver.stage_kernel = args.kernel
    solver.ctas_per_sm = args.ctas_per_sm
    solver.start(sc.dt_max, sc.dt_init)
    spin_steps = 0
    while float(solver.sim_time[0]) < args.spin_up:
        solver.run_steps(solver.steps_per_graph)
        spin_steps += solver.steps_per_graph
        if spin_steps > 200_000:
            raise RuntimeError("the spin-up did not reach its simulated time")
    t_spun = float(solver.sim_time[0])
    spun = {name: solver.download_state(name) for name in ("h", "hu", "hv")}
    if args.kernel == "auto":  # the choice "auto" makes for this state, fixed for the timed region
        solver.stage_kernel = {v: k for k, v in KERNELS.items()}[solver._kernel]
    kernel = solver.stage_kernel
    _timed_steps(solver, args.warmup, max(1, args.warmup))
    computed0 = solver.computed_cells
    steps0 = solver.steps.copy()
    t0_sim = float(solver.sim_time[0])
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ms = _timed_steps(solver, args.steps, args.chunk)
    clock = clocks.stop()
    barrier(world)
    ms_max = reduce_max(ms, world)
    done = solver.steps - steps0
    if int(done[0]) != args.steps:
        raise RuntimeError(f"timed region ran {int(done[0])} real steps, expected {args.steps}")
    computed = solver.computed_cells - computed0
    t_sim = float(solver.sim_time[0]) - t0_sim
    bpc = algorithmic_bytes_per_cell_step(g)
    peak, peak_kind = peaks()
    achieved = computed * bpc / (ms * 1e-3) / 1e9
    stage_launches = 2 * args.steps if kernel != "persistent" else -(-args.steps // args.chunk)
    traffic = None
    tfile = ROOT / "profiles" / "stage_kernel_traffic.json"
    if tfile.exists():
        per_cell = json.loads(tfile.read_text()).get(kernel, {}).get("dram_bytes_per_computed_cell_step")
        if per_cell:
            traffic = per_cell * computed / stage_launches
    per_step_launches = {"persistent": 0, "plain": 5, "staged": 5, "tiled": 5}[kernel]  # stages, sources (2), dilation

    # End to end through the public calls: the spun-up state from host arrays, a clock restart, the
    # same number of steps (the timed region's graphs, already captured), the final depth back.
    zeros = np.zeros(g.N, np.float32)
    solver._stream.synchronize()
    t0 = time.perf_counter()
    for name in ("h", "hu", "hv"):
        solver.upload_state(name, spun[name])
    solver.upload_state("h_lo", zeros)
    solver.start(sc.dt_max, sc.dt_init)
    e2e_steps0 = solver.steps.copy()
    solver.run_steps(args.steps)
    final_h = solver.download_h(0)
    e2e_done = int((solver.steps - e2e_steps0)[0])
    e2e_wall = time.perf_counter() - t0
    del final_h
    line = {
        "metric": METRIC,
        "value": world * g.N * args.steps / (ms_max * 1e-3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic: seeded Voronoi mesh, fractal DEM, seeded roughness (no real DEM or mesh files)",
        "config": {**workload_config(sc, args), "spin_up_s": t_spun, "spin_up_steps": spin_steps,
                   "sources": int(np.count_nonzero(sc.source_rate)), "hydrographs": len(sc.hydrographs)},
        "mode": "forward with sources, plain (one mesh per GPU)",
        "computed_cell_steps_per_s": world * computed / (ms_max * 1e-3),
        "active_fraction": computed / (g.N * args.steps),
        "simulated_s": t_sim,
        "gpu_launches": per_step_launches * args.steps if kernel != "persistent" else stage_launches,
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "kernel": f"whole step ({kernel} stage kernel, sources, dilation): algorithmic bytes of the stages "
                      "over the step time",
            "algorithmic_bytes_per_cell_step": bpc,
            "launches": stage_launches,
            "peak_kind": f"{peak_kind} HBM copy bandwidth",
        },
        "clocks": clock,
        "e2e": {
            "value": g.N * e2e_done / e2e_wall,
            "unit": UNIT,
            "steps": e2e_done,
            "wall_s": e2e_wall,
            "h2d_bytes_per_step": (16 * g.N + 48) / max(e2e_done, 1),
            "d2h_bytes_per_step": (4 * g.N + 3 * (48 + 64)) / max(e2e_done, 1),
            "path": "BatchedSolver.upload_state(host h, hu, hv, h_lo) + start + run_steps + download_h",
        },
        "build_s": t_build,
    }
    del solver
    torch.cuda.empty_cache()
    return line


# -- batched scenarios -------------------------------------------------------------------------------
def _batch_scenario(n_seed: tuple[int, int]):
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, str(ROOT))
    from inundation_b200 import scenarios

    return scenarios.batch_member(*n_seed)


def build_batch(count: int) -> list:
    """The batched workload: ``count`` seeded scenarios, N log-uniform in [20k, 500k], built in parallel."""
    import multiprocessing as mp

    from inundation_b200 import scenarios

    sizes = scenarios.batch_sizes(count)
    jobs = [(n, 1000 + i) for i, n in enumerate(sizes)]
    procs = max(1, min(os.cpu_count() or 1, 16, count))
    with mp.get_context("spawn").Pool(procs) as pool:
        return pool.map(_batch_scenario, jobs, chunksize=1)


def _timed_steps(solver, steps: int, graph_steps: int) -> float:
    """Device milliseconds of ``steps`` steps replayed as graphs of ``graph_steps`` (captured beforehand)."""
    import torch

    solver.steps_per_graph = graph_steps
    full, rest = divmod(steps, graph_steps)
    graphs = ([solver._graph()] * full) + ([solver._graph(rest)] if rest else [])
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(solver._stream):
        ev0.record(solver._stream)
        for g in graphs:
            g.replay()
        ev1.record(solver._stream)
    ev1.synchronize()
    return ev0.elapsed_time(ev1)


def run_batch(args, world: int, local: int) -> dict:
    """Batched forward against the same scenarios run one at a time (both on this GPU).

    Every scenario: a seeded Voronoi mesh of N cells (log-uniform in
    [20k, 500k]) at 10 m spacing on its own fractal DEM, n uniform in
    [0.02, 0.06], initially dry, fed by a triangular inflow hydrograph
    (peak 10-300 m^3/s at 20 min) at its highest cell; ``--batch-steps``
    steps each, every scenario with its own CFL dt.
    """
    import torch

    from inundation_b200.batch import BatchedSolver, BatchMember, autotune
    from inundation_b200.layout import algorithmic_bytes_per_cell_step

    t_build = time.perf_counter()
    scs = build_batch(args.batch_count)
    t_build = time.perf_counter() - t_build
    members = [BatchMember(s.geom, s.h0, s.hu0, s.hv0, s.manning, hydrographs=s.hydrographs) for s in scs]
    cells = int(sum(s.geom.N for s in scs))
    steps = args.batch_steps
    dt_max, dt_init = scs[0].dt_max, scs[0].dt_init
    device = f"cuda:{local}"

    solver = BatchedSolver(members, device=device)
    tune = autotune(solver, dt_max=dt_max, dt_init=dt_init, steps=40)
    solver.reset()
    solver.start(dt_max, dt_init)
    _timed_steps(solver, args.warmup, max(1, args.warmup))  # warm-up steps, not timed
    computed0 = solver.computed_cells
    steps0 = solver.steps.copy()
    clocks = ClockSampler(local)
    clocks.start()
    ms = _timed_steps(solver, steps, 200)
    clock = clocks.stop()
    done = solver.steps - steps0
    if not (done == steps).all():
        raise RuntimeError(f"batched run: scenarios ran {sorted(set(done.tolist()))} steps, expected {steps}")
    computed = solver.computed_cells - computed0
    ms_max = reduce_max(ms, world)
    bpc = algorithmic_bytes_per_cell_step([s.geom for s in scs])
    peak, peak_kind = peaks()

    # End to end through the public calls: host initial states in, final depths out.
    t0 = time.perf_counter()
    solver.reset()
    solver.start(dt_max, dt_init)
    solver.run_steps(steps)
    finals = [solver.download_h(i) for i in range(solver.n_inst)]
    n_done = solver.steps
    e2e_wall = time.perf_counter() - t0
    if not (n_done == steps).all():
        raise RuntimeError("batched end-to-end run stalled")
    del finals
    kernel = solver.stage_kernel
    launches_per_step = 3 + (2 if solver._src_count else 0)  # stages, dilation (+ source increments and bounds)
    del solver
    torch.cuda.empty_cache()

    # The same scenarios one at a time, each with its own solver and graphs.
    plain_ms = 0.0
    plain_computed = 0
    for m in members:
        one = BatchedSolver([m], device=device)
        one.stage_kernel = kernel
        one.start(dt_max, dt_init)
        _timed_steps(one, args.warmup, max(1, args.warmup))
        c0 = one.computed_cells
        plain_ms += _timed_steps(one, steps, 200)
        plain_computed += one.computed_cells - c0
        del one
    torch.cuda.empty_cache()
    value = world * cells * steps / (ms_max * 1e-3)
    achieved = computed * bpc / (ms * 1e-3) / 1e9
    return {
        "workload": f"batch{args.batch_count}_voronoi_inflow",
        "scenarios": args.batch_count,
        "cells": cells,
        "steps_per_scenario": steps,
        "value": value,
        "unit": UNIT,
        "ms_per_step": ms_max / steps,
        "computed_cell_steps_per_s": world * computed / (ms_max * 1e-3),
        "active_fraction": computed / (cells * steps),
        "achieved_gbs_over_step": achieved,
        "hbm_frac_of_step": achieved / peak,
        "peak_kind": f"{peak_kind} HBM copy bandwidth",
        "plain": {
            "value": cells * steps / (plain_ms * 1e-3),
            "ms_total": plain_ms,
            "computed_cell_steps_per_s": plain_computed / (plain_ms * 1e-3),
            "note": "each scenario alone through the same kernels, one after another",
        },
        "speedup_vs_plain": plain_ms / ms,
        "autotune": {"stage_kernel": tune["stage_kernel"], "ctas_per_sm": tune["ctas_per_sm"],
                     "candidates": [(r["stage_kernel"], r["ctas_per_sm"], round(r["ms_per_step"], 5))
                                    for r in tune["results"]]},
        "e2e": {
            "value": cells * steps / e2e_wall,
            "unit": UNIT,
            "wall_s": e2e_wall,
            "h2d_bytes_per_step": (12 * cells + 48 * args.batch_count) / steps,
            "d2h_bytes_per_step": (4 * cells + 2 * 48 * args.batch_count) / steps,
            "path": "BatchedSolver.reset(host states) + start + run_steps + download_h per scenario",
        },
        "build_s": t_build,
        "gpu_launches": launches_per_step * steps,
        "clocks": clock,
    }


# -- forward + adjoint --------------------------------------------------------------------------------
def _adjoint_problem(cells: int, steps: int, knots: int, gauges: int, device: str, seed: int = 5,
                     checkpoint_every: int = 50):
    from inundation_b200.adjoint import GaugeCalibration
    from inundation_b200.scenarios import calibration

    sc = calibration(cells, seed=seed, knots=knots, gauges=gauges)
    prob = GaugeCalibration(sc.geom, sc.h0, sc.hu0, sc.hv0, gauges=sc.meta["gauges"], steps=steps,
                            hydrographs=sc.hydrographs, checkpoint_every=checkpoint_every, dt_max=sc.dt_max,
                            dt_init=sc.dt_init, device=device)
    prob.cut_depth = 4.0 * sc.dry_tol
    z = sc.geom.zb.astype(np.float32)
    q = sc.hydrographs[0].knot_q.astype(np.float32)
    prob.observe(sc.meta["n_true"], z, q)
    return sc, prob, sc.manning.copy(), z, q


def _gradient_error(device: str) -> dict:
    """The CUDA gradient against float64 torch autograd of the same discrete step (dt frozen, the
    same film-depth cut), on a 4000-cell instance of the calibration problem over 120 steps. Each
    model is compared on its own observations (the float64 reference recomputes the gauge depths
    of the "true" run with that run's clock), so residuals share each model's rounding. The
    float64 reference runs on the host CPU."""
    import torch

    from oracle.torch_step import TorchStep, hydrograph_value, misfit

    sc, prob, n, z, q = _adjoint_problem(4000, 120, 8, 40, device, seed=7)
    true_dts, true_ts = prob.clock()
    loss32 = prob.loss(n, z, q)
    gn, gz, gq = prob.gradient()
    dts, ts = prob.clock()
    g = sc.geom
    model = TorchStep(g, dry_tol=sc.dry_tol, cut_depth=prob.cut_depth)
    t64 = lambda a: torch.as_tensor(np.asarray(a, np.float64))  # noqa: E731
    hg = sc.hydrographs[0]
    cells = torch.as_tensor(np.asarray(hg.cells, np.int64))
    hscale = t64((hg.shares() * (1.0 / np.asarray(g.area, np.float32)[hg.cells]).astype(np.float32)).astype(np.float64))
    gauges = torch.as_tensor(np.asarray(sc.meta["gauges"], np.int64))
    obs = []
    with torch.no_grad():
        dzL, dzR = model.bed_steps(t64(z))
        h, hu, hv = t64(sc.h0), t64(sc.hu0), t64(sc.hv0)
        for dt, t in zip(true_dts, true_ts, strict=True):
            h, hu, hv = model.step(h, hu, hv, t64(sc.meta["n_true"]), dzL, dzR, dt, cells,
                                   hscale * hydrograph_value(t64(hg.knot_t), t64(q), t))
            obs.append(h[gauges].numpy().copy())
    n_t, z_t, q_t = (t64(v).requires_grad_(True) for v in (n, z, q))
    loss = misfit(model, t64(sc.h0), t64(sc.hu0), t64(sc.hv0), n_t, z_t, q_t, dts, ts, gauges, t64(np.array(obs)),
                  hydro=[(cells, hscale, t64(hg.knot_t), slice(0, hg.knot_q.size))])
    loss.backward()
    rel = lambda a, b: float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))  # noqa: E731
    return {
        "reference": "float64 torch autograd of the same discrete step, dt frozen, same film-depth cut; "
        "4000 cells, 120 steps, 8 knots, 40 gauges",
        "loss_rel": abs(loss32 - float(loss.detach())) / float(loss.detach()),
        "grad_rel_n": rel(gn, n_t.grad.numpy()),
        "grad_rel_z": rel(gz, z_t.grad.numpy()),
        "grad_rel_q": rel(gq, q_t.grad.numpy()),
        "tolerance": 1e-3,
    }


def run_adjoint(args, world: int, local: int) -> dict:
    """Forward and forward+adjoint of the calibration problem, device time of each.

    A seeded 250k-cell Voronoi mesh (10 m spacing) on a fractal DEM, a 1 m pond and a
    triangular inflow hydrograph of 32 knots, 200 gauges, 2000 steps; the misfit against a run
    with a seeded Manning field, its gradient with respect to n, bed and knots with a
    checkpoint every 50 steps.
    """
    import torch

    device = f"cuda:{local}"
    sc, prob, n, z, q = _adjoint_problem(args.adjoint_cells, args.adjoint_steps, 32, 200, device)
    prob.loss(n, z, q)  # capture the graphs and warm up
    prob.backward()
    prob.set_parameters(n, z, q)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    ev[0].record(prob._stream)
    prob._run(record=0, checkpoints=False)
    ev[1].record(prob._stream)
    ev[1].synchronize()
    ev[2].record(prob._stream)
    prob._run(record=0, checkpoints=True)
    prob._has_forward = True
    prob.backward()
    ev[3].record(prob._stream)
    ev[3].synchronize()
    fwd_ms = ev[0].elapsed_time(ev[1])
    both_ms = ev[2].elapsed_time(ev[3])
    gn, gz, gq = prob.gradient()
    cells, steps = int(sc.geom.N), prob.steps
    out = {
        "workload": f"calibration_{cells // 1000}k_voronoi",
        "cells": cells,
        "steps": steps,
        "gauges": int(prob.gauges.size),
        "knots": prob.n_knots,
        "checkpoint_every": prob.K,
        "fwd_ms": fwd_ms,
        "fwd_adj_ms": both_ms,
        "fwd_cell_steps_per_s": cells * steps / (fwd_ms * 1e-3),
        "fwd_adj_cell_steps_per_s": cells * steps / (both_ms * 1e-3),
        "ratio_fwd_adj_over_fwd": both_ms / fwd_ms,
        "target_ratio": 4.0,
        "grad_norms": {"n": float(np.linalg.norm(gn)), "z": float(np.linalg.norm(gz)), "q": float(np.linalg.norm(gq))},
        "grad_finite": bool(np.isfinite(gn).all() and np.isfinite(gz).all() and np.isfinite(gq).all()),
        "cut_depth_m": prob.cut_depth,
        "note": "fwd = the misfit run alone; fwd+adj = the run with checkpoints, then every segment taped "
        "again and reversed",
    }
    del prob
    torch.cuda.empty_cache()
    out["gradient_error"] = _gradient_error(device)
    return out


def adjoint_fd_check(args, local: int) -> dict:
    """The adjoint of the calibration problem at its benchmark size (250k cells, 32 knots, 200
    gauges, checkpoints every 50 steps) over a shorter run (``--fd-steps``), against float64:

    * directional derivatives along ``--fd-directions`` seeded random directions of (n, z, q)
      by central differences of the float64 loss (the same discrete step in float64 on the GPU,
      ``oracle/torch_step.py``, with the CUDA run's dt frozen), at the two step sizes of
      ``--fd-eps``, the direction counted as smooth where they agree to 1e-2 (with wetting fronts
      the loss has kinks: too small a step measures them instead of the slope);
    * the CUDA gradient (derivatives cut below the film depth, 4 dry_tol) against those
      differences of the exact loss: the cut surrogate's bias and the float32 error together;
    * float64 autograd with the same cut against the same differences (the bias alone) and
      against the CUDA gradient (the implementation's error alone).
    Errors are relative to the summed size of the n, z and q terms of a direction.
    """
    import torch

    from oracle.torch_step import TorchStep, hydrograph_value, misfit

    device = f"cuda:{local}"
    t_all = time.perf_counter()
    sc, prob, n, z, q = _adjoint_problem(args.adjoint_cells, args.fd_steps, 32, 200, device)
    true_dts, true_ts = prob.clock()
    loss32 = prob.loss(n, z, q)
    gn, gz, gq = prob.gradient()
    dts, ts = prob.clock()
    g = sc.geom
    t64 = lambda a: torch.as_tensor(np.asarray(a, np.float64), device=device)  # noqa: E731
    hg = sc.hydrographs[0]
    cells = torch.as_tensor(np.asarray(hg.cells, np.int64), device=device)
    hscale = t64((hg.shares() * (1.0 / np.asarray(g.area, np.float32)[hg.cells]).astype(np.float32)).astype(np.float64))
    hydro = [(cells, hscale, t64(hg.knot_t), slice(0, hg.knot_q.size))]
    gauges = torch.as_tensor(np.asarray(sc.meta["gauges"], np.int64), device=device)
    exact = TorchStep(g, dry_tol=sc.dry_tol, device=device)
    cut = TorchStep(g, dry_tol=sc.dry_tol, device=device, cut_depth=prob.cut_depth)
    with torch.no_grad():  # the float64 model's own observations, with the "true" run's clock
        dzL, dzR = exact.bed_steps(t64(z))
        h, hu, hv = t64(sc.h0), t64(sc.hu0), t64(sc.hv0)
        obs = []
        for dt, t in zip(true_dts, true_ts, strict=True):
            h, hu, hv = exact.step(h, hu, hv, t64(sc.meta["n_true"]), dzL, dzR, dt, cells,
                                   hscale * hydrograph_value(t64(hg.knot_t), t64(q), t))
            obs.append(h[gauges])
        obs = torch.stack(obs)

    def loss64(model, nn, zz, qq, grad=False):
        return misfit(model, t64(sc.h0), t64(sc.hu0), t64(sc.hv0), nn, zz, qq, dts, ts, gauges, obs, hydro=hydro,
                      checkpoint=grad)

    n_t, z_t, q_t = (t64(v).requires_grad_(True) for v in (n, z, q))
    loss_cut = loss64(cut, n_t, z_t, q_t, grad=True)
    loss_cut.backward()
    an, az, aq = (v.grad.cpu().numpy() for v in (n_t, z_t, q_t))
    n0, z0, q0 = (np.asarray(v, np.float64) for v in (n, z, q))
    eps_a, eps_b = (float(v) for v in args.fd_eps.split(","))
    rows = []
    with torch.no_grad():
        base = float(loss64(exact, t64(n0), t64(z0), t64(q0)))

        def fd(dn, dz, dq, eps):
            plus = float(loss64(exact, t64(n0 + eps * dn), t64(z0 + eps * dz), t64(q0 + eps * dq)))
            minus = float(loss64(exact, t64(n0 - eps * dn), t64(z0 - eps * dz), t64(q0 - eps * dq)))
            return (plus - minus) / (2.0 * eps)

        for k in range(args.fd_directions):
            rng = np.random.default_rng(500 + k)
            dn = rng.standard_normal(n0.size) * 0.005
            dz = rng.standard_normal(z0.size) * 0.01
            dq = rng.standard_normal(q0.size) * 2.0
            d1, d2 = fd(dn, dz, dq, eps_a), fd(dn, dz, dq, eps_b)
            cuda = (float(np.dot(gn, dn)), float(np.dot(gz, dz)), float(np.dot(gq, dq)))
            ref = (float(np.dot(an, dn)), float(np.dot(az, dz)), float(np.dot(aq, dq)))
            scale = sum(abs(v) for v in cuda)
            rows.append({
                "direction": k,
                "fd": d1,
                "fd_fine": d2,
                "smooth": abs(d1 - d2) <= 1e-2 * max(abs(d1), 1e-300),
                "cuda_cut": sum(cuda),
                "f64_cut": sum(ref),
                "err_cuda_cut_vs_fd": abs(sum(cuda) - d1) / scale,
                "err_f64_cut_vs_fd": abs(sum(ref) - d1) / scale,
                "err_cuda_vs_f64_cut": abs(sum(cuda) - sum(ref)) / scale,
            })
    smooth = [r for r in rows if r["smooth"]]
    rel = lambda a, b: float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))  # noqa: E731
    med = lambda key, rs: float(np.median([r[key] for r in rs])) if rs else None  # noqa: E731
    mx = lambda key, rs: float(np.max([r[key] for r in rs])) if rs else None  # noqa: E731
    return {
        "workload": f"calibration_{g.N // 1000}k_voronoi",
        "cells": int(g.N),
        "steps": int(prob.steps),
        "checkpoint_every": int(prob.K),
        "knots": int(prob.n_knots),
        "gauges": int(prob.gauges.size),
        "cut_depth_m": prob.cut_depth,
        "loss_f32": loss32,
        "loss_f64": base,
        "grad_rel_vs_f64_cut_autograd": {"n": rel(gn, an), "z": rel(gz, az), "q": rel(gq, aq)},
        "directions": len(rows),
        "smooth_directions": len(smooth),
        "smooth": {
            "err_cuda_cut_vs_fd_median": med("err_cuda_cut_vs_fd", smooth),
            "err_cuda_cut_vs_fd_max": mx("err_cuda_cut_vs_fd", smooth),
            "err_f64_cut_vs_fd_median": med("err_f64_cut_vs_fd", smooth),
            "err_f64_cut_vs_fd_max": mx("err_f64_cut_vs_fd", smooth),
            "err_cuda_vs_f64_cut_max": mx("err_cuda_vs_f64_cut", smooth),
        },
        "all_directions": {
            "err_cuda_cut_vs_fd_median": med("err_cuda_cut_vs_fd", rows),
            "err_f64_cut_vs_fd_median": med("err_f64_cut_vs_fd", rows),
            "err_cuda_vs_f64_cut_max": mx("err_cuda_vs_f64_cut", rows),
        },
        "rows": rows,
        "wall_s": time.perf_counter() - t_all,
        "fd_eps": [eps_a, eps_b],
        "reference": "float64 torch restatement of the same discrete step on the GPU (oracle/torch_step.py), dt "
        "frozen at the CUDA run's values; central differences of the exact (uncut) loss",
    }


# -- reference arm ---------------------------------------------------------------------------------
_WORKER: dict = {}


def _ref_worker_init(workload: str, cells: int, seed: int, spin_up: float) -> None:
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, str(ROOT))
    from oracle import fp64_step

    sc = build_scenario(workload, cells, seed)  # the workload at the sample's size, same cell size
    if workload == "rain_inflow":
        # the timed CUDA steps start from a mesh the rain has wetted: a film of the rain's depth by then
        # (the float64 step has no source term)
        sc.h0 = np.full(sc.geom.N, sc.meta["rain_m_per_s"] * spin_up, np.float32)
    s = fp64_step.State(*(a.astype(np.float64) for a in (sc.h0, sc.hu0, sc.hv0)))
    cfl = float(sc.meta.get("cfl", 0.8))
    dt = min(fp64_step.cfl_dt(sc.geom, s, g=9.81, dry_tol=sc.dry_tol, cfl=cfl), sc.dt_max)
    _WORKER.update(geom=sc.geom, state=s, n=sc.manning.astype(np.float64), dt=dt, dry=sc.dry_tol)


def _ref_worker_step(_: int) -> int:
    from oracle import fp64_step

    w = _WORKER
    w["state"] = fp64_step.heun_step(w["geom"], w["state"], w["n"], w["dt"], g=9.81, dry_tol=w["dry"])
    return int(w["geom"].N)


def run_reference(args, world: int, rank: int) -> None:
    if rank != 0:
        return
    import multiprocessing as mp

    procs = max(1, min(os.cpu_count() or 1, 64))
    budget_s = 150.0
    per_core_rate = 3.0e5
    cells = int(np.clip(budget_s * per_core_rate / (args.steps + args.warmup), 2000, args.cells))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs, initializer=_ref_worker_init,
                  initargs=(args.workload, cells, args.seed, args.spin_up)) as pool:
        # the full workload's description, as the CUDA arm states it (built while the workers start)
        full = build_scenario(args.workload, args.cells, args.seed)
        config = workload_config(full, args, float(full.meta.get("cfl", 0.8)))
        del full
        for _ in range(args.warmup):
            pool.map(_ref_worker_step, range(procs), chunksize=1)
        t0 = time.perf_counter()
        total = 0
        for _ in range(args.steps):
            total += sum(pool.map(_ref_worker_step, range(procs), chunksize=1))
        wall = time.perf_counter() - t0
    value = total / wall
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": wall * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded Voronoi mesh, fractal DEM",
        "config": config,
        "cpu_baseline": {
            "value": value,
            "unit": UNIT,
            "cores": procs,
            "kind": "port",
            "source": "oracle/fp64_step.py: the reference's float64 CPU step tests/unit/_cpu_step.py restated, "
            "pinned to that file's outputs to 1e-12 by tests/golden/cpu_step.npz (the reference keeps the step in "
            "its test tree, which a package install does not carry, so the restatement runs)",
            "sample_cells_per_process": cells,
            "processes": procs,
            "sample": f"each step: one float64 Heun step of a {cells}-cell sample of the workload (same cell "
            f"size, terrain and water) in each of {procs} processes"
            + (f"; rain_inflow: a {1000 * 0.05 / 3600 * args.spin_up:.2f} mm film for the state the rain leaves "
               f"after {args.spin_up:g} s (the float64 step has no source term)" if args.workload == "rain_inflow"
               else ""),
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    args = parse_args()
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup()
    if args.adjoint_fd:
        import torch

        torch.cuda.set_device(local)
        if rank == 0:
            print(json.dumps(adjoint_fd_check(args, local)), flush=True)
        return
    try:
        run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
