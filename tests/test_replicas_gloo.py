"""The multi-rank plumbing of ``bench.py --gpus N`` on CPU ranks (``gloo``, world size 2).

The single-mesh path does not shard: N ranks run N independent replicas, and
the only collectives are a barrier around the timed region and the maximum of
the ranks' times. The reference arm prints from rank 0 alone.
"""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return int(s.getsockname()[1])


def _rank(rank: int, world: int, port: int, out) -> None:
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        out.put((rank, bench.reduce_max(1.5 + rank, world), bench.reduce_max(10.0 - rank, world)))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_on_two_gloo_ranks() -> None:
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(out.get(timeout=5) for _ in range(2))
    assert got == [(0, 2.5, 10.0), (1, 2.5, 10.0)]  # every rank sees the slowest time


def test_reference_arm_prints_from_rank_zero_only(capsys: pytest.CaptureFixture[str]) -> None:
    sys.path.insert(0, str(ROOT))
    import bench

    sys_argv = sys.argv
    try:
        sys.argv = ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "3", "--warmup", "3"]
        args = bench.parse_args()
    finally:
        sys.argv = sys_argv
    bench.run_reference(args, world=2, rank=1)  # no pool, no work, no line
    assert capsys.readouterr().out == ""


def test_single_rank_needs_no_process_group() -> None:
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.reduce_max(3.25, 1) == 3.25
    bench.barrier(1)
