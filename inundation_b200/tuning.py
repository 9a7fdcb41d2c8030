"""Physical constants, solver defaults and the integer simulated-time clock.

Values and semantics follow the reference's ``inundation/tuning.py`` (constants
at lines 26-69, tick helpers at lines 121-152). Simulated time is a uint64
count of 2^-20 s ticks; every step's dt is a whole number of ticks no larger
than 2^24, so ``float32(ticks) * 2^-20`` is exact and the device clock advances
by exactly the dt the physics used.
"""

from __future__ import annotations

import math
import struct
from collections.abc import Iterator

GRAVITY_G = 9.81
DRY_TOL_DEFAULT = 1e-4
# dt_i = CFL * A_i / sum_j(max|S_j| * len_j) over the cell's edges, with the
# wave speeds the flux assumed (reference tuning.py:28-33).
CFL_DEFAULT = 0.8
# CFL number of backends that reuse one dt for several steps.
CFL_HOST_DRIVEN = 0.45
# Below this many dry_tol the velocity is desingularised and film momentum
# decays at a rate (reference tuning.py:37-39).
FILM_DEPTHS = 4.0

CFL_EPSILON_MIN = 1e-10
CFL_SANITY_MAX = 1e10
DT_SENTINEL = 1e30

SIM_TICKS_PER_SECOND = 1 << 20
SIM_DT_MAX_TICKS = 1 << 24

# Active-set block: this many consecutive Hilbert-ordered cells. One CUDA
# thread block owns one mesh block in every per-cell kernel.
ACTIVE_BLOCK_CELLS = 256

# Cells at or below this area get no CFL bound (reference tuning.py:88-92).
MIN_CELL_AREA = 1e-10

# Open-boundary condition codes (reference tuning.py:63-68).
OPEN_WALL = 0
OPEN_FREE = 1
OPEN_NORMAL = 2
OPEN_STAGE = 3
OPEN_INFLOW = 4

# Backend names the workflow accepts. ``b200_resident`` is the CUDA backend of
# this package; the reference's Vulkan names are accepted by the config and
# refused at ``prepare()`` because no Vulkan path exists here.
B200_BACKEND = "b200_resident"
SOLVER_IMPLS = frozenset({"baseline", "fixed_dt_batch_barrier", "gpu_resident_batch", B200_BACKEND})
MOMENTUM_SNAPSHOT_BACKENDS = frozenset({"baseline", "gpu_resident_batch", B200_BACKEND})
OPEN_BOUNDARY_BACKENDS = frozenset({"baseline", "gpu_resident_batch", B200_BACKEND})


def float_bits(value: float) -> int:
    """The uint32 bit pattern of ``value`` rounded to float32."""
    return struct.unpack("<I", struct.pack("<f", value))[0]


def bits_float(bits: int) -> float:
    """The float32 whose bit pattern is ``bits``, as a Python float."""
    return struct.unpack("<f", struct.pack("<I", bits & 0xFFFFFFFF))[0]


DT_SENTINEL_BITS = float_bits(DT_SENTINEL)


def seconds_to_ticks(seconds: float) -> int:
    """Simulated time in seconds -> nearest whole tick (reference tuning.py:121-125)."""
    if not math.isfinite(seconds) or seconds < 0.0:
        raise ValueError(f"simulated time must be finite and non-negative, got {seconds}")
    return round(seconds * SIM_TICKS_PER_SECOND)


def ticks_to_seconds(ticks: int) -> float:
    """Whole ticks -> simulated seconds (float64)."""
    return ticks / SIM_TICKS_PER_SECOND


def dt_to_ticks(dt: float) -> int:
    """A timestep -> whole ticks, rounded down so a bound is never exceeded.

    Range [1, 2^24] ticks (reference tuning.py:133-142).
    """
    if not math.isfinite(dt) or dt <= 0.0:
        raise ValueError(f"dt must be finite and positive, got {dt}")
    ticks = math.floor(dt * SIM_TICKS_PER_SECOND)
    if ticks < 1 or ticks > SIM_DT_MAX_TICKS:
        raise ValueError(
            f"dt must be between one tick and {SIM_DT_MAX_TICKS / SIM_TICKS_PER_SECOND} s, got {dt}"
        )
    return ticks


def output_window_stops(start_ticks: int, end_ticks: int, interval_ticks: int) -> Iterator[int]:
    """Stop tick of each output window: every interval after the start, then the end."""
    if interval_ticks <= 0:
        raise ValueError(f"output interval must be positive, got {interval_ticks} ticks")
    stop = start_ticks
    while stop < end_ticks:
        stop = min(stop + interval_ticks, end_ticks)
        yield stop


def num_blocks(n_cells: int, block_cells: int = ACTIVE_BLOCK_CELLS) -> int:
    """Blocks covering ``n_cells`` cells; the last may be partial."""
    if block_cells < 1:
        raise ValueError(f"block_cells must be positive, got {block_cells}")
    return -(-n_cells // block_cells)
