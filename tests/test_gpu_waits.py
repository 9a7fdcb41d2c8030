"""A bounded device wait runs out with an error status, not a hang (no GPU fault involved).

The persistent kernel's seats wait for the step control's published (dt, epoch)
pair. ``swe_dt_wait_probe`` makes that same wait once: with the pair carrying the
asked epoch it returns the dt at once; for an epoch that nothing publishes (a flag
nothing sets) it gives up after its 2 s limit, returns 0 and records error bit 4,
and the host turns the control block's error into an exception.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np
import pytest

from tests._valley import DRY_TOL, MANNING, valley_grid

pytestmark = pytest.mark.gpu


def test_a_dt_that_is_never_published_times_out_with_an_error() -> None:
    import torch

    from inundation_b200.backend import SWESolverB200Resident

    grid = valley_grid(nx=16, ny=16)
    z = np.zeros(grid.N, np.float32)
    solver = SWESolverB200Resident(grid, None, z, z, z, np.full(grid.N, MANNING, np.float32), dry_tol=DRY_TOL,
                                   device="cuda:0")
    lib = solver._lib
    out = torch.full((1,), -1, dtype=torch.int32, device="cuda:0")
    dt_bits = int(np.float32(0.25).view(np.int32))
    solver._dt_buf[2] = dt_bits  # the pair (dt, epoch 7), little-endian words 2 and 3
    solver._dt_buf[3] = 7
    torch.cuda.synchronize()
    stream = ctypes.c_void_p(solver._stream.cuda_stream)
    out_ptr = ctypes.c_void_p(out.data_ptr())

    assert lib.swe_dt_wait_probe(ctypes.byref(solver._state), 7, out_ptr, stream) == 0
    solver._stream.synchronize()
    assert int(out.item()) == dt_bits
    solver._read_ctrl()  # no error recorded

    t0 = time.perf_counter()
    assert lib.swe_dt_wait_probe(ctypes.byref(solver._state), 8, out_ptr, stream) == 0
    solver._stream.synchronize()
    waited = time.perf_counter() - t0
    assert int(out.item()) == 0
    assert 1.9 < waited < 60.0, waited
    with pytest.raises(RuntimeError, match="for a step's dt"):
        solver._read_ctrl()

