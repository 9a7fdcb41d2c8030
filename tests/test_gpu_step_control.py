"""The reference's ``step_control`` known answers on the device kernel.

The reference runs these cases through its GLSL kernel
(``tests/unit/test_gpu_resident_clock.py:118-214``); here each one fills a
48-byte control block and four dt words on the device, calls
``swe_step_control`` through the C ABI, and checks every field against the
known answer and, word for word, against the FP32 oracle's restatement.
The cases run once alone and once as instances of one launch (each
instance has its own control block and dt words).
"""

from __future__ import annotations

import ctypes
import struct

import numpy as np
import pytest

from inundation_b200.tuning import SIM_TICKS_PER_SECOND
from oracle.resident_oracle import CTRL_DTYPE, step_control

pytestmark = pytest.mark.gpu

START, STEP, RETARGET = 0, 1, 2


def _bits(v: float) -> int:
    return struct.unpack("<I", struct.pack("<f", v))[0]


def _ticks(raw: float, safety: float = 0.8) -> int:
    """Ticks from a CFL bound in float32, as the kernel computes them."""
    return int(np.float32(raw) * np.float32(safety) * np.float32(SIM_TICKS_PER_SECOND))


def _inputs(slot0: float = 0.0, slot1: float = 1e30, **fields):
    c = np.zeros(1, CTRL_DTYPE)
    c["dt_max_ticks"] = SIM_TICKS_PER_SECOND  # 1 s
    c["dry_dt_ticks"] = SIM_TICKS_PER_SECOND // 100
    c["cfl_safety"] = 0.8
    c["stop_ticks"] = 10**9
    for k, v in fields.items():
        c[k] = v
    return c, np.array([_bits(slot0), _bits(slot1), 0, 0], np.uint32)


# (name, mode, inputs, known answer: {field: value} with "dt0"/"dt1" for the dt words)
CASES = [
    ("start_takes_the_prologue_bound_with_safety", START, dict(slot0=0.05, now_ticks=123),
     dict(dt_ticks=_ticks(0.05), now_ticks=123, steps=0, dt0=_bits(_ticks(0.05) / SIM_TICKS_PER_SECOND),
          dt1=_bits(1e30))),
    ("dt_is_exactly_the_tick_count", START, dict(slot0=0.0314),
     dict(dt_ticks=_ticks(0.0314), dt0=_bits(_ticks(0.0314) / SIM_TICKS_PER_SECOND))),
    ("step_advances_by_the_previous_ticks_and_counts", STEP,
     dict(slot1=0.02, now_ticks=1000, dt_ticks=777, steps=5),
     dict(now_ticks=1777, steps=6, dt_ticks=_ticks(0.02), last_raw=np.float32(0.02))),
    ("noop_step_keeps_clock_count_and_bound", STEP, dict(now_ticks=1000, dt_ticks=0, steps=5, last_raw=0.03),
     dict(now_ticks=1000, steps=5, dt_ticks=_ticks(0.03))),
    ("retarget_replans_from_the_last_bound", RETARGET, dict(slot1=0.5, now_ticks=1000, dt_ticks=0, last_raw=0.03),
     dict(now_ticks=1000, dt_ticks=_ticks(0.03))),
    ("capped_by_dt_max", START, dict(slot0=50.0, dt_max_ticks=4096), dict(dt_ticks=4096)),
    ("last_step_lands_exactly_on_the_stop", START, dict(slot0=0.05, now_ticks=10_000, stop_ticks=10_005),
     dict(dt_ticks=5)),
    ("window_done_gives_a_zero_dt", STEP, dict(slot1=0.05, now_ticks=9_000, dt_ticks=1_000, stop_ticks=10_000),
     dict(now_ticks=10_000, dt_ticks=0, dt0=0)),
    ("all_dry_falls_back_to_the_dry_dt", START, dict(slot0=1e30, dry_dt_ticks=2048), dict(dt_ticks=2048)),
    ("degenerate_bound_stalls_instead_of_stepping", START, dict(slot0=1e-12), dict(dt_ticks=0, dt0=0)),
    ("clock_carries_past_32_bits", STEP, dict(slot1=0.05, now_ticks=2**32 - 3, dt_ticks=10, stop_ticks=2**40),
     dict(now_ticks=2**32 + 7, steps=1)),
]


def _device_step_control(ctrls: np.ndarray, dts: np.ndarray, mode: int) -> tuple[np.ndarray, np.ndarray]:
    """One launch of swe_step_control over len(ctrls) instances; returns the device's words."""
    import torch

    from inundation_b200 import native

    lib = native.load()
    c_dev = torch.from_numpy(ctrls.view(np.int64).copy()).cuda()
    d_dev = torch.from_numpy(dts.view(np.int32).copy()).cuda()
    stream = torch.cuda.current_stream()
    rc = lib.swe_step_control(c_dev.data_ptr(), d_dev.data_ptr(), len(ctrls), mode,
                              ctypes.c_void_p(stream.cuda_stream))
    native.check(rc, "swe_step_control")
    torch.cuda.synchronize()
    return c_dev.cpu().numpy().view(CTRL_DTYPE), d_dev.cpu().numpy().view(np.uint32)


def _check_known(ctrl, dt, want: dict) -> None:
    for k, v in want.items():
        if k == "dt0":
            assert int(dt[0]) == v
        elif k == "dt1":
            assert int(dt[1]) == v
        else:
            assert ctrl[k] == v, (k, ctrl[k], v)


@pytest.mark.parametrize("name, mode, inputs, want", CASES, ids=[c[0] for c in CASES])
def test_known_answer_on_the_device(name, mode, inputs, want) -> None:
    c, dt = _inputs(**inputs)
    got_c, got_dt = _device_step_control(c, dt, mode)
    _check_known(got_c[0], got_dt, want)
    oc, odt = c.copy(), dt.copy()
    step_control(oc, odt, mode)  # the oracle's restatement, word for word
    np.testing.assert_array_equal(got_c.view(np.uint64), oc.view(np.uint64))
    np.testing.assert_array_equal(got_dt, odt)
    # the dt word is the tick count exactly
    dt_s = struct.unpack("<f", struct.pack("<I", int(got_dt[0])))[0]
    assert dt_s * SIM_TICKS_PER_SECOND == int(got_c[0]["dt_ticks"])


@pytest.mark.parametrize("mode", [START, STEP, RETARGET])
def test_every_instance_keeps_its_own_clock(mode: int) -> None:
    """All cases of one mode as instances of a single launch: each gets its own answer."""
    rows = [_inputs(**inputs) for _, m, inputs, _ in CASES if m == mode]
    ctrls = np.concatenate([r[0] for r in rows])
    dts = np.concatenate([r[1] for r in rows])
    got_c, got_dt = _device_step_control(ctrls, dts, mode)
    want_c, want_dt = ctrls.copy(), dts.copy()
    for i in range(len(rows)):
        c1, d1 = want_c[i : i + 1].copy(), want_dt[4 * i : 4 * i + 4].copy()
        step_control(c1, d1, mode)
        want_c[i], want_dt[4 * i : 4 * i + 4] = c1[0], d1
    np.testing.assert_array_equal(got_c.view(np.uint64), want_c.view(np.uint64))
    np.testing.assert_array_equal(got_dt, want_dt)
    known = [w for _, m, _, w in CASES if m == mode]
    for i, w in enumerate(known):
        _check_known(got_c[i], got_dt[4 * i : 4 * i + 4], w)
