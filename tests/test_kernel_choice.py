"""The ``stage_kernel = "auto"`` rule and the persistent kernel's capacity, on a stub engine (no device).

The rule: the persistent whole-step kernel while at most a quarter of the blocks
are active, or while every active 64-cell tile has a CTA of its grid to itself
(a small mesh); the staged 256-cell block kernel otherwise, and always when the
persistent grid cannot hold a step (one seat and 512 other tiles per CTA).
Also the two-sum guard's verdict on a probe's words.
"""

from __future__ import annotations

import pytest

from inundation_b200.engine import KERNELS, PERSISTENT_EXTRA_TILES, ResidentEngine

PERSISTENT, STAGED = KERNELS["persistent"], KERNELS["staged"]


def engine(n_blocks: int, active: int, sms: int = 148, per_sm: int = 4, max_grid: int | None = None):
    e = ResidentEngine.__new__(ResidentEngine)  # the rule reads only these fields
    e.stage_kernel = "auto"
    e.n_blocks = n_blocks
    e._active_blocks = active
    e._sms = sms
    e._per_sm = {k: per_sm for k in KERNELS.values()}
    e.ctas_per_sm = None
    e.max_grid = max_grid
    e._staged_fits = True
    return e


@pytest.mark.parametrize(
    ("n_blocks", "active", "want"),
    [
        (3907, 140, PERSISTENT),  # 1M-cell dam break: 3.6 % of the blocks
        (3907, 976, PERSISTENT),  # a quarter active (976.75), no more
        (3907, 977, STAGED),  # past a quarter: issue-bound work for the block kernel
        (3907, 3907, STAGED),  # all wet
        (32, 32, PERSISTENT),  # 8k-cell lake at rest: 128 tiles, one CTA each
        (148, 148, PERSISTENT),  # 592 tiles on 592 CTAs
        (149, 149, STAGED),  # one tile more than CTAs, all active
    ],
)
def test_auto_rule(n_blocks: int, active: int, want: int) -> None:
    assert engine(n_blocks, active)._kernel == want


def test_persistent_needs_room_for_every_tile() -> None:
    grid = 148 * 4
    fits = grid * (1 + PERSISTENT_EXTRA_TILES) // 4
    assert engine(fits, 1)._persistent_fits
    assert engine(fits, 1)._kernel == PERSISTENT
    too_many = fits + 1
    assert not engine(too_many, 1)._persistent_fits
    assert engine(too_many, 1)._kernel == STAGED  # sparse, but a step could not find every tile a CTA
    # a capped grid shrinks both the capacity and the "one CTA per tile" case
    assert engine(32, 32, max_grid=64)._kernel == STAGED


def test_blocks_too_large_for_the_staged_kernel_run_the_plain_one() -> None:
    e = engine(3907, 3907)
    e._staged_fits = False
    assert e._kernel == KERNELS["plain"]
    assert engine(3907, 140)._kernel == PERSISTENT


def test_explicit_choice_and_unknown_names() -> None:
    e = engine(3907, 3907)
    e.stage_kernel = "persistent"
    assert e._kernel == PERSISTENT
    e.stage_kernel = "fastest"
    with pytest.raises(ValueError, match="stage_kernel"):
        _ = e._kernel


def test_two_sum_probe_verdicts() -> None:
    """The guard's decision on the probe's words (the device half runs in the GPU tests)."""
    import numpy as np

    from inundation_b200.engine import check_eft_probe

    check_eft_probe(np.array([1.0, 1e-9, 1e-9], np.float32))  # the exact error term: accepted
    for words in ([1.0, 1e-9, 0.0], [1.0, 1e-9, np.nan], [1.0, 1e-9, 2e-9], [1.0, 1e-9]):
        with pytest.raises(RuntimeError, match="error-free arithmetic is broken"):
            check_eft_probe(np.array(words, np.float32))
