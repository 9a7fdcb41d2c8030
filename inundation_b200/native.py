"""ctypes binding of ``lib/libinundation_b200.so`` (the C ABI in ``include/inundation_b200.h``).

The library is the only compute path: if it is missing or cannot be loaded,
``load()`` raises. There is no CPU fallback.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

from .build import LIB_PATH

_P = ctypes.c_void_p
_U32 = ctypes.c_uint32

STATUS_MESSAGES = {
    1: "invalid argument",
    2: "CUDA launch or runtime error",
    3: "size beyond a fixed limit (an edge tile larger than shared memory or than a work item's fields, "
    "or more cells than the allocation-free volume's static scratch holds)",
    4: "device arithmetic lost the two-sum error term",
}

# Every function the header declares, with its argument and result types.
_SIGNATURES: dict[str, tuple[list, object]] = {
    "swe_workspace_bytes": ([_U32, _U32], ctypes.c_size_t),
    "swe_configure": ([_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "swe_stage": ([_P, _P, _P, ctypes.c_int, _P], ctypes.c_int),
    "swe_apply_sources": ([_P, _P, _P, _P, _P], ctypes.c_int),
    "swe_block_dilate_compact": ([_P, _P, _P, ctypes.c_int, ctypes.c_int, _P], ctypes.c_int),
    "swe_block_mark": ([_P, _P, _P, _P], ctypes.c_int),
    "swe_cfl_prologue": ([_P, _P, _P, _P], ctypes.c_int),
    "swe_step_control": ([_P, _P, _U32, ctypes.c_int, _P], ctypes.c_int),
    "swe_prologue": ([_P, _P, _P, _P], ctypes.c_int),
    "swe_step": ([_P, _P, _P, _P, _P], ctypes.c_int),
    "swe_steps": ([_P, _P, _P, _P, _U32, _P], ctypes.c_int),
    "swe_volume_partials": ([_U32], _U32),
    "swe_volume_fp64": ([_P, _P, _P, _U32, _P, _P, _P], ctypes.c_int),
    "swe_volume_fp64_noalloc": ([_P, _P, _P, _U32, _P, _P], ctypes.c_int),
    "swe_eft_probe": ([_P, _P], ctypes.c_int),
    "swe_dt_wait_probe": ([_P, _U32, _P, _P], ctypes.c_int),
    "swe_inv_pow43": ([_P, _P, _U32, _P], ctypes.c_int),
    "swe_open_ghost_probe": ([_P, _P, _P, _U32, ctypes.c_float, ctypes.c_float, _P], ctypes.c_int),
    "swe_status_string": ([ctypes.c_int], ctypes.c_char_p),
    "swe_bed_steps": ([_P, _P, _P, _P, _U32, _P, _P, _U32, _P], ctypes.c_int),
    "swe_stage_taped": ([_P, _P, _P, ctypes.c_int, _P, _P], ctypes.c_int),
    "swe_tape_record": ([_P, _P, _P, _U32, _P], ctypes.c_int),
    "swe_gauge_misfit": ([_P, _P, ctypes.c_int, _P], ctypes.c_int),
    "swe_adjoint_segment": ([_P, _P, _P, _P, _P, _P, _U32, _U32, _U32, _P], ctypes.c_int),
}


class SweMesh(ctypes.Structure):
    _fields_ = [
        ("n_cells", _U32),
        ("n_blocks", _U32),
        ("max_tile_edges", _U32),
        ("n_inst", _U32),
        *[(name, _P) for name in (
            "tile_cl", "tile_cr", "tile_nx", "tile_ny", "tile_len", "tile_dzl", "tile_dzr", "tile_ptr",
            "tile_count", "cptr", "lcsr", "area", "n_mann", "ring_ptr", "ring_idx", "block_inst", "block_cells",
        )],
        ("max_sub_edges", _U32),
        ("max_sub_slots", _U32),
        *[(name, _P) for name in (
            "sub_cl", "sub_cr", "sub_nx", "sub_ny", "sub_len", "sub_dzl", "sub_dzr", "sub_ptr", "sub_count",
            "sub_lcsr", "sub_lcsr_ptr",
        )],
        ("n_open", _U32),
        ("open_cond", _P),
        ("max_blk_slots", _U32),
        ("blk_lcsr", _P),
        ("blk_lcsr_ptr", _P),
    ]


class SweState(ctypes.Structure):
    _fields_ = [
        (name, _P)
        for name in (
            "h", "hu", "hv", "h_lo", "h1", "hu1", "hv1", "h1_lo", "clamp_mass", "blk", "active_list", "items",
            "sched", "dt_buf", "ctrl", "sync", "marks", "open_vol",
        )
    ]


class SweParams(ctypes.Structure):
    _fields_ = [
        ("g", ctypes.c_float),
        ("dry_tol", ctypes.c_float),
        ("cfl", ctypes.c_float),
        ("compensated", _U32),
        ("track_clamp", _U32),
        ("active_set", _U32),
        ("grid", _U32),
        ("kernel", _U32),
    ]


class SweSources(ctypes.Structure):
    _fields_ = [
        *[(name, _P) for name in ("cells", "rate", "hydro", "hscale", "knot_ptr", "knot_t", "knot_q")],
        ("count", _U32),
        ("n_hydro", _U32),
    ]


class SweTape(ctypes.Structure):
    _fields_ = [
        *[(name, _P) for name in ("h", "hu", "hv", "h_lo", "s0", "s1", "dt", "t", "list", "count")],
        ("capacity", _U32),
    ]


class SweAdjoint(ctypes.Structure):
    _fields_ = [
        *[(name, _P) for name in (
            "lh", "lhu", "lhv", "ls", "lsh", "lshu", "lshv", "uh", "ulo", "uhu", "uhv", "mark", "gn", "gz", "gq", "sync",
        )],
        ("cut_depth", ctypes.c_float),
    ]


class SweGauges(ctypes.Structure):
    _fields_ = [("cells", _P), ("obs", _P), ("loss", _P), ("count", _U32), ("steps", _U32)]


_LIB: ctypes.CDLL | None = None


def library_path() -> Path:
    return LIB_PATH


def load() -> ctypes.CDLL:
    """Load the CUDA library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"CUDA extension {LIB_PATH} is missing: build it with `python -m inundation_b200.build`"
            )
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _LIB = lib
    return _LIB


def check(rc: int, what: str) -> None:
    """Turn a status code into an exception (0 is success)."""
    if rc != 0:
        raise RuntimeError(f"{what} failed: {STATUS_MESSAGES.get(rc, f'status {rc}')}")


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)
