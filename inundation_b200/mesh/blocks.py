"""Active-set block topology (host side).

A block is ``ACTIVE_BLOCK_CELLS`` consecutive Hilbert-ordered cells. The device
skips every block outside the two-ring of blocks that hold water; that is exact
because one Heun step moves water at most two cell rings. The helpers here
follow the reference's ``inundation/mesh/blocks.py:21-128`` (same names,
arguments and results) and are checked against it.
"""

from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

from ..tuning import num_blocks

__all__ = [
    "block_adjacency",
    "block_two_ring",
    "dilate_blocks",
    "edge_order_by_block",
    "edge_workgroup_block_ranges",
    "num_blocks",
    "remap_cell_edges",
]


def edge_order_by_block(edge_cell_l: NDArray[np.int32], block_cells: int) -> NDArray[np.int64]:
    """Stable permutation of edges by the block of their left cell (blocks.py:28-30)."""
    return np.argsort(np.asarray(edge_cell_l) // block_cells, kind="stable")


def remap_cell_edges(cell_edge_idx_signed: NDArray[np.int32], order: NDArray[np.int64]) -> NDArray[np.uint32]:
    """Signed CSR entries after the edges are permuted by ``order`` (``order[new] = old``).

    Each cell keeps the order of its entries; only edge ids change (blocks.py:33-44).
    """
    new_of_old = np.empty(order.size, dtype=np.int64)
    new_of_old[order] = np.arange(order.size, dtype=np.int64)
    s = np.asarray(cell_edge_idx_signed, dtype=np.int64)
    return ((new_of_old[s >> 1] << 1) | (s & 1)).astype(np.uint32)


def edge_workgroup_block_ranges(
    sorted_cell_l: NDArray[np.int32], workgroup: int, block_cells: int
) -> NDArray[np.uint32]:
    """First and last left-cell block of each run of ``workgroup`` block-sorted edges."""
    blocks = np.asarray(sorted_cell_l, dtype=np.int64) // block_cells
    if blocks.size and np.any(np.diff(blocks) < 0):
        raise ValueError("edges must be sorted by the block of their left cell")
    first = np.arange(0, blocks.size, workgroup)
    last = np.minimum(first + workgroup, blocks.size) - 1
    return np.column_stack([blocks[first], blocks[last]]).astype(np.uint32)


def block_adjacency(
    edge_cell_l: NDArray[np.int32], edge_cell_r: NDArray[np.int32], n_cells: int, block_cells: int
) -> tuple[NDArray[np.uint32], NDArray[np.uint32]]:
    """CSR of the other blocks each block shares an interior edge with (sorted, unique)."""
    n_blk = num_blocks(n_cells, block_cells)
    inner = np.asarray(edge_cell_r) >= 0
    bl = np.asarray(edge_cell_l)[inner].astype(np.int64) // block_cells
    br = np.asarray(edge_cell_r)[inner].astype(np.int64) // block_cells
    cross = bl != br
    pairs = np.concatenate([np.column_stack([bl[cross], br[cross]]), np.column_stack([br[cross], bl[cross]])])
    pairs = np.unique(pairs, axis=0) if pairs.size else np.zeros((0, 2), dtype=np.int64)
    ptr = np.zeros(n_blk + 1, dtype=np.uint32)
    np.cumsum(np.bincount(pairs[:, 0], minlength=n_blk), out=ptr[1:])
    return ptr, pairs[:, 1].astype(np.uint32)


def block_two_ring(ptr: NDArray[np.uint32], idx: NDArray[np.uint32]) -> tuple[NDArray[np.uint32], NDArray[np.uint32]]:
    """CSR of the blocks within two adjacency steps of each block, itself excluded."""
    n_blk = ptr.size - 1
    deg = np.diff(ptr.astype(np.int64))
    src1 = np.repeat(np.arange(n_blk), deg)
    dst1 = idx.astype(np.int64)
    deg2 = deg[dst1]
    src2 = np.repeat(src1, deg2)
    base = np.repeat(ptr[dst1].astype(np.int64), deg2)
    within = np.arange(int(deg2.sum())) - np.repeat(np.cumsum(deg2) - deg2, deg2)
    dst2 = idx[base + within].astype(np.int64)
    src = np.concatenate([src1, src2])
    dst = np.concatenate([dst1, dst2])
    keep = src != dst
    pairs = np.column_stack([src[keep], dst[keep]])
    pairs = np.unique(pairs, axis=0) if pairs.size else np.zeros((0, 2), dtype=np.int64)
    out = np.zeros(n_blk + 1, dtype=np.uint32)
    np.cumsum(np.bincount(pairs[:, 0], minlength=n_blk), out=out[1:])
    return out, pairs[:, 1].astype(np.uint32)


def dilate_blocks(flags: NDArray[np.bool_], ptr: NDArray[np.uint32], idx: NDArray[np.uint32]) -> NDArray[np.bool_]:
    """One dilation: a block is set if it or any block in its CSR row is set."""
    out = flags.copy()
    rows = np.repeat(np.arange(flags.size), np.diff(ptr.astype(np.int64)))
    np.logical_or.at(out, rows, flags[idx.astype(np.int64)])
    return out
