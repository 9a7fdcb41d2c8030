"""Active-set block topology (host side), built as sparse boolean matrices.

A block is ``ACTIVE_BLOCK_CELLS`` consecutive Hilbert-ordered cells. The device
skips every block outside the two-ring of blocks that hold water; that is exact
because one Heun step moves water at most two cell rings.

The block graph is the symmetric boolean matrix A with A[b, c] set when an
interior edge joins a cell of block b to a cell of block c != b. Its CSR
(``indptr``, sorted ``indices``) is the adjacency the kernels read; the two-ring
is the off-diagonal pattern of A + A @ A, and one dilation is ``f | (A f)``.

The results equal those of the reference's helpers of the same names
(``inundation/mesh/blocks.py:21-128``): ``tests/golden/blocks.npz`` holds the
reference's outputs and the tests compare them array for array.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
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
    """``order[new] = old``: edges grouped by the block of their left cell, each group in edge order."""
    block = np.asarray(edge_cell_l, dtype=np.int64) // block_cells
    # lexsort sorts by the last key first: block, ties broken by the edge's own index
    return np.lexsort((np.arange(block.size, dtype=np.int64), block)).astype(np.int64)


def remap_cell_edges(cell_edge_idx_signed: NDArray[np.int32], order: NDArray[np.int64]) -> NDArray[np.uint32]:
    """Signed CSR entries ``(edge << 1) | is_right`` renamed to the edge numbering of ``order``.

    Each cell keeps its entries in their order; only edge ids change.
    """
    order = np.asarray(order, dtype=np.int64)
    renamed = np.argsort(order)  # the inverse permutation: renamed[old] = new
    entry = np.asarray(cell_edge_idx_signed, dtype=np.int64)
    edge, side = np.divmod(entry, 2)
    return (2 * renamed[edge] + side).astype(np.uint32)


def edge_workgroup_block_ranges(
    sorted_cell_l: NDArray[np.int32], workgroup: int, block_cells: int
) -> NDArray[np.uint32]:
    """``(groups, 2)``: the first and last left-cell block of each run of ``workgroup`` edges."""
    block = np.asarray(sorted_cell_l, dtype=np.int64) // block_cells
    if (block[1:] < block[:-1]).any():
        raise ValueError("edges must be sorted by the block of their left cell")
    if block.size == 0:
        return np.zeros((0, 2), dtype=np.uint32)
    groups = -(-block.size // workgroup)
    # pad the last run with its own last block, so every row of the table is a full run
    table = np.pad(block, (0, groups * workgroup - block.size), mode="edge").reshape(groups, workgroup)
    return np.stack([table[:, 0], table[:, -1]], axis=1).astype(np.uint32)


def _pattern(matrix: sp.spmatrix, n_blk: int) -> tuple[NDArray[np.uint32], NDArray[np.uint32]]:
    """CSR of the nonzero pattern without the diagonal, columns ascending."""
    m = sp.csr_matrix(matrix, shape=(n_blk, n_blk), dtype=np.int64)
    m.setdiag(0)
    m.eliminate_zeros()
    m.sort_indices()
    return m.indptr.astype(np.uint32), m.indices.astype(np.uint32)


def _graph(ptr: NDArray[np.uint32], idx: NDArray[np.uint32]) -> sp.csr_matrix:
    n_blk = ptr.size - 1
    ones = np.ones(idx.size, dtype=np.int64)
    return sp.csr_matrix((ones, idx.astype(np.int64), ptr.astype(np.int64)), shape=(n_blk, n_blk))


def block_adjacency(
    edge_cell_l: NDArray[np.int32], edge_cell_r: NDArray[np.int32], n_cells: int, block_cells: int
) -> tuple[NDArray[np.uint32], NDArray[np.uint32]]:
    """CSR ``(ptr, idx)`` of the other blocks each block shares an interior edge with (sorted, unique)."""
    n_blk = num_blocks(n_cells, block_cells)
    right = np.asarray(edge_cell_r, dtype=np.int64)
    interior = right >= 0
    a = np.asarray(edge_cell_l, dtype=np.int64)[interior] // block_cells
    b = right[interior] // block_cells
    ones = np.ones(a.size, dtype=np.int64)
    one_way = sp.coo_matrix((ones, (a, b)), shape=(n_blk, n_blk))
    return _pattern(one_way + one_way.T, n_blk)


def block_two_ring(ptr: NDArray[np.uint32], idx: NDArray[np.uint32]) -> tuple[NDArray[np.uint32], NDArray[np.uint32]]:
    """CSR of the blocks at most two adjacency steps from each block, itself excluded.

    One dilation over this graph equals two dilations over ``(ptr, idx)``.
    """
    a = _graph(ptr, idx)
    return _pattern(a + a @ a, ptr.size - 1)


def dilate_blocks(flags: NDArray[np.bool_], ptr: NDArray[np.uint32], idx: NDArray[np.uint32]) -> NDArray[np.bool_]:
    """One dilation: a block is set if it or any block in its CSR row is set."""
    flags = np.asarray(flags, dtype=bool)
    reached = _graph(ptr, idx) @ flags.astype(np.int64)
    return flags | (reached > 0)
