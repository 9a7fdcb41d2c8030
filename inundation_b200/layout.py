"""Block-tile layout of a mesh for the device kernels (host side, NumPy).

Cells stay in Hilbert order; block ``b`` is cells ``[256 b, 256 b + 256)``.
Edges take the reference's resident order (sorted stably by the block of the
left cell, ``inundation/vulkan/gpu_resident_batch.py:175``). Each block gets
one contiguous *tile* of edge records, structure-of-arrays:

* its own edges (left cell in the block), in resident order, then
* the edges whose right cell is in the block and left cell is not, in
  resident order,

padded to a multiple of ``TILE_ALIGN`` records so every tile starts on a
128-byte boundary of every array. One CTA then finds, in one tile, every edge
its 256 cells touch. ``lcsr`` replaces the reference's remapped CSR
(``inundation/mesh/blocks.py:33-44``) with each slot's position in its
cell's tile (plus the side bit), in the same per-cell order, so the gather
sums the same terms in the same order as the reference.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from numpy.typing import NDArray

from .mesh.blocks import block_adjacency, block_two_ring, edge_order_by_block, remap_cell_edges
from .mesh.geometry import MeshGeometry
from .tuning import ACTIVE_BLOCK_CELLS, num_blocks

TILE_ALIGN = 32
MAX_TILE_EDGES = 32767


@dataclass
class TileLayout:
    n_cells: int
    n_edges: int
    n_blocks: int
    max_tile_edges: int
    edge_order: NDArray[np.int64]  # resident order: order[new] = geometry edge
    tile_cl: NDArray[np.int32]
    tile_cr: NDArray[np.int32]
    tile_nx: NDArray[np.float32]
    tile_ny: NDArray[np.float32]
    tile_len: NDArray[np.float32]
    tile_dzl: NDArray[np.float32]
    tile_dzr: NDArray[np.float32]
    tile_ptr: NDArray[np.uint32]  # n_blocks + 1: tile b is [tile_ptr[b], tile_ptr[b + 1]) with padding
    tile_count: NDArray[np.uint32]
    tile_edge: NDArray[np.int64]  # resident edge id of every tile record (-1 on padding)
    cptr: NDArray[np.uint32]  # n_blocks * 256 + 4 entries; past n_cells they repeat the total
    lcsr: NDArray[np.uint16]
    lcsr_blk: NDArray[np.uint16]  # lcsr regrouped per block, block b's slots from lcsr_ptr[b]
    lcsr_ptr: NDArray[np.uint32]  # n_blocks + 1, multiples of 8 (16-byte aligned segments)
    max_block_slots: int  # the largest padded slot segment of a block
    ring_ptr: NDArray[np.uint32]
    ring_idx: NDArray[np.uint32]
    area: NDArray[np.float32]

    @property
    def n_padded_cells(self) -> int:
        return self.n_blocks * ACTIVE_BLOCK_CELLS

    @property
    def n_tile_records(self) -> int:
        return int(self.tile_cl.size)

    @property
    def foreign_edges(self) -> int:
        return int(self.tile_count.sum()) - self.n_edges


def build_tile_layout(geom: MeshGeometry) -> TileLayout:
    """Tiles, local CSR and block two-ring of a Hilbert-ordered geometry."""
    n, n_e = int(geom.N), int(geom.E)
    if n == 0 or n_e == 0:
        raise ValueError("mesh has no cells or no edges")
    bc = ACTIVE_BLOCK_CELLS
    n_blk = num_blocks(n, bc)
    order = edge_order_by_block(geom.edge_cellL, bc)
    ecl = geom.edge_cellL[order].astype(np.int64)
    ecr = geom.edge_cellR[order].astype(np.int64)
    if (ecr < -1).any():
        raise ValueError("open boundary edges are not supported by this layout")
    blk_l = ecl // bc
    blk_r = np.where(ecr >= 0, ecr // bc, -1)
    own_lo = np.searchsorted(blk_l, np.arange(n_blk), side="left")
    n_own = np.bincount(blk_l, minlength=n_blk)

    foreign = np.flatnonzero((blk_r >= 0) & (blk_r != blk_l))
    f_sorted = foreign[np.argsort(blk_r[foreign], kind="stable")]
    f_block = blk_r[f_sorted]
    n_for = np.bincount(f_block, minlength=n_blk)
    f_first = np.zeros(n_blk + 1, dtype=np.int64)
    np.cumsum(n_for, out=f_first[1:])
    f_rank = np.zeros(n_e, dtype=np.int64)
    f_rank[f_sorted] = np.arange(f_sorted.size) - f_first[f_block]

    count = n_own + n_for
    if int(count.max()) > MAX_TILE_EDGES:
        raise ValueError(f"a block touches {int(count.max())} edges; the tile limit is {MAX_TILE_EDGES}")
    padded = (count + TILE_ALIGN - 1) // TILE_ALIGN * TILE_ALIGN
    ptr = np.zeros(n_blk + 1, dtype=np.int64)
    np.cumsum(padded, out=ptr[1:])
    total = int(ptr[-1])

    rec = np.full(total, -1, dtype=np.int64)
    own_pos = np.arange(n_e) - own_lo[blk_l]
    rec[ptr[blk_l] + own_pos] = np.arange(n_e)
    rec[ptr[f_block] + n_own[f_block] + f_rank[f_sorted]] = f_sorted
    valid = rec >= 0
    src = np.where(valid, rec, 0)

    def gather(values: NDArray, fill: float | int, dtype: type) -> NDArray:
        out = np.asarray(values)[src].astype(dtype)
        out[~valid] = fill
        return out

    signed = remap_cell_edges(geom.cell_edge_idx_signed, order).astype(np.int64)
    slot_edge = signed >> 1
    slot_side = signed & 1
    slot_cell = np.repeat(np.arange(n, dtype=np.int64), np.diff(geom.cell_edge_ptr.astype(np.int64)))
    slot_block = slot_cell // bc
    owned = blk_l[slot_edge] == slot_block
    local = np.where(owned, slot_edge - own_lo[slot_block], n_own[slot_block] + f_rank[slot_edge])
    if local.size and int(local.max()) > MAX_TILE_EDGES:
        raise ValueError("local tile index overflows 15 bits")
    lcsr = ((local << 1) | slot_side).astype(np.uint16)

    cptr64 = geom.cell_edge_ptr.astype(np.int64)
    first_slot = cptr64[np.minimum(np.arange(n_blk + 1) * bc, n)]
    seg = np.diff(first_slot)
    seg_pad = (seg + 7) // 8 * 8
    lptr = np.zeros(n_blk + 1, dtype=np.int64)
    np.cumsum(seg_pad, out=lptr[1:])
    lcsr_blk = np.zeros(int(lptr[-1]) + 8, dtype=np.uint16)
    dest = lptr[slot_block] + (np.arange(slot_cell.size) - first_slot[slot_block])
    lcsr_blk[dest] = lcsr
    cptr_pad = np.full(n_blk * bc + 4, cptr64[-1], dtype=np.int64)
    cptr_pad[: n + 1] = cptr64

    rptr, ridx = block_two_ring(*block_adjacency(ecl.astype(np.int32), ecr.astype(np.int32), n, bc))
    return TileLayout(
        n_cells=n,
        n_edges=n_e,
        n_blocks=n_blk,
        max_tile_edges=int(count.max()),
        edge_order=order,
        tile_cl=gather(ecl, 0, np.int32),
        tile_cr=gather(ecr, -1, np.int32),
        tile_nx=gather(geom.edge_nx[order], 0.0, np.float32),
        tile_ny=gather(geom.edge_ny[order], 0.0, np.float32),
        tile_len=gather(geom.edge_len[order], 0.0, np.float32),
        tile_dzl=gather(geom.edge_dzL[order], 0.0, np.float32),
        tile_dzr=gather(geom.edge_dzR[order], 0.0, np.float32),
        tile_ptr=ptr.astype(np.uint32),
        tile_count=count.astype(np.uint32),
        tile_edge=rec,
        cptr=cptr_pad.astype(np.uint32),
        lcsr=lcsr,
        lcsr_blk=lcsr_blk,
        lcsr_ptr=lptr.astype(np.uint32),
        max_block_slots=int(seg_pad.max()),
        ring_ptr=rptr.astype(np.uint32),
        ring_idx=ridx.astype(np.uint32) if ridx.size else np.zeros(1, np.uint32),
        area=np.concatenate([geom.area.astype(np.float32), np.ones(n_blk * bc - n, np.float32)]),
    )


def algorithmic_bytes_per_cell_step(geom: MeshGeometry) -> float:
    """Compulsory HBM bytes of one Heun step per cell.

    Per stage: edge geometry 28 B per edge (cL, cR, nx, ny, len, dzL, dzR),
    cell data 12 B (area, n, cptr), CSR 4 B per slot; state (h, hu, hv, h_lo):
    the predictor reads U^n and writes U* (32 B), the corrector reads U* and
    U^n and writes U^{n+1} (48 B). B = 2 (28 E/N + 12 + 4 S/N) + 80.
    """
    e_per_n = geom.E / geom.N
    s_per_n = float(geom.cell_edge_ptr[-1]) / geom.N
    return 2.0 * (28.0 * e_per_n + 12.0 + 4.0 * s_per_n) + 80.0
