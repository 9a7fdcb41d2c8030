"""Tile layouts of a mesh for the device kernels (host side, NumPy).

Cells stay in Hilbert order. Edges take the reference's resident order (sorted
stably by the 256-cell block of the left cell,
``inundation/vulkan/gpu_resident_batch.py:175``). For a tile size of T cells,
tile ``t`` is cells ``[T t, T t + T)`` and owns one contiguous segment of edge
records, structure-of-arrays:

* the edges whose left cell is in the tile and whose right cell is in it too
  (or is a boundary), then
* the edges whose left cell is in the tile and right cell in another tile, then
* the edges whose right cell is in the tile and left cell is not,

each group in resident order, so the records that read another tile's state
come last and fill the last warps of a tile pass,
padded to a multiple of ``TILE_ALIGN`` records so every segment starts on a
128-byte boundary of every array. One CTA then finds, in one segment, every
edge its cells touch. ``lcsr`` replaces the reference's remapped CSR
(``inundation/mesh/blocks.py:33-44``) with each slot's position in its cell's
tile segment (plus the side bit), in the same per-cell order, so a gather sums
the same terms in the same order as the reference.

Two tile sizes are built: 256 cells (one active-set block; the kernels of
the prologue, the sources and the plain stage kernel) and 64 cells (four
compute tiles per block; the tiled stage kernel).

Open boundary edges keep the reference's numbering (``inundation/vulkan/solver.py:236-243``):
an edge whose right cell is ``-2 - k`` is open edge ``k``. Like a wall it sits
in the tile of its left cell only.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from numpy.typing import NDArray

from .mesh.blocks import block_adjacency, block_two_ring, edge_order_by_block, remap_cell_edges
from .mesh.geometry import MeshGeometry
from .tuning import ACTIVE_BLOCK_CELLS, num_blocks

TILE_ALIGN = 32
SUB_TILE_CELLS = 64
MAX_TILE_EDGES = 32767


@dataclass
class TileSet:
    """Edge segments and local CSR of one tile size."""

    tile_cells: int
    n_tiles: int
    max_edges: int  # the largest count
    max_slots: int  # the largest padded lcsr segment
    ptr: NDArray[np.uint32]  # n_tiles + 1: segment t is [ptr[t], ptr[t + 1]), count[t] records then padding
    count: NDArray[np.uint32]
    edge: NDArray[np.int64]  # resident edge id of every record (-1 on padding)
    cl: NDArray[np.int32]
    cr: NDArray[np.int32]
    nx: NDArray[np.float32]
    ny: NDArray[np.float32]
    len: NDArray[np.float32]
    dzl: NDArray[np.float32]
    dzr: NDArray[np.float32]
    lcsr: NDArray[np.uint16]  # per CSR slot, flat in global slot order
    lcsr_blk: NDArray[np.uint16]  # the same, regrouped per tile from lcsr_ptr[t]
    lcsr_ptr: NDArray[np.uint32]  # n_tiles + 1, multiples of 8 (16-byte aligned segments)


@dataclass
class TileLayout:
    n_cells: int
    n_edges: int
    n_blocks: int
    edge_order: NDArray[np.int64]  # resident order: order[new] = geometry edge
    blocks: TileSet  # 256-cell tiles
    subs: TileSet  # 64-cell tiles
    cptr: NDArray[np.uint32]  # n_blocks * 256 + 4 entries; past n_cells they repeat the total
    ring_ptr: NDArray[np.uint32]
    ring_idx: NDArray[np.uint32]
    area: NDArray[np.float32]  # padded to n_blocks * 256 with 1.0
    block_inst: NDArray[np.uint32]  # instance of every block (all 0 for one mesh)
    block_cells: NDArray[np.uint32]  # real cells of every block
    inst_cell_offset: NDArray[np.int64]  # first cell of every instance (a multiple of 256)
    inst_cells: NDArray[np.int64]  # real cells of every instance
    open_cells: NDArray[np.int64] | None = None  # left (padded) cell of every open edge, by open index

    @property
    def n_open(self) -> int:
        return 0 if self.open_cells is None else int(self.open_cells.size)

    @property
    def n_inst(self) -> int:
        return int(self.inst_cells.size)

    @property
    def n_padded_cells(self) -> int:
        return self.n_blocks * ACTIVE_BLOCK_CELLS

    @property
    def max_tile_edges(self) -> int:
        return self.blocks.max_edges

    @property
    def foreign_edges(self) -> int:
        return int(self.blocks.count.sum()) - self.n_edges


def _tile_set(geom: MeshGeometry, order: NDArray[np.int64], signed: NDArray[np.int64], tile_cells: int) -> TileSet:
    n, n_e = int(geom.N), int(geom.E)
    ecl = geom.edge_cellL[order].astype(np.int64)
    ecr = geom.edge_cellR[order].astype(np.int64)
    n_t = num_blocks(n, tile_cells)
    t_l = ecl // tile_cells
    t_r = np.where(ecr >= 0, ecr // tile_cells, -1)

    # a tile's own edges whose right cell lies in another tile go after the others: the records
    # that read state from outside the tile sit together at the segment's end
    outside = (t_r >= 0) & (t_r != t_l)
    own_sorted = np.lexsort((np.arange(n_e), outside, t_l))
    n_own = np.bincount(t_l, minlength=n_t)
    own_first = np.zeros(n_t + 1, dtype=np.int64)
    np.cumsum(n_own, out=own_first[1:])
    own_rank = np.empty(n_e, dtype=np.int64)
    own_rank[own_sorted] = np.arange(n_e) - own_first[t_l[own_sorted]]

    foreign = np.flatnonzero((t_r >= 0) & (t_r != t_l))
    f_sorted = foreign[np.argsort(t_r[foreign], kind="stable")]
    f_tile = t_r[f_sorted]
    n_for = np.bincount(f_tile, minlength=n_t)
    f_first = np.zeros(n_t + 1, dtype=np.int64)
    np.cumsum(n_for, out=f_first[1:])
    f_rank = np.zeros(n_e, dtype=np.int64)
    f_rank[f_sorted] = np.arange(f_sorted.size) - f_first[f_tile]

    count = n_own + n_for
    if int(count.max()) > MAX_TILE_EDGES:
        raise ValueError(f"a tile touches {int(count.max())} edges; the limit is {MAX_TILE_EDGES}")
    padded = (count + TILE_ALIGN - 1) // TILE_ALIGN * TILE_ALIGN
    ptr = np.zeros(n_t + 1, dtype=np.int64)
    np.cumsum(padded, out=ptr[1:])
    rec = np.full(int(ptr[-1]), -1, dtype=np.int64)
    rec[ptr[t_l] + own_rank] = np.arange(n_e)
    rec[ptr[f_tile] + n_own[f_tile] + f_rank[f_sorted]] = f_sorted
    valid = rec >= 0
    src = np.where(valid, rec, 0)

    def gather(values: NDArray, fill: float | int, dtype: type) -> NDArray:
        out = np.asarray(values)[src].astype(dtype)
        out[~valid] = fill
        return out

    slot_edge = signed >> 1
    slot_side = signed & 1
    cptr64 = geom.cell_edge_ptr.astype(np.int64)
    slot_cell = np.repeat(np.arange(n, dtype=np.int64), np.diff(cptr64))
    slot_tile = slot_cell // tile_cells
    owned = t_l[slot_edge] == slot_tile
    local = np.where(owned, own_rank[slot_edge], n_own[slot_tile] + f_rank[slot_edge])
    if local.size and int(local.max()) > MAX_TILE_EDGES:
        raise ValueError("local tile index overflows 15 bits")
    lcsr = ((local << 1) | slot_side).astype(np.uint16)

    first_slot = cptr64[np.minimum(np.arange(n_t + 1) * tile_cells, n)]
    seg_pad = (np.diff(first_slot) + 7) // 8 * 8
    lptr = np.zeros(n_t + 1, dtype=np.int64)
    np.cumsum(seg_pad, out=lptr[1:])
    lcsr_blk = np.zeros(int(lptr[-1]) + 8, dtype=np.uint16)
    lcsr_blk[lptr[slot_tile] + (np.arange(slot_cell.size) - first_slot[slot_tile])] = lcsr

    return TileSet(
        tile_cells=tile_cells,
        n_tiles=n_t,
        max_edges=int(count.max()),
        max_slots=int(seg_pad.max()),
        ptr=ptr.astype(np.uint32),
        count=count.astype(np.uint32),
        edge=rec,
        cl=gather(ecl, 0, np.int32),
        cr=gather(ecr, -1, np.int32),
        nx=gather(geom.edge_nx[order], 0.0, np.float32),
        ny=gather(geom.edge_ny[order], 0.0, np.float32),
        len=gather(geom.edge_len[order], 0.0, np.float32),
        dzl=gather(geom.edge_dzL[order], 0.0, np.float32),
        dzr=gather(geom.edge_dzR[order], 0.0, np.float32),
        lcsr=lcsr,
        lcsr_blk=lcsr_blk,
        lcsr_ptr=lptr.astype(np.uint32),
    )


def build_tile_layout(geom: MeshGeometry) -> TileLayout:
    """Both tile sets, the padded CSR pointers and the block two-ring of a Hilbert-ordered geometry."""
    n = int(geom.N)
    layout = _build(geom)
    first = np.arange(layout.n_blocks, dtype=np.int64) * ACTIVE_BLOCK_CELLS
    layout.block_cells = np.minimum(ACTIVE_BLOCK_CELLS, n - first).astype(np.uint32)
    layout.inst_cells = np.array([n], dtype=np.int64)
    return layout


def _build(geom) -> TileLayout:
    n, n_e = int(geom.N), int(geom.E)
    if n == 0 or n_e == 0:
        raise ValueError("mesh has no cells or no edges")
    open_mask = np.asarray(geom.edge_cellR) < -1
    open_k = (-2 - np.asarray(geom.edge_cellR)[open_mask]).astype(np.int64)
    if open_k.size and not np.array_equal(np.sort(open_k), np.arange(open_k.size)):
        raise ValueError("open edges must be numbered -2 - k for k = 0 .. n_open - 1, each once")
    open_cells = np.empty(open_k.size, dtype=np.int64)
    open_cells[open_k] = np.asarray(geom.edge_cellL)[open_mask]
    bc = ACTIVE_BLOCK_CELLS
    n_blk = num_blocks(n, bc)
    order = edge_order_by_block(geom.edge_cellL, bc)
    signed = remap_cell_edges(geom.cell_edge_idx_signed, order).astype(np.int64)
    cptr64 = geom.cell_edge_ptr.astype(np.int64)
    cptr_pad = np.full(n_blk * bc + 4, cptr64[-1], dtype=np.int64)
    cptr_pad[: n + 1] = cptr64
    ecl = geom.edge_cellL[order].astype(np.int32)
    ecr = geom.edge_cellR[order].astype(np.int32)
    rptr, ridx = block_two_ring(*block_adjacency(ecl, ecr, n, bc))
    return TileLayout(
        n_cells=n,
        n_edges=n_e,
        n_blocks=n_blk,
        edge_order=order,
        blocks=_tile_set(geom, order, signed, bc),
        subs=_tile_set(geom, order, signed, SUB_TILE_CELLS),
        cptr=cptr_pad.astype(np.uint32),
        ring_ptr=rptr.astype(np.uint32),
        ring_idx=ridx.astype(np.uint32) if ridx.size else np.zeros(1, np.uint32),
        area=np.concatenate([geom.area.astype(np.float32), np.ones(n_blk * bc - n, np.float32)]),
        block_inst=np.zeros(n_blk, np.uint32),
        block_cells=np.full(n_blk, bc, np.uint32),
        inst_cell_offset=np.zeros(1, np.int64),
        inst_cells=np.array([n], np.int64),
        open_cells=open_cells,
    )


@dataclass
class _Concatenated:
    """The fields of ``MeshGeometry`` the layout reads, for a batch of meshes."""

    N: int
    E: int
    edge_cellL: NDArray[np.int32]
    edge_cellR: NDArray[np.int32]
    edge_nx: NDArray[np.float32]
    edge_ny: NDArray[np.float32]
    edge_len: NDArray[np.float32]
    edge_dzL: NDArray[np.float32]
    edge_dzR: NDArray[np.float32]
    cell_edge_ptr: NDArray[np.int64]
    cell_edge_idx_signed: NDArray[np.int64]
    area: NDArray[np.float32]


def build_batch_layout(geoms: list[MeshGeometry]) -> TileLayout:
    """One layout for a batch of independent Hilbert-ordered meshes.

    Instance ``i`` takes whole blocks from cell ``inst_cell_offset[i]``; the
    cells that pad its last block have no edges and are never updated. Every
    instance keeps the tiles, edge segments and per-cell CSR order it has on
    its own, so its results are bit-identical to a run of that mesh alone.
    """
    if not geoms:
        raise ValueError("a batch needs at least one mesh")
    bc = ACTIVE_BLOCK_CELLS
    sizes = np.array([int(g.N) for g in geoms], dtype=np.int64)
    padded = (sizes + bc - 1) // bc * bc
    offs = np.zeros(len(geoms) + 1, dtype=np.int64)
    np.cumsum(padded, out=offs[1:])
    e_offs = np.zeros(len(geoms) + 1, dtype=np.int64)
    np.cumsum([int(g.E) for g in geoms], out=e_offs[1:])
    total = int(offs[-1])
    ptr = np.zeros(total + 1, dtype=np.int64)
    area = np.ones(total, dtype=np.float32)
    signed, cl, cr = [], [], []
    open_base = 0  # open edges keep their order, numbered on from the previous instances'
    for i, g in enumerate(geoms):
        o, n = int(offs[i]), int(g.N)
        gptr = g.cell_edge_ptr.astype(np.int64)
        ptr[o + 1 : o + n + 1] = ptr[o] + gptr[1:]
        ptr[o + n + 1 : int(offs[i + 1]) + 1] = ptr[o] + gptr[-1]
        area[o : o + n] = g.area
        signed.append(g.cell_edge_idx_signed.astype(np.int64) + 2 * int(e_offs[i]))
        cl.append(g.edge_cellL.astype(np.int64) + o)
        r = g.edge_cellR.astype(np.int64)
        cr.append(np.where(r >= 0, r + o, np.where(r < -1, r - open_base, r)))
        open_base += int((r < -1).sum())
    cat = lambda name: np.concatenate([getattr(g, name) for g in geoms]).astype(np.float32)  # noqa: E731
    geom = _Concatenated(
        N=total,
        E=int(e_offs[-1]),
        edge_cellL=np.concatenate(cl).astype(np.int32),
        edge_cellR=np.concatenate(cr).astype(np.int32),
        edge_nx=cat("edge_nx"),
        edge_ny=cat("edge_ny"),
        edge_len=cat("edge_len"),
        edge_dzL=cat("edge_dzL"),
        edge_dzR=cat("edge_dzR"),
        cell_edge_ptr=ptr,
        cell_edge_idx_signed=np.concatenate(signed),
        area=area,
    )
    layout = _build(geom)
    blocks = padded // bc
    layout.block_inst = np.repeat(np.arange(len(geoms), dtype=np.uint32), blocks)
    cells = np.full(layout.n_blocks, bc, dtype=np.int64)
    last = np.cumsum(blocks) - 1
    cells[last] = sizes - (blocks - 1) * bc
    layout.block_cells = cells.astype(np.uint32)
    layout.inst_cell_offset = offs[:-1].copy()
    layout.inst_cells = sizes
    return layout


def algorithmic_bytes_per_cell_step(geom: MeshGeometry | list[MeshGeometry]) -> float:
    """Compulsory HBM bytes of one Heun step per cell.

    Per stage: edge geometry 28 B per edge (cL, cR, nx, ny, len, dzL, dzR),
    cell data 12 B (area, n, cptr), CSR 4 B per slot; state (h, hu, hv, h_lo):
    the predictor reads U^n and writes U* (32 B), the corrector reads U* and
    U^n and writes U^{n+1} (48 B). B = 2 (28 E/N + 12 + 4 S/N) + 80.
    """
    geoms = geom if isinstance(geom, list) else [geom]
    n = sum(int(g.N) for g in geoms)
    e_per_n = sum(int(g.E) for g in geoms) / n
    s_per_n = sum(float(g.cell_edge_ptr[-1]) for g in geoms) / n
    return 2.0 * (28.0 * e_per_n + 12.0 + 4.0 * s_per_n) + 80.0
