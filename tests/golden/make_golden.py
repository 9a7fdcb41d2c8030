"""Generate the golden fixtures of ``tests/golden/*.npz`` from the reference.

Run in a container where the reference tree is importable:

    python tests/golden/make_golden.py /path/to/reference [--parts geometry blocks ticks step cache]

It imports the reference's own geometry builder (``inundation/mesh/geometry.py``),
block helpers (``inundation/mesh/blocks.py``), tick helpers
(``inundation/tuning.py``) and float64 CPU step (``tests/unit/_cpu_step.py``),
runs them on small seeded inputs made by this package's generators, and saves
inputs and outputs. The tests then pin this package's geometry, blocks, ticks
and FP64 oracle to these outputs without the reference present.
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

GEOM_FIELDS = (
    "origin", "centroid", "area", "zb", "cell_vertices", "cell_vertex_ptr", "cell_bbox", "edge_len", "edge_nx",
    "edge_ny", "edge_dzL", "edge_dzR", "edge_cellL", "edge_cellR", "edge_sideL", "edge_sideR", "cell_edge_ptr",
    "cell_edge_idx", "cell_nbr_idx", "cell_edge_side", "cell_edge_idx_signed",
)

VALLEY_NX, VALLEY_NY, VALLEY_DX = 64, 32, 2.0
DRY_TOL = 1e-3
MANNING = 0.03
DT = 2.0**-10


def valley_inputs(datum: float):
    from inundation_b200.mesh.synthetic import quad_grid

    nx, ny, dx = VALLEY_NX, VALLEY_NY, VALLEY_DX
    q = quad_grid(nx, ny, dx)
    cx = (np.arange(nx * ny) % nx + 0.5) * dx
    cy = (np.arange(nx * ny) // nx + 0.5) * dx
    zb = (datum - 0.002 * cx - 0.3 * np.exp(-(((cy - ny * dx / 2) / (0.2 * ny * dx)) ** 2))).astype(np.float32)
    return q.verts.astype(np.float32), q.faces.reshape(-1, 4).astype(np.int32), None, zb


def voronoi_inputs():
    from inundation_b200.mesh.synthetic import gaussian_bumps, voronoi_mesh

    m = voronoi_mesh(2000, 1000.0, seed=11)
    approx = np.array([m.verts[m.faces[a:b]].mean(axis=0) for a, b in zip(m.offsets[:-1], m.offsets[1:])])
    zb = gaussian_bumps(approx, 1000.0, count=6, seed=11).astype(np.float32)
    return m.verts, m.faces, m.offsets, zb


def mixed_inputs():
    """Two quads, a triangle and a pentagon, some listed clockwise."""
    verts = np.array(
        [[0, 0], [2, 0], [4, 0], [0, 2], [2, 2], [4, 2], [1, 3.5], [3, 3.5], [5, 1]], dtype=np.float64
    ) + np.array([100.0, 50.0])
    faces = np.array([0, 1, 4, 3, 4, 1, 2, 5, 3, 4, 6, 5, 2, 8, 4, 5, 7, 6], dtype=np.int32)
    offsets = np.array([0, 4, 8, 11, 14, 18], dtype=np.int32)
    # cell 1 (4,1,2,5) is clockwise; cell 4 (4,5,7,6) counter-clockwise
    zb = np.array([0.1, 0.2, 0.0, 0.3, 0.15], dtype=np.float32)
    return verts, faces, offsets, zb


def geometry_record(prefix: str, geom) -> dict[str, np.ndarray]:
    out = {f"{prefix}{f}": np.asarray(getattr(geom, f)) for f in GEOM_FIELDS}
    out[f"{prefix}NEV"] = np.array([geom.N, geom.E, geom.V, geom.max_degree], dtype=np.int64)
    return out


def cases(geom, nx: int, ny: int, dx: float):
    x, y = geom.centroid[:, 0].astype(np.float64), geom.centroid[:, 1].astype(np.float64)
    dam = np.where((x < nx * dx * 0.25) & (np.abs(y - ny * dx / 2) < ny * dx * 0.15), 1.0, 0.0)
    sheet = np.where(x < nx * dx * 0.3, 0.02, 0.0)
    h_lake = float(geom.zb.max()) + 0.5 - geom.zb.astype(np.float64)
    far = x > nx * dx * 0.8
    z = np.zeros_like(x)
    return {
        "wet_lake": (h_lake, 0.1 * np.sin(2 * np.pi * x / (nx * dx)) * h_lake, z),
        "dam_break": (dam, z, z),
        "draining": (sheet, np.where(sheet > 0.0, 0.05, 0.0), z),
        "dry_momentum": (dam, np.where(far, 0.1, 0.0), -np.where(far, 0.1, 0.0)),
    }


CACHE_MESH = "cache_mesh.obj"


def write_cache_mesh(path: Path) -> None:
    """A 12 x 6 quad grid with a bumpy bed, at a UTM-sized offset, as a Wavefront OBJ (z per vertex)."""
    nx, ny, dx = 12, 6, 5.0
    x0, y0 = 512_000.0, 4_180_000.0
    lines = ["# 12 x 6 quads, 5 m, bed from the vertex elevations"]
    for j in range(ny + 1):
        for i in range(nx + 1):
            z = 0.01 * i + 0.3 * np.sin(0.7 * i) * np.cos(0.9 * j)
            lines.append(f"v {x0 + i * dx:.3f} {y0 + j * dx:.3f} {z:.6f}")
    row = nx + 1
    for j in range(ny):
        for i in range(nx):
            a = j * row + i + 1
            lines.append(f"f {a} {a + 1} {a + row + 1} {a + row}")
    path.write_text("\n".join(lines) + "\n")


def cache_fixtures() -> None:
    """Geometry-cache files written by the reference's own writer (``inundation/mesh/cache.py:103-191``):
    explicit artifacts in Hilbert and file order, and one key-addressed directory entry."""
    from inundation.mesh import cache as RC

    os.chdir(ROOT)  # the artifacts record the mesh source as given: a path relative to the repository
    mesh = Path("tests/golden") / CACHE_MESH
    write_cache_mesh(mesh)
    RC.build_geometry_cache(mesh, HERE / "ref_cache_hilbert.npz", use_hilbert_reorder=True)
    RC.build_geometry_cache(mesh, HERE / "ref_cache_file_order.npz", use_hilbert_reorder=False)
    key = RC.geometry_cache_key(mesh, use_hilbert_reorder=True)
    geom, perm, _ = RC.load_geometry_cache_artifact(HERE / "ref_cache_hilbert.npz")
    written = RC.save_geometry_cache(HERE / "ref_cache_dir", key, geom, perm)
    print("wrote", written.relative_to(ROOT), "and the two artifacts")


PARTS = ("geometry", "blocks", "ticks", "step", "cache")


def main(reference: str, parts: tuple[str, ...] = PARTS) -> None:
    sys.path.insert(0, reference)
    if "cache" in parts:
        cache_fixtures()
    from inundation import tuning as T
    from inundation.mesh import blocks as B
    from inundation.mesh.geometry import build_geometry, hilbert_reorder
    import importlib.util

    spec = importlib.util.spec_from_file_location("reference_cpu_step", Path(reference) / "tests/unit/_cpu_step.py")
    C = importlib.util.module_from_spec(spec)
    sys.modules["reference_cpu_step"] = C
    spec.loader.exec_module(C)

    if "geometry" in parts:
        rec: dict[str, np.ndarray] = {}
        # Geometry: raw and Hilbert-reordered, for a quad valley, a Voronoi mesh and a mixed mesh.
        for name, (verts, faces, offsets, zb) in {
            "valley": valley_inputs(0.0),
            "valley300": valley_inputs(300.0),
            "voronoi": voronoi_inputs(),
            "mixed": mixed_inputs(),
        }.items():
            rec[f"{name}_in_verts"] = verts
            rec[f"{name}_in_faces"] = faces
            rec[f"{name}_in_offsets"] = offsets if offsets is not None else np.zeros(0, np.int32)
            rec[f"{name}_in_zb"] = zb
            raw = build_geometry(verts, faces, offsets, zb_from_file=zb)
            ordered, perm = hilbert_reorder(raw, verbose=False)
            rec.update(geometry_record(f"{name}_raw_", raw))
            rec.update(geometry_record(f"{name}_hil_", ordered))
            rec[f"{name}_perm"] = perm
        np.savez_compressed(HERE / "geometry.npz", **rec)

    if "blocks" in parts:
        # Active-set block topology of the reordered Voronoi mesh (256-cell blocks) and of 16-cell blocks.
        rec = {}
        vor, _ = hilbert_reorder(build_geometry(*voronoi_inputs()[:3], zb_from_file=voronoi_inputs()[3]), verbose=False)
        for bc in (256, 16):
            order = B.edge_order_by_block(vor.edge_cellL, bc)
            ecl, ecr = vor.edge_cellL[order], vor.edge_cellR[order]
            ptr, idx = B.block_adjacency(ecl, ecr, vor.N, bc)
            p2, i2 = B.block_two_ring(ptr, idx)
            rec[f"b{bc}_order"] = order
            rec[f"b{bc}_remap"] = B.remap_cell_edges(vor.cell_edge_idx_signed, order)
            rec[f"b{bc}_ranges"] = B.edge_workgroup_block_ranges(ecl, 256, bc)
            rec[f"b{bc}_adj_ptr"], rec[f"b{bc}_adj_idx"] = ptr, idx
            rec[f"b{bc}_ring_ptr"], rec[f"b{bc}_ring_idx"] = p2, i2
            flags = np.random.default_rng(bc).random(ptr.size - 1) < 0.1
            rec[f"b{bc}_flags"] = flags
            rec[f"b{bc}_dilated"] = B.dilate_blocks(flags, p2, i2)
        np.savez_compressed(HERE / "blocks.npz", **rec)

    if "ticks" in parts:
        # Tick helpers.
        secs = np.array([0.0, 0.1, 0.5, 1.0, 600.0, 1800.0, 7200.0, 86400.0, 12345.678, 2.0**-20 * 3.4])
        dts = np.array([2.0**-20, 0.0314, 0.05, 0.5, 1.0, 2.0**-10, 15.999, 16.0])
        rec = {
            "seconds": secs,
            "seconds_ticks": np.array([T.seconds_to_ticks(s) for s in secs], dtype=np.int64),
            "dts": dts,
            "dt_ticks": np.array([T.dt_to_ticks(d) for d in dts], dtype=np.int64),
            "windows_a": np.array(list(T.output_window_stops(0, 1000, 600)), dtype=np.int64),
            "windows_b": np.array(list(T.output_window_stops(7200 << 20, (7200 + 3600) << 20, 1800 << 20)), dtype=np.int64),
        }
        np.savez_compressed(HERE / "ticks.npz", **rec)

    if "step" in parts:
        # The float64 step: 8 steps of dt = 2^-10 on the small valley (and 64 at a 300 m datum),
        # a Voronoi dam break, the prologue CFL bound, HLLC and its wave speeds.
        rec = {}
        rng = np.random.default_rng(5)
        for grid_name, datum, steps in (("valley", 0.0, 8), ("valley300", 300.0, 64)):
            v, f, _, zb = valley_inputs(datum)
            grid = hilbert_reorder(build_geometry(v, f, zb_from_file=zb), verbose=False)[0]
            n = np.full(grid.N, MANNING, np.float32)
            for case, (h, hu, hv) in cases(grid, VALLEY_NX, VALLEY_NY, VALLEY_DX).items():
                h32, hu32, hv32 = (a.astype(np.float32) for a in (h, hu, hv))
                key = f"{grid_name}_{case}"
                rec[f"{key}_h0"], rec[f"{key}_hu0"], rec[f"{key}_hv0"] = h32, hu32, hv32
                s = C.run_steps(grid, h32, hu32, hv32, n, DT, steps, g=T.GRAVITY_G, dry_tol=DRY_TOL)
                rec[f"{key}_h"], rec[f"{key}_hu"], rec[f"{key}_hv"] = s.h, s.hu, s.hv
                s0 = C.State(h32.astype(np.float64), hu32.astype(np.float64), hv32.astype(np.float64))
                rec[f"{key}_cfl"] = np.array(C.cfl_dt(grid, s0, g=T.GRAVITY_G, dry_tol=DRY_TOL, cfl=T.CFL_DEFAULT))
        vv, vf, vo, vz = voronoi_inputs()
        vor = hilbert_reorder(build_geometry(vv, vf, vo, zb_from_file=vz), verbose=False)[0]
        x, y = vor.centroid[:, 0].astype(np.float64), vor.centroid[:, 1].astype(np.float64)
        h0 = np.where(np.hypot(x - 500.0, y - 500.0) < 150.0, 2.0, 0.0) + np.maximum(0.0, 0.5 - vor.zb)
        h0 = h0.astype(np.float32)
        z = np.zeros(vor.N, np.float32)
        nv = rng.uniform(0.02, 0.06, vor.N).astype(np.float32)
        rec["voronoi_h0"], rec["voronoi_n"] = h0, nv
        s = C.run_steps(vor, h0, z, z, nv, 0.05, 8, g=T.GRAVITY_G, dry_tol=1e-4)
        rec["voronoi_h"], rec["voronoi_hu"], rec["voronoi_hv"] = s.h, s.hu, s.hv
        st = rng.uniform([0.0, -1.0, -1.0, 0.0, -1.0, -1.0], [2.0, 1.0, 1.0, 2.0, 1.0, 1.0], (200, 6))
        st[::7, 0] = 0.0
        st[::11, 3] = 5e-4
        rec["hllc_in"] = st
        out = C.hllc(*(st[:, k] for k in range(6)), g=T.GRAVITY_G, dry_tol=DRY_TOL)
        rec["hllc_out"] = np.column_stack(out)
        sp = rng.uniform([0.0, -2.0, 0.0, -2.0], [1.0, 2.0, 1.0, 2.0], (200, 4))
        sp[::5, 0] = DRY_TOL * np.linspace(0.5, 2.5, sp[::5].shape[0])
        rec["speeds_in"] = sp
        rec["speeds_out"] = np.column_stack(C.hllc_speeds(sp[:, 0], sp[:, 1], sp[:, 2], sp[:, 3], g=T.GRAVITY_G, dry_tol=DRY_TOL))
        np.savez_compressed(HERE / "cpu_step.npz", **rec)
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("reference", help="root of the reference's source tree (the directory holding inundation/)")
    ap.add_argument("--parts", nargs="+", choices=PARTS, default=list(PARTS))
    args = ap.parse_args()
    main(os.path.abspath(args.reference), tuple(args.parts))
