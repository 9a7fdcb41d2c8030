"""Host side of the workflow API (no GPU): config validation, sources, initial state, caches, loaders.

Restates the reference's CPU-runnable workflow checks (``inundation/workflow.py:191-227`` validation,
``:294-358`` source cell selection, ``:450-596`` initial state, ``inundation/mesh/cache.py`` artifacts).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from inundation_b200.mesh.cache import (
    GEOMETRY_CACHE_VERSION,
    build_geometry_cache,
    geometry_cache_key,
    load_geometry_cache,
    load_geometry_cache_artifact,
    save_geometry_cache,
)
from inundation_b200.mesh.geometry import build_geometry, hilbert_reorder
from inundation_b200.mesh.loader import load_mesh_file, save_mesh_npz
from inundation_b200.mesh.synthetic import quad_grid
from inundation_b200.workflow import (
    PointSource,
    SimulationPhase,
    SWEWorkflow,
    WorkflowConfig,
    build_phase_source_rate,
    load_initial_state,
    select_cells_within_radius,
)

GEO = np.load(Path(__file__).parent / "golden" / "geometry.npz")
FIELDS = ("origin", "centroid", "area", "zb", "edge_len", "edge_nx", "edge_cellL", "edge_cellR", "cell_edge_idx_signed")


def cfg(**kw) -> WorkflowConfig:
    base = {"mesh_source": "mesh.obj", "manning_n": 0.03, "output_interval_s": 10.0, "dt_max": 1.0, "cfl_interval": 1}
    base.update(kw)
    return WorkflowConfig(**base)


@pytest.mark.parametrize(
    ("kw", "match"),
    [
        ({"mesh_source": None}, "mesh_source"),
        ({"manning_n": 0.0}, "manning_n"),
        ({"output_interval_s": 0.0}, "output_interval_s"),
        ({"dt_max": -1.0}, "dt_max"),
        ({"cfl_interval": 0}, "cfl_interval"),
        ({"steps_per_graph": 0}, "steps_per_graph"),
        ({"solver_impl": "cuda"}, "solver_impl"),
        ({"capture_momentum_snapshots": True, "solver_impl": "fixed_dt_batch_barrier"}, "capture_momentum"),
    ],
)
def test_config_rejects(kw: dict, match: str) -> None:
    with pytest.raises(ValueError, match=match):
        cfg(**kw)


def test_config_defaults_to_the_b200_backend() -> None:
    c = cfg()
    assert c.solver_impl == "b200_resident" and c.cfl is None and c.dry_tol == 1e-4


def test_vulkan_backends_are_refused_at_prepare(tmp_path: Path) -> None:
    with pytest.raises(RuntimeError, match="Vulkan"):
        SWEWorkflow(cfg(solver_impl="gpu_resident_batch")).prepare()


def test_source_selection_includes_the_containing_cell() -> None:
    q = quad_grid(10, 10, 1.0)
    g = build_geometry(q.verts, q.faces.reshape(-1, 4), zb_from_file=np.zeros(100, np.float32))
    # A radius smaller than any centroid distance still selects the cell containing the centre.
    m = select_cells_within_radius(g.centroid, (3.2, 4.7), 0.01, None, g.cell_vertices, g.cell_vertex_ptr, g.cell_bbox)
    assert m.sum() == 1 and int(np.flatnonzero(m)[0]) == 4 * 10 + 3
    assert not select_cells_within_radius(g.centroid, (3.2, 4.7), -1.0).any()
    phase = SimulationPhase(10.0, [PointSource(2.0, (5.0, 5.0), 1.6)])
    src = build_phase_source_rate(g, phase, np.ones(100, bool))
    assert src.sum() == pytest.approx(2.0, rel=1e-6)
    assert (src > 0).sum() >= 4


def test_initial_state_forms_and_checks() -> None:
    n = 5
    zb = np.arange(n, dtype=np.float32)
    perm = np.array([4, 3, 2, 1, 0], np.int32)
    h, hu, hv, nm = load_initial_state({"wse": zb + 1.0, "u": np.ones(n), "v": np.zeros(n), "n_mann": np.full(n, 1e-6)},
                                       n, zb, order="solver", id_col="cell_id", perm=perm, dry_tol=1e-4)
    np.testing.assert_array_equal(h, np.ones(n, np.float32))
    np.testing.assert_array_equal(hu, np.ones(n, np.float32))
    assert (nm == np.float32(1e-4)).all()
    h, *_ = load_initial_state({"h": np.arange(n), "hu": np.zeros(n), "hv": np.zeros(n)}, n, zb, order="original",
                               id_col="cell_id", perm=perm, dry_tol=1e-4)
    np.testing.assert_array_equal(h, np.arange(n)[perm].astype(np.float32))
    h, *_ = load_initial_state({"cell_id": [4, 3, 2, 1, 0], "h": np.arange(n), "hu": np.zeros(n), "hv": np.zeros(n)},
                               n, zb, order="solver", id_col="cell_id", perm=perm, dry_tol=1e-4)
    np.testing.assert_array_equal(h, np.arange(n)[::-1].astype(np.float32))
    with pytest.raises(ValueError, match="unsupported"):
        load_initial_state({"h": np.ones(n), "hu": 0, "hv": 0, "zz": 1}, n, zb, order="solver", id_col="c", perm=perm, dry_tol=1e-4)
    with pytest.raises(ValueError, match="'h' or 'wse'"):
        load_initial_state({"hu": np.ones(n), "hv": np.ones(n)}, n, zb, order="solver", id_col="c", perm=perm, dry_tol=1e-4)
    with pytest.raises(ValueError, match="unique"):
        load_initial_state({"cell_id": [0, 0, 1, 2, 3], "h": np.ones(n), "hu": np.ones(n), "hv": np.ones(n)},
                           n, zb, order="solver", id_col="cell_id", perm=perm, dry_tol=1e-4)


def test_artifact_round_trip_and_reference_format(tmp_path: Path) -> None:
    offsets = GEO["voronoi_in_offsets"]
    save_mesh_npz(tmp_path / "m.npz", GEO["voronoi_in_verts"], GEO["voronoi_in_faces"], offsets, GEO["voronoi_in_zb"])
    art = build_geometry_cache(tmp_path / "m.npz", tmp_path / "art.npz")
    geom, perm, meta = load_geometry_cache_artifact(art)
    assert meta.version == GEOMETRY_CACHE_VERSION == 6 and meta.use_hilbert_reorder
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(geom, f), GEO[f"voronoi_hil_{f}"])
    np.testing.assert_array_equal(perm, GEO["voronoi_perm"])
    with np.load(art) as npz:
        assert {"meta", "perm", "N", "E", "V", "max_degree", "manning_n"} <= set(npz.files)
    key = geometry_cache_key(tmp_path / "m.npz", use_hilbert_reorder=True)
    assert load_geometry_cache(tmp_path, key) is None
    save_geometry_cache(tmp_path, key, geom, perm)
    g2, p2 = load_geometry_cache(tmp_path, key)
    np.testing.assert_array_equal(g2.edge_nx, geom.edge_nx)
    with pytest.raises(FileNotFoundError):
        load_geometry_cache_artifact(tmp_path / "missing.npz")


def test_obj_loader_averages_vertex_elevations(tmp_path: Path) -> None:
    obj = tmp_path / "m.obj"
    obj.write_text("v 0 0 1\nv 1 0 2\nv 1 1 3\nv 0 1 4\nf 1 2 3 4\nf 1/1 3/3 4/4\n")
    verts, faces, offsets, zb, manning = load_mesh_file(str(obj))
    assert offsets.tolist() == [0, 4, 7] and faces.tolist() == [0, 1, 2, 3, 0, 2, 3]
    np.testing.assert_allclose(zb, [2.5, 8.0 / 3.0], rtol=1e-6)
    assert manning is None
    obj.write_text("v 0 0\nf 1 2 3\n")
    with pytest.raises(ValueError, match="Z"):
        load_mesh_file(str(obj))
    with pytest.raises(ValueError, match="Unsupported"):
        load_mesh_file(str(tmp_path / "m.shp"))


def test_hilbert_built_geometry_round_trips_through_an_obj(tmp_path: Path) -> None:
    q = quad_grid(8, 4, 2.0)
    lines = [f"v {x} {y} 0.5" for x, y in q.verts] + [
        "f " + " ".join(str(i + 1) for i in q.faces[a:b]) for a, b in zip(q.offsets[:-1], q.offsets[1:])
    ]
    (tmp_path / "g.obj").write_text("\n".join(lines) + "\n")
    verts, faces, offsets, zb, _ = load_mesh_file(str(tmp_path / "g.obj"))
    g = hilbert_reorder(build_geometry(verts, faces, offsets, zb_from_file=zb), verbose=False)[0]
    assert g.N == 32 and (g.zb == np.float32(0.5)).all()
