"""Geometry-cache files written by the reference load here, and this package writes the same format.

The fixtures under ``tests/golden/`` were written by the reference's own
``build_geometry_cache`` and ``save_geometry_cache``
(``inundation/mesh/cache.py:103-191``, cache version 6) from
``tests/golden/cache_mesh.obj``, by ``tests/golden/make_golden.py --parts cache``.
"""

from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np
import pytest

from inundation_b200.layout import build_tile_layout
from inundation_b200.mesh.cache import (
    ARRAY_FIELDS,
    GEOMETRY_CACHE_VERSION,
    SCALAR_FIELDS,
    build_geometry_cache,
    geometry_cache_key,
    load_geometry_cache,
    load_geometry_cache_artifact,
)

GOLD = Path(__file__).resolve().parent / "golden"
ROOT = GOLD.parent.parent
MESH = "tests/golden/cache_mesh.obj"


@pytest.fixture()
def at_root():
    """Mesh sources are recorded as given: run from the repository root like the fixture writer."""
    here = os.getcwd()
    os.chdir(ROOT)
    yield
    os.chdir(here)


def assert_same_geometry(a, b) -> None:
    for name in ARRAY_FIELDS:
        x, y = getattr(a, name), getattr(b, name)
        if x is None or y is None:
            assert x is None and y is None, name
            continue
        assert x.dtype == y.dtype and x.shape == y.shape, name
        np.testing.assert_array_equal(x, y, err_msg=name)
    for name in SCALAR_FIELDS:
        assert getattr(a, name) == getattr(b, name), name


@pytest.mark.parametrize("artifact, hilbert", [("ref_cache_hilbert.npz", True), ("ref_cache_file_order.npz", False)])
def test_reference_artifacts_load_and_equal_this_builder(artifact: str, hilbert: bool, tmp_path, at_root) -> None:
    geom, perm, meta = load_geometry_cache_artifact(GOLD / artifact)
    assert meta.version == GEOMETRY_CACHE_VERSION == 6
    assert meta.use_hilbert_reorder is hilbert and meta.mesh_source == MESH
    assert geom.N == 72 and perm.shape == (72,)
    if not hilbert:
        np.testing.assert_array_equal(perm, np.arange(72))
    ours = build_geometry_cache(MESH, tmp_path / "ours.npz", use_hilbert_reorder=hilbert)
    g2, p2, m2 = load_geometry_cache_artifact(ours)
    assert m2 == meta
    np.testing.assert_array_equal(p2, perm)
    assert_same_geometry(g2, geom)
    build_tile_layout(geom)  # the artifact's geometry lays out for the kernels


def test_this_writer_uses_the_reference_format(tmp_path, at_root) -> None:
    """Same entries, dtypes, shapes and metadata as the reference's artifact, so its loader reads ours."""
    ours = build_geometry_cache(MESH, tmp_path / "ours.npz", use_hilbert_reorder=True)
    with np.load(GOLD / "ref_cache_hilbert.npz") as ref, np.load(ours) as mine:
        assert sorted(ref.files) == sorted(mine.files)
        for name in ref.files:
            assert ref[name].dtype == mine[name].dtype and ref[name].shape == mine[name].shape, name
            if name == "meta":
                assert json.loads(str(ref[name].item())) == json.loads(str(mine[name].item()))
            else:
                np.testing.assert_array_equal(ref[name], mine[name], err_msg=name)


def test_reference_directory_cache_entry_is_found_by_its_key(at_root) -> None:
    key = geometry_cache_key(MESH, use_hilbert_reorder=True)
    assert (GOLD / "ref_cache_dir" / f"geometry_{key}.npz").exists()
    hit = load_geometry_cache(GOLD / "ref_cache_dir", key)
    assert hit is not None
    geom, perm = hit
    ref, ref_perm, _ = load_geometry_cache_artifact(GOLD / "ref_cache_hilbert.npz")
    assert_same_geometry(geom, ref)
    np.testing.assert_array_equal(perm, ref_perm)
    assert load_geometry_cache(GOLD / "ref_cache_dir", geometry_cache_key(MESH, use_hilbert_reorder=False)) is None
