"""Geometry-cache artifacts: a prebuilt ``MeshGeometry`` on disk.

The file format is the reference's (``inundation/mesh/cache.py:40-67,194-293``):
an ``.npz`` with one entry per ``MeshGeometry`` array (``manning_n`` empty when
absent), the scalars ``N, E, V, max_degree``, the Hilbert permutation ``perm``
and, for explicit artifacts, a JSON ``meta`` blob ``{version, mesh_source,
use_hilbert_reorder}`` with cache version 6. Artifacts written by either
package load in the other, so a pipeline that preprocessed its meshes for the
reference can run them on this backend without the mesh files.
"""

from __future__ import annotations

import hashlib
import json
import os
import zipfile
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np
from numpy.typing import NDArray

from .geometry import MeshGeometry, build_geometry, hilbert_reorder
from .loader import load_mesh_file

GEOMETRY_CACHE_VERSION = 6

ARRAY_FIELDS = (
    "origin", "centroid", "area", "zb", "manning_n", "cell_vertices", "cell_vertex_ptr", "cell_bbox", "edge_len",
    "edge_nx", "edge_ny", "edge_dzL", "edge_dzR", "edge_cellL", "edge_cellR", "edge_sideL", "edge_sideR",
    "cell_edge_ptr", "cell_edge_idx", "cell_nbr_idx", "cell_edge_side", "cell_edge_idx_signed",
)
SCALAR_FIELDS = ("N", "E", "V", "max_degree")


@dataclass(frozen=True)
class GeometryCacheMeta:
    version: int
    mesh_source: str
    use_hilbert_reorder: bool


def geometry_cache_key(mesh_path: str | os.PathLike[str], *, use_hilbert_reorder: bool) -> str:
    """Key of a mesh file's cache entry: the file's bytes, the format version and the order."""
    h = hashlib.blake2b(digest_size=32)
    h.update(f"v{GEOMETRY_CACHE_VERSION}|hilbert={use_hilbert_reorder}|".encode())
    with Path(mesh_path).open("rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def geometry_cache_path(cache_dir: str | os.PathLike[str], cache_key: str) -> Path:
    return Path(cache_dir) / f"geometry_{cache_key}.npz"


def write_geometry_npz(path: Path, geom: MeshGeometry, perm: NDArray[np.int32], meta: GeometryCacheMeta | None = None) -> Path:
    """Write ``geom`` and ``perm`` (and ``meta``) atomically through a temporary file."""
    payload: dict[str, Any] = {}
    for name in ARRAY_FIELDS:
        value = getattr(geom, name)
        payload[name] = np.empty(0, np.float32) if value is None else value
    payload.update({name: np.int64(getattr(geom, name)) for name in SCALAR_FIELDS})
    payload["perm"] = np.asarray(perm, np.int32)
    if meta is not None:
        payload["meta"] = np.asarray(json.dumps(
            {"version": meta.version, "mesh_source": meta.mesh_source, "use_hilbert_reorder": meta.use_hilbert_reorder}
        ))
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_name(path.name + ".tmp")
    with tmp.open("wb") as f:
        np.savez(f, **payload)
    tmp.replace(path)
    return path


def geometry_from_payload(payload: dict[str, Any]) -> MeshGeometry:
    arrays = {name: payload[name] for name in ARRAY_FIELDS}
    arrays["manning_n"] = None if arrays["manning_n"].size == 0 else arrays["manning_n"]
    return MeshGeometry(**arrays, **{name: int(payload[name]) for name in SCALAR_FIELDS})


def _read(path: Path) -> dict[str, Any]:
    with np.load(path) as npz:
        return {name: npz[name] for name in npz.files}


def _meta(raw: NDArray[Any]) -> GeometryCacheMeta:
    try:
        data = json.loads(str(raw.item()))
        return GeometryCacheMeta(int(data["version"]), str(data["mesh_source"]), bool(data["use_hilbert_reorder"]))
    except (AttributeError, TypeError, ValueError, KeyError) as exc:
        raise ValueError(f"invalid geometry cache metadata: {raw!r}") from exc


def build_geometry_cache(
    mesh_source: str | os.PathLike[str], out_path: str | os.PathLike[str], *, use_hilbert_reorder: bool = True,
    progress: bool = False,
) -> Path:
    """Load a mesh file, build (and Hilbert-order) its geometry and write an artifact."""
    verts, faces, offsets, zb, manning = load_mesh_file(os.fspath(mesh_source))
    geom = build_geometry(verts, faces, offsets, zb_from_file=zb, manning_n_from_file=manning, progress=progress)
    perm = np.arange(geom.N, dtype=np.int32)
    if use_hilbert_reorder:
        geom, perm = hilbert_reorder(geom, verbose=progress)
    meta = GeometryCacheMeta(GEOMETRY_CACHE_VERSION, os.fspath(mesh_source), use_hilbert_reorder)
    return write_geometry_npz(Path(out_path), geom, perm, meta)


def load_geometry_cache_artifact(path: str | os.PathLike[str]) -> tuple[MeshGeometry, NDArray[np.int32], GeometryCacheMeta]:
    """An explicit artifact: raises on a missing, unreadable or stale file."""
    p = Path(path)
    if not p.exists():
        raise FileNotFoundError(f"geometry cache artifact not found: {p}")
    try:
        payload = _read(p)
    except (OSError, ValueError, KeyError, EOFError, zipfile.BadZipFile) as exc:
        raise ValueError(f"unreadable geometry cache artifact {p}: {exc}") from exc
    missing = [n for n in (*ARRAY_FIELDS, *SCALAR_FIELDS, "perm", "meta") if n not in payload]
    if missing:
        raise ValueError(f"geometry cache artifact {p} is missing fields: {missing}")
    meta = _meta(payload["meta"])
    if meta.version != GEOMETRY_CACHE_VERSION:
        raise ValueError(
            f"geometry cache artifact {p} was written with cache version {meta.version}, this build expects "
            f"{GEOMETRY_CACHE_VERSION}: rebuild it with build_geometry_cache()"
        )
    return geometry_from_payload(payload), payload["perm"], meta


def save_geometry_cache(cache_dir: str | os.PathLike[str], cache_key: str, geom: MeshGeometry, perm: NDArray[np.int32]) -> Path:
    return write_geometry_npz(geometry_cache_path(cache_dir, cache_key), geom, perm)


def load_geometry_cache(cache_dir: str | os.PathLike[str], cache_key: str) -> tuple[MeshGeometry, NDArray[np.int32]] | None:
    """A directory cache entry, or None on any miss (a cache is only an optimisation)."""
    p = geometry_cache_path(cache_dir, cache_key)
    if not p.exists():
        return None
    try:
        payload = _read(p)
    except (OSError, ValueError, KeyError, EOFError, zipfile.BadZipFile):
        return None
    if any(n not in payload for n in (*ARRAY_FIELDS, *SCALAR_FIELDS, "perm")):
        return None
    return geometry_from_payload(payload), payload["perm"]
