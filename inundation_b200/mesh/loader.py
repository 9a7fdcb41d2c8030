"""Mesh files: Wavefront OBJ (as the reference reads it) and a plain ``.npz``.

* ``.obj``: ``v x y z`` records (z required) and ``f i j k ...`` polygons
  (1-based, ``i/t/n`` accepted); the bed of a cell is the mean of its vertices'
  z, in float32 (the reference's ``inundation/mesh/loader.py:177-211``).
* ``.npz``: arrays ``verts (V, 2)``, ``faces`` (flat) with ``face_offsets``
  (N+1) or ``faces (N, d)``, ``zb (N,)`` and optionally ``manning_n (N,)``.

The reference's GIS readers (GeoPackage, shapefile, GeoParquet) need
geopandas/shapely and sit outside the step's scope.
"""

from __future__ import annotations

import os
from pathlib import Path

import numpy as np
from numpy.typing import NDArray

MIN_POLYGON_VERTICES = 3


def _optional_manning(values: object) -> NDArray[np.float32]:
    n = np.asarray(values, dtype=np.float32).reshape(-1)
    if not np.isfinite(n).all() or not (n > 0.0).all():
        raise ValueError("manning_n must contain finite positive values")
    return n


def load_mesh_file(path: str) -> tuple[NDArray[np.float64], NDArray[np.int32], NDArray[np.int32], NDArray[np.float32], NDArray[np.float32] | None]:
    """``(verts, faces, face_offsets, zb, manning_n or None)`` of a mesh file."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".obj":
        xy: list[list[float]] = []
        z: list[float] = []
        polys: list[list[int]] = []
        with open(path) as fh:
            for line in fh:
                parts = line.strip().split()
                if not parts or parts[0].startswith("#"):
                    continue
                if parts[0] == "v":
                    if len(parts) < 4:
                        raise ValueError(f"OBJ file '{path}' has a vertex without required Z elevation")
                    xy.append([float(parts[1]), float(parts[2])])
                    z.append(float(parts[3]))
                elif parts[0] == "f":
                    idx = [int(p.split("/")[0]) - 1 for p in parts[1:]]
                    if len(idx) < MIN_POLYGON_VERTICES:
                        raise ValueError(f"OBJ face has {len(idx)} vertices — need at least 3.")
                    polys.append(idx)
        if not polys:
            raise ValueError(f"OBJ file '{path}' contains no face ('f') records.")
        vz = np.asarray(z, dtype=np.float32)
        if not np.isfinite(vz).all():
            raise ValueError(f"OBJ file '{path}' contains non-finite vertex elevations")
        faces = np.concatenate([np.asarray(f, np.int32) for f in polys])
        offsets = np.zeros(len(polys) + 1, np.int32)
        np.cumsum([len(f) for f in polys], out=offsets[1:])
        zb = np.asarray([vz[f].mean() for f in polys], dtype=np.float32)
        return np.asarray(xy, np.float64), faces, offsets, zb, None
    if ext == ".npz":
        with np.load(path) as npz:
            data = {k: npz[k] for k in npz.files}
        for key in ("verts", "faces", "zb"):
            if key not in data:
                raise ValueError(f"mesh file '{path}' is missing '{key}'")
        faces = np.asarray(data["faces"], np.int32)
        if faces.ndim == 2:
            offsets = np.arange(0, faces.size + 1, faces.shape[1], dtype=np.int32)
            faces = faces.ravel()
        elif "face_offsets" in data:
            offsets = np.asarray(data["face_offsets"], np.int32)
        else:
            raise ValueError(f"mesh file '{path}' has flat 'faces' without 'face_offsets'")
        zb = np.asarray(data["zb"], np.float32)
        if not np.isfinite(zb).all():
            raise ValueError(f"mesh file '{path}' contains non-finite bed elevations")
        manning = _optional_manning(data["manning_n"]) if "manning_n" in data else None
        return np.asarray(data["verts"], np.float64)[:, :2], faces, offsets, zb, manning
    raise ValueError(f"Unsupported format: '{ext}'. Supported here: .obj, .npz")


def save_mesh_npz(path: str | os.PathLike[str], verts, faces, face_offsets, zb, manning_n=None) -> Path:
    """Write a mesh in the ``.npz`` form ``load_mesh_file`` reads."""
    out = {"verts": np.asarray(verts), "faces": np.asarray(faces), "face_offsets": np.asarray(face_offsets), "zb": np.asarray(zb)}
    if manning_n is not None:
        out["manning_n"] = np.asarray(manning_n)
    p = Path(path)
    np.savez(p, **out)
    return p
