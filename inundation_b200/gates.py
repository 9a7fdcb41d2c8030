"""Physical validation gates of the B200 backend: analytic and reference solutions.

The cases and thresholds of the reference's benchmark harnesses
(``inundation/bench/dambreak.py``, ``radial_dambreak.py``, ``parabolic_bowl.py``,
``lake_at_rest.py``, ``open_boundary.py``), run on ``SWESolverB200Resident``:

* ``stoker`` / ``ritter``: the wet- and dry-bed 1-D dam breaks on a flat
  frictionless 1000 m x 10 m channel (dam at 500 m, 10 m upstream, 1 m or dry
  downstream, 20 s), against Stoker's (1957) and Ritter's (1892) exact
  solutions: relative L1 depth error of the column means <= 5 %, Ritter wet
  front within 15 % of its travel, volume drift <= 1e-5.
* ``radial``: the circular dam break (2.5 m inside r = 2.5 m, 0.5 m outside, a
  40 m square, 1.5 s) against a fine 1-D axisymmetric finite-volume solution:
  azimuthal-mean L1 <= 10 %, bore radius within 5 %, the bore radius of 12
  angular sectors within 8 % of each other, volume drift <= 1e-5.
* ``bowl``: Thacker's (1981) planar surface rotating in a frictionless
  paraboloid, wetting and drying every period: mean relative L1 depth error
  over the snapshots < 0.18 at nx = 200, films below 1 mm slower than 1 m/s,
  no positivity clamp, volume drift < 1e-7.
* ``lake``: still water over Gaussian bumps: max speed over wet cells and the
  volume drift at round-off.
* ``uniform``: 10 m^3/s into a dry channel sloped 1e-3 (2 km x 40 m, n = 0.03)
  through an inflow, out through a normal-depth outlet, 4 h: mean depth over
  the middle fifth within 1 % of Manning's normal depth, the last window's
  outflow within 1e-3 of the discharge, the inflow volume within 1e-7.
* ``held_lake``: still water at 12 m over a bed of two sines, held by its own
  level as a stage at both ends, 300 s: level within 1e-4 m, speeds below
  1e-3 m/s.
* ``backwater_m1`` / ``backwater_m2``: the inflow into a 3 km channel held at its
  outlet 0.8 m or 0.25 m above the bed, 6 h, against the gradually varied flow
  profile (within 1.5 %).
* ``basins``: a hydrograph through a 4 km channel run whole, and cut in two with
  the upper half's outflow passed into the lower half by ``inflow_phases``.

``python -m inundation_b200.gates [case ...]`` prints one JSON line per case.
"""

from __future__ import annotations

import argparse
import json
import math
import sys
import time
from collections.abc import Callable

import numpy as np
from numpy.typing import NDArray

from .mesh.geometry import MeshGeometry, build_geometry, hilbert_reorder
from .mesh.synthetic import channel_grid, quad_grid
from .tuning import GRAVITY_G, OPEN_INFLOW, OPEN_NORMAL, OPEN_STAGE

MANNING_FLOOR = 1e-4  # the solver-wide floor: a frictionless case runs at this n

# -- analytic and reference solutions --------------------------------------------------------


def ritter(x: NDArray, t: float, *, h_up: float, dam_x: float, g: float = GRAVITY_G) -> tuple[NDArray, NDArray]:
    """Ritter's dry-bed dam break at time t: still water upstream of the fan x - dam_x <= -c0 t,
    the fan h = (2 c0 - xi)^2 / 9g, u = 2 (xi + c0) / 3 up to the front xi = 2 c0, dry beyond."""
    if t <= 0.0:
        raise ValueError(f"t must be positive, got {t}")
    xi = (np.asarray(x, np.float64) - dam_x) / t
    c0 = math.sqrt(g * h_up)
    h, u = np.zeros_like(xi), np.zeros_like(xi)
    h[xi <= -c0] = h_up
    fan = (xi > -c0) & (xi < 2.0 * c0)
    h[fan] = (2.0 * c0 - xi[fan]) ** 2 / (9.0 * g)
    u[fan] = 2.0 * (xi[fan] + c0) / 3.0
    return h, u


def stoker_middle_depth(h_up: float, h_down: float, g: float = GRAVITY_G) -> float:
    """The plateau depth of Stoker's wet-bed dam break: where the rarefaction's velocity
    2 (c0 - cm) equals the bore's (hm - h_down) sqrt(g (hm + h_down) / (2 hm h_down)); bisection."""
    if not 0.0 < h_down < h_up:
        raise ValueError(f"need 0 < h_down < h_up, got {h_down}, {h_up}")
    c0 = math.sqrt(g * h_up)

    def mismatch(hm: float) -> float:
        return 2.0 * (c0 - math.sqrt(g * hm)) - (hm - h_down) * math.sqrt(g * (hm + h_down) / (2.0 * hm * h_down))

    lo, hi = h_down, h_up
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if mismatch(mid) > 0.0 else (lo, mid)
    return 0.5 * (lo + hi)


def stoker(x: NDArray, t: float, *, h_up: float, h_down: float, dam_x: float,
           g: float = GRAVITY_G) -> tuple[NDArray, NDArray]:
    """Stoker's wet-bed dam break at time t: still upstream, rarefaction fan, plateau (hm, um)
    up to the bore at speed um hm / (hm - h_down), still downstream."""
    if t <= 0.0:
        raise ValueError(f"t must be positive, got {t}")
    xi = (np.asarray(x, np.float64) - dam_x) / t
    c0 = math.sqrt(g * h_up)
    hm = stoker_middle_depth(h_up, h_down, g)
    cm = math.sqrt(g * hm)
    um = 2.0 * (c0 - cm)
    bore = um * hm / (hm - h_down)
    h, u = np.full_like(xi, h_down), np.zeros_like(xi)
    h[xi <= -c0] = h_up
    fan = (xi > -c0) & (xi < um - cm)
    h[fan] = (2.0 * c0 - xi[fan]) ** 2 / (9.0 * g)
    u[fan] = 2.0 * (xi[fan] + c0) / 3.0
    plateau = (xi >= um - cm) & (xi < bore)
    h[plateau], u[plateau] = hm, um
    return h, u


def radial_reference(t: float, *, h_in: float, h_out: float, r_dam: float, r_max: float, cells: int = 2000,
                     cfl: float = 0.9, g: float = GRAVITY_G, dry_tol: float = 1e-8) -> tuple[NDArray, NDArray, NDArray]:
    """The axisymmetric dam break on [0, r_max] by a fine 1-D finite-volume scheme.

    Conservative form in r: d(r h)/dt + d(r h u)/dr = 0 and d(r h u)/dt +
    d(r (h u^2 + g h^2 / 2))/dr = g h^2 / 2, with HLL fluxes (Harten, Lax and
    van Leer; Davis speed estimates), Heun steps at CFL ``cfl``, no flux of
    mass through r = 0 and a transmissive outer face. Returns the cell
    centres, depth and velocity at time t; no closed form exists.
    """
    dr = r_max / cells
    rc = (np.arange(cells) + 0.5) * dr
    rf = np.arange(cells + 1) * dr
    h = np.where(rc < r_dam, h_in, h_out).astype(np.float64)
    m = np.zeros(cells)

    def vel(hh: NDArray, mm: NDArray) -> NDArray:
        return np.where(hh > dry_tol, mm / np.maximum(hh, dry_tol), 0.0)

    def rates(hh: NDArray, mm: NDArray) -> tuple[NDArray, NDArray]:
        uu = vel(hh, mm)
        c = np.sqrt(g * np.maximum(hh, 0.0))
        fh = np.empty(cells + 1)
        fm = np.empty(cells + 1)
        hl, hr, ml, mr, ul, ur, cl, cr = hh[:-1], hh[1:], mm[:-1], mm[1:], uu[:-1], uu[1:], c[:-1], c[1:]
        pl, pr = ml * ul + 0.5 * g * hl * hl, mr * ur + 0.5 * g * hr * hr
        sl, sr = np.minimum(ul - cl, ur - cr), np.maximum(ul + cl, ur + cr)
        span = np.where(sr > sl, sr - sl, 1.0)
        mid_h = (sr * ml - sl * mr + sl * sr * (hr - hl)) / span
        mid_m = (sr * pl - sl * pr + sl * sr * (mr - ml)) / span
        fh[1:-1] = np.where(sl >= 0.0, ml, np.where(sr <= 0.0, mr, mid_h))
        fm[1:-1] = np.where(sl >= 0.0, pl, np.where(sr <= 0.0, pr, mid_m))
        fh[0], fm[0] = 0.0, 0.5 * g * hh[0] ** 2
        fh[-1], fm[-1] = mm[-1], mm[-1] * uu[-1] + 0.5 * g * hh[-1] ** 2
        dh = -(rf[1:] * fh[1:] - rf[:-1] * fh[:-1]) / (dr * rc)
        dm = (-(rf[1:] * fm[1:] - rf[:-1] * fm[:-1]) / dr + 0.5 * g * hh * hh) / rc
        return dh, dm

    now = 0.0
    while now < t:
        speed = float((np.abs(vel(h, m)) + np.sqrt(g * np.maximum(h, 0.0))).max())
        dt = min(cfl * dr / speed if speed > 0.0 else t, t - now)
        dh1, dm1 = rates(h, m)
        h1 = np.maximum(h + dt * dh1, 0.0)
        m1 = np.where(h1 > dry_tol, m + dt * dm1, 0.0)
        dh2, dm2 = rates(h1, m1)
        h = np.maximum(h + 0.5 * dt * (dh1 + dh2), 0.0)
        m = np.where(h > dry_tol, m + 0.5 * dt * (dm1 + dm2), 0.0)
        now += dt
    return rc, h, vel(h, m)


def thacker_omega(centre_depth: float, radius: float, g: float = GRAVITY_G) -> float:
    return math.sqrt(2.0 * g * centre_depth) / radius


def thacker(x: NDArray, y: NDArray, t: float, *, centre_depth: float, radius: float, swing: float,
            g: float = GRAVITY_G) -> tuple[NDArray, NDArray, NDArray]:
    """Thacker's planar surface in the paraboloid z = -D (1 - r^2 / R^2): the surface
    eta = (swing D / R^2)(2 x cos wt + 2 y sin wt - swing) and the uniform velocity
    (-swing w sin wt, swing w cos wt) over the wet region."""
    w = thacker_omega(centre_depth, radius, g)
    c, s = math.cos(w * t), math.sin(w * t)
    bed = -centre_depth * (1.0 - (x * x + y * y) / radius**2)
    eta = swing * centre_depth / radius**2 * (2.0 * x * c + 2.0 * y * s - swing)
    h = np.maximum(eta - bed, 0.0)
    wet = h > 0.0
    return h, np.where(wet, -swing * w * s, 0.0), np.where(wet, swing * w * c, 0.0)


def normal_depth(discharge: float, width: float, slope: float, manning: float) -> float:
    """Manning's normal depth of a wide channel: q = h^(5/3) sqrt(S) / n, q = Q / width."""
    return (discharge / width * manning / math.sqrt(slope)) ** 0.6


# -- meshes ----------------------------------------------------------------------------------


def _geometry(verts: NDArray, faces: NDArray, offsets: NDArray | None, zb: NDArray) -> MeshGeometry:
    g = build_geometry(verts, faces, offsets, zb_from_file=np.asarray(zb, np.float32))
    return hilbert_reorder(g, verbose=False)[0]


def channel_geometry(cells: int, across: int, length: float, width: float,
                     bed: Callable[[NDArray], NDArray] | None = None, x0: float = 0.0) -> MeshGeometry:
    """A channel of ``cells`` x ``across`` rectangles from x = x0, its bed a function of x."""
    mesh = channel_grid(cells, across, length, width)
    x = np.tile((np.arange(cells) + 0.5) * (length / cells), across) + x0
    zb = np.zeros(x.size) if bed is None else bed(x)
    verts = mesh.verts.copy()
    verts[:, 0] += x0
    return _geometry(verts, mesh.faces, mesh.offsets, zb)


def column_profile(geom: MeshGeometry, h: NDArray) -> tuple[NDArray, NDArray]:
    """Depth averaged across a channel, by position along it."""
    x, inverse = np.unique(np.round(geom.world_centroid[:, 0], 6), return_inverse=True)
    return x, np.bincount(inverse, weights=np.asarray(h, np.float64)) / np.bincount(inverse)


def gradually_varied_profile(x: NDArray, depth_at_end: float, end_x: float, unit_discharge: float, slope: float,
                             manning: float, g: float = GRAVITY_G) -> NDArray:
    """Steady depth at ascending x, integrated upstream from ``end_x`` by classical RK4 steps
    of at most 1 m on dh/dx = (S - Sf) / (1 - Fr^2), Sf = n^2 q^2 / h^(10/3), Fr^2 = q^2 / (g h^3)."""

    def dhdx(h: float) -> float:
        return (slope - manning**2 * unit_discharge**2 / h ** (10.0 / 3.0)) / (1.0 - unit_discharge**2 / (g * h**3))

    out = np.empty(len(x))
    h, pos = depth_at_end, end_x
    for k in range(len(x) - 1, -1, -1):
        dist = pos - float(x[k])
        n = max(1, math.ceil(dist))
        dx = -dist / n
        for _ in range(n):
            k1 = dhdx(h)
            k2 = dhdx(h + 0.5 * dx * k1)
            k3 = dhdx(h + 0.5 * dx * k2)
            k4 = dhdx(h + dx * k3)
            h += dx * (k1 + 2.0 * k2 + 2.0 * k3 + k4) / 6.0
        out[k] = h
        pos = float(x[k])
    return out


def square_geometry(n: int, side: float, origin: float = 0.0,
                    bed: Callable[[NDArray, NDArray], NDArray] | None = None) -> MeshGeometry:
    mesh = quad_grid(n, n, side / n)
    c = (np.arange(n) + 0.5) * (side / n) + origin
    cx, cy = np.tile(c, n), np.repeat(c, n)
    zb = np.zeros(n * n) if bed is None else bed(cx, cy)
    return _geometry(mesh.verts + origin, mesh.faces, mesh.offsets, zb)


# -- the cases -------------------------------------------------------------------------------


def _solver(geom, h, hu, hv, n, **kw):
    from .backend import SWESolverB200Resident

    dry_tol = kw.pop("dry_tol", 1e-4)
    cfl = kw.pop("cfl", None)
    s = SWESolverB200Resident(geom, None, np.asarray(h, np.float32), np.asarray(hu, np.float32),
                              np.asarray(hv, np.float32), np.asarray(n, np.float32), dry_tol=dry_tol, cfl=cfl, **kw)
    s.track_clamp = True
    return s


def _volume(geom, h) -> float:
    return float((np.asarray(h, np.float64) * geom.area.astype(np.float64)).sum())


def _l1(num: NDArray, ref: NDArray) -> float:
    return float(np.abs(num - ref).sum() / max(np.abs(ref).sum(), 1e-300))


def dambreak(case: str = "stoker", nx: int = 500, ny: int = 5, t_end: float = 20.0) -> dict:
    """``inundation/bench/dambreak.py``: 1000 m x 10 m, dam at 500 m, 10 m up, 1 m (Stoker) or dry (Ritter)."""
    length, width, dam, h_up = 1000.0, 10.0, 500.0, 10.0
    h_down = 0.0 if case == "ritter" else 1.0
    geom = channel_geometry(nx, ny, length, width)
    x = geom.world_centroid[:, 0]
    h0 = np.where(x < dam, h_up, h_down)
    z = np.zeros(geom.N)
    s = _solver(geom, h0, z, z, np.full(geom.N, MANNING_FLOOR))
    t0 = time.perf_counter()
    s.run(t_end=t_end, output_interval_s=t_end, dt_max=0.02, dt_init=1e-3, cfl_interval=1, progress=False)
    wall = time.perf_counter() - t0
    h = s.download_h().astype(np.float64)
    dx = length / nx
    col = np.clip((x / dx).astype(np.int64), 0, nx - 1)
    h_num = np.bincount(col, weights=h, minlength=nx) / np.maximum(np.bincount(col, minlength=nx), 1)
    xc = (np.arange(nx) + 0.5) * dx
    h_ex = (ritter(xc, t_end, h_up=h_up, dam_x=dam) if case == "ritter"
            else stoker(xc, t_end, h_up=h_up, h_down=h_down, dam_x=dam))[0]
    out = {"case": case, "cells": geom.N, "steps": s.steps_total, "wall_s": wall, "l1_rel": _l1(h_num, h_ex),
           "volume_drift_rel": abs(s.volume_fp64() - _volume(geom, h0.astype(np.float32))) / _volume(geom, h0),
           "min_depth_m": float(h.min()), "finite": bool(np.isfinite(h).all())}
    gates = {"l1_rel": 0.05, "volume_drift_rel": 1e-5}
    if case == "ritter":
        wet = xc[h_num > 1e-3]
        travel = 2.0 * math.sqrt(GRAVITY_G * h_up) * t_end
        out["front_rel_err"] = abs((float(wet.max()) if wet.size else dam) - (dam + travel)) / travel
        gates["front_rel_err"] = 0.15
    return _gate_result(out, gates)


def radial(n: int = 200, t_end: float = 1.5) -> dict:
    """``inundation/bench/radial_dambreak.py``: a 40 m square, 2.5 m inside r = 2.5 m, 0.5 m outside."""
    side, r_dam, h_in, h_out = 40.0, 2.5, 2.5, 0.5
    centre = side / 2.0
    geom = square_geometry(n, side)
    cx, cy = geom.world_centroid[:, 0] - centre, geom.world_centroid[:, 1] - centre
    r = np.hypot(cx, cy)
    h0 = np.where(r < r_dam, h_in, h_out)
    z = np.zeros(geom.N)
    s = _solver(geom, h0, z, z, np.full(geom.N, MANNING_FLOOR))
    t0 = time.perf_counter()
    s.run(t_end=t_end, output_interval_s=t_end, dt_max=0.05, dt_init=1e-3, cfl_interval=1, progress=False)
    wall = time.perf_counter() - t0
    h = s.download_h().astype(np.float64)
    dx = side / n
    r_max = centre  # annuli inside the inscribed circle only
    nb = max(1, round(r_max / dx))
    idx = (r / (r_max / nb)).astype(np.int64)
    inside = idx < nb
    counts = np.bincount(idx[inside], minlength=nb)
    h_num = np.bincount(idx[inside], weights=h[inside], minlength=nb) / np.maximum(counts, 1)
    rb = (np.arange(nb) + 0.5) * (r_max / nb)
    rc, h_ref_fine, _ = radial_reference(t_end, h_in=h_in, h_out=h_out, r_dam=r_dam, r_max=r_max)
    h_ref = np.interp(rb, rc, h_ref_fine)
    valid = counts > 0
    threshold = 1.2 * h_out

    def front(rr: NDArray, hh: NDArray, ok: NDArray) -> float:
        wet = (hh > threshold) & ok
        return float(rr[wet].max()) if wet.any() else r_dam

    front_ref = front(rc, h_ref_fine, np.ones(rc.size, bool))
    theta = np.arctan2(cy, cx)
    sector = ((theta + np.pi) / (2.0 * np.pi) * 12).astype(np.int64) % 12
    bw = 2.0 * dx
    nbs = max(1, round(r_max / bw))
    rs = (np.arange(nbs) + 0.5) * bw
    fronts = []
    for k in range(12):
        sel = (r < r_max) & (sector == k)
        i = np.clip((r[sel] / bw).astype(np.int64), 0, nbs - 1)
        cnt = np.bincount(i, minlength=nbs)
        fronts.append(front(rs, np.bincount(i, weights=h[sel], minlength=nbs) / np.maximum(cnt, 1), cnt > 0))
    fronts_a = np.asarray(fronts)
    out = {"case": "radial", "cells": geom.N, "steps": s.steps_total, "wall_s": wall,
           "l1_rel": _l1(h_num[valid], h_ref[valid]),
           "front_rel_err": abs(front(rb, h_num, valid) - front_ref) / front_ref,
           "isotropy_spread": float((fronts_a.max() - fronts_a.min()) / fronts_a.mean()),
           "volume_drift_rel": abs(s.volume_fp64() - _volume(geom, h0.astype(np.float32))) / _volume(geom, h0),
           "min_depth_m": float(h.min()), "finite": bool(np.isfinite(h).all())}
    return _gate_result(out, {"l1_rel": 0.10, "front_rel_err": 0.05, "isotropy_spread": 0.08, "volume_drift_rel": 1e-5})


def bowl(n: int = 200, periods: int = 3, cfl: float | None = None) -> dict:
    """``inundation/bench/parabolic_bowl.py``: R = 1 m, D = 0.1 m, swing 0.5 m, a 4 m square."""
    radius, depth, swing, side = 1.0, 0.1, 0.5, 4.0
    paraboloid = lambda x, y: -depth * (1.0 - (x * x + y * y) / radius**2)  # noqa: E731
    geom = square_geometry(n, side, origin=-side / 2.0, bed=paraboloid)
    x, y = geom.world_centroid[:, 0], geom.world_centroid[:, 1]
    area = geom.area.astype(np.float64)
    h0, u0, v0 = thacker(x, y, 0.0, centre_depth=depth, radius=radius, swing=swing)
    s = _solver(geom, h0, h0 * u0, h0 * v0, np.full(geom.N, MANNING_FLOOR), cfl=cfl)
    t_end = periods * 2.0 * math.pi / thacker_omega(depth, radius)
    t0 = time.perf_counter()
    snaps, times = s.run(t_end=t_end, output_interval_s=t_end / (8 * periods), dt_max=0.05, dt_init=1e-3,
                         cfl_interval=1, progress=False)
    wall = time.perf_counter() - t0
    errors = []
    for snap, t in zip(snaps[1:], times[1:], strict=True):
        he = thacker(x, y, t, centre_depth=depth, radius=radius, swing=swing)[0]
        errors.append(float((np.abs(np.asarray(snap, np.float64) - he) * area).sum() / (he * area).sum()))
    h = s.download_h().astype(np.float64)
    qx, qy = s.download_hu().astype(np.float64), s.download_hv().astype(np.float64)
    film = (h >= 1e-4) & (h < 1e-3)
    film_speed = float((np.hypot(qx[film], qy[film]) / h[film]).max()) if film.any() else 0.0
    v0_total = _volume(geom, h0.astype(np.float32))
    out = {"case": "bowl", "cells": geom.N, "steps": s.steps_total, "wall_s": wall,
           "depth_l1_rel_mean": float(np.mean(errors)), "depth_l1_rel_final": errors[-1],
           "film_speed_max_ms": film_speed,
           "clamp_rel": float(np.asarray(s.download_clamp_mass(), np.float64).sum()) / v0_total,
           "volume_drift_rel": abs(s.volume_fp64() - v0_total) / v0_total}
    gates = {"film_speed_max_ms": 1.0, "volume_drift_rel": 1e-7, "clamp_rel": 0.0}
    if n == 200:
        gates["depth_l1_rel_mean"] = 0.18
    return _gate_result(out, gates, strict=("depth_l1_rel_mean", "film_speed_max_ms", "volume_drift_rel"))


def lake(cells: int = 8000, t_end: float = 600.0) -> dict:
    """``inundation/bench/lake_at_rest.py``: still water at 1 m over six Gaussian bumps, CFL 0.9."""
    from .scenarios import lake_at_rest

    sc = lake_at_rest(cells, seed=1)
    s = _solver(sc.geom, sc.h0, sc.hu0, sc.hv0, sc.manning, dry_tol=sc.dry_tol, cfl=sc.meta["cfl"])
    v0 = s.volume_fp64()
    t0 = time.perf_counter()
    s.run(t_end=t_end, output_interval_s=t_end, dt_max=1.0, dt_init=0.01, cfl_interval=10, progress=False)
    wall = time.perf_counter() - t0
    h, hu, hv = s.download_h(), s.download_hu(), s.download_hv()
    wet = h > 10 * sc.dry_tol
    max_u = float(max((np.abs(hu[wet]) / h[wet]).max(), (np.abs(hv[wet]) / h[wet]).max()))
    out = {"case": "lake", "cells": sc.geom.N, "steps": s.steps_total, "wall_s": wall, "max_speed_ms": max_u,
           "volume_drift_rel": abs(s.volume_fp64() - v0) / v0}
    return _gate_result(out, {"max_speed_ms": 0.01, "volume_drift_rel": 1e-9})


def uniform(cells: int = 200, length: float = 2000.0, width: float = 40.0, across: int = 2,
            discharge: float = 10.0, slope: float = 1e-3, manning: float = 0.03, hours: float = 4.0) -> dict:
    """``inundation/bench/open_boundary.py`` uniform case: a dry sloped channel fed through an
    inflow and drained through a normal-depth outlet, against Manning's normal depth."""
    from .mesh.boundaries import conveyance_split, select_boundary_edges

    geom = channel_geometry(cells, across, length, width, bed=lambda x: 10.0 - slope * x)
    dx = length / cells
    up = select_boundary_edges(geom, [(0.0, 0.0), (0.0, width)], 0.25 * dx)
    down = select_boundary_edges(geom, [(length, 0.0), (length, width)], 0.25 * dx)
    n = np.full(geom.N, manning, np.float32)
    z = np.zeros(geom.N)
    s = _solver(geom, z, z, z, n, open_edges=[up, down])
    q = conveyance_split(discharge, geom.edge_len[up], geom.zb[geom.edge_cellL[up]], n[geom.edge_cellL[up]], slope)
    kinds = np.concatenate([np.full(up.size, OPEN_INFLOW), np.full(down.size, OPEN_NORMAL)]).astype(np.uint32)
    values = np.concatenate([q, np.full(down.size, math.sqrt(slope) / manning)]).astype(np.float32)
    s.set_open_conditions(kinds, values)
    t_end = hours * 3600.0
    t0 = time.perf_counter()
    s.run(t_end=t_end, output_interval_s=t_end / 8.0, dt_max=5.0, dt_init=1e-2, cfl_interval=1, progress=False)
    wall = time.perf_counter() - t0
    h = s.download_h().astype(np.float64)
    x = geom.world_centroid[:, 0]
    middle = (x > 0.4 * length) & (x < 0.6 * length)
    hn = normal_depth(discharge, width, slope, manning)
    went_out = np.array([v[1, 0] for v in s.open_volume_snapshots])
    out = {"case": "uniform", "cells": geom.N, "steps": s.steps_total, "wall_s": wall, "normal_depth_m": hn,
           "depth_error_rel": abs(float(h[middle].mean()) / hn - 1.0),
           "discharge_error_rel": abs((went_out[-1] - went_out[-2]) / (t_end / 8.0) / discharge - 1.0),
           "inflow_error_rel": abs(s.download_open_volumes()[0, 1] / (discharge * t_end) - 1.0)}
    return _gate_result(out, {"depth_error_rel": 0.01, "discharge_error_rel": 1e-3, "inflow_error_rel": 1e-7},
                    strict=("depth_error_rel", "discharge_error_rel", "inflow_error_rel"))


def held_lake(cells: int = 200, length: float = 1000.0, width: float = 40.0, across: int = 2, level: float = 12.0,
              t_end: float = 300.0) -> dict:
    """``inundation/bench/open_boundary.py`` lake case: still water over a bed of two sines
    held by its own level as a stage at both ends."""
    from .mesh.boundaries import select_boundary_edges

    bed = lambda x: 10.0 + np.sin(2.0 * np.pi * x / 200.0) + 0.5 * np.sin(2.0 * np.pi * x / 73.0)  # noqa: E731
    geom = channel_geometry(cells, across, length, width, bed=bed)
    dx = length / cells
    ends = [select_boundary_edges(geom, [(xe, 0.0), (xe, width)], 0.25 * dx) for xe in (0.0, length)]
    zb = geom.zb.astype(np.float64)
    h0 = np.maximum(level - zb, 0.0)
    z = np.zeros(geom.N)
    s = _solver(geom, h0, z, z, np.full(geom.N, 0.03), open_edges=ends)
    ids = np.concatenate(ends)
    s.set_open_conditions(np.full(ids.size, OPEN_STAGE, np.uint32),
                          np.maximum(level - zb[geom.edge_cellL[ids]], 0.0).astype(np.float32))
    t0 = time.perf_counter()
    s.run(t_end=t_end, output_interval_s=t_end, dt_max=5.0, dt_init=1e-2, cfl_interval=1, progress=False)
    wall = time.perf_counter() - t0
    h = s.download_h().astype(np.float64)
    speed = float(np.hypot(s.download_hu(), s.download_hv()).max() / h.min())
    out = {"case": "held_lake", "cells": geom.N, "steps": s.steps_total, "wall_s": wall,
           "level_error_m": float(np.abs(h + zb - level).max()), "speed_max_ms": speed}
    return _gate_result(out, {"level_error_m": 1e-4, "speed_max_ms": 1e-3}, strict=("level_error_m", "speed_max_ms"))


def _workflow(geom: MeshGeometry, ends: list, *, output_interval_s: float, manning: float = 0.03):
    from .workflow import SWEWorkflow, WorkflowConfig

    wf = SWEWorkflow(WorkflowConfig(mesh_source="channel", manning_n=manning, output_interval_s=output_interval_s,
                                    dt_max=5.0, cfl_interval=1, progress=False, track_clamp_mass=True,
                                    open_boundaries=ends), geometry=geom)
    wf.prepare()
    return wf


def _end(name: str, x: float, width: float, dx: float):
    from .workflow import OpenBoundary

    return OpenBoundary(name, [(x, 0.0), (x, width)], 0.25 * dx)


def _balance_rel(result, initial: float = 0.0) -> float:
    last = [v[-1] for v in result.boundary_volumes_m3.values()]
    went_out, went_in = float(sum(v[0] for v in last)), float(sum(v[1] for v in last))
    return abs(initial + went_in - went_out - result.volume_final_m3) / max(initial + went_in, 1e-30)


def backwater(end_depth: float = 0.8, cells: int = 600, length: float = 3000.0, width: float = 40.0,
              discharge: float = 10.0, slope: float = 1e-3, manning: float = 0.03, hours: float = 6.0) -> dict:
    """``inundation/bench/open_boundary.py`` backwater case: an inflow into a sloped channel held at
    its outlet by a stage ``end_depth`` over the bed (0.8 m: an M1 profile, 0.25 m: M2), against the
    gradually varied flow profile: interior columns within 1.5 %, last window's outflow within 1e-3."""
    from .workflow import Inflow, SimulationPhase, Stage

    sloped = lambda x: 10.0 - slope * x  # noqa: E731
    geom = channel_geometry(cells, 2, length, width, bed=sloped)
    dx = length / cells
    wf = _workflow(geom, [_end("up", 0.0, width, dx), _end("down", length, width, dx)],
                   output_interval_s=hours * 3600.0 / 6.0, manning=manning)
    t0 = time.perf_counter()
    r = wf.run([SimulationPhase(hours * 3600.0, [], {"up": Inflow(discharge, slope),
                                                      "down": Stage(float(sloped(length)) + end_depth)})])
    wall = time.perf_counter() - t0
    x, h = column_profile(geom, r.h_final)
    ref = gradually_varied_profile(x, end_depth, length, discharge / width, slope, manning)
    went_out = r.boundary_volumes_m3["down"][:, 0]
    window = hours * 3600.0 / 6.0
    out = {"case": f"backwater_{'m1' if end_depth > normal_depth(discharge, width, slope, manning) else 'm2'}",
           "cells": geom.N, "steps": r.steps_total, "wall_s": wall,
           "profile_error_rel": float((np.abs(h - ref) / ref)[1:-1].max()),
           "discharge_error_rel": abs((went_out[-1] - went_out[-2]) / window / discharge - 1.0),
           "balance_rel": _balance_rel(r)}
    return _gate_result(out, {"profile_error_rel": 0.015, "discharge_error_rel": 1e-3, "balance_rel": 1e-7},
                    strict=("profile_error_rel", "discharge_error_rel", "balance_rel"))


def basins(cells: int = 400, length: float = 4000.0, width: float = 40.0, slope: float = 1e-3,
           phase_s: float = 900.0, discharges: tuple[float, ...] = (5.0, 10.0, 15.0, 20.0, 15.0, 10.0, 5.0, 5.0),
           output_s: float = 60.0) -> dict:
    """``inundation/bench/open_boundary.py`` basins case: one channel run whole, then cut in two and
    run upstream first, its outflow passed into the lower half through ``inflow_phases``: the volume
    passed arrives (1e-6), the lower half's depths match the whole run's (1 %), and so does its
    outflow (2 %); both halves' balances close (1e-7)."""
    from .workflow import Inflow, NormalDepth, SimulationPhase, inflow_phases

    sloped = lambda x: 10.0 - slope * x  # noqa: E731
    cut = 0.5 * length
    dx = length / cells

    def hydrograph(down: str) -> list:
        return [SimulationPhase(phase_s, [], {"up": Inflow(q, slope), down: NormalDepth(slope)}) for q in discharges]

    t0 = time.perf_counter()
    whole_g = channel_geometry(cells, 2, length, width, bed=sloped)
    whole = _workflow(whole_g, [_end("up", 0.0, width, dx), _end("down", length, width, dx)],
                      output_interval_s=output_s).run(hydrograph("down"))
    upper_g = channel_geometry(cells // 2, 2, cut, width, bed=sloped)
    first = _workflow(upper_g, [_end("up", 0.0, width, dx), _end("cut", cut, width, dx)],
                      output_interval_s=output_s).run(hydrograph("cut"))
    lower_g = channel_geometry(cells // 2, 2, cut, width, bed=sloped, x0=cut)
    second = _workflow(lower_g, [_end("from_upper", cut, width, dx), _end("down", length, width, dx)],
                       output_interval_s=output_s).run(
        inflow_phases(first, "cut", "from_upper", slope, {"down": NormalDepth(slope)}))
    wall = time.perf_counter() - t0
    passed = float(first.boundary_volumes_m3["cut"][-1, 0])
    received = float(second.boundary_volumes_m3["from_upper"][-1, 1])
    xl, hl = column_profile(lower_g, second.h_final)
    xw, hw = column_profile(whole_g, whole.h_final)
    shared = hw[np.searchsorted(xw, xl - 1e-6)]
    wet = shared > 0.01
    out_whole = float(whole.boundary_volumes_m3["down"][-1, 0])
    out_lower = float(second.boundary_volumes_m3["down"][-1, 0])
    out = {"case": "basins", "cells": whole_g.N, "steps": whole.steps_total + first.steps_total + second.steps_total,
           "wall_s": wall, "volume_passed_m3": passed, "passed_error_rel": abs(received / passed - 1.0),
           "depth_difference_rel": float((np.abs(hl - shared)[wet] / shared[wet]).max()),
           "outflow_difference_rel": abs(out_lower / out_whole - 1.0),
           "upper_balance_rel": _balance_rel(first), "balance_rel": _balance_rel(second)}
    gates = {"passed_error_rel": 1e-6, "depth_difference_rel": 0.01, "outflow_difference_rel": 0.02,
             "upper_balance_rel": 1e-7, "balance_rel": 1e-7}
    return _gate_result(out, gates, strict=tuple(gates))


def _gate_result(out: dict, gates: dict, strict: tuple[str, ...] = ()) -> dict:
    """``passed`` and the failed gates: a value above its gate fails (at or above for ``strict``)."""
    failed = []
    for key, bound in gates.items():
        v = out[key]
        if not math.isfinite(v) or v > bound or (key in strict and v >= bound and bound > 0.0):
            failed.append(f"{key}={v:.4g} > {bound:g}")
    if "finite" in out and not out["finite"]:
        failed.append("non-finite depth")
    if "min_depth_m" in out and out["min_depth_m"] < 0.0:
        failed.append("negative depth")
    out["gates"] = gates
    out["failed"] = failed
    out["passed"] = not failed
    return out


CASES: dict[str, Callable[[], dict]] = {
    "stoker": lambda: dambreak("stoker"),
    "ritter": lambda: dambreak("ritter"),
    "radial": radial,
    "bowl": bowl,
    "lake": lake,
    "uniform": uniform,
    "held_lake": held_lake,
    "backwater_m1": lambda: backwater(0.8),
    "backwater_m2": lambda: backwater(0.25),
    "basins": basins,
}


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description="physical validation gates of the B200 backend")
    ap.add_argument("cases", nargs="*", metavar="case", help=f"any of {', '.join(CASES)} (default: all)")
    args = ap.parse_args(argv)
    unknown = sorted(set(args.cases) - set(CASES))
    if unknown:
        ap.error(f"unknown cases {unknown}; choose from {list(CASES)}")
    ok = True
    for name in args.cases or list(CASES):
        res = CASES[name]()
        ok &= res["passed"]
        print(json.dumps(res), flush=True)
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
