"""FP64 oracle of one Heun shallow-water step (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline arm may import it.
It restates, in float64 NumPy, the reference's CPU step
``tests/unit/_cpu_step.py`` (the reference's own oracle of its GPU kernels):

* ``safe_vel``        -- ``_cpu_step.py:36-41`` (Kurganov-Petrova velocity)
* ``hllc_speeds``     -- ``_cpu_step.py:44-79`` (Roe / Toro dry-bed blend)
* ``hllc``            -- ``_cpu_step.py:82-127`` (HLLC flux in the face frame)
* ``edge_states``     -- ``_cpu_step.py:130-169`` (Audusse reconstruction, walls)
* ``flux_divergence`` -- ``_cpu_step.py:172-199``
* ``cfl_dt``          -- ``_cpu_step.py:202-216``
* ``stage``           -- ``_cpu_step.py:219-248`` (clamp, dry test, film drag, Manning)
* ``heun_step``       -- ``_cpu_step.py:251-267``
* ``run_steps``       -- ``_cpu_step.py:270-285``

Pinned against the reference by ``tests/golden/cpu_step_*.npz`` (outputs of the
reference's ``_cpu_step`` on the same inputs, made by
``tests/golden/make_golden.py``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from numpy.typing import NDArray

FILM_DEPTHS = 4.0
F64 = np.float64


@dataclass(frozen=True)
class State:
    h: NDArray[np.float64]
    hu: NDArray[np.float64]
    hv: NDArray[np.float64]


def safe_vel(h: NDArray[np.float64], hq: NDArray[np.float64], dry_tol: float) -> NDArray[np.float64]:
    film = FILM_DEPTHS * dry_tol
    return np.where(h > dry_tol, 2.0 * h * hq / (h * h + np.maximum(h * h, film * film)), 0.0)


def hllc_speeds(hL, unL, hR, unR, *, g: float, dry_tol: float):
    """Left/right wave-speed bounds: Roe average blended into the dry-bed ``u -+ 2c``."""
    cL = np.sqrt(g * np.maximum(hL, 0.0))
    cR = np.sqrt(g * np.maximum(hR, 0.0))
    sqL = np.sqrt(np.maximum(hL, 0.0))
    sqR = np.sqrt(np.maximum(hR, 0.0))
    den = sqL + sqR
    u_roe = np.where(den > 1e-12, (sqL * unL + sqR * unR) / np.where(den > 1e-12, den, 1.0), 0.0)
    c_roe = np.sqrt(g * 0.5 * (hL + hR))
    sl = np.minimum(unL - cL, u_roe - c_roe)
    sr = np.maximum(unR + cR, u_roe + c_roe)
    wl = np.clip(hL / dry_tol - 1.0, 0.0, 1.0)
    wr = np.clip(hR / dry_tol - 1.0, 0.0, 1.0)
    dry_l = (1.0 - wl) * wr
    dry_r = (1.0 - wr) * wl
    roe = 1.0 - dry_l - dry_r
    return (
        roe * sl + dry_l * (unR - 2.0 * cR) + dry_r * (unL - cL),
        roe * sr + dry_l * (unR + cR) + dry_r * (unL + 2.0 * cL),
    )


def hllc(hL, hqnL, hqtL, hR, hqnR, hqtR, *, g: float, dry_tol: float):
    """(Fh, Fhn, Fht, max |S|) of the HLLC solver in the face frame."""
    unL, utL = safe_vel(hL, hqnL, dry_tol), safe_vel(hL, hqtL, dry_tol)
    unR, utR = safe_vel(hR, hqnR, dry_tol), safe_vel(hR, hqtR, dry_tol)
    SL, SR = hllc_speeds(hL, unL, hR, unR, g=g, dry_tol=dry_tol)
    num = SL * hR * (unR - SR) - SR * hL * (unL - SL)
    den = hR * (unR - SR) - hL * (unL - SL)
    ok = np.abs(den) > 1e-12
    SM = np.where(ok, num / np.where(ok, den, 1.0), 0.0)
    FLh, FLn, FLt = hL * unL, hL * unL * unL + 0.5 * g * hL * hL, hL * unL * utL
    FRh, FRn, FRt = hR * unR, hR * unR * unR + 0.5 * g * hR * hR, hR * unR * utR
    dSL, dSR = SL - SM, SR - SM
    kL = hL * (SL - unL) / np.where(np.abs(dSL) > 1e-14, dSL, 1e-14)
    kR = hR * (SR - unR) / np.where(np.abs(dSR) > 1e-14, dSR, 1e-14)
    starL = (FLh + SL * (kL - hL), FLn + SL * (kL * SM - hL * unL), FLt + SL * (kL * utL - hL * utL))
    starR = (FRh + SR * (kR - hR), FRn + SR * (kR * SM - hR * unR), FRt + SR * (kR * utR - hR * utR))
    out = []
    for fl, fsl, fsr, fr in zip((FLh, FLn, FLt), starL, starR, (FRh, FRn, FRt), strict=True):
        out.append(np.where(SL >= 0, fl, np.where(SM >= 0, fsl, np.where(SR >= 0, fsr, fr))))
    return out[0], out[1], out[2], np.maximum(np.abs(SL), np.abs(SR))


def edge_states(geom, s: State, *, dry_tol: float):
    """Reconstructed face states (hLs, hqnL, hqtL, hRs, hqnR, hqtR, hL, hR, live)."""
    cL, cR = geom.edge_cellL, geom.edge_cellR
    nx, ny = geom.edge_nx.astype(F64), geom.edge_ny.astype(F64)
    wall = cR < 0
    cRi = np.where(wall, cL, cR)
    zb = geom.zb.astype(F64)
    hL, huL, hvL, zL = s.h[cL], s.hu[cL], s.hv[cL], zb[cL]
    hR, huR, hvR, zR = s.h[cRi], s.hu[cRi], s.hv[cRi], zb[cRi]
    qn = huL * nx + hvL * ny
    huR = np.where(wall, huL - 2.0 * qn * nx, huR)
    hvR = np.where(wall, hvL - 2.0 * qn * ny, hvR)
    live = ~((hL < dry_tol) & (hR < dry_tol))
    zf = np.maximum(zL, zR)
    hLs = np.maximum(0.0, hL + zL - zf)
    hRs = np.maximum(0.0, hR + zR - zf)
    uL, vL = safe_vel(hL, huL, dry_tol), safe_vel(hL, hvL, dry_tol)
    uR, vR = safe_vel(hR, huR, dry_tol), safe_vel(hR, hvR, dry_tol)
    huLs, hvLs, huRs, hvRs = hLs * uL, hLs * vL, hRs * uR, hRs * vR
    return (
        hLs,
        huLs * nx + hvLs * ny,
        -huLs * ny + hvLs * nx,
        hRs,
        huRs * nx + hvRs * ny,
        -huRs * ny + hvRs * nx,
        hL,
        hR,
        live,
    )


def flux_divergence(geom, s: State, *, g: float, dry_tol: float):
    """Per-cell sums of outward edge fluxes with the hydrostatic correction."""
    nx, ny = geom.edge_nx.astype(F64), geom.edge_ny.astype(F64)
    length = geom.edge_len.astype(F64)
    hLs, hqnL, hqtL, hRs, hqnR, hqtR, hL, hR, live = edge_states(geom, s, dry_tol=dry_tol)
    Fh, Fhn, Fht, _ = hllc(hLs, hqnL, hqtL, hRs, hqnR, hqtR, g=g, dry_tol=dry_tol)
    Fh = np.where(geom.edge_cellR < 0, 0.0, Fh)
    Fhu = Fhn * nx - Fht * ny
    Fhv = Fhn * ny + Fht * nx
    gL = 0.5 * g * (hL * hL - hLs * hLs)
    gR = 0.5 * g * (hR * hR - hRs * hRs)
    w = live.astype(F64)
    n = geom.N
    dh, dhu, dhv = np.zeros(n), np.zeros(n), np.zeros(n)
    cL, cR = geom.edge_cellL, geom.edge_cellR
    np.add.at(dh, cL, Fh * length * w)
    np.add.at(dhu, cL, (Fhu + gL * nx) * length * w)
    np.add.at(dhv, cL, (Fhv + gL * ny) * length * w)
    inner = cR >= 0
    np.add.at(dh, cR[inner], (-Fh * length * w)[inner])
    np.add.at(dhu, cR[inner], ((-Fhu - gR * nx) * length * w)[inner])
    np.add.at(dhv, cR[inner], ((-Fhv - gR * ny) * length * w)[inner])
    return dh, dhu, dhv


def cfl_dt(geom, s: State, *, g: float, dry_tol: float, cfl: float) -> float:
    """Smallest ``cfl * A / sum(max|S| * len)`` over cells with a live edge."""
    length = geom.edge_len.astype(F64)
    hLs, hqnL, hqtL, hRs, hqnR, hqtR, _, _, live = edge_states(geom, s, dry_tol=dry_tol)
    smax = hllc(hLs, hqnL, hqtL, hRs, hqnR, hqtR, g=g, dry_tol=dry_tol)[3]
    term = smax * length * live.astype(F64)
    lam = np.zeros(geom.N)
    np.add.at(lam, geom.edge_cellL, term)
    inner = geom.edge_cellR >= 0
    np.add.at(lam, geom.edge_cellR[inner], term[inner])
    area = geom.area.astype(F64)
    ok = (lam > 1e-30) & (area > 1e-10)
    if not ok.any():
        return float("inf")
    return float(np.min(cfl * area[ok] / lam[ok]))


def stage(geom, s: State, n: NDArray[np.float64], dt: float, *, g: float, dry_tol: float) -> State:
    """One forward-Euler stage: fluxes, positivity clamp, dry test, film drag, Manning."""
    dh, dhu, dhv = flux_divergence(geom, s, g=g, dry_tol=dry_tol)
    dti = dt / geom.area.astype(F64)
    h = np.maximum(s.h - dti * dh, 0.0)
    hu = s.hu - dti * dhu
    hv = s.hv - dti * dhv
    wet = h >= dry_tol
    hu = np.where(wet, hu, 0.0)
    hv = np.where(wet, hv, 0.0)
    film = FILM_DEPTHS * dry_tol
    hf = np.where(wet & (h < film), h, film)
    rate = (film * film - hf * hf) / (2.0 * hf * hf) * np.sqrt(g / film)
    hu = hu / (1.0 + dt * rate)
    hv = hv / (1.0 + dt * rate)
    hs = np.where(wet, h, 1.0)
    u, v = hu / hs, hv / hs
    sf = g * n * n * np.sqrt(u * u + v * v) / hs ** (4.0 / 3.0)
    den = np.where(wet, 1.0 + dt * sf, 1.0)
    return State(h, hu / den, hv / den)


def heun_step(geom, s: State, n: NDArray[np.float64], dt: float, *, g: float, dry_tol: float) -> State:
    """SSP-RK2 step; a cell that ends dry carries no momentum."""
    s1 = stage(geom, s, n, dt, g=g, dry_tol=dry_tol)
    s2 = stage(geom, s1, n, dt, g=g, dry_tol=dry_tol)
    h = 0.5 * (s.h + s2.h)
    wet = h >= dry_tol
    return State(h, np.where(wet, 0.5 * (s.hu + s2.hu), 0.0), np.where(wet, 0.5 * (s.hv + s2.hv), 0.0))


def run_steps(geom, h, hu, hv, n, dt: float, steps: int, *, g: float, dry_tol: float) -> State:
    s = State(np.asarray(h, F64), np.asarray(hu, F64), np.asarray(hv, F64))
    n64 = np.asarray(n, F64)
    for _ in range(steps):
        s = heun_step(geom, s, n64, dt, g=g, dry_tol=dry_tol)
    return s


@dataclass(frozen=True)
class Region:
    """The cells ``cells`` of a mesh as a mesh of their own, for the step functions above.

    Edges keep their order; an edge with one cell outside the region becomes a
    wall of the inside cell (oriented outward from it). The steps above give
    the same values on a region as on the whole mesh for as long as no water
    reaches a cell with such an edge: every edge across the region's rim is
    then dry on both sides, which the whole-mesh step skips as well.
    """

    N: int
    edge_cellL: NDArray[np.int64]
    edge_cellR: NDArray[np.int64]
    edge_nx: NDArray[np.float32]
    edge_ny: NDArray[np.float32]
    edge_len: NDArray[np.float32]
    zb: NDArray[np.float32]
    area: NDArray[np.float32]
    cells: NDArray[np.int64]  # region cell -> mesh cell
    rim: NDArray[np.int64]  # region cells with an edge to a cell outside


def restrict(geom, cells: NDArray[np.int64]) -> Region:
    cells = np.unique(np.asarray(cells, np.int64))
    inside = np.zeros(geom.N, bool)
    inside[cells] = True
    local = np.full(geom.N, -1, np.int64)
    local[cells] = np.arange(cells.size)
    cL = np.asarray(geom.edge_cellL, np.int64)
    cR = np.asarray(geom.edge_cellR, np.int64)
    in_l = inside[cL]
    in_r = (cR >= 0) & inside[np.where(cR >= 0, cR, 0)]
    keep = in_l | in_r
    flip = keep & ~in_l  # the right cell is the inside one: it becomes the left cell of a wall
    cut = keep & in_l & (cR >= 0) & ~in_r
    new_l = np.where(flip, local[np.where(cR >= 0, cR, 0)], local[cL])[keep]
    new_r = np.where(flip | cut, -1, np.where(cR >= 0, local[np.where(cR >= 0, cR, 0)], -1))[keep]
    sign = np.where(flip, -1.0, 1.0)[keep].astype(np.float32)
    rim = np.unique(np.concatenate([local[cL[cut]], local[cR[flip]]]))
    return Region(
        N=int(cells.size),
        edge_cellL=new_l,
        edge_cellR=new_r,
        edge_nx=np.asarray(geom.edge_nx)[keep] * sign,
        edge_ny=np.asarray(geom.edge_ny)[keep] * sign,
        edge_len=np.asarray(geom.edge_len)[keep],
        zb=np.asarray(geom.zb)[cells],
        area=np.asarray(geom.area)[cells],
        cells=cells,
        rim=rim,
    )
