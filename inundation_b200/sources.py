"""Inflow hydrographs: time-varying point sources evaluated on the device.

The reference feeds inflows as per-phase constant rates
(``inundation/workflow.py:258-291``, ``inundation/bench/flood_propagation.py:322-341``);
here a hydrograph's knots go to the device and every step evaluates the
discharge at its own clock, which keeps the rate a differentiable function
of the knots.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from numpy.typing import NDArray

NO_HYDROGRAPH = 0xFFFFFFFF


@dataclass
class Hydrograph:
    """An inflow whose discharge follows knots (t seconds, q m^3/s), shared among cells.

    Cell ``cells[k]`` gains ``share[k] * q(t) / area`` metres of depth per
    second (``share`` defaults to equal parts summing to 1); q is piecewise
    linear between the knots and holds its end values outside them.
    """

    cells: NDArray[np.int64]
    knot_t: NDArray[np.float32]
    knot_q: NDArray[np.float32]
    share: NDArray[np.float32] | None = None

    def shares(self) -> NDArray[np.float32]:
        cells = np.asarray(self.cells).ravel()
        if self.share is None:
            return np.full(cells.size, 1.0 / max(cells.size, 1), np.float32)
        return np.asarray(self.share, np.float32).ravel()

    def validate(self, n_cells: int) -> None:
        t = np.asarray(self.knot_t, np.float32).ravel()
        q = np.asarray(self.knot_q, np.float32).ravel()
        cells = np.asarray(self.cells).ravel()
        if t.size == 0 or t.size != q.size:
            raise ValueError(f"a hydrograph needs matching, non-empty knot arrays (got {t.size} and {q.size})")
        if t.size > 1 and not (np.diff(t) > 0).all():
            raise ValueError("hydrograph knot times must increase strictly")
        if cells.size == 0 or cells.min() < 0 or cells.max() >= n_cells:
            raise ValueError(f"hydrograph cells must be in [0, {n_cells})")
        if np.unique(cells).size != cells.size:
            raise ValueError("a hydrograph lists a cell twice")
        if self.shares().size != cells.size:
            raise ValueError("hydrograph share must have one value per cell")


def triangular_knots(peak: float, t_peak: float, t_end: float) -> tuple[NDArray[np.float32], NDArray[np.float32]]:
    """Knots of a triangle rising from 0 at t=0 to ``peak`` at ``t_peak`` and back to 0 at ``t_end``."""
    return np.array([0.0, t_peak, t_end], np.float32), np.array([0.0, peak, 0.0], np.float32)


__all__ = ["NO_HYDROGRAPH", "Hydrograph", "triangular_knots"]
