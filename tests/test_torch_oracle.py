"""The float64 torch step (the adjoint's autograd reference) against the pinned float64 step oracle."""

from __future__ import annotations

import numpy as np
import torch

from oracle import fp64_step
from oracle.torch_step import TorchStep, hydrograph_value

from ._valley import DRY_TOL, MANNING, dam, valley_grid


def test_torch_heun_steps_match_the_numpy_oracle() -> None:
    g = valley_grid(nx=48, ny=24)
    h0 = dam(g, 48, 24).astype(np.float64)
    rng = np.random.default_rng(3)
    hu0 = np.where(h0 > 0, rng.normal(0.0, 0.05, g.N), 0.0)
    hv0 = np.where(h0 > 0, rng.normal(0.0, 0.05, g.N), 0.0)
    n = np.full(g.N, MANNING)
    dt = 2.0**-6
    want = fp64_step.State(h0, hu0, hv0)
    model = TorchStep(g, dry_tol=DRY_TOL)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64)  # noqa: E731
    h, hu, hv = t(h0), t(hu0), t(hv0)
    dzL, dzR = model.bed_steps(t(g.zb.astype(np.float64)))
    np.testing.assert_allclose(dzL.numpy(), g.edge_dzL, atol=1e-6)
    for _ in range(6):
        want = fp64_step.heun_step(g, want, n, dt, g=9.81, dry_tol=DRY_TOL)
        h, hu, hv = model.step(h, hu, hv, t(n), dzL, dzR, dt)
    assert np.abs(h.numpy() - want.h).max() < 1e-6
    assert np.abs(hu.numpy() - want.hu).max() < 1e-6
    assert np.abs(hv.numpy() - want.hv).max() < 1e-6


def test_hydrograph_value_is_piecewise_linear_with_flat_ends() -> None:
    kt = torch.tensor([0.0, 10.0, 30.0], dtype=torch.float64)
    kq = torch.tensor([1.0, 5.0, 2.0], dtype=torch.float64)
    assert float(hydrograph_value(kt, kq, -1.0)) == 1.0
    assert float(hydrograph_value(kt, kq, 5.0)) == 3.0
    assert float(hydrograph_value(kt, kq, 20.0)) == 3.5
    assert float(hydrograph_value(kt, kq, 40.0)) == 2.0
