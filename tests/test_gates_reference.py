"""The analytic and reference solutions the validation gates compare with (CPU).

Each is checked against a property that holds exactly: conservation of the
volume the solution holds, the published plateau depth of the Stoker case,
Manning's relation at the normal depth, and the wet-region velocity of
Thacker's solution.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from inundation_b200.gates import normal_depth, radial_reference, ritter, stoker, stoker_middle_depth, thacker, thacker_omega
from inundation_b200.tuning import GRAVITY_G


def test_ritter_keeps_the_volume_of_the_reservoir() -> None:
    x = np.linspace(0.0, 1000.0, 2_000_001)
    h, u = ritter(x, 20.0, h_up=10.0, dam_x=500.0)
    assert np.trapezoid(h, x) == pytest.approx(10.0 * 500.0, rel=1e-6)
    front = 500.0 + 2.0 * math.sqrt(GRAVITY_G * 10.0) * 20.0
    assert h[x > front + 1.0].max() == 0.0 and h[x < 500.0 - math.sqrt(GRAVITY_G * 10.0) * 20.0].min() == 10.0
    assert u.max() == pytest.approx(2.0 * math.sqrt(GRAVITY_G * 10.0), rel=1e-4)


def test_stoker_plateau_and_volume() -> None:
    hm = stoker_middle_depth(10.0, 1.0)
    assert hm == pytest.approx(3.9618, abs=2e-4)
    x = np.linspace(0.0, 1000.0, 2_000_001)
    h, _ = stoker(x, 20.0, h_up=10.0, h_down=1.0, dam_x=500.0)
    assert np.trapezoid(h, x) == pytest.approx(10.0 * 500.0 + 1.0 * 500.0, rel=1e-5)
    assert h.max() == 10.0 and h.min() == 1.0


def test_the_radial_reference_conserves_the_annular_volume() -> None:
    r, h, _ = radial_reference(1.5, h_in=2.5, h_out=0.5, r_dam=2.5, r_max=20.0, cells=2000)
    dr = r[1] - r[0]
    v0 = math.pi * 2.5**2 * 2.5 + math.pi * (20.0**2 - 2.5**2) * 0.5
    assert float((2.0 * math.pi * r * h * dr).sum()) == pytest.approx(v0, rel=1e-9)
    assert h[-1] == pytest.approx(0.5, abs=1e-12)  # the bore has not reached the outer face
    assert 0.5 < h.max() < 2.5


def test_thacker_keeps_its_volume_and_moves_as_one_body() -> None:
    c = np.linspace(-2.0, 2.0, 2001)
    x, y = np.meshgrid(c, c)
    dx = c[1] - c[0]
    vols = []
    period = 2.0 * math.pi / thacker_omega(0.1, 1.0)
    for t in np.linspace(0.0, period, 7):
        h, u, v = thacker(x, y, float(t), centre_depth=0.1, radius=1.0, swing=0.5)
        vols.append(float(h.sum()) * dx * dx)
        wet = h > 0.0
        w = thacker_omega(0.1, 1.0)
        assert np.allclose(u[wet], -0.5 * w * math.sin(w * t)) and np.allclose(v[wet], 0.5 * w * math.cos(w * t))
    assert max(vols) / min(vols) - 1.0 < 1e-3


def test_normal_depth_carries_the_discharge() -> None:
    h = normal_depth(10.0, 40.0, 1e-3, 0.03)
    assert h ** (5.0 / 3.0) * math.sqrt(1e-3) / 0.03 * 40.0 == pytest.approx(10.0, rel=1e-12)


def test_the_backwater_reference_holds_normal_depth() -> None:
    from inundation_b200.gates import gradually_varied_profile

    target = normal_depth(10.0, 40.0, 1e-3, 0.03)
    x = np.linspace(100.0, 2900.0, 8)
    np.testing.assert_allclose(gradually_varied_profile(x, target, 3000.0, 0.25, 1e-3, 0.03), target, rtol=1e-9)


def test_the_backwater_reference_rises_towards_a_high_level() -> None:
    from inundation_b200.gates import gradually_varied_profile

    x = np.linspace(100.0, 2900.0, 8)
    assert (np.diff(gradually_varied_profile(x, 0.8, 3000.0, 0.25, 1e-3, 0.03)) > 0.0).all()
