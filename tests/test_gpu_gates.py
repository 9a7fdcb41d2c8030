"""The physical validation gates on the device (``inundation_b200.gates``): each case
of the reference's benchmark harnesses, at its own size, must pass the
reference's thresholds."""

from __future__ import annotations

import pytest

from inundation_b200 import gates

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", sorted(gates.CASES))
def test_gate_passes(case: str) -> None:
    result = gates.CASES[case]()
    assert result["passed"], result
