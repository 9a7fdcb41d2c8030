"""The allocation-free volume entry point agrees with the allocating one.

``swe_volume_fp64_noalloc`` is for callers that cannot allocate device memory
while they run (a host held to a fixed device-memory budget, an application
that owns the CUDA allocator, code running where cudaMalloc is not allowed):
it keeps its partial sums in a static device array of the library instead of
a caller buffer. This test calls it through the C ABI twice in a row, on
different data, and checks each result against ``swe_volume_fp64`` on the same
data; then that a mesh beyond the array's 4,194,304-cell limit is refused.
The file name sorts last so a run that stops at the first failure has already
run every other test; it also passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 4_194_304


def _volume_pair(lib, torch, n: int, seed: int) -> tuple[float, float]:
    gen = torch.Generator(device="cuda").manual_seed(seed)
    h = torch.rand(n, device="cuda", generator=gen, dtype=torch.float32) * 3.0
    lo = (torch.rand(n, device="cuda", generator=gen, dtype=torch.float32) - 0.5) * 1e-7
    area = torch.rand(n, device="cuda", generator=gen, dtype=torch.float32) * 100.0 + 1.0
    partials = torch.zeros(int(lib.swe_volume_partials(n)), dtype=torch.float64, device="cuda")
    want = torch.zeros(1, dtype=torch.float64, device="cuda")
    got = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.swe_volume_fp64(h.data_ptr(), lo.data_ptr(), area.data_ptr(), n, partials.data_ptr(), want.data_ptr(), stream) == 0
    assert lib.swe_volume_fp64_noalloc(h.data_ptr(), lo.data_ptr(), area.data_ptr(), n, got.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    host = float(((h.double() + lo.double()) * area.double()).sum().item())
    assert float(want.item()) == pytest.approx(host, rel=1e-12)
    return float(got.item()), float(want.item())


@pytest.mark.parametrize("n", [1, 1000, 1_000_003, LIMIT])
def test_noalloc_volume_matches_the_allocating_entry_point_twice(n: int) -> None:
    import torch

    from inundation_b200 import native

    lib = native.load()
    for seed in (n, n + 17):  # two calls in a row, on different data
        got, want = _volume_pair(lib, torch, n, seed)
        assert got == pytest.approx(want, rel=1e-12, abs=0.0)


def test_noalloc_volume_refuses_more_cells_than_its_scratch_holds() -> None:
    import torch

    from inundation_b200 import native

    lib = native.load()
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = buf.data_ptr()
    assert lib.swe_volume_fp64_noalloc(p, p, p, LIMIT + 1, p, stream) == 3
    assert b"scratch" in lib.swe_status_string(3)
    assert lib.swe_volume_fp64_noalloc(None, None, None, 10, p, stream) == 1
    np.testing.assert_array_equal(buf.cpu().numpy(), np.zeros(4))
