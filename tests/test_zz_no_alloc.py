"""Allocation-free COO -> CSR (pm_coo_to_csr_static_*).

Some callers cannot allocate device memory while they run: a host application that fixes
the device-memory budget at start-up and owns every allocation afterwards, or a
latency-critical loop in which a cudaMalloc could block or fail part-way.  For them the
library offers a COO -> CSR entry point whose scratch is a fixed device array inside the
library.  These tests call it through the C ABI twice in a row (the second call runs on
the scratch left behind by the first) and require bit-for-bit the same CSR as the regular,
workspace-based entry point.  They pass on their own in a fresh process and after the rest
of the suite.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from plamatrix_b200 import _native as N
from plamatrix_b200 import sparse as S

pytestmark = pytest.mark.gpu

MAX_TRIPLETS = 65536
MAX_ROWS = 65536


def _static_csr(rows, cols, r, c, v):
    count = int(v.numel())
    sfx = "f32" if v.dtype == torch.float32 else "f64"
    capacity = max(count, 1)
    ro = torch.full((rows + 1,), -7, dtype=torch.int64, device="cuda")
    co = torch.full((capacity,), -7, dtype=torch.int64, device="cuda")
    vo = torch.full((capacity,), -7, dtype=v.dtype, device="cuda")
    nnz = C.c_int64(-1)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    N.call(f"pm_coo_to_csr_static_{sfx}", stream, rows, cols, count, C.c_void_p(r.data_ptr()),
           C.c_void_p(c.data_ptr()), C.c_void_p(v.data_ptr()), capacity, C.c_void_p(ro.data_ptr()),
           C.c_void_p(co.data_ptr()), C.c_void_p(vo.data_ptr()), C.byref(nnz))
    k = nnz.value
    return ro.cpu().numpy(), co[:k].cpu().numpy(), vo[:k].cpu().numpy()


def _triplets(seed, rows, cols, count, dtype):
    rng = np.random.default_rng(seed)
    r = rng.integers(0, rows, count)
    c = rng.integers(0, cols, count)
    # a few long rows and many duplicates, with values spanning many magnitudes
    r[: count // 8] = rng.integers(0, 3, count // 8)
    v = rng.standard_normal(count) * 10.0 ** rng.integers(-4, 8, count)
    to = lambda a, t: torch.as_tensor(a, dtype=t).cuda()  # noqa: E731
    return to(r, torch.int64), to(c, torch.int64), to(v, dtype)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_static_scratch_matches_workspace_entry_point_on_consecutive_calls(checkers, dtype):
    """Two calls in a row, the second at the stated maximum: bit for bit the workspace entry
    point's CSR and the oracle's (the reference CPU conversion restated)."""
    cases = [(5000, 700, 40000, 1), (MAX_ROWS, 300, MAX_TRIPLETS, 2)]  # second call: the stated maximum
    for rows, cols, count, seed in cases:
        r, c, v = _triplets(seed, rows, cols, count, dtype)
        got = _static_csr(rows, cols, r, c, v)
        for ref in (S.coo_to_csr(rows, cols, r, c, v).cpu(),
                    checkers.coo_to_csr(rows, cols, r.cpu().numpy(), c.cpu().numpy(), v.cpu().numpy())):
            assert np.array_equal(got[0], ref[0])
            assert np.array_equal(got[1], ref[1])
            assert np.array_equal(got[2].view(np.uint8), np.asarray(ref[2]).view(np.uint8))


def test_static_scratch_rejects_sizes_beyond_its_maximum():
    r, c, v = _triplets(3, 10, 10, MAX_TRIPLETS + 1, torch.float64)
    with pytest.raises(N.InvalidArgument, match="at most 65536 triplets"):
        _static_csr(10, 10, r, c, v)
    r, c, v = _triplets(4, 10, 10, 8, torch.float64)
    with pytest.raises(N.InvalidArgument, match="65536 rows"):
        _static_csr(MAX_ROWS + 1, 10, r, c, v)


def test_static_scratch_reports_coordinate_errors():
    r = torch.tensor([0, 5], dtype=torch.int64, device="cuda")
    c = torch.tensor([0, 0], dtype=torch.int64, device="cuda")
    v = torch.tensor([1.0, 2.0], dtype=torch.float64, device="cuda")
    with pytest.raises(N.OutOfRange, match="source offset 1"):
        _static_csr(2, 2, r, c, v)
    # the scratch is usable again right after an error
    r[1] = 1
    ro, co, vo = _static_csr(2, 2, r, c, v)
    assert ro.tolist() == [0, 1, 2] and co.tolist() == [0, 0] and vo.tolist() == [1.0, 2.0]
