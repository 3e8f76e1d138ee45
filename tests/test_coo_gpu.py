"""Device COO -> CSR: bit-exact against the oracle (pinned to the reference) and the
known answers of the reference's unit tests; deferred error semantics of cooToCsrAsync."""
import numpy as np
import pytest
import torch

import known_answers as KA
from gpu_util import dev, host, tdtype
from plamatrix_b200 import _native as N
from plamatrix_b200 import sparse as S
from plamatrix_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _gpu_csr(rows, cols, r, c, v, dtype):
    return S.coo_to_csr(rows, cols, dev(np.asarray(r, np.int64)), dev(np.asarray(c, np.int64)),
                        dev(np.asarray(v, dtype)))


def _assert_bitwise(gpu, ref):
    ro, ci, v = gpu.cpu()
    assert np.array_equal(ro, ref[0])
    assert np.array_equal(ci, ref[1])
    assert np.array_equal(v.view(np.uint8), np.asarray(ref[2], v.dtype).view(np.uint8))


@pytest.mark.parametrize("case", KA.COO_CASES, ids=lambda c: c["name"])
def test_known_answers_sync(case):
    out = _gpu_csr(case["rows"], case["cols"], case["r"], case["c"], case["v"], case["dtype"])
    ro, ci, v = out.cpu()
    assert ro.tolist() == case["row_offsets"]
    assert ci.tolist() == case["col_indices"]
    assert v.tolist() == case["values"]


@pytest.mark.parametrize("case", KA.COO_CASES, ids=lambda c: c["name"])
def test_known_answers_async_on_side_stream(case):
    stream = torch.cuda.Stream()
    ws = S.SparseOpsWorkspace()
    dtype = tdtype(case["dtype"])
    r, c = dev(np.asarray(case["r"], np.int64)), dev(np.asarray(case["c"], np.int64))
    v = dev(np.asarray(case["v"], case["dtype"]))
    out = S.CSRMatrix.empty(case["rows"], case["cols"], len(case["values"]), dtype)
    torch.cuda.synchronize()
    for _ in range(2):  # reuse of workspace and output
        S.coo_to_csr_async(case["rows"], case["cols"], r, c, v, out, ws, stream=stream)
        stream.synchronize()
        ws.check_status("cooToCsrAsync")
    ro, ci, vv = out.cpu()
    assert ro.tolist() == case["row_offsets"] and ci.tolist() == case["col_indices"]
    assert vv.tolist() == case["values"]
    # inputs are not modified
    assert host(r).tolist() == case["r"] and host(v).tolist() == list(np.asarray(case["v"], case["dtype"]))
    ws.close()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", ["short", "long", "huge", "dup_heavy", "large", "large_skew"])
def test_random_matches_oracle_bitwise(checkers, dtype, shape):
    """Shapes of every bucketing tier: short rows, shared-memory and merged long rows, heavy
    duplicates, and large inputs (1.2M triplets over 500k rows; 600k triplets with a third of them
    in three rows)."""
    rng = np.random.default_rng(sum(map(ord, shape)))
    if shape == "short":
        rows, cols, n = 5000, 300, 30000
        r = rng.integers(0, rows, n)
    elif shape == "long":          # rows of 17..2048 entries (shared-memory tier)
        rows, cols, n = 64, 5000, 60000
        r = rng.integers(0, rows, n)
    elif shape == "huge":          # rows longer than one 2048-entry chunk (merge tier)
        rows, cols, n = 3, 100000, 50000
        r = rng.choice(rows, n, p=[0.8, 0.15, 0.05])
    elif shape == "dup_heavy":     # many duplicates with cancellation
        rows, cols, n = 200, 4, 40000
        r = rng.integers(0, rows, n)
    elif shape == "large":
        rows, cols, n = 500_000, 3000, 1_200_000
        r = rng.integers(0, rows, n)
    else:                          # a few rows holding a third of the triplets (merge tier)
        rows, cols, n = 300_000, 200_000, 600_000
        r = rng.integers(0, rows, n)
        r[: n // 3] = rng.choice([7, 123_456, 299_999], n // 3)
    c = rng.integers(0, cols, n)
    v = (rng.standard_normal(n) * 10.0 ** rng.integers(-4, 9, n)).astype(dtype)
    ref = checkers.coo_to_csr(rows, cols, r, c, v)
    _assert_bitwise(_gpu_csr(rows, cols, r, c, v, dtype), ref)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_laplacian_with_split_duplicates_matches_oracle(checkers, dtype):
    lap = W.laplacian_coo(48, seed=2, dtype=dtype)
    ref = checkers.coo_to_csr(lap["rows"], lap["cols"], lap["row_indices"], lap["col_indices"], lap["values"])
    out = _gpu_csr(lap["rows"], lap["cols"], lap["row_indices"], lap["col_indices"], lap["values"], dtype)
    _assert_bitwise(out, ref)
    assert out.nnz == lap["nnz"]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_full_size_laplacian_matches_oracle_bitwise(checkers, dtype):
    """The 128^3 7-point Laplacian + 1e-2 shift as permuted COO with 10% of the entries split
    into two duplicates (16,040,764 triplets -> 14,581,760 nonzeros): byte for byte the oracle's
    CSR, whose duplicate sums follow the reference CPU conversion (first value verbatim, the
    rest added in input order), plus the structural properties of the result."""
    lap = W.laplacian_coo(128, seed=0, dtype=dtype)
    ref = checkers.coo_to_csr(lap["rows"], lap["cols"], lap["row_indices"], lap["col_indices"], lap["values"])
    out = _gpu_csr(lap["rows"], lap["cols"], lap["row_indices"], lap["col_indices"], lap["values"], dtype)
    assert out.nnz == lap["nnz"] == 14_581_760
    _assert_bitwise(out, ref)
    ro, ci, v = out.cpu()
    assert ro[0] == 0 and ro[-1] == out.nnz and np.all(np.diff(ro) >= 1)
    row_of = np.repeat(np.arange(lap["rows"]), np.diff(ro))
    key = row_of * lap["cols"] + ci
    assert np.all(np.diff(key) > 0)            # strictly increasing (row, col): sorted and unique
    tol = 1e-12 if dtype == np.float64 else 1e-5
    assert np.allclose(v[ci == row_of], 6.01, rtol=0, atol=tol)
    assert np.allclose(v[ci != row_of], -1.0, rtol=0, atol=tol)


def test_deferred_nnz_and_coordinate_errors():
    """sparse_ops_test.cpp:468-497."""
    ws = S.SparseOpsWorkspace()
    r, c, v = dev(np.array([0, 0])), dev(np.array([1, 1])), dev(np.array([2.0, 3.0]))
    wrong = S.CSRMatrix.empty(2, 2, 2)
    S.coo_to_csr_async(2, 2, r, c, v, wrong, ws)
    torch.cuda.synchronize()
    with pytest.raises(N.PlamatrixError):
        ws.check_status("cooToCsrAsync")
    bad = dev(np.array([0, 2]))
    ok = S.CSRMatrix.empty(2, 2, 1)
    S.coo_to_csr_async(2, 2, bad, c, v, ok, ws)
    torch.cuda.synchronize()
    with pytest.raises(N.OutOfRange) as err:
        ws.check_status("cooToCsrAsync")
    assert "source offset 1" in str(err.value)


def test_status_must_be_checked_and_stream_finished():
    ws = S.SparseOpsWorkspace()
    r, c, v = dev(np.array([0])), dev(np.array([0])), dev(np.array([1.0]))
    out = S.CSRMatrix.empty(1, 1, 1)
    S.coo_to_csr_async(1, 1, r, c, v, out, ws)
    with pytest.raises(N.LogicError):
        S.coo_to_csr_async(1, 1, r, c, v, out, ws)
    torch.cuda.synchronize()
    ws.check_status()
    other = torch.cuda.Stream()
    with pytest.raises(N.LogicError):
        S.coo_to_csr_async(1, 1, r, c, v, out, ws, stream=other)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rejects_non_finite_input_and_sum(dtype):
    """sparse_ops_test.cpp:499-522."""
    r, c = np.zeros(2, np.int64), np.zeros(2, np.int64)
    with pytest.raises(N.InvalidArgument):
        _gpu_csr(1, 1, r, c, np.array([np.inf, 1.0], dtype), dtype)
    big = np.finfo(dtype).max
    with pytest.raises(N.InvalidArgument):
        _gpu_csr(1, 1, r, c, np.array([big, big], dtype), dtype)


def test_empty_input():
    out = _gpu_csr(3, 4, [], [], np.zeros(0), np.float64)
    assert out.nnz == 0 and host(out.row_offsets).tolist() == [0, 0, 0, 0]
    ws = S.SparseOpsWorkspace()
    e = torch.empty(0, dtype=torch.int64, device="cuda")
    with pytest.raises(N.PlamatrixError):
        S.coo_to_csr_async(3, 4, e, e, torch.empty(0, device="cuda", dtype=torch.float64),
                           S.CSRMatrix.empty(3, 4, 1), ws)
