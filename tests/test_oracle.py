"""CPU oracle pinned against the reference: known answers of the reference's unit
tests and bit-for-bit agreement with the reference library built from its sources."""
import numpy as np
import pytest

import known_answers as KA
from plamatrix_b200 import workloads as W

IMPLS = ["orc", "ref"]


def _impls(checkers):
    return [i for i in IMPLS if checkers.available(i)]


@pytest.mark.parametrize("case", KA.COO_CASES, ids=lambda c: c["name"])
def test_coo_known_answers(checkers, case):
    for impl in _impls(checkers):
        ro, ci, v = checkers.coo_to_csr(case["rows"], case["cols"], case["r"], case["c"],
                                        np.array(case["v"], case["dtype"]), impl=impl)
        assert ro.tolist() == case["row_offsets"]
        assert ci.tolist() == case["col_indices"]
        assert v.tolist() == case["values"]


@pytest.mark.parametrize("case", KA.COO_ERRORS)
def test_coo_rejects_coordinates(checkers, case):
    for impl in _impls(checkers):
        with pytest.raises(checkers.CheckerError) as err:
            checkers.coo_to_csr(case["rows"], case["cols"], case["r"], case["c"], np.array(case["v"]), impl=impl)
        assert err.value.kind == case["kind"]


def test_coo_random_matches_reference_bitwise(checkers):
    if not checkers.available("ref"):
        pytest.skip("reference library not built")
    rng = np.random.default_rng(3)
    for dtype in (np.float32, np.float64):
        n = 20000
        r = rng.integers(0, 300, n)
        c = rng.integers(0, 50, n)
        v = rng.standard_normal(n).astype(dtype) * 10.0 ** rng.integers(-3, 8, n)
        a = checkers.coo_to_csr(300, 50, r, c, v.astype(dtype), impl="orc")
        b = checkers.coo_to_csr(300, 50, r, c, v.astype(dtype), impl="ref")
        for x, y in zip(a, b):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8))


def _coo_edge_shapes(dtype):
    rng = np.random.default_rng(7)
    n = 5000
    yield "one_coordinate", 3, 3, np.full(n, 1), np.full(n, 2), \
        (rng.standard_normal(n) * 10.0 ** rng.integers(-4, 9, n)).astype(dtype)
    yield "signed_zeros", 2, 2, np.array([0, 0, 1, 1, 1, 0]), np.array([0, 0, 1, 1, 1, 1]), \
        np.array([0.0, -0.0, -0.0, 0.0, -0.0, -0.0], dtype)
    yield "zero_rows", 0, 5, np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, dtype)
    yield "mostly_empty_rows", 1000, 1000, rng.integers(0, 3, 200), rng.integers(0, 1000, 200), \
        rng.standard_normal(200).astype(dtype)
    yield "wide_rows", 4, 100000, rng.integers(0, 4, 50000), rng.integers(0, 100000, 50000), \
        rng.standard_normal(50000).astype(dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_coo_edge_shapes_match_reference_bitwise(checkers, dtype):
    """One coordinate repeated 5,000 times (the summation order of a long duplicate run), signed
    zeros, zero rows, mostly empty rows and 12,500-entry rows: byte for byte the reference's CSR."""
    if not checkers.available("ref"):
        pytest.skip("reference library not built")
    for name, rows, cols, r, c, v in _coo_edge_shapes(dtype):
        a = checkers.coo_to_csr(rows, cols, r, c, v, impl="orc")
        b = checkers.coo_to_csr(rows, cols, r, c, v, impl="ref")
        assert len(a[0]) == rows + 1, name
        for x, y in zip(a, b):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), name


@pytest.mark.parametrize("case", KA.SPMV_CASES)
def test_spmv_known_answers(checkers, case):
    for impl in _impls(checkers):
        ro, ci, v = checkers.coo_to_csr(case["rows"], case["cols"], case["r"], case["c"],
                                        np.array(case["v"], case["dtype"]), impl=impl)
        y = checkers.csr_spmv(ro, ci, v, np.array(case["x"], case["dtype"]), impl=impl)
        assert y.tolist() == case["y"]


@pytest.mark.parametrize("case", KA.SPMM_CASES)
def test_spmm_known_answers(checkers, case):
    for impl in _impls(checkers):
        ro, ci, v = checkers.coo_to_csr(case["rows"], case["cols"], case["r"], case["c"],
                                        np.array(case["v"], case["dtype"]), impl=impl)
        B = np.array(case["B"], case["dtype"]).T
        out = checkers.csr_spmm(ro, ci, v, case["cols"], B, impl=impl)
        assert out.T.tolist() == case["out"]


def test_spmm_matches_reference_bitwise(checkers):
    if not checkers.available("ref"):
        pytest.skip("reference library not built")
    rng = np.random.default_rng(8)
    for dtype in (np.float32, np.float64):
        r, c = rng.integers(0, 200, 3000), rng.integers(0, 150, 3000)
        ro, ci, v = checkers.coo_to_csr(200, 150, r, c, rng.standard_normal(3000).astype(dtype))
        B = rng.standard_normal((150, 5)).astype(dtype)
        a = checkers.csr_spmm(ro, ci, v, 150, B, impl="orc")
        b = checkers.csr_spmm(ro, ci, v, 150, B, impl="ref")
        assert np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_pcg_diagonal_and_poisson(checkers, dtype):
    tol = 2e-4 if dtype == np.float32 else 1e-10
    for impl in _impls(checkers):
        d = KA.DIAGONAL_PCG
        ro, ci, v = checkers.coo_to_csr(3, 3, d["r"], d["c"], np.array(d["v"], dtype), impl=impl)
        x, rep = checkers.pcg(ro, ci, v, np.array(d["rhs"], dtype), impl=impl)
        assert rep["converged"] and rep["iterations"] == d["iterations"]
        assert np.allclose(x, d["solution"], atol=tol)
        for scale in (1e-3, 1.0, 1e3):
            r, c, vv = KA.poisson1d(8, scale)
            ro, ci, v = checkers.coo_to_csr(8, 8, r, c, np.array(vv, dtype), impl=impl)
            expected = np.arange(1, 9, dtype=dtype)
            rhs = checkers.csr_spmv(ro, ci, v, expected, impl=impl)
            rel = 1e-5 if dtype == np.float32 else 1e-12
            for pre in (False, True):
                x, rep = checkers.pcg(ro, ci, v, rhs, relative_tolerance=rel, preconditioned=pre, impl=impl)
                assert rep["converged"]
                assert np.all(np.abs(x - expected) <= tol * np.arange(1, 9))


def test_pcg_matches_reference_bitwise(checkers):
    if not checkers.available("ref"):
        pytest.skip("reference library not built")
    lap = W.laplacian_coo(12, seed=5)
    for dtype in (np.float32, np.float64):
        ro, ci, v = checkers.coo_to_csr(lap["rows"], lap["cols"], lap["row_indices"], lap["col_indices"],
                                        lap["values"].astype(dtype))
        b = lap["rhs"].astype(dtype)
        for pre in (True, False):   # Jacobi PCG and plain CG
            xa, ra = checkers.pcg(ro, ci, v, b, relative_tolerance=1e-8, preconditioned=pre, impl="orc")
            xb, rb = checkers.pcg(ro, ci, v, b, relative_tolerance=1e-8, preconditioned=pre, impl="ref")
            assert ra == rb and ra["converged"]
            assert np.array_equal(xa, xb)


def test_pcg_error_paths(checkers):
    for impl in _impls(checkers):
        ro, ci, v = checkers.coo_to_csr(2, 2, [0, 1], [1, 0], np.array([1.0, 1.0]), impl=impl)
        with pytest.raises(checkers.CheckerError) as err:
            checkers.pcg(ro, ci, v, np.ones(2), impl=impl)
        assert err.value.kind == "runtime_error"
        ro, ci, v = checkers.coo_to_csr(2, 2, [0, 1], [0, 1], np.array([1.0, 0.0]), impl=impl)
        with pytest.raises(checkers.CheckerError):
            checkers.pcg(ro, ci, v, np.ones(2), impl=impl)
        with pytest.raises(checkers.CheckerError) as err:
            checkers.pcg(ro, ci, v, np.ones(2), max_iterations=-1, impl=impl)
        assert err.value.kind == "invalid_argument"


def test_huber_known_answers(checkers):
    for impl in _impls(checkers):
        for case in KA.HUBER:
            cost, weight = checkers.huber(case["s"], case["delta"], impl=impl)
            assert cost == pytest.approx(case["cost"], rel=1e-15)
            assert weight == pytest.approx(case["weight"], rel=1e-15)
        with pytest.raises(checkers.CheckerError):
            checkers.huber(-1.0, 3.0, impl=impl)
        with pytest.raises(checkers.CheckerError):
            checkers.huber(1.0, -1.0, impl=impl)


def _build(checkers, builder, impl, dtype=np.float64):
    P, L, bp, bl, residuals = builder()
    ne = checkers.NormalEquations(P, L, bp, bl, dtype=dtype, impl=impl)
    for prims, pj, elim, ej, r, w in residuals:
        ne.add_residual(prims, pj, elim, ej, r, w)
    return ne


@pytest.mark.parametrize("backend", ["cpu", "dense_cpu"])
def test_schur_known_answers(checkers, backend):
    for impl in _impls(checkers):
        ne = _build(checkers, KA.synthetic_residuals, impl)
        dp, dl, rep = ne.solve(0.1, backend=backend, max_iterations=50, relative_tolerance=1e-13,
                               absolute_tolerance=1e-14)
        assert rep["converged"], rep["message"]
        assert np.allclose(np.concatenate([dp, dl]), KA.SYNTHETIC_EXPECTED, atol=1e-11, rtol=0)
        ne = _build(checkers, KA.multi_primary_residuals, impl)
        dp, dl, rep = ne.solve(0.1, backend=backend, max_iterations=50, relative_tolerance=1e-13,
                               absolute_tolerance=1e-14)
        assert rep["converged"]
        assert np.allclose(dp, KA.MULTI_PRIMARY_EXPECTED["primary"], atol=1e-11, rtol=0)
        assert np.allclose(dl, KA.MULTI_PRIMARY_EXPECTED["eliminated"], atol=1e-11, rtol=0)
        ne = _build(checkers, KA.aggregation_residuals, impl)
        dp, dl, rep = ne.solve(0.5, backend=backend)
        assert rep["converged"]
        assert np.allclose(dp, KA.AGGREGATION_EXPECTED["primary"], atol=1e-12, rtol=0)
        assert np.allclose(dl, KA.AGGREGATION_EXPECTED["eliminated"], atol=1e-12, rtol=0)


def test_schur_point_only_float(checkers):
    c = KA.POINT_ONLY
    for impl in _impls(checkers):
        ne = checkers.NormalEquations(c["P"], c["L"], c["bp"], c["bl"], dtype=np.float32, impl=impl)
        ne.add_residual([], None, 0, [c["jacobian"]], [c["residual"]], 1.0)
        dp, dl, rep = ne.solve(c["damping"])
        assert rep["converged"] and len(dp) == 0
        assert dl[0] == pytest.approx(c["eliminated"], abs=1e-6)


def test_schur_rejects_invalid_input(checkers):
    for impl in _impls(checkers):
        ne = checkers.NormalEquations(1, 1, 2, 1, impl=impl)
        with pytest.raises(checkers.CheckerError) as err:
            ne.add_residual([1], [1.0, 0.0], 0, [1.0], [0.0])
        assert err.value.kind == "out_of_range"
        with pytest.raises(checkers.CheckerError) as err:
            ne.add_residual([0], [1.0, 0.0], 0, [1.0], [0.0], weight=float("inf"))
        assert err.value.kind == "invalid_argument"


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_small_bundle_matches_reference_bitwise(checkers, dtype):
    """C0-shaped problem: oracle and reference agree bit for bit on the accumulated normal
    equations, the Schur pattern/values/RHS and the PCG solution."""
    if not checkers.available("ref"):
        pytest.skip("reference library not built")
    prob = W.small_bundle(seed=11, dtype=dtype)
    a = checkers.normal_equations_from_observations(prob, dtype=dtype, impl="orc")
    b = checkers.normal_equations_from_observations(prob, dtype=dtype, impl="ref")
    ea, eb = a.export(), b.export()
    for key in ea:
        assert np.array_equal(ea[key], eb[key]), key
    sa = a.schur_system(1e-3, with_preconditioner=False)
    sb = b.schur_system(1e-3)
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)
    ra = a.solve(1e-3, relative_tolerance=1e-10, max_iterations=500)
    rb = b.solve(1e-3, relative_tolerance=1e-10, max_iterations=500)
    assert np.array_equal(ra[0], rb[0]) and np.array_equal(ra[1], rb[1])
    assert ra[2]["iterations"] == rb[2]["iterations"]


BUNDLE_SHAPES = {
    # the large workload's distribution (2 + Poisson(4) distinct primaries from a wrapped window
    # of 40, 5% outliers under the Huber loss) at 1/667 of its size
    "windowed_2_poisson4": dict(P=60, L=3000, per_eliminated="2+poisson4", window=40),
    # block sizes other than 6 x 3 and three rows per residual: the generic paths
    "blocks_4x2_m3": dict(P=30, L=1500, per_eliminated=3, bp=4, bl=2, residual_size=3),
    # most primaries observed by nothing: rows held up by the damping alone
    "unobserved_primaries": dict(P=60, L=12, per_eliminated=1),
}


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", sorted(BUNDLE_SHAPES))
def test_bundle_shapes_match_reference_bitwise(checkers, shape, dtype):
    """Ragged and non-default problems: oracle and reference agree bit for bit on the normal
    equations, the Schur system and the PCG solution with its iteration count."""
    if not checkers.available("ref"):
        pytest.skip("reference library not built")
    kw = dict(BUNDLE_SHAPES[shape])
    prob = W.bundle_problem(kw.pop("P"), kw.pop("L"), seed=5, dtype=dtype, **kw)
    a = checkers.normal_equations_from_observations(prob, dtype=dtype, impl="orc")
    b = checkers.normal_equations_from_observations(prob, dtype=dtype, impl="ref")
    ea, eb = a.export(), b.export()
    for key in ea:
        assert np.array_equal(ea[key], eb[key]), key
    for x, y in zip(a.schur_system(1e-3, with_preconditioner=False), b.schur_system(1e-3)):
        assert np.array_equal(x, y)
    ra = a.solve(1e-3, relative_tolerance=1e-10, max_iterations=500)
    rb = b.solve(1e-3, relative_tolerance=1e-10, max_iterations=500)
    assert ra[2]["converged"] and rb[2]["converged"]
    assert np.array_equal(ra[0], rb[0]) and np.array_equal(ra[1], rb[1])
    assert ra[2]["iterations"] == rb[2]["iterations"]


def test_merge_matches_serial(checkers):
    for impl in _impls(checkers):
        serial = _build(checkers, KA.synthetic_residuals, impl)
        merged = checkers.NormalEquations(2, 2, 2, 1, impl=impl)
        merged.merge_from(_build(checkers, KA.synthetic_residuals, impl))
        a = serial.solve(0.1, backend="dense_cpu", relative_tolerance=1e-13, absolute_tolerance=1e-14)
        b = merged.solve(0.1, backend="dense_cpu", relative_tolerance=1e-13, absolute_tolerance=1e-14)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
