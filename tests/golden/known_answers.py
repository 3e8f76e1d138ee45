"""Known-answer cases of the reference's own unit tests for this path, restated as data.

Each entry cites the reference test it comes from (paths inside the reference
project).  The CPU oracle, the reference library and the CUDA path are all
checked against these numbers.
"""
import numpy as np

# ------------------------------------------------------------------ COO -> CSR
COO_CASES = [
    {   # test/unit/sparse/sparse_ops_test.cpp:22-46 (insertion-order duplicate sums, 1e16 cancellation)
        "name": "insertion_order_cancellation_f64", "dtype": np.float64, "rows": 4, "cols": 5,
        "r": [2, 0, 2, 1, 2, 0, 2], "c": [4, 3, 1, 2, 1, 3, 1],
        "v": [5.0, 2.0, 1.0e16, 4.0, -1.0e16, -2.0, 1.0],
        "row_offsets": [0, 1, 2, 4, 4], "col_indices": [3, 2, 1, 4], "values": [0.0, 4.0, 1.0, 5.0],
    },
    {   # test/unit/sparse/sparse_ops_test.cpp:320-369 (device variant, float uses 1e8)
        "name": "insertion_order_cancellation_f32", "dtype": np.float32, "rows": 4, "cols": 5,
        "r": [2, 0, 2, 1, 2, 0, 2], "c": [4, 3, 1, 2, 1, 3, 1],
        "v": [5.0, 2.0, 1.0e8, 4.0, -1.0e8, -2.0, 1.0],
        "row_offsets": [0, 1, 2, 4, 4], "col_indices": [3, 2, 1, 4], "values": [0.0, 4.0, 1.0, 5.0],
    },
    {   # test/unit/sparse/sparse_ops_test.cpp:49-71 (float, output reuse)
        "name": "reuse_f32", "dtype": np.float32, "rows": 2, "cols": 2,
        "r": [1, 0, 1], "c": [0, 1, 0], "v": [2.0, 3.0, 4.0],
        "row_offsets": [0, 1, 2], "col_indices": [1, 0], "values": [3.0, 6.0],
    },
    {   # test/unit/sparse/sparse_ops_test.cpp:371-430 (async, non-default stream)
        "name": "async_stream", "dtype": np.float64, "rows": 3, "cols": 3,
        "r": [1, 0, 1, 2, 1], "c": [0, 2, 0, 1, 0], "v": [2.0, 3.0, 4.0, 5.0, -1.0],
        "row_offsets": [0, 1, 2, 3], "col_indices": [2, 0, 1], "values": [3.0, 5.0, 5.0],
    },
    {   # test/unit/sparse/sparse_ops_test.cpp:73-86 (empty matrix 0x5)
        "name": "empty", "dtype": np.float32, "rows": 0, "cols": 5, "r": [], "c": [], "v": [],
        "row_offsets": [0], "col_indices": [], "values": [],
    },
]

# coordinate errors, test/unit/sparse/sparse_ops_test.cpp:87-104
COO_ERRORS = [
    {"rows": 1, "cols": 1, "r": [-1], "c": [0], "v": [1.0], "kind": "out_of_range"},
    {"rows": 1, "cols": 1, "r": [0], "c": [-1], "v": [1.0], "kind": "out_of_range"},
    {"rows": 1, "cols": 1, "r": [1], "c": [0], "v": [1.0], "kind": "out_of_range"},
    {"rows": 1, "cols": 1, "r": [0], "c": [1], "v": [1.0], "kind": "out_of_range"},
]

# ------------------------------------------------------------------ SpMV
SPMV_CASES = [
    {   # test/unit/sparse/sparse_ops_test.cpp:120-150
        "dtype": np.float32, "rows": 3, "cols": 4, "r": [2, 0, 1, 0], "c": [3, 2, 1, 0],
        "v": [5.0, 2.0, -1.0, 3.0], "x": [1.0, 2.0, 3.0, 4.0], "y": [9.0, -2.0, 20.0],
    },
    {   # test/unit/sparse/sparse_ops_test.cpp:153-170 (empty rows)
        "dtype": np.float64, "rows": 3, "cols": 2, "r": [1], "c": [0], "v": [2.0], "x": [3.0, 4.0],
        "y": [0.0, 6.0, 0.0],
    },
]

# dense matrices column-major: "B" and "out" list their columns
SPMM_CASES = [
    {   # test/unit/sparse/sparse_ops_test.cpp:196-233 and :704-735 (GPU)
        "dtype": np.float64, "rows": 3, "cols": 3, "r": [1, 0, 2, 0], "c": [1, 2, 0, 0],
        "v": [4.0, 2.0, -1.0, 3.0], "B": [[1.0, 2.0, 3.0], [10.0, 20.0, 30.0]],
        "out": [[9.0, 8.0, -1.0], [90.0, 80.0, -10.0]],
    },
    {   # test/unit/sparse/sparse_ops_test.cpp:737-760 (GPU, synchronous spmm)
        "dtype": np.float32, "rows": 2, "cols": 2, "r": [0, 1], "c": [0, 1], "v": [2.0, 3.0],
        "B": [[4.0, 5.0], [6.0, 7.0]], "out": [[8.0, 15.0], [12.0, 21.0]],
    },
]

# ------------------------------------------------------------------ iterative solvers
# test/unit/sparse/iterative_solver_test.cpp:103-123: diagonal PCG converges in one iteration
DIAGONAL_PCG = {"r": [0, 1, 2], "c": [0, 1, 2], "v": [2.0, 4.0, 8.0], "rhs": [2.0, 8.0, 24.0],
                "solution": [1.0, 2.0, 3.0], "iterations": 1}

# test/unit/sparse/iterative_solver_test.cpp:78-101, 394-424: caller-supplied 2x2 inverse blocks
COUPLED_BLOCK = {
    "r": [0, 0, 1, 1, 2, 2, 3, 3], "c": [0, 1, 0, 1, 2, 3, 2, 3],
    "v": [4.0, 1.0, 1.0, 3.0, 2.0, 0.5, 0.5, 1.5],
    "inverse": [3.0 / 11.0, -1.0 / 11.0, -1.0 / 11.0, 4.0 / 11.0,
                1.5 / 2.75, -0.5 / 2.75, -0.5 / 2.75, 2.0 / 2.75],
    "expected": [1.0, 2.0, -1.0, 3.0], "block_size": 2, "iterations": 1,
}


def poisson1d(size: int, scale: float = 1.0):
    """test/unit/sparse/iterative_solver_test.cpp:44-69 (COO triplets of the 1-D Poisson matrix)."""
    rows, cols, vals = [], [], []
    for row in range(size):
        if row > 0:
            rows.append(row); cols.append(row - 1); vals.append(-scale)
        rows.append(row); cols.append(row); vals.append(2.0 * scale)
        if row + 1 < size:
            rows.append(row); cols.append(row + 1); vals.append(-scale)
    return rows, cols, vals


# ------------------------------------------------------------------ Huber / LM
HUBER = [  # test/unit/optimization/block_schur_test.cpp:24-33
    {"s": 4.0, "delta": 3.0, "cost": 2.0, "weight": 1.0},
    {"s": 25.0, "delta": 3.0, "cost": 10.5, "weight": 0.6},
]
LM_STEPS = {  # test/unit/optimization/block_schur_test.cpp:550-569
    "options": {"initial": 1e-3, "minimum": 1e-8, "maximum": 1e4, "decrease": 0.25, "increase": 8.0},
    "after_accept": 2.5e-4, "after_reject": 2e-3,
}


# ------------------------------------------------------------------ Schur systems
def synthetic_residuals():
    """makeSyntheticEquations, test/unit/optimization/block_schur_test.cpp:41-75.

    Returns (P, L, bp, bl, residuals) with residuals as
    (primaries, primary_jacobians(flat), eliminated, eliminated_jacobian, residual, weight)."""
    res = []
    for p, l, jp, jl, r in ((0, 0, [1.0, 2.0], 0.5, -1.0), (1, 0, [-0.5, 1.0], 1.5, 0.25),
                            (0, 1, [2.0, -1.0], -0.75, 2.0), (1, 1, [1.25, 0.5], 2.0, -0.5)):
        res.append(([p], jp, l, [jl], [r], 1.0))
    res.append(([0], [0.4, -0.2], -1, None, [0.75], 2.0))   # addPrimaryResidualBlock
    res.append(([], None, 1, [0.8], [-0.3], 1.5))           # addEliminatedResidualBlock
    return 2, 2, 2, 1, res


SYNTHETIC_EXPECTED = [  # block_schur_test.cpp:142-149 and :216-224, damping 0.1
    -0.532196868252671, 0.717080672008074, 0.078633780070238, -0.210823022930113,
    0.017900956933130, 0.253200998620430]


def multi_primary_residuals():
    """expectMultiPrimaryReference, block_schur_test.cpp:77-117 (damping 0.1)."""
    res = [([0, 1], [1.0, 2.0], 0, [3.0], [4.0], 1.0),        # addResidualBlocks
           ([0, 1], [0.5, -1.0], -1, None, [0.2], 1.0)]       # addPrimaryResidualBlocks
    return 2, 1, 1, 1, res


MULTI_PRIMARY_EXPECTED = {"primary": [-1.345185185185185, -0.512592592592593],
                          "eliminated": [-0.493827160493827]}


def coupled_chain_residuals():
    """DenseCpuSolvesParallelSizeCoupledSystemDeterministically, block_schur_test.cpp:275-331:
    24 primary blocks of size 6, identity blocks with residuals 0.01 (1 + block + component),
    and a 1-row residual coupling every block with the next."""
    P, bp = 24, 6
    identity = np.eye(bp).reshape(-1).tolist()
    res = []
    for b in range(P):
        res.append(([b], identity, -1, None, [0.01 * (1 + b + c) for c in range(bp)], 1.0))
    left = [1.0, 0.2, -0.1, 0.3, 0.05, -0.2]
    right = [-0.8, 0.1, 0.25, -0.2, 0.15, 0.3]
    for b in range(P - 1):
        res.append(([b, b + 1], left + right, -1, None, [0.02 * (b + 1)], 1.0))
    return P, 0, bp, 1, res


def aggregation_residuals():
    """AggregatesRepeatedVariablePairsBeforeElimination, block_schur_test.cpp:482-504 (damping 0.5)."""
    return 1, 1, 1, 1, [([0], [1.0, 0.0][:1], 0, [1.0], [1.0], 1.0),
                        ([0], [2.0], 0, [-1.0], [-0.5], 1.0)]


AGGREGATION_EXPECTED = {"primary": [-0.069767441860465], "eliminated": [-0.523255813953488]}

# FloatPointOnlySystemUsesDirectEliminatedSolve, block_schur_test.cpp:531-548
POINT_ONLY = {"P": 0, "L": 1, "bp": 6, "bl": 1, "jacobian": 2.0, "residual": 4.0, "damping": 0.5,
              "eliminated": -4.0 / 3.0}
