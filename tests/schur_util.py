"""Shared helpers of the Schur tests: oracle-built normal equations and canonical comparisons."""
import numpy as np


def canonical(state: dict) -> dict:
    """Cross blocks of every eliminated block sorted by primary index (the device observation
    path stores them in that order; the reference keeps first-appearance order)."""
    offs = state["adjacency_offsets"]
    order = []
    for l in range(len(offs) - 1):
        idx = np.arange(offs[l], offs[l + 1])
        order.append(idx[np.argsort(state["cross_primary"][idx], kind="stable")])
    order = np.concatenate(order) if order else np.zeros(0, np.int64)
    out = dict(state)
    out["cross_primary"] = state["cross_primary"][order]
    out["cross_values"] = state["cross_values"][order]
    return out


def dense_from_csr(ro, ci, v, n):
    A = np.zeros((n, n))
    for r in range(n):
        A[r, ci[ro[r]:ro[r + 1]]] += v[ro[r]:ro[r + 1]]
    return A


def csr_matvec(ro, ci, v, x):
    n = len(ro) - 1
    rows = np.repeat(np.arange(n), np.diff(ro))
    y = np.zeros(n)
    np.add.at(y, rows, v.astype(np.float64) * x[ci])
    return y
