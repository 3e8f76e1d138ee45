"""Seeded synthetic workloads with the shapes and value distributions of the
LM normal-equation benchmarks (no dataset is involved anywhere).

* ``bundle_problem``   -- two-block LM observations: each eliminated (3-dof) block
  is observed by distinct primary (6-dof) blocks; Jacobian blocks J_p (m x 6) and
  J_l (m x 3) with i.i.d. N(0,1) entries; residuals N(0, 0.5^2) with a fraction of
  N(0, 20^2) outliers; Huber delta 1.  Observations arrive in shuffled order.
  - small  : P=20,   L=2,000,     4 uniform distinct primaries per eliminated block
  - large  : P=4,000, L=2,000,000, 2+Poisson(4) distinct primaries drawn from a
             window of 40 consecutive primaries (indices wrap modulo P) around a
             uniform random centre.
* ``laplacian_coo``    -- 3-D 7-point Laplacian on an n^3 grid plus a diagonal shift,
  delivered as randomly permuted COO with a fraction of entries split in two
  duplicate triplets (split at a U(0,1) fraction).

Every generator is a pure function of its arguments (numpy PCG64 seeded).
"""
from __future__ import annotations

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _distinct_from_window(rng, count: np.ndarray, centre: np.ndarray, window: int, P: int) -> list:
    """For each eliminated block pick `count[l]` distinct primaries in the wrapped window."""
    kmax = int(count.max())
    chunks = []
    step = 1 << 18
    for start in range(0, len(count), step):
        stop = min(start + step, len(count))
        keys = rng.random((stop - start, window), dtype=np.float32)
        picks = np.argsort(keys, axis=1)[:, :kmax].astype(np.int64)
        chunks.append(picks)
    picks = np.concatenate(chunks, axis=0)
    offsets = picks - window // 2
    primaries = (centre[:, None] + offsets) % P
    return primaries  # (L, kmax); only the first count[l] columns are used


def bundle_problem(P: int, L: int, *, per_eliminated: str | int = 4, window: int | None = None,
                   residual_size: int = 2, bp: int = 6, bl: int = 3, outlier_fraction: float = 0.05,
                   huber_delta: float = 1.0, seed: int = 0, dtype=np.float64, shuffle: bool = True) -> dict:
    """Synthetic two-block LM observation problem.

    per_eliminated: an int k (exactly k distinct primaries, uniform over all P, or over
    the window when `window` is set) or "2+poisson4" (k = 2 + Poisson(4), clipped to the
    window / P).
    """
    rng = _rng(seed)
    if isinstance(per_eliminated, str):
        assert per_eliminated == "2+poisson4"
        count = 2 + rng.poisson(4.0, size=L)
    else:
        count = np.full(L, int(per_eliminated), dtype=np.int64)
    limit = min(P, window) if window else P
    count = np.minimum(count, limit).astype(np.int64)
    if window:
        centre = rng.integers(0, P, size=L)
        table = _distinct_from_window(rng, count, centre, window, P)
    else:
        kmax = int(count.max())
        keys = rng.random((L, P), dtype=np.float32) if P <= 4096 else None
        if keys is None:
            raise ValueError("uniform distinct primaries need P <= 4096; use a window")
        table = np.argsort(keys, axis=1)[:, :kmax].astype(np.int64)
    col = np.arange(table.shape[1])[None, :]
    mask = col < count[:, None]
    obs_primary = table[mask]
    obs_eliminated = np.repeat(np.arange(L, dtype=np.int64), count)
    n = len(obs_primary)
    jp = rng.standard_normal((n, residual_size, bp))
    jl = rng.standard_normal((n, residual_size, bl))
    r = rng.standard_normal((n, residual_size)) * 0.5
    outliers = rng.random(n) < outlier_fraction
    r[outliers] = rng.standard_normal((int(outliers.sum()), residual_size)) * 20.0
    if shuffle:
        order = rng.permutation(n)
        obs_primary, obs_eliminated = obs_primary[order], obs_eliminated[order]
        jp, jl, r = jp[order], jl[order], r[order]
    return {
        "P": P, "L": L, "bp": bp, "bl": bl, "m": residual_size, "huber_delta": huber_delta,
        "obs_primary": np.ascontiguousarray(obs_primary), "obs_eliminated": np.ascontiguousarray(obs_eliminated),
        "jp": np.ascontiguousarray(jp.astype(dtype)), "jl": np.ascontiguousarray(jl.astype(dtype)),
        "residual": np.ascontiguousarray(r.astype(dtype)), "seed": seed,
    }


def small_bundle(seed: int = 0, dtype=np.float64, **kw) -> dict:
    """P=20, L=2,000, 4 distinct uniform primaries per eliminated block (8,000 observations)."""
    return bundle_problem(20, 2000, per_eliminated=4, seed=seed, dtype=dtype, **kw)


def large_bundle(seed: int = 0, dtype=np.float64, P: int = 4000, L: int = 2_000_000, **kw) -> dict:
    """P=4,000, L=2,000,000, 2+Poisson(4) distinct primaries from a wrapped window of 40."""
    return bundle_problem(P, L, per_eliminated="2+poisson4", window=40, seed=seed, dtype=dtype, **kw)


def laplacian_coo(n: int = 128, *, shift: float = 1e-2, split_fraction: float = 0.1, seed: int = 0,
                  dtype=np.float64) -> dict:
    """3-D 7-point Laplacian (diag 6 + shift, off-diagonals -1) on an n^3 grid, as permuted COO."""
    rng = _rng(seed)
    N = n ** 3
    idx = np.arange(N, dtype=np.int64)
    i, j, k = idx // (n * n), (idx // n) % n, idx % n
    rows = [idx]
    cols = [idx]
    vals = [np.full(N, 6.0 + shift)]
    for axis, coord, stride in ((0, i, n * n), (1, j, n), (2, k, 1)):
        lo = coord > 0
        rows.append(idx[lo]); cols.append(idx[lo] - stride); vals.append(np.full(int(lo.sum()), -1.0))
        hi = coord < n - 1
        rows.append(idx[hi]); cols.append(idx[hi] + stride); vals.append(np.full(int(hi.sum()), -1.0))
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    nnz = len(v)
    split = rng.random(nnz) < split_fraction
    frac = rng.random(int(split.sum()))
    r2, c2 = r[split], c[split]
    v2 = v[split] * (1.0 - frac)
    v[split] = v[split] * frac
    r = np.concatenate([r, r2])
    c = np.concatenate([c, c2])
    v = np.concatenate([v, v2])
    order = rng.permutation(len(v))
    b = rng.uniform(-1.0, 1.0, size=N)
    return {"rows": N, "cols": N, "nnz": nnz, "row_indices": np.ascontiguousarray(r[order]),
            "col_indices": np.ascontiguousarray(c[order]), "values": np.ascontiguousarray(v[order].astype(dtype)),
            "rhs": b.astype(dtype), "seed": seed, "n": n}


def uneven_batch(count: int = 512, seed: int = 0, dtype=np.float64, p_range=(8, 512), l_range=(500, 50_000),
                 per_eliminated: int = 4) -> list:
    """Independent systems with P ~ U{p_range} and L ~ U{l_range}, 4 observations per eliminated block."""
    rng = _rng(seed)
    out = []
    for s in range(count):
        P = int(rng.integers(p_range[0], p_range[1] + 1))
        L = int(rng.integers(l_range[0], l_range[1] + 1))
        k = min(per_eliminated, P)
        out.append(bundle_problem(P, L, per_eliminated=k, window=min(P, 40), seed=seed * 100003 + s, dtype=dtype))
    return out


def uneven_family_sizes(count: int = 512, seed: int = 12345) -> list:
    """(P, L) of the batched uneven-systems workload: P ~ U{8..512}, L ~ U{500..50,000}."""
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(8, 513)), int(rng.integers(500, 50_001))) for _ in range(count)]


def uneven_family_system(index: int, P: int, L: int, device="cuda") -> dict:
    """System `index` of the batched uneven-systems workload (4 uniform distinct primaries per
    eliminated block, drawn on the device)."""
    return bundle_problem_device(P, L, per_eliminated=4, seed=50_000 + index, device=device)


def bundle_problem_device(P: int, L: int, *, per_eliminated: str | int = 4, window: int | None = None,
                          residual_size: int = 2, outlier_fraction: float = 0.05, huber_delta: float = 1.0,
                          seed: int = 0, device="cuda") -> dict:
    """`bundle_problem` drawn on the device with torch's generator (same distributions and
    structure, different values): for the large learned-preconditioner and batched workloads,
    whose host generation would dominate a benchmark run.  Arrays are device tensors."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    if isinstance(per_eliminated, str):
        assert per_eliminated == "2+poisson4"
        count = 2 + torch.poisson(torch.full((L,), 4.0, device=device), generator=g).to(torch.int64)
    else:
        count = torch.full((L,), int(per_eliminated), dtype=torch.int64, device=device)
    limit = min(P, window) if window else P
    count = count.clamp(max=limit)
    kmax = int(count.max().item()) if L else 0
    width = window if window else P
    cols = []
    step = max(1, (1 << 26) // max(width, 1))
    for start in range(0, L, step):
        stop = min(start + step, L)
        keys = torch.rand((stop - start, width), generator=g, device=device)
        cols.append(keys.argsort(dim=1)[:, :kmax])
    picks = torch.cat(cols, 0) if cols else torch.zeros((0, kmax), dtype=torch.int64, device=device)
    if window:
        centre = torch.randint(0, P, (L,), generator=g, device=device)
        table = (centre[:, None] + picks - window // 2) % P
    else:
        table = picks
    mask = torch.arange(kmax, device=device)[None, :] < count[:, None]
    obs_primary = table[mask]
    obs_eliminated = torch.arange(L, device=device).repeat_interleave(count)
    n = obs_primary.numel()
    jp = torch.randn((n, residual_size, 6), generator=g, device=device, dtype=torch.float64)
    jl = torch.randn((n, residual_size, 3), generator=g, device=device, dtype=torch.float64)
    r = torch.randn((n, residual_size), generator=g, device=device, dtype=torch.float64) * 0.5
    out_mask = torch.rand(n, generator=g, device=device) < outlier_fraction
    r[out_mask] = torch.randn((int(out_mask.sum().item()), residual_size), generator=g, device=device,
                              dtype=torch.float64) * 20.0
    order = torch.randperm(n, generator=g, device=device)
    return {"P": P, "L": L, "bp": 6, "bl": 3, "m": residual_size, "huber_delta": huber_delta,
            "obs_primary": obs_primary[order].contiguous(), "obs_eliminated": obs_eliminated[order].contiguous(),
            "jp": jp[order].contiguous(), "jl": jl[order].contiguous(), "residual": r[order].contiguous(),
            "seed": seed}
