"""Learned block-Jacobi correction on the device against the FP64 oracle (features, forward,
loss and gradients with BF16 operands emulated), its preconditioner contract (a zero network is
block Jacobi; a bad network falls back), and what training gains on unseen systems."""
import numpy as np
import pytest
import torch

import oracle as O
from gpu_util import dev, host
from plamatrix_b200 import schur as SC
from plamatrix_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _solved(prob, damping=1e-3, options=None):
    ne = SC.DeviceNormalEquations(prob["P"], prob["L"], prob["bp"], prob["bl"])
    ne.accumulate_observations(dev(prob["obs_primary"]), dev(prob["obs_eliminated"]), dev(prob["jp"]),
                               dev(prob["jl"]), dev(prob["residual"]), prob["huber_delta"])
    ws = SC.SchurComplementSolverWorkspace()
    opts = options or SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10)
    dp, dl, rep = SC.solve_damped_schur_complement(ne, damping, opts, ws)
    return ne, ws, dp, rep


def _blocks(ws):
    """6x6 block-CSR (row pointers, columns, blocks) of the exported reduced system."""
    sysd = ws.export()
    ro, ci, v = host(sysd["row_offsets"]), host(sysd["col_indices"]), host(sysd["values"])
    n = len(ro) - 1
    P = n // 6
    dense = np.zeros((n, n))
    for r in range(n):
        dense[r, ci[ro[r]:ro[r + 1]]] = v[ro[r]:ro[r + 1]]
    bptr, bcol, blocks = [0], [], []
    for p in range(P):
        cols = sorted({c // 6 for r in range(6 * p, 6 * p + 6) for c in ci[ro[r]:ro[r + 1]]})
        for q in cols:
            bcol.append(q)
            blocks.append(dense[6 * p:6 * p + 6, 6 * q:6 * q + 6].reshape(36))
        bptr.append(len(bcol))
    diag = np.stack([dense[6 * p:6 * p + 6, 6 * p:6 * p + 6].reshape(36) for p in range(P)])
    return np.array(bptr), np.array(bcol), np.array(blocks), diag, host(sysd["rhs"])


def _random_params(seed, scale=0.15):
    rng = np.random.default_rng(seed)
    p = (scale * rng.standard_normal(SC.LearnedPreconditioner.param_count())).astype(np.float32)
    return p


def test_features_and_forward_match_oracle():
    _, ws, _, rep = _solved(W.small_bundle(seed=31))
    assert rep["converged"]
    net = SC.LearnedPreconditioner(seed=1)
    params = _random_params(2)
    net.set_params(params)
    got = net.forward(ws)
    bptr, bcol, blocks, _, _ = _blocks(ws)
    ref_f = O.mlp_features(bptr, bcol, blocks)
    assert np.abs(got["features"] - ref_f).max() <= 1e-5 * max(1.0, np.abs(ref_f).max())
    ref = O.mlp_forward(got["features"].astype(np.float64), params.astype(np.float64), bf16=True)
    err = np.abs(got["outputs"] - ref["out"]).max() / np.abs(ref["out"]).max()
    assert err <= 2e-2, err


def test_loss_and_gradients_match_oracle():
    _, ws, dp, rep = _solved(W.small_bundle(seed=33))
    assert rep["converged"]
    bptr, bcol, blocks, diag, rhs = _blocks(ws)
    net = SC.LearnedPreconditioner(seed=3)
    params = _random_params(4, scale=0.1)
    net.set_params(params)
    x = dp.to(torch.float64)
    b = torch.from_numpy(rhs).cuda()
    loss = net.train_step(ws, x, b, learning_rate=0.0)
    got = net.inspect()
    f64 = got["features"].astype(np.float64)
    cache = O.mlp_forward(f64, params.astype(np.float64), bf16=True)
    ref_loss, dout = O.mlp_loss_grad(diag, got["outputs"].astype(np.float64), host(x).reshape(-1, 6),
                                     rhs.reshape(-1, 6))
    assert loss == pytest.approx(ref_loss, rel=1e-6)
    ref_g = O.mlp_backward(f64, params.astype(np.float64), cache, dout, bf16=True)
    g = got["gradients"].astype(np.float64)
    for lo, hi in [(0, 3200), (3200, 3328), (3328, 19712), (19712, 19840), (19840, 22528), (22528, 22549)]:
        err = np.linalg.norm(g[lo:hi] - ref_g[lo:hi]) / max(np.linalg.norm(ref_g[lo:hi]), 1e-30)
        assert err <= 3e-2, (lo, err)


def test_probe_loss_and_gradients_match_oracle():
    """||(I - M S) v||^2 / ||v||^2 along a Rademacher probe v with S v from the device SpMV: loss and
    per-section parameter gradients against the FP64 oracle (BF16 operands emulated)."""
    _, ws, _, rep = _solved(W.small_bundle(seed=41))
    assert rep["converged"]
    bptr, bcol, blocks, diag, _ = _blocks(ws)
    net = SC.LearnedPreconditioner(seed=13)
    params = _random_params(14, scale=0.1)
    net.set_params(params)
    n = diag.shape[0] * 6
    v = torch.from_numpy(np.random.default_rng(15).choice([-1.0, 1.0], n)).cuda()
    sv = ws.spmv(v)
    loss = net.train_probe_step(ws, v, sv, learning_rate=0.0)
    got = net.inspect()
    f64 = got["features"].astype(np.float64)
    cache = O.mlp_forward(f64, params.astype(np.float64), bf16=True)
    ref_loss, dout = O.mlp_probe_loss_grad(diag, got["outputs"].astype(np.float64), host(v).reshape(-1, 6),
                                           host(sv).reshape(-1, 6))
    assert loss == pytest.approx(ref_loss, rel=1e-6)
    ref_g = O.mlp_backward(f64, params.astype(np.float64), cache, dout, bf16=True)
    g = got["gradients"].astype(np.float64)
    for lo, hi in [(0, 3200), (3200, 3328), (3328, 19712), (19712, 19840), (19840, 22528), (22528, 22549)]:
        err = np.linalg.norm(g[lo:hi] - ref_g[lo:hi]) / max(np.linalg.norm(ref_g[lo:hi]), 1e-30)
        assert err <= 3e-2, (lo, err)


def test_gemm_stage_wait_that_runs_out_is_an_error_and_the_network_stays_usable():
    """A stage wait limit of 0 makes the 128-deep hidden-layer GEMM (four K steps) give up at its
    first stage wait: the call fails with the GEMM error, and with the default limit back the
    same forward pass gives the normal outputs."""
    import plamatrix_b200._native as N
    _, ws, _, rep = _solved(W.small_bundle(seed=39))
    assert rep["converged"]
    net = SC.LearnedPreconditioner(seed=9)
    net.set_params(_random_params(10))
    want = net.forward(ws)["outputs"].copy()
    net.set_wait_limit(0)
    with pytest.raises(N.PlamatrixError, match="tensor-core GEMM did not complete"):
        net.forward(ws)
    net.set_wait_limit(1 << 20)
    got = net.forward(ws)["outputs"]
    assert np.array_equal(got, want)
    with pytest.raises(N.InvalidArgument):
        net.set_wait_limit(-1)


@pytest.mark.parametrize("precision", ["native", "mixed"])
def test_network_that_gives_up_inside_a_solve_falls_back_on_the_device(precision):
    """A GEMM stage wait that runs out inside a solve: the device puts plain block Jacobi back
    before the PCG (no host round trip), the report says so, and the solve is block Jacobi's."""
    prob = W.small_bundle(seed=41)
    net = SC.LearnedPreconditioner(seed=9)
    net.set_params(_random_params(10))
    net.set_wait_limit(0)
    try:
        opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10, learned=net,
                                               precision=precision)
        _, _, dp, rep = _solved(prob, options=opts)
    finally:
        net.set_wait_limit(1 << 20)
    _, _, dp_plain, rep_plain = _solved(prob, options=SC.SchurComplementSolverOptions(
        max_iterations=500, relative_tolerance=1e-10, precision=precision))
    assert rep["converged"], rep["message"]
    assert rep["learned_fallback"] and not rep["learned_used"]
    assert rep["iterations"] == rep_plain["iterations"]
    assert torch.allclose(dp, dp_plain, rtol=1e-9, atol=1e-12)


def test_zero_network_matches_block_jacobi():
    prob = W.small_bundle(seed=35)
    _, _, dp_plain, rep_plain = _solved(prob)
    net = SC.LearnedPreconditioner(seed=5)  # output layer starts at zero
    opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10, learned=net)
    _, _, dp, rep = _solved(prob, options=opts)
    assert rep["converged"] and rep["learned_used"] and not rep["learned_fallback"]
    assert rep["iterations"] == rep_plain["iterations"]
    assert torch.allclose(dp, dp_plain, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("precision", ["native", "mixed"])
def test_bad_network_falls_back_to_block_jacobi(precision):
    prob = W.small_bundle(seed=37)
    net = SC.LearnedPreconditioner(seed=7)
    net.set_params(_random_params(8, scale=3.0))
    opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10, learned=net,
                                           stagnation_window=5, precision=precision)
    _, _, dp, rep = _solved(prob, options=opts)
    _, _, dp_plain, _ = _solved(prob)
    assert rep["converged"], rep["message"]
    # either its blocks are rejected when built, or its PCG stagnates: block Jacobi finishes
    assert rep["learned_fallback"]
    assert torch.allclose(dp, dp_plain, rtol=1e-6, atol=1e-9)


def test_training_reduces_loss_and_reports_its_gain():
    """Train on windowed systems of 6 seeds, test on 2 unseen seeds: the training loss falls and
    the solves with the trained network converge; the iteration counts are the reported gain."""
    net = SC.LearnedPreconditioner(seed=11)
    systems = []
    for seed in range(8):
        prob = W.large_bundle(seed=100 + seed, P=200, L=6000)
        _, ws, dp, rep = _solved(prob)
        _, _, _, _, rhs = _blocks(ws) if seed >= 6 else (None, None, None, None, None)
        sysd = ws.export()
        systems.append((prob, ws, dp.to(torch.float64), sysd["rhs"]))
    first = None
    for epoch in range(60):
        losses = [net.train_step(ws, x, b, learning_rate=2e-3) for _, ws, x, b in systems[:6]]
        if first is None:
            first = float(np.mean(losses))
    last = float(np.mean([net.train_step(ws, x, b, learning_rate=0.0) for _, ws, x, b in systems[:6]]))
    assert last < 0.95 * first, (first, last)
    for prob, _, _, _ in systems[6:]:
        _, _, dp_plain, plain = _solved(prob)
        opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10, learned=net)
        _, _, dp, learned = _solved(prob, options=opts)
        assert learned["converged"] and plain["converged"]
        assert torch.allclose(dp, dp_plain, rtol=1e-6, atol=1e-9)
        print("unseen system: block Jacobi", plain["iterations"], "iterations, learned", learned["iterations"],
              "(fallback)" if learned["learned_fallback"] else "")


def test_probe_training_on_the_uneven_family_and_its_measured_gain():
    """Probe-loss training (||(I - M S) v||^2 / ||v||^2, Rademacher v) on 12 systems of the 512-system
    uneven family, evaluated on 4 held-out systems of the family.  Asserted: every solve converges to
    the same steps as block Jacobi, and the held-out iteration count does not grow (mean change
    <= 0.5).  The change itself is what the network gains; measured here and in the benchmark it
    is zero: a block-diagonal correction has no room on these families (the probe loss of block
    Jacobi is ~0.006 and training leaves it there)."""
    sizes = W.uneven_family_sizes(512)
    rows = []
    for i in range(16):
        P, L = sizes[i]
        prob = W.uneven_family_system(i, P, L)
        ne = SC.DeviceNormalEquations(P, L, 6, 3)
        ne.accumulate_observations(prob["obs_primary"], prob["obs_eliminated"], prob["jp"], prob["jl"],
                                   prob["residual"], 1.0)
        ws = SC.SchurComplementSolverWorkspace()
        opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-8)
        dp, _, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
        assert rep["converged"]
        rows.append((ne, ws, P, dp.clone(), rep["iterations"]))
    net = SC.LearnedPreconditioner(seed=17)
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    losses = []
    for epoch in range(10):
        epoch_losses = []
        for ne, ws, P, _, _ in rows[:12]:
            SC.solve_damped_schur_complement(ne, 1e-3, SC.SchurComplementSolverOptions(max_iterations=1,
                                                                                        relative_tolerance=1e-30), ws)
            for _ in range(4):
                v = torch.randint(0, 2, (6 * P,), generator=g, device="cuda").to(torch.float64) * 2.0 - 1.0
                epoch_losses.append(net.train_probe_step(ws, v, ws.spmv(v), learning_rate=1e-3))
        losses.append(float(np.mean(epoch_losses)))
    assert all(np.isfinite(losses)) and losses[-1] <= 1.5 * losses[0], losses
    plain_it, learned_it = [], []
    for ne, ws, P, dp_plain, it_plain in rows[12:]:
        opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-8, learned=net)
        dp, _, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
        assert rep["converged"], rep["message"]
        assert torch.linalg.norm(dp - dp_plain) <= 1e-6 * torch.linalg.norm(dp_plain)
        plain_it.append(it_plain)
        learned_it.append(rep["iterations"])
    gain = float(np.mean(plain_it) - np.mean(learned_it))
    print(f"probe loss per epoch {losses[0]:.5f} -> {losses[-1]:.5f}; held-out iterations block Jacobi "
          f"{plain_it}, learned {learned_it}; mean gain {gain:+.2f} iterations")
    assert gain >= -0.5, (plain_it, learned_it)

