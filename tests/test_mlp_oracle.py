"""FP64 oracle of the learned block-Jacobi correction, pinned by finite differences: the
analytic gradients of loss(params) (loss -> output -> three layers) against central differences,
the zero network against plain block Jacobi, and the SPD property of the corrected blocks."""
import numpy as np
import pytest

import oracle as O


def _system(P=12, seed=0):
    rng = np.random.default_rng(seed)
    blocks, x, b = [], [], []
    for _ in range(P):
        A = rng.standard_normal((6, 6))
        blocks.append(A @ A.T + 6 * np.eye(6))
    D = np.array(blocks).reshape(P, 36)
    x = rng.standard_normal((P, 6))
    b = np.einsum("pij,pj->pi", np.array(blocks), x) + 0.3 * rng.standard_normal((P, 6))
    feats = rng.standard_normal((P, O.MLP_IN))
    return D, x, b, feats


def _params(seed=1, scale=0.2):
    rng = np.random.default_rng(seed)
    return scale * rng.standard_normal(O.mlp_param_count())


def _loss(params, feats, D, x, b):
    out = O.mlp_forward(feats, params)["out"]
    return O.mlp_loss_grad(D, out, x, b)[0]


def test_param_count():
    assert O.mlp_param_count() == 25 * 128 + 128 + 128 * 128 + 128 + 128 * 21 + 21


def test_zero_network_is_block_jacobi():
    D, x, b, feats = _system()
    minv = O.mlp_preconditioner(D, np.zeros((len(D), O.MLP_OUT)))
    for p in range(len(D)):
        assert np.allclose(minv[p].reshape(6, 6), np.linalg.inv(D[p].reshape(6, 6)), rtol=1e-12, atol=1e-14)


def test_corrected_blocks_stay_spd():
    D, x, b, feats = _system(seed=3)
    out = 3.0 * np.random.default_rng(4).standard_normal((len(D), O.MLP_OUT))
    minv = O.mlp_preconditioner(D, out)
    for p in range(len(D)):
        m = minv[p].reshape(6, 6)
        assert np.allclose(m, m.T, rtol=1e-10, atol=1e-12)
        assert np.linalg.eigvalsh(0.5 * (m + m.T)).min() > 0


def test_output_gradient_matches_finite_differences():
    D, x, b, feats = _system(seed=5)
    out = 0.5 * np.random.default_rng(6).standard_normal((len(D), O.MLP_OUT))
    _, dout = O.mlp_loss_grad(D, out, x, b)
    h = 1e-6
    for p, k in [(0, 0), (1, 4), (3, 20), (7, 11), (11, 2), (5, 14)]:
        e = np.zeros_like(out)
        e[p, k] = h
        fd = (O.mlp_loss_grad(D, out + e, x, b)[0] - O.mlp_loss_grad(D, out - e, x, b)[0]) / (2 * h)
        assert dout[p, k] == pytest.approx(fd, rel=1e-6, abs=1e-10)


def test_probe_loss_gradient_matches_finite_differences_and_numpy():
    """||(I - M S) v||^2 / ||v||^2 with M = blockdiag((L'L'^T)^-1): the loss equals a numpy
    evaluation with explicit inverses, and its output gradient matches central differences."""
    D, x, _, _ = _system(seed=9)
    rng = np.random.default_rng(10)
    v = rng.standard_normal((len(D), 6))
    sv = v @ rng.standard_normal((6, 6)) + 2.0 * v   # any vector field plays u = S v here
    out = 0.4 * rng.standard_normal((len(D), O.MLP_OUT))
    loss, dout = O.mlp_probe_loss_grad(D, out, v, sv)
    minv = O.mlp_preconditioner(D, out).reshape(-1, 6, 6)
    e = v - np.einsum("pij,pj->pi", minv, sv)
    assert loss == pytest.approx((e ** 2).sum() / (v ** 2).sum(), rel=1e-10)
    h = 1e-6
    for p, k in [(0, 0), (2, 5), (4, 20), (8, 9), (11, 1)]:
        d = np.zeros_like(out)
        d[p, k] = h
        fd = (O.mlp_probe_loss_grad(D, out + d, v, sv)[0] - O.mlp_probe_loss_grad(D, out - d, v, sv)[0]) / (2 * h)
        assert dout[p, k] == pytest.approx(fd, rel=1e-6, abs=1e-10)


def test_parameter_gradient_matches_finite_differences():
    D, x, b, feats = _system(seed=7)
    params = _params()
    cache = O.mlp_forward(feats, params)
    _, dout = O.mlp_loss_grad(D, cache["out"], x, b)
    grads = O.mlp_backward(feats, params, cache, dout)
    rng = np.random.default_rng(8)
    n = O.mlp_param_count()
    sections = [(0, 3200), (3200, 3328), (3328, 19712), (19712, 19840), (19840, 22528), (22528, n)]
    h = 1e-6
    for lo, hi in sections:
        for i in rng.integers(lo, hi, size=4):
            e = np.zeros(n)
            e[i] = h
            fd = (_loss(params + e, feats, D, x, b) - _loss(params - e, feats, D, x, b)) / (2 * h)
            assert grads[i] == pytest.approx(fd, rel=1e-5, abs=1e-9), (lo, i)


def test_features_of_a_small_block_matrix():
    rng = np.random.default_rng(9)
    A = rng.standard_normal((6, 6))
    d0 = A @ A.T + 6 * np.eye(6)
    off = rng.standard_normal(36)
    ro = np.array([0, 2, 3])
    col = np.array([0, 1, 1])
    blocks = np.stack([d0.reshape(36), off, (2 * np.eye(6)).reshape(36)])
    f = O.mlp_features(ro, col, blocks)
    s = np.trace(d0) / 6
    a = d0[3, 1] / s
    assert f[0, 3 * 4 // 2 + 1] == pytest.approx(np.sign(a) * np.log1p(abs(a)))
    fro = np.linalg.norm(off) / s
    assert f[0, 21] == pytest.approx(np.log1p(fro)) and f[0, 22] == f[0, 21] and f[0, 23] == f[0, 21]
    assert f[0, 24] == pytest.approx(np.log1p(1) / 4)
    assert f[1, 21:24].tolist() == [0.0, 0.0, 0.0] and f[1, 24] == 0.0
