"""Device damped Schur solve against the oracle (pinned to the reference) and the reference's
known answers: normal-equation accumulation, Schur pattern (bit-exact), values, RHS,
block-Jacobi PCG, mixed precision, pattern reuse."""
import numpy as np
import pytest
import torch

import known_answers as KA
from gpu_util import dev, host
from schur_util import canonical, csr_matvec
from plamatrix_b200 import _native as N
from plamatrix_b200 import schur as SC
from plamatrix_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _oracle_ne(checkers, builder, dtype=np.float64):
    P, L, bp, bl, residuals = builder()
    ne = checkers.NormalEquations(P, L, bp, bl, dtype=dtype)
    for prims, pj, elim, ej, r, w in residuals:
        ne.add_residual(prims, pj, elim, ej, r, w)
    return ne


def _device_ne(oracle_ne, dtype=np.float64):
    d = SC.DeviceNormalEquations(oracle_ne.P, oracle_ne.L, oracle_ne.bp, oracle_ne.bl, dtype=dtype)
    d.upload(oracle_ne.export())
    return d


def _opts(**kw):
    base = dict(max_iterations=50, relative_tolerance=1e-13, absolute_tolerance=1e-14)
    base.update(kw)
    return SC.SchurComplementSolverOptions(**base)


@pytest.mark.parametrize("precision", ["native", "mixed"])
def test_known_answers(checkers, precision):
    """block_schur_test.cpp:119-158 (synthetic), :77-117 (multi-primary), :482-504 (aggregation)."""
    ne = _device_ne(_oracle_ne(checkers, KA.synthetic_residuals))
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 0.1, _opts(precision=precision))
    assert rep["converged"], rep["message"]
    assert np.allclose(np.concatenate([host(dp), host(dl)]), KA.SYNTHETIC_EXPECTED, atol=1e-10, rtol=0)
    ne = _device_ne(_oracle_ne(checkers, KA.multi_primary_residuals))
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 0.1, _opts(precision=precision))
    assert rep["converged"]
    assert np.allclose(host(dp), KA.MULTI_PRIMARY_EXPECTED["primary"], atol=1e-10, rtol=0)
    assert np.allclose(host(dl), KA.MULTI_PRIMARY_EXPECTED["eliminated"], atol=1e-10, rtol=0)
    ne = _device_ne(_oracle_ne(checkers, KA.aggregation_residuals))
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 0.5, SC.SchurComplementSolverOptions(precision=precision))
    assert rep["converged"]
    assert np.allclose(host(dp), KA.AGGREGATION_EXPECTED["primary"], atol=1e-12, rtol=0)
    assert np.allclose(host(dl), KA.AGGREGATION_EXPECTED["eliminated"], atol=1e-12, rtol=0)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_dense_backend_known_answers(checkers, dtype):
    """DenseCpuMatchesDenseDampedNormalEquation (block_schur_test.cpp:268-273): the synthetic and
    multi-primary systems through the dense backend; one 'iteration'."""
    tol = 1e-5 if dtype == np.float32 else 1e-10
    opts = _opts(linear_backend="dense")
    ne = _device_ne(_oracle_ne(checkers, KA.synthetic_residuals, dtype), dtype)
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 0.1, opts)
    assert rep["converged"] and rep["iterations"] == 1, rep["message"]
    assert np.allclose(np.concatenate([host(dp), host(dl)]), KA.SYNTHETIC_EXPECTED, atol=tol, rtol=0)
    ne = _device_ne(_oracle_ne(checkers, KA.multi_primary_residuals, dtype), dtype)
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 0.1, opts)
    assert rep["converged"]
    assert np.allclose(host(dp), KA.MULTI_PRIMARY_EXPECTED["primary"], atol=tol, rtol=0)
    assert np.allclose(host(dl), KA.MULTI_PRIMARY_EXPECTED["eliminated"], atol=tol, rtol=0)


def test_dense_backend_coupled_chain_is_deterministic(checkers):
    """block_schur_test.cpp:275-331: 24 coupled 6x6 primary blocks, no eliminated blocks; two
    dense solves agree bit for bit and with the oracle's reduced PCG."""
    orc = _oracle_ne(checkers, KA.coupled_chain_residuals)
    ne = _device_ne(orc)
    opts = SC.SchurComplementSolverOptions(relative_tolerance=1e-12, absolute_tolerance=1e-14,
                                           linear_backend="dense")
    a, _, rep1 = SC.solve_damped_schur_complement(ne, 0.01, opts)
    b, _, rep2 = SC.solve_damped_schur_complement(ne, 0.01, opts)
    assert rep1["converged"] and rep2["converged"], rep1["message"]
    assert torch.equal(a, b) and np.all(np.isfinite(host(a)))
    ref, _, rep_ref = orc.solve(0.01, relative_tolerance=1e-13, max_iterations=500)
    assert rep_ref["converged"]
    assert np.linalg.norm(host(a) - ref) <= 1e-9 * np.linalg.norm(ref)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("size", ["small", "windowed"])
def test_dense_backend_matches_direct_solve(checkers, dtype, size):
    """Device Cholesky over many panels and tiles (n = 120 and 2,400 primary unknowns) against a
    direct solve of the reference's reduced system and the oracle's PCG solution."""
    prob = (W.small_bundle(seed=11, dtype=dtype) if size == "small"
            else W.large_bundle(seed=7, P=400, L=20000, dtype=dtype))
    orc = checkers.normal_equations_from_observations(prob, dtype=dtype)
    ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
    n = len(ro) - 1
    dense = np.zeros((n, n))
    dense[np.repeat(np.arange(n), np.diff(ro)), ci] = vals
    direct = np.linalg.solve(dense, rhs.astype(np.float64))
    ne = _device_from_observations(prob, dtype)
    dp, dl, rep = SC.solve_damped_schur_complement(
        ne, 1e-3, SC.SchurComplementSolverOptions(relative_tolerance=1e-10, linear_backend="dense"))
    assert rep["converged"] and rep["iterations"] == 1, rep["message"]
    tol = 1e-4 if dtype == np.float32 else 1e-9
    assert np.linalg.norm(host(dp).astype(np.float64) - direct) <= tol * np.linalg.norm(direct)
    assert rep["true_relative_residual"] <= (1e-5 if dtype == np.float32 else 1e-12)
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=1e-10, max_iterations=1000)
    stol = 1e-4 if dtype == np.float32 else 1e-6
    assert np.linalg.norm(host(dl).astype(np.float64) - dl_ref) <= stol * np.linalg.norm(dl_ref)


def test_dense_backend_rejections(checkers):
    # a primary block without observations and no damping: a zero pivot
    o = checkers.NormalEquations(2, 1, 1, 1)
    o.add_residual([0], [1.0], 0, [2.0], [1.0])
    dp, dl, rep = SC.solve_damped_schur_complement(_device_ne(o), 0.0, _opts(linear_backend="dense"))
    assert not rep["converged"] and rep["message"] == "reduced Schur complement is not positive definite"
    # a zero pivot in a later panel (column 69 of 70): found when that panel's diagonal block is
    # factored after the trailing update that finishes it
    o = checkers.NormalEquations(70, 1, 1, 1)
    for p in range(69):
        o.add_residual([p], [1.0], -1, None, [1.0])
    o.add_residual([], None, 0, [1.0], [1.0])
    dp, dl, rep = SC.solve_damped_schur_complement(_device_ne(o), 0.0, _opts(linear_backend="dense"))
    assert not rep["converged"] and rep["message"] == "reduced Schur complement is not positive definite"
    big =SC.DeviceNormalEquations(SC.DENSE_MAX_UNKNOWNS // 6 + 1, 1, 6, 3)
    with pytest.raises(N.InvalidArgument, match="16,384"):
        SC.solve_damped_schur_complement(big, 1e-3, _opts(linear_backend="dense"))


def test_mixed_precision_falls_back_to_fp64_when_fp32_fails():
    """The guarded FP32 pass (block_schur_accelerated.cpp:160-195): a system whose reduced values
    overflow FP32 (Jacobians scaled by 1e20) breaks the FP32 inner solve, and the solve finishes
    in FP64 PCG without reporting mixed precision as used; a well-scaled system keeps it."""
    prob = W.small_bundle(seed=13)
    big = dict(prob)
    for key in ("jp", "jl"):
        big[key] = prob[key] * 1e20
    opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10, precision="mixed")
    dp, dl, rep = SC.solve_damped_schur_complement(_device_from_observations(big), 1e-3, opts)
    assert rep["converged"], rep["message"]
    assert not rep["mixed_precision_used"]
    ref, _, rep_ref = SC.solve_damped_schur_complement(
        _device_from_observations(big), 1e-3, SC.SchurComplementSolverOptions(max_iterations=500,
                                                                              relative_tolerance=1e-10))
    assert rep_ref["converged"]
    assert np.linalg.norm(host(dp) - host(ref)) <= 1e-6 * np.linalg.norm(host(ref))
    dp, dl, rep = SC.solve_damped_schur_complement(_device_from_observations(prob), 1e-3, opts)
    assert rep["converged"] and rep["mixed_precision_used"]


def test_primary_coupling_blocks_in_the_pair_assembly(checkers):
    """6x3 systems with primary-primary residual blocks: one coupling adds to blocks the crosses
    also fill, two create blocks that no eliminated block touches (their only terms); the reduced
    system (both triangles) and the step match the reference."""
    prob = W.large_bundle(seed=3, P=400, L=2000)
    orc = checkers.normal_equations_from_observations(prob)
    rng = np.random.default_rng(0)
    for a, b in ((0, 200), (5, 6), (100, 399)):
        orc.add_residual([a, b], rng.standard_normal(24), -1, None, rng.standard_normal(2))
    ne = _device_ne(orc)
    ws = SC.SchurComplementSolverWorkspace()
    dp, dl, rep = SC.solve_damped_schur_complement(
        ne, 1e-3, SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10), ws)
    assert rep["converged"], rep["message"]
    ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
    sysd = ws.export()
    assert np.array_equal(host(sysd["row_offsets"]), ro) and np.array_equal(host(sysd["col_indices"]), ci)
    assert np.abs(host(sysd["values"]) - vals).max() <= 1e-12 * np.abs(vals).max()
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=1e-10, max_iterations=500)
    assert np.linalg.norm(host(dp) - dp_ref) <= 1e-6 * np.linalg.norm(dp_ref)


def test_point_only_float(checkers):
    """block_schur_test.cpp:531-548."""
    c = KA.POINT_ONLY
    o = checkers.NormalEquations(c["P"], c["L"], c["bp"], c["bl"], dtype=np.float32)
    o.add_residual([], None, 0, [c["jacobian"]], [c["residual"]], 1.0)
    ne = _device_ne(o, np.float32)
    dp, dl, rep = SC.solve_damped_schur_complement(ne, c["damping"])
    assert rep["converged"] and dp.numel() == 0
    assert host(dl)[0] == pytest.approx(c["eliminated"], abs=1e-6)


def test_pattern_reuse_counts(checkers):
    """block_schur_test.cpp:160-196."""
    ne = _device_ne(_oracle_ne(checkers, KA.synthetic_residuals))
    ws = SC.SchurComplementSolverWorkspace()
    _, _, first = SC.solve_damped_schur_complement(ne, 0.1, _opts(), ws)
    assert first["converged"] and not first["pattern_reused"] and ws.pattern_build_count() == 1
    _, _, second = SC.solve_damped_schur_complement(ne, 0.2, _opts(), ws)
    assert second["converged"] and second["pattern_reused"] and ws.pattern_build_count() == 1
    # same topology in a different object is still a reuse (signature comparison)
    ne2 = _device_ne(_oracle_ne(checkers, KA.synthetic_residuals))
    _, _, third = SC.solve_damped_schur_complement(ne2, 0.2, _opts(), ws)
    assert third["pattern_reused"] and ws.pattern_build_count() == 1
    o = checkers.NormalEquations(1, 1, 1, 1)
    o.add_residual([0], [1.0], 0, [1.0], [-0.5])
    o.add_residual([0], [1.0], -1, None, [-0.5])
    changed = _device_ne(o)
    _, _, fourth = SC.solve_damped_schur_complement(changed, 0.2, _opts(), ws)
    assert fourth["converged"] and not fourth["pattern_reused"] and ws.pattern_build_count() == 2


def test_invalid_options_and_aliasing(checkers):
    ne = _device_ne(_oracle_ne(checkers, KA.synthetic_residuals))
    with pytest.raises(N.InvalidArgument):
        SC.solve_damped_schur_complement(ne, -1.0)
    with pytest.raises(N.InvalidArgument):
        SC.solve_damped_schur_complement(ne, 0.1, SC.SchurComplementSolverOptions(minimum_diagonal=0.0))
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(N.InvalidArgument):
        SC.solve_damped_schur_complement(ne, 0.1, primary_step=buf, eliminated_step=buf)


def test_accumulation_rejects_bad_indices_sizes_and_delta():
    """RejectsDimensionMismatchAndNonFiniteInput (block_schur_test.cpp:506-529) on the
    observation path: a primary index past the last block, a zero residual size and a
    non-finite Huber delta."""
    prob = W.small_bundle(seed=2)
    ne = SC.DeviceNormalEquations(prob["P"], prob["L"], 6, 3)
    args = [dev(prob[k]) for k in ("obs_primary", "obs_eliminated", "jp", "jl", "residual")]
    bad_p = args[0].clone()
    bad_p[5] = prob["P"]
    with pytest.raises(N.OutOfRange):
        ne.accumulate_observations(bad_p, *args[1:], 1.0)
    with pytest.raises(N.InvalidArgument):
        ne.accumulate_observations(*args, float("inf"))
    n = len(prob["obs_primary"])
    with pytest.raises(N.InvalidArgument):
        N.call("pm_ne_accumulate_observations_f64", ne._h, None, n, 0, *[a.data_ptr() for a in args], 1.0)


def test_dense_backend_generic_blocks_are_repeatable(checkers):
    """DenseCpuEliminatedAssemblyIsBitwiseStableAcrossThreadCounts (block_schur_test.cpp:334-405):
    36 primaries of size 9, 240 eliminated blocks of size 3; repeated dense solves agree bit for
    bit and with the oracle's reduced PCG."""
    P, L, bp, bl = 36, 240, 9, 3
    o = checkers.NormalEquations(P, L, bp, bl)
    identity = np.eye(bp).reshape(-1)
    for p in range(P):
        o.add_residual([p], identity, -1, None, np.zeros(bp), 0.25)
    for l in range(L):
        for obs in range(4):
            p = (l * 7 + obs * 5) % P
            jp = [0.01 * (1 + (i + l + obs) % 13) for i in range(2 * bp)]
            jl = [0.02 * (1 + (i + l + 2 * obs) % 7) for i in range(2 * bl)]
            o.add_residual([p], jp, l, jl, [0.001 * (l + 1), -0.002 * (obs + 1)])
    ne = _device_ne(o)
    opts = SC.SchurComplementSolverOptions(relative_tolerance=1e-11, absolute_tolerance=1e-13,
                                           linear_backend="dense")
    a1, b1, r1 = SC.solve_damped_schur_complement(ne, 0.1, opts)
    a2, b2, r2 = SC.solve_damped_schur_complement(ne, 0.1, opts)
    assert r1["converged"] and r2["converged"], r1["message"]
    assert torch.equal(a1, a2) and torch.equal(b1, b2)
    ref_p, ref_l, rep = o.solve(0.1, relative_tolerance=1e-13, max_iterations=1000)
    assert rep["converged"]
    assert np.linalg.norm(host(a1) - ref_p) <= 1e-8 * np.linalg.norm(ref_p)
    assert np.linalg.norm(host(b1) - ref_l) <= 1e-8 * np.linalg.norm(ref_l)


def test_non_spd_eliminated_block_reports_message(checkers):
    o = checkers.NormalEquations(1, 1, 1, 1)
    o.add_residual([0], [1.0], -1, None, [1.0])
    ne = _device_ne(o)  # eliminated block stays zero: damping of zero is zero -> not SPD
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 0.0)
    assert not rep["converged"] and rep["message"] == "eliminated block is not positive definite"


def _device_from_observations(prob, dtype=np.float64):
    ne = SC.DeviceNormalEquations(prob["P"], prob["L"], prob["bp"], prob["bl"], dtype=dtype)
    ne.accumulate_observations(dev(prob["obs_primary"]), dev(prob["obs_eliminated"]), dev(prob["jp"]),
                               dev(prob["jl"]), dev(prob["residual"]), prob["huber_delta"])
    return ne


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_observation_accumulation_matches_reference(checkers, dtype):
    """Huber weights + addResidualBlock on the device: eliminated blocks, gradients and cross
    blocks bit-exact with the reference's accumulation; primary blocks within rounding."""
    prob = W.small_bundle(seed=21, dtype=dtype)
    ref = canonical(checkers.normal_equations_from_observations(prob, dtype=dtype).export())
    got = _device_from_observations(prob, dtype).download()
    for key in ("eliminated_diagonal", "eliminated_gradient", "adjacency_offsets", "cross_primary", "cross_values"):
        assert np.array_equal(got[key], ref[key]), key
    tol = 1e-5 if dtype == np.float32 else 1e-12
    for key in ("primary_diagonal", "primary_gradient"):
        scale = np.abs(ref[key]).max()
        assert np.abs(got[key] - ref[key]).max() <= tol * scale, key


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_repeated_pairs_and_unaligned_rows_match_reference(checkers, dtype):
    """Crosses with several observations (the first 600 observations repeated with new values
    and interleaved) and Jacobian / residual rows that do not start on a 16-byte boundary (the
    generic path): eliminated, gradient and cross blocks bit-exact."""
    base = W.small_bundle(seed=23, dtype=dtype)
    rng = np.random.default_rng(5)
    k = 600
    prob = dict(base)
    prob["obs_primary"] = np.concatenate([base["obs_primary"], base["obs_primary"][:k]])
    prob["obs_eliminated"] = np.concatenate([base["obs_eliminated"], base["obs_eliminated"][:k]])
    for key in ("jp", "jl", "residual"):
        extra = rng.standard_normal(base[key][:k].shape).astype(dtype)
        prob[key] = np.concatenate([base[key], extra])
    order = rng.permutation(len(prob["obs_primary"]))
    for key in ("obs_primary", "obs_eliminated", "jp", "jl", "residual"):
        prob[key] = np.ascontiguousarray(prob[key][order])
    ref = canonical(checkers.normal_equations_from_observations(prob, dtype=dtype).export())
    dne = _device_from_observations(prob, dtype)
    assert dne.counts()[0] < len(prob["obs_primary"])  # some crosses have several observations
    got = dne.download()
    for key in ("eliminated_diagonal", "eliminated_gradient", "adjacency_offsets", "cross_primary", "cross_values"):
        assert np.array_equal(got[key], ref[key]), key

    def shifted(a):  # same values, device row pointer one scalar past an aligned allocation
        t = torch.zeros(a.size + 1, dtype=torch.float32 if dtype == np.float32 else torch.float64, device="cuda")
        t[1:] = torch.as_tensor(a.reshape(-1)).cuda()
        return t[1:].view(a.shape)

    ne = SC.DeviceNormalEquations(prob["P"], prob["L"], prob["bp"], prob["bl"], dtype=dtype)
    ne.accumulate_observations(dev(prob["obs_primary"]), dev(prob["obs_eliminated"]), shifted(prob["jp"]),
                               shifted(prob["jl"]), shifted(prob["residual"]), prob["huber_delta"])
    got2 = ne.download()
    for key in ("eliminated_diagonal", "eliminated_gradient", "cross_values"):
        assert np.array_equal(got2[key], ref[key]), key
    tol = 1e-5 if dtype == np.float32 else 1e-12
    for key in ("primary_diagonal", "primary_gradient"):
        assert np.abs(got2[key] - got[key]).max() <= tol * np.abs(ref[key]).max(), key


@pytest.mark.parametrize("residual_size", [2, 3])
def test_nonfinite_residual_is_rejected(residual_size):
    """A residual whose squared norm is NaN or overflows is rejected as evaluateHuberLoss
    rejects it: by the explicit check and by the next solve, naming the first such observation;
    a clean accumulation clears the report."""
    prob = W.bundle_problem(30, 400, per_eliminated=4, residual_size=residual_size, seed=4)
    bad = dict(prob)
    bad["residual"] = prob["residual"].copy()
    bad["residual"][7, 0] = np.nan
    bad["residual"][19, -1] = 1e200
    ne = _device_from_observations(bad)
    with pytest.raises(N.InvalidArgument, match="observation 7"):
        ne.check_observations()
    with pytest.raises(N.InvalidArgument, match="observation 7"):
        SC.solve_damped_schur_complement(ne, 1e-3)
    bad["residual"][7, 0] = 0.5
    ne.accumulate_observations(dev(bad["obs_primary"]), dev(bad["obs_eliminated"]), dev(bad["jp"]), dev(bad["jl"]),
                               dev(bad["residual"]), bad["huber_delta"])
    with pytest.raises(N.InvalidArgument, match="observation 19"):
        ne.check_observations()
    ne.accumulate_observations(dev(prob["obs_primary"]), dev(prob["obs_eliminated"]), dev(prob["jp"]),
                               dev(prob["jl"]), dev(prob["residual"]), prob["huber_delta"])
    ne.check_observations()
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 1e-3, SC.SchurComplementSolverOptions(max_iterations=500))
    assert rep["converged"]


def _join(a, b):
    """Observations of b appended to those of a, b's eliminated blocks numbered after a's."""
    out = dict(a)
    out["L"] = a["L"] + b["L"]
    out["obs_primary"] = np.concatenate([a["obs_primary"], b["obs_primary"]])
    out["obs_eliminated"] = np.concatenate([a["obs_eliminated"], b["obs_eliminated"] + a["L"]])
    for k in ("jp", "jl", "residual"):
        out[k] = np.ascontiguousarray(np.concatenate([a[k], b[k]]))
    return out


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_generic_block_sizes_match_reference(checkers, dtype):
    """Block sizes 4 / 2 with 3-row residuals: the generic accumulation and assembly kernels."""
    prob = W.bundle_problem(24, 1500, per_eliminated=4, residual_size=3, bp=4, bl=2, seed=41, dtype=dtype)
    orc = checkers.normal_equations_from_observations(prob, dtype=dtype)
    ref = canonical(orc.export())
    ne = _device_from_observations(prob, dtype)
    got = ne.download()
    for key in ("eliminated_diagonal", "eliminated_gradient", "adjacency_offsets", "cross_primary", "cross_values"):
        assert np.array_equal(got[key], ref[key]), key
    tol = 1e-5 if dtype == np.float32 else 1e-12
    for key in ("primary_diagonal", "primary_gradient"):
        assert np.abs(got[key] - ref[key]).max() <= tol * np.abs(ref[key]).max(), key
    rtol = 1e-5 if dtype == np.float32 else 1e-10
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=rtol, max_iterations=500)
    ws = SC.SchurComplementSolverWorkspace()
    dp, dl, rep = SC.solve_damped_schur_complement(
        ne, 1e-3, SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=rtol), ws)
    assert rep["converged"] and rep_ref["converged"], rep["message"]
    stol = 1e-4 if dtype == np.float32 else 1e-6
    assert np.linalg.norm(host(dp) - dp_ref) <= stol * np.linalg.norm(dp_ref)
    assert np.linalg.norm(host(dl) - dl_ref) <= stol * np.linalg.norm(dl_ref)
    if dtype == np.float64:
        ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
        sysd = ws.export()
        assert np.array_equal(host(sysd["row_offsets"]), ro) and np.array_equal(host(sysd["col_indices"]), ci)
        assert np.abs(host(sysd["values"]) - vals).max() <= 1e-12 * np.abs(vals).max()
        assert np.abs(host(sysd["rhs"]) - rhs).max() <= 1e-12 * np.abs(rhs).max()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_hub_point_and_wide_rows_match_reference(checkers, dtype):
    """Two points seen by all 320 primaries: cross lists longer than the assembly's shared-memory
    staging area, block rows with 319 upper neighbours (several owner groups per row), and
    eliminated buckets longer than the input-order selection window."""
    base = W.bundle_problem(320, 3000, per_eliminated=3, seed=31, dtype=dtype)
    hub = W.bundle_problem(320, 2, per_eliminated=320, seed=32, dtype=dtype)
    prob = _join(base, hub)
    orc = checkers.normal_equations_from_observations(prob, dtype=dtype)
    ref = canonical(orc.export())
    ne = _device_from_observations(prob, dtype)
    got = ne.download()
    for key in ("adjacency_offsets", "cross_primary", "cross_values"):
        assert np.array_equal(got[key], ref[key]), key
    tol = 1e-5 if dtype == np.float32 else 1e-12
    for key in ("eliminated_diagonal", "eliminated_gradient", "primary_diagonal", "primary_gradient"):
        assert np.abs(got[key] - ref[key]).max() <= tol * np.abs(ref[key]).max(), key
    rtol = 1e-5 if dtype == np.float32 else 1e-10
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=rtol, max_iterations=1000)
    ws = SC.SchurComplementSolverWorkspace()
    dp, dl, rep = SC.solve_damped_schur_complement(
        ne, 1e-3, SC.SchurComplementSolverOptions(max_iterations=1000, relative_tolerance=rtol), ws)
    assert rep["converged"] and rep_ref["converged"], rep["message"]
    stol = 1e-4 if dtype == np.float32 else 1e-6
    assert np.linalg.norm(host(dp) - dp_ref) <= stol * np.linalg.norm(dp_ref)
    assert np.linalg.norm(host(dl) - dl_ref) <= stol * np.linalg.norm(dl_ref)
    ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
    sysd = ws.export(torch.float32 if dtype == np.float32 else torch.float64)
    assert np.array_equal(host(sysd["row_offsets"]), ro) and np.array_equal(host(sysd["col_indices"]), ci)
    vtol = 1e-5 if dtype == np.float32 else 1e-12
    assert np.abs(host(sysd["values"]).astype(np.float64) - vals).max() <= vtol * np.abs(vals).max()
    assert np.abs(host(sysd["rhs"]).astype(np.float64) - rhs).max() <= vtol * np.abs(rhs).max()


def test_observation_topology_is_cached_and_rebuilt(checkers):
    prob = W.small_bundle(seed=3)
    ne = _device_from_observations(prob)
    _, _, v1 = ne.counts()
    ne.accumulate_observations(dev(prob["obs_primary"]), dev(prob["obs_eliminated"]), dev(prob["jp"]),
                               dev(prob["jl"]), dev(prob["residual"] * 0.5), prob["huber_delta"])
    assert ne.counts()[2] == v1
    shuffled = prob["obs_primary"].copy()
    shuffled[[0, 1]] = shuffled[[1, 0]]
    ne.accumulate_observations(dev(shuffled), dev(prob["obs_eliminated"]), dev(prob["jp"]), dev(prob["jl"]),
                               dev(prob["residual"]), prob["huber_delta"])
    assert ne.counts()[2] == v1 + 1


@pytest.mark.parametrize("precision", ["native", "mixed"])
def test_small_bundle_solve_matches_reference(checkers, precision):
    """P=20, L=2,000, 8,000 observations, lambda 1e-3, tol 1e-10, <=500 iterations."""
    prob = W.small_bundle(seed=1)
    orc = checkers.normal_equations_from_observations(prob)
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=1e-10, max_iterations=500)
    ne = _device_from_observations(prob)
    ws = SC.SchurComplementSolverWorkspace()
    opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10, precision=precision)
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
    assert rep["converged"] and rep_ref["converged"], rep["message"]
    if precision == "native":
        assert abs(rep["iterations"] - rep_ref["iterations"]) <= 1
    # solutions within 1e-6 relative (FP64)
    assert np.linalg.norm(host(dp) - dp_ref) <= 1e-6 * np.linalg.norm(dp_ref)
    assert np.linalg.norm(host(dl) - dl_ref) <= 1e-6 * np.linalg.norm(dl_ref)
    # reduced system: pattern bit-exact, values / RHS within rounding of the reference assembly
    ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
    sysd = ws.export()
    assert np.array_equal(host(sysd["row_offsets"]), ro)
    assert np.array_equal(host(sysd["col_indices"]), ci)
    assert np.abs(host(sysd["values"]) - vals).max() <= 1e-12 * np.abs(vals).max()
    assert np.abs(host(sysd["rhs"]) - rhs).max() <= 1e-12 * np.abs(rhs).max()
    # FP64 true relative residual of the device step on the reference's reduced system
    res = rhs - csr_matvec(ro, ci, vals, host(dp))
    assert np.linalg.norm(res) / np.linalg.norm(rhs) <= 1e-9


def test_fp32_assembly_products_match_reference(checkers):
    """Mixed precision with FP32 assembly products (6x6 / 3x3): the FP32-assembled reduced system
    within FP32 rounding of the reference's (pattern bit-exact, values within 1e-6 of the largest
    entry, RHS summed in FP64 within 1e-12), and the step refined to the FP64 tolerance by the
    matrix-free FP64 residual: within 1e-6 of the reference's steps, FP64 true residual <= 1e-10."""
    prob = W.small_bundle(seed=2)
    orc = checkers.normal_equations_from_observations(prob)
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=1e-10, max_iterations=500)
    ne = _device_from_observations(prob)
    ws = SC.SchurComplementSolverWorkspace()
    opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10,
                                           precision="mixed_fp32_assembly")
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
    assert rep["converged"] and rep["mixed_precision_used"], rep["message"]
    assert rep["true_relative_residual"] <= 1e-10 * 1.01
    assert np.linalg.norm(host(dp) - dp_ref) <= 1e-6 * np.linalg.norm(dp_ref)
    assert np.linalg.norm(host(dl) - dl_ref) <= 1e-6 * np.linalg.norm(dl_ref)
    ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
    res = rhs - csr_matvec(ro, ci, vals, host(dp))
    assert np.linalg.norm(res) / np.linalg.norm(rhs) <= 1e-10 * 1.5
    sysd = ws.export()
    assert np.array_equal(host(sysd["row_offsets"]), ro) and np.array_equal(host(sysd["col_indices"]), ci)
    assert np.abs(host(sysd["values"]) - vals).max() <= 1e-6 * np.abs(vals).max()
    assert np.abs(host(sysd["rhs"]) - rhs).max() <= 1e-12 * np.abs(rhs).max()
    # the workspace now holds FP32 values: the float SpMV reads them, the double one refuses
    x = np.random.default_rng(1).standard_normal(len(ro) - 1)
    y = host(ws.spmv(dev(x.astype(np.float32))))
    ref = csr_matvec(ro, ci, vals, x)
    assert np.abs(y - ref).max() <= 1e-5 * np.abs(ref).max()
    with pytest.raises(N.LogicError):
        ws.spmv(dev(x))
    # a plain solve on the same workspace assembles FP64 values again
    dp2, _, rep2 = SC.solve_damped_schur_complement(
        ne, 1e-3, SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10), ws)
    assert rep2["converged"]
    assert np.abs(host(ws.export()["values"]) - vals).max() <= 1e-12 * np.abs(vals).max()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reduced_system_spmv_matches_reference(checkers, dtype):
    """y = S x through the block-CSR SpMV of the assembled system against the reference's
    scalar CSR of the same reduced system; errors on type mismatch and aliasing."""
    prob = W.small_bundle(seed=3, dtype=dtype)
    orc = checkers.normal_equations_from_observations(prob, dtype=dtype)
    ne = _device_from_observations(prob, dtype)
    ws = SC.SchurComplementSolverWorkspace()
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    with pytest.raises(N.LogicError):
        ws.spmv(torch.ones(6, dtype=tdt, device="cuda"))
    SC.solve_damped_schur_complement(ne, 1e-3, SC.SchurComplementSolverOptions(max_iterations=5), ws)
    ro, ci, vals, _ = orc.schur_system(1e-3, with_preconditioner=False)
    x = np.random.default_rng(0).standard_normal(len(ro) - 1).astype(dtype)
    y = host(ws.spmv(dev(x)))
    ref = csr_matvec(ro, ci, vals.astype(np.float64), x.astype(np.float64))
    tol = 1e-5 if dtype == np.float32 else 1e-12
    assert np.abs(y - ref).max() <= tol * np.abs(ref).max()
    other = torch.float64 if dtype == np.float32 else torch.float32
    with pytest.raises(N.InvalidArgument):
        ws.spmv(torch.ones(len(x), dtype=other, device="cuda"))
    xd = dev(x)
    with pytest.raises(N.InvalidArgument):
        ws.spmv(xd, out=xd)


def test_float_pipeline_matches_reference(checkers):
    prob = W.small_bundle(seed=5, dtype=np.float32)
    orc = checkers.normal_equations_from_observations(prob, dtype=np.float32)
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=1e-5, max_iterations=500)
    ne = _device_from_observations(prob, np.float32)
    dp, dl, rep = SC.solve_damped_schur_complement(
        ne, 1e-3, SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-5))
    assert rep["converged"] and rep_ref["converged"]
    assert np.linalg.norm(host(dp) - dp_ref) <= 1e-4 * np.linalg.norm(dp_ref)
    assert np.linalg.norm(host(dl) - dl_ref) <= 1e-4 * np.linalg.norm(dl_ref)


def test_windowed_bundle_matches_oracle(checkers):
    """Large-system generator at 1/10 of the primaries and 1/100 of the eliminated blocks."""
    prob = W.large_bundle(seed=7, P=400, L=20000)
    orc = checkers.normal_equations_from_observations(prob)
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=1e-8, max_iterations=200)
    ne = _device_from_observations(prob)
    ws = SC.SchurComplementSolverWorkspace()
    dp, dl, rep = SC.solve_damped_schur_complement(
        ne, 1e-3, SC.SchurComplementSolverOptions(max_iterations=200), ws)
    assert rep["converged"] and rep_ref["converged"]
    assert abs(rep["iterations"] - rep_ref["iterations"]) <= 1
    assert np.linalg.norm(host(dp) - dp_ref) <= 1e-6 * np.linalg.norm(dp_ref)
    assert np.linalg.norm(host(dl) - dl_ref) <= 1e-6 * np.linalg.norm(dl_ref)
    ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
    sysd = ws.export()
    assert np.array_equal(host(sysd["row_offsets"]), ro) and np.array_equal(host(sysd["col_indices"]), ci)
    assert rep["true_relative_residual"] <= 1e-8 * 1.01


@pytest.mark.parametrize("precision", ["native", "mixed_fp32_assembly"])
def test_assembly_does_not_depend_on_the_order_of_crosses(precision):
    """The same normal equations with every eliminated block's crosses in ascending primary order
    (as the observation path stores them) and reversed (an uploaded state in another adjacency
    order): same pattern, values within rounding, same steps."""
    prob = W.large_bundle(seed=13, P=300, L=12000)
    ne_sorted = _device_from_observations(prob)
    state = ne_sorted.download()
    offs = state["adjacency_offsets"]
    order = np.concatenate([np.arange(offs[l], offs[l + 1])[::-1] for l in range(len(offs) - 1)])
    shuffled = dict(state)
    shuffled["cross_primary"] = state["cross_primary"][order]
    shuffled["cross_values"] = state["cross_values"][order]
    ne_rev = SC.DeviceNormalEquations(prob["P"], prob["L"], 6, 3)
    ne_rev.upload(shuffled)
    opts = SC.SchurComplementSolverOptions(max_iterations=200, relative_tolerance=1e-10, precision=precision)
    got = []
    for ne in (ne_sorted, ne_rev):
        ws = SC.SchurComplementSolverWorkspace()
        dp, dl, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
        assert rep["converged"], rep["message"]
        got.append((host(dp), host(dl), ws.export()))
    (dp_a, dl_a, sa), (dp_b, dl_b, sb) = got
    assert np.array_equal(host(sa["row_offsets"]), host(sb["row_offsets"]))
    assert np.array_equal(host(sa["col_indices"]), host(sb["col_indices"]))
    va, vb = host(sa["values"]), host(sb["values"])
    tol = 1e-12 if precision == "native" else 1e-6
    assert np.abs(va - vb).max() <= tol * np.abs(vb).max()
    assert np.abs(host(sa["rhs"]) - host(sb["rhs"])).max() <= 1e-12 * np.abs(host(sb["rhs"])).max()
    assert np.linalg.norm(dp_a - dp_b) <= 1e-8 * np.linalg.norm(dp_b)
    assert np.linalg.norm(dl_a - dl_b) <= 1e-8 * np.linalg.norm(dl_b)


def test_repeated_solves_are_bitwise_identical(checkers):
    prob = W.large_bundle(seed=9, P=300, L=10000)
    ne = _device_from_observations(prob)
    ws = SC.SchurComplementSolverWorkspace()
    a = SC.solve_damped_schur_complement(ne, 1e-3, workspace=ws)
    b = SC.solve_damped_schur_complement(ne, 1e-3, workspace=ws)
    ne2 = _device_from_observations(prob)
    c = SC.solve_damped_schur_complement(ne2, 1e-3)
    for x, y in ((a, b), (a, c)):
        assert torch.equal(x[0], y[0]) and torch.equal(x[1], y[1])


def test_empty_observations_give_zero_normal_equations():
    ne = SC.DeviceNormalEquations(3, 4, 6, 3)
    e = torch.empty(0, dtype=torch.int64, device="cuda")
    f = torch.empty(0, dtype=torch.float64, device="cuda")
    ne.accumulate_observations(e, e, f, f, f, 1.0)
    got = ne.download()
    assert ne.counts()[0] == 0
    assert not got["primary_diagonal"].any() and not got["eliminated_diagonal"].any()
    assert got["adjacency_offsets"].tolist() == [0, 0, 0, 0, 0]


@pytest.mark.parametrize("precision", ["native", "mixed_fp32_assembly"])
def test_every_assembly_shape_matches_reference(checkers, precision):
    """Each launch shape of the upper-block assembly pass (pair streams x lanes per pair) on a
    windowed system against the reference's reduced system: pattern bit-exact, values within
    rounding (FP64: 1e-12 of the largest entry; FP32 products: 1e-6), repeatable bit for bit per
    shape, and the steps within 1e-8 of each other across shapes."""
    prob = W.large_bundle(seed=17, P=200, L=8000)
    orc = checkers.normal_equations_from_observations(prob)
    ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
    ne = _device_from_observations(prob)
    opts = SC.SchurComplementSolverOptions(max_iterations=200, relative_tolerance=1e-10, precision=precision)
    shapes = SC.SchurComplementSolverWorkspace.assembly_shape_count()
    assert shapes >= 2
    tol = 1e-12 if precision == "native" else 1e-6
    steps = []
    for shape in range(shapes):
        ws = SC.SchurComplementSolverWorkspace()
        ws.assembly_shape = shape
        assert ws.assembly_shape == shape
        dp, dl, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
        assert rep["converged"], (shape, rep["message"])
        sysd = ws.export()
        assert np.array_equal(host(sysd["row_offsets"]), ro) and np.array_equal(host(sysd["col_indices"]), ci)
        v = host(sysd["values"])
        assert np.abs(v - vals).max() <= tol * np.abs(vals).max(), shape
        dp2, dl2, _ = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
        assert torch.equal(dp, dp2) and torch.equal(dl, dl2), shape
        assert np.array_equal(host(ws.export()["values"]), v), shape
        steps.append(host(dp))
    for s in steps[1:]:
        assert np.linalg.norm(s - steps[0]) <= 1e-8 * np.linalg.norm(steps[0])
    with pytest.raises(N.InvalidArgument):
        SC.SchurComplementSolverWorkspace().assembly_shape = shapes


def test_assembly_autotune_keeps_the_fastest_shape(checkers):
    """The autotuner times every shape on the solved system, keeps the fastest, leaves the
    workspace needing a new solve, and that solve matches the reference."""
    prob = W.large_bundle(seed=19, P=200, L=8000)
    orc = checkers.normal_equations_from_observations(prob)
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=1e-8, max_iterations=200)
    ne = _device_from_observations(prob)
    ws = SC.SchurComplementSolverWorkspace()
    other = SC.DeviceNormalEquations(3, 4, 6, 3)
    with pytest.raises(N.LogicError):
        ws.autotune_assembly(ne)  # nothing solved yet
    opts = SC.SchurComplementSolverOptions(max_iterations=200)
    SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
    with pytest.raises(N.LogicError):
        ws.autotune_assembly(other)  # not the system last solved
    with pytest.raises(N.InvalidArgument):
        ws.autotune_assembly(ne, repeats=0)
    tuned = ws.autotune_assembly(ne, repeats=2)
    count = SC.SchurComplementSolverWorkspace.assembly_shape_count()
    assert 0 <= tuned["shape"] < count and len(tuned["shape_ms"]) == count
    assert all(t > 0 for t in tuned["shape_ms"])
    assert tuned["ms"] == min(tuned["shape_ms"])
    assert ws.assembly_shape == tuned["shape"]
    with pytest.raises(N.LogicError):
        ws.export()  # reassembled by the autotuner: a new solve comes first
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
    assert rep["converged"] and rep["pattern_reused"]
    assert np.linalg.norm(host(dp) - dp_ref) <= 1e-6 * np.linalg.norm(dp_ref)
    assert np.linalg.norm(host(dl) - dl_ref) <= 1e-6 * np.linalg.norm(dl_ref)


def test_one_workspace_alternating_systems_matches_fresh_workspaces():
    """The PCG iteration graphs a workspace keeps (one per operand set) follow the system: solves
    that alternate between two systems of different sizes, and between plain and mixed
    precision, on one workspace equal solves on fresh workspaces bit for bit."""
    probs = [W.large_bundle(seed=21, P=150, L=6000), W.small_bundle(seed=22)]
    nes = [_device_from_observations(p) for p in probs]
    plain = SC.SchurComplementSolverOptions(max_iterations=300, relative_tolerance=1e-10)
    mixed = SC.SchurComplementSolverOptions(max_iterations=300, relative_tolerance=1e-10, precision="mixed")
    shared = SC.SchurComplementSolverWorkspace()
    for ne, opts in [(nes[0], plain), (nes[1], plain), (nes[0], mixed), (nes[1], mixed), (nes[0], plain)]:
        dp, dl, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, shared)
        dp_f, dl_f, rep_f = SC.solve_damped_schur_complement(ne, 1e-3, opts, SC.SchurComplementSolverWorkspace())
        assert rep["converged"] and rep_f["converged"]
        assert rep["iterations"] == rep_f["iterations"]
        assert torch.equal(dp, dp_f) and torch.equal(dl, dl_f)


@pytest.mark.parametrize("precision", ["native", "mixed", "mixed_fp32_assembly"])
def test_step_vectors_need_no_16_byte_alignment(precision):
    """The caller's step vectors may start 8 bytes past a 16-byte boundary (a view one element
    into a buffer): every kernel reads and writes them element by element, and the steps equal
    those of aligned vectors bit for bit."""
    prob = W.large_bundle(seed=29, P=120, L=6000)
    ne = _device_from_observations(prob)
    n, m = 120 * 6, 6000 * 3
    opts = SC.SchurComplementSolverOptions(max_iterations=300, relative_tolerance=1e-9, precision=precision)
    ws = SC.SchurComplementSolverWorkspace()
    dp, dl, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
    assert rep["converged"], rep["message"]
    pbuf = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    lbuf = torch.zeros(m + 1, dtype=torch.float64, device="cuda")
    dp1, dl1 = pbuf[1:], lbuf[1:]
    assert dp1.data_ptr() % 16 == 8 and dl1.data_ptr() % 16 == 8
    ws2 = SC.SchurComplementSolverWorkspace()
    _, _, rep2 = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws2, dp1, dl1)
    assert rep2["converged"] and rep2["iterations"] == rep["iterations"]
    assert torch.equal(dp1, dp) and torch.equal(dl1, dl)


def test_step_vectors_are_checked():
    """Step vectors of the wrong type, device or length are refused before any device work."""
    prob = W.large_bundle(seed=29, P=40, L=600)
    ne = _device_from_observations(prob)
    ws = SC.SchurComplementSolverWorkspace()
    n, m = 40 * 6, 600 * 3
    good_p = torch.zeros(n, dtype=torch.float64, device="cuda")
    good_l = torch.zeros(m, dtype=torch.float64, device="cuda")
    for dp, dl in ((good_p[:-1], good_l), (good_p, good_l[:-1]), (good_p.float(), good_l),
                   (good_p.cpu(), good_l), (torch.zeros(2 * n, dtype=torch.float64, device="cuda")[::2], good_l)):
        with pytest.raises(N.InvalidArgument):
            SC.solve_damped_schur_complement(ne, 1e-3, SC.SchurComplementSolverOptions(), ws, dp, dl)
    _, _, rep = SC.solve_damped_schur_complement(ne, 1e-3, SC.SchurComplementSolverOptions(), ws, good_p, good_l)
    assert rep["converged"]
