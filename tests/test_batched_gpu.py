"""Batched independent Schur solves (one block-diagonal union, per-system PCG state on the
device, graph-replayed iterations) against the same systems solved one by one."""
import numpy as np
import pytest
import torch

from gpu_util import dev
from plamatrix_b200 import _native as N
from plamatrix_b200 import schur as SC
from plamatrix_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _ne(prob):
    ne = SC.DeviceNormalEquations(prob["P"], prob["L"], prob["bp"], prob["bl"])
    ne.accumulate_observations(dev(prob["obs_primary"]), dev(prob["obs_eliminated"]), dev(prob["jp"]),
                               dev(prob["jl"]), dev(prob["residual"]), prob["huber_delta"])
    return ne


def _problems(count=12, seed=0):
    rng = np.random.default_rng(seed)
    return [W.bundle_problem(int(rng.integers(8, 40)), int(rng.integers(200, 1500)), per_eliminated=4,
                             seed=1000 + seed * 100 + i) for i in range(count)]


def test_batched_matches_individual_solves():
    probs = _problems()
    union = SC.pack_observation_systems(probs)
    ne = _ne(union)
    opts = SC.SchurComplementSolverOptions(max_iterations=300, relative_tolerance=1e-10)
    dp, dl, rep, per = SC.solve_batched_schur_complement(ne, 1e-3, union["primary_offsets"], opts)
    assert rep["converged"], rep["message"]
    P_off, L_off = union["primary_offsets"], union["eliminated_offsets"]
    for s, prob in enumerate(probs):
        ref_dp, ref_dl, ref = SC.solve_damped_schur_complement(_ne(prob), 1e-3, opts)
        assert ref["converged"] and per[s]["converged"]
        assert abs(per[s]["iterations"] - ref["iterations"]) <= 1
        a, b = dp[6 * P_off[s]:6 * P_off[s + 1]], ref_dp
        assert torch.linalg.norm(a - b) <= 1e-6 * torch.linalg.norm(b)
        a, b = dl[3 * L_off[s]:3 * L_off[s + 1]], ref_dl
        assert torch.linalg.norm(a - b) <= 1e-6 * torch.linalg.norm(b)
        assert per[s]["time_ms"] >= 0.0


def test_batched_family_matches_oracle_per_system(checkers):
    """Eight systems of the 512-system uneven family (P ~ U{8..512}, L ~ U{500..50,000}, 4 uniform
    distinct primaries per eliminated block) solved in one batched call; every system's steps
    against the oracle's per-system solve (the reference's solveDampedSchurComplement, Cpu backend,
    restated): within 1e-6 relative, iteration counts within 1."""
    sizes = W.uneven_family_sizes(512)
    picks = [0, 1, 2, 3, 100, 200, 300, 511]
    probs = []
    for i in picks:
        P, L = sizes[i]
        d = W.uneven_family_system(i, P, L)
        probs.append({k: (v.cpu().numpy() if torch.is_tensor(v) else v) for k, v in d.items()})
    union = SC.pack_observation_systems(probs)
    ne = _ne(union)
    opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-8)
    dp, dl, rep, per = SC.solve_batched_schur_complement(ne, 1e-3, union["primary_offsets"], opts)
    assert rep["converged"], rep["message"]
    P_off, L_off = union["primary_offsets"], union["eliminated_offsets"]
    dp_h, dl_h = dp.cpu().numpy(), dl.cpu().numpy()
    for s, prob in enumerate(probs):
        orc = checkers.normal_equations_from_observations(prob)
        ref_dp, ref_dl, ref = orc.solve(1e-3, relative_tolerance=1e-8, max_iterations=500)
        assert ref["converged"] and per[s]["converged"]
        assert abs(per[s]["iterations"] - ref["iterations"]) <= 1, (s, per[s]["iterations"], ref["iterations"])
        a = dp_h[6 * P_off[s]:6 * P_off[s + 1]]
        assert np.linalg.norm(a - ref_dp) <= 1e-6 * np.linalg.norm(ref_dp)
        a = dl_h[3 * L_off[s]:3 * L_off[s + 1]]
        assert np.linalg.norm(a - ref_dl) <= 1e-6 * np.linalg.norm(ref_dl)


def test_batched_rejects_coupled_systems():
    probs = _problems(3, seed=1)
    union = SC.pack_observation_systems(probs)
    ne = _ne(union)
    bad = union["primary_offsets"].copy()
    bad[1] += 1  # the first two systems now share a block row boundary that their observations cross
    with pytest.raises(N.InvalidArgument):
        SC.solve_batched_schur_complement(ne, 1e-3, bad)


def test_batched_learned_with_per_system_fallback():
    probs = _problems(6, seed=2)
    union = SC.pack_observation_systems(probs)
    ne = _ne(union)
    net = SC.LearnedPreconditioner(seed=3)
    rng = np.random.default_rng(4)
    net.set_params((0.8 * rng.standard_normal(net.param_count())).astype(np.float32))
    opts = SC.SchurComplementSolverOptions(max_iterations=400, relative_tolerance=1e-10, learned=net,
                                           stagnation_window=4)
    dp, _, rep, per = SC.solve_batched_schur_complement(ne, 1e-3, union["primary_offsets"], opts)
    plain_dp, _, plain, _ = SC.solve_batched_schur_complement(
        _ne(union), 1e-3, union["primary_offsets"], SC.SchurComplementSolverOptions(max_iterations=400,
                                                                                    relative_tolerance=1e-10))
    assert plain["converged"], plain["message"]
    assert rep["converged"], [(s["converged"], s["iterations"], s["learned_fallback"], s["breakdown"]) for s in per]
    assert torch.linalg.norm(dp - plain_dp) <= 1e-6 * torch.linalg.norm(plain_dp)


@pytest.mark.parametrize("learned", [False, True])
def test_batched_mixed_precision_meets_the_fp64_tolerance_per_system(checkers, learned):
    """Mixed precision in the batched solve: FP64 assembly, iterations on the FP32 values and
    preconditioner blocks (FP64 vectors and dots), then an FP64 true-residual check of every system
    that converged, which iterates on from the FP64 residual when the check misses.  Every system
    meets its tolerance on the reference's FP64 reduced system, and its steps agree with the
    oracle's per-system solve within 1e-6."""
    sizes = W.uneven_family_sizes(512)
    picks = [0, 5, 150, 400]
    probs = []
    for i in picks:
        P, L = sizes[i]
        d = W.uneven_family_system(i, P, L)
        probs.append({k: (v.cpu().numpy() if torch.is_tensor(v) else v) for k, v in d.items()})
    union = SC.pack_observation_systems(probs)
    ne = _ne(union)
    net = SC.LearnedPreconditioner(seed=5) if learned else None
    opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-8, precision="mixed",
                                           learned=net)
    dp, dl, rep, per = SC.solve_batched_schur_complement(ne, 1e-3, union["primary_offsets"], opts)
    assert rep["converged"], rep["message"]
    assert rep["mixed_precision_used"] and rep["refinement_steps"] >= 1
    P_off, L_off = union["primary_offsets"], union["eliminated_offsets"]
    dp_h, dl_h = dp.cpu().numpy(), dl.cpu().numpy()
    for s, prob in enumerate(probs):
        orc = checkers.normal_equations_from_observations(prob)
        ref_dp, ref_dl, ref = orc.solve(1e-3, relative_tolerance=1e-8, max_iterations=500)
        assert ref["converged"] and per[s]["converged"]
        a = dp_h[6 * P_off[s]:6 * P_off[s + 1]]
        ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
        res = rhs - np.array([vals[ro[i]:ro[i + 1]] @ a[ci[ro[i]:ro[i + 1]]] for i in range(len(ro) - 1)])
        assert np.linalg.norm(res) <= 1e-8 * 1.01 * np.linalg.norm(rhs), s
        assert np.linalg.norm(a - ref_dp) <= 1e-6 * np.linalg.norm(ref_dp)
        b = dl_h[3 * L_off[s]:3 * L_off[s + 1]]
        assert np.linalg.norm(b - ref_dl) <= 1e-6 * np.linalg.norm(ref_dl)
