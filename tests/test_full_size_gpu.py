"""The large Schur LM workload at its stated size against the oracle: P=4,000 primary 6-dof
blocks, L=2,000,000 eliminated 3-dof blocks, 2+Poisson(4) primaries per eliminated block from a
wrapped window of 40 (11,998,722 shuffled two-row observations), Huber delta 1, lambda 1e-3,
tolerance 1e-8.  The oracle restates the reference's CPU path (BlockNormalEquations accumulation,
rebuild of the Schur pattern, solveDampedSchurComplement with the Cpu backend) and is pinned bit
for bit to the reference library at smaller sizes.

Checked here at full size: the reduced system's scalar-CSR pattern bit for bit, its values and
RHS within 1e-12 of the largest entry, and the primary / eliminated steps of the plain FP64,
mixed-precision (FP64 assembly, and FP32 assembly products) and learned + mixed (FP32 assembly
products) solves within 1e-6 relative of the oracle's steps."""
import numpy as np
import pytest
import torch

from gpu_util import dev, host
from plamatrix_b200 import schur as SC
from plamatrix_b200 import workloads as W

pytestmark = pytest.mark.gpu

P_FULL, L_FULL = 4000, 2_000_000


@pytest.fixture(scope="module")
def full_size(checkers):
    prob = W.large_bundle(seed=0, P=P_FULL, L=L_FULL)
    orc = checkers.normal_equations_from_observations(prob)
    dp_ref, dl_ref, rep_ref = orc.solve(1e-3, relative_tolerance=1e-8, max_iterations=200)
    ro, ci, vals, rhs = orc.schur_system(1e-3, with_preconditioner=False)
    del orc
    ne = SC.DeviceNormalEquations(P_FULL, L_FULL, 6, 3)
    ne.accumulate_observations(dev(prob["obs_primary"]), dev(prob["obs_eliminated"]), dev(prob["jp"]),
                               dev(prob["jl"]), dev(prob["residual"]), prob["huber_delta"])
    del prob
    return {"ne": ne, "dp": dp_ref, "dl": dl_ref, "rep": rep_ref, "system": (ro, ci, vals, rhs)}


def _learned_net():
    net = SC.LearnedPreconditioner(seed=21)
    rng = np.random.default_rng(22)
    net.set_params((0.05 * rng.standard_normal(net.param_count())).astype(np.float32))
    return net


@pytest.mark.parametrize("variant", ["plain", "mixed", "mixed_fp32_assembly", "learned_mixed"])
def test_full_size_step_matches_oracle(full_size, variant):
    kw = {"max_iterations": 200, "relative_tolerance": 1e-8}
    if variant != "plain":
        kw["precision"] = "mixed" if variant == "mixed" else "mixed_fp32_assembly"
    if variant == "learned_mixed":
        kw["learned"] = _learned_net()
    ws = SC.SchurComplementSolverWorkspace()
    dp, dl, rep = SC.solve_damped_schur_complement(full_size["ne"], 1e-3, SC.SchurComplementSolverOptions(**kw), ws)
    ref = full_size["rep"]
    assert rep["converged"] and ref["converged"], rep["message"]
    if variant == "plain":
        assert abs(rep["iterations"] - ref["iterations"]) <= 1
    dp_ref, dl_ref = full_size["dp"], full_size["dl"]
    assert np.linalg.norm(host(dp) - dp_ref) <= 1e-6 * np.linalg.norm(dp_ref)
    assert np.linalg.norm(host(dl) - dl_ref) <= 1e-6 * np.linalg.norm(dl_ref)
    if variant == "plain":
        ro, ci, vals, rhs = full_size["system"]
        sysd = ws.export()
        assert np.array_equal(host(sysd["row_offsets"]), ro)
        assert np.array_equal(host(sysd["col_indices"]), ci)
        assert np.abs(host(sysd["values"]) - vals).max() <= 1e-12 * np.abs(vals).max()
        assert np.abs(host(sysd["rhs"]) - rhs).max() <= 1e-12 * np.abs(rhs).max()
        del sysd
    torch.cuda.empty_cache()
