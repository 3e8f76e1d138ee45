// C-ABI harness around the reference's own CPU library (TEST INFRASTRUCTURE ONLY).
//
// oracle/Makefile compiles the reference's CPU sources for this path (listed there)
// together with this file into oracle/_ref/libplamatrix_ref.so.  Nothing here is
// product code: the tests use it to pin the C oracle to the real reference, and
// bench.py's reference arm times it on the host cores.
//
// The harness needs the accumulated BlockNormalEquations state and the reduced
// Schur CSR that block_schur_detail::assembleReducedSchurCsr builds.  Both live
// behind `private`; this translation unit (and only it) opens them up so the real
// reference routines can be called on the real reference state.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <algorithm>
#include <array>
#include <chrono>
#include <limits>
#include <map>
#include <mutex>
#include <sstream>
#include <unordered_map>
#include <utility>

#define private public
#include "plamatrix/optimization/block_schur.h"
#undef private
#include "plamatrix/optimization/robust_loss.h"
#include "plamatrix/sparse/coo_matrix.h"
#include "plamatrix/sparse/iterative_solver.h"
#include "plamatrix/sparse/sparse_ops.h"

#include "optimization/block_schur_linear_algebra.h"
#include "optimization/block_schur_sparse_assembly.h"

using plamatrix::Index;

namespace
{
thread_local std::string g_error;

int fail(int status, const char* what)
{
    g_error = what;
    return status;
}

template <typename Fn>
int guarded(Fn&& fn)
{
    try
    {
        fn();
        return 0;
    }
    catch (const std::out_of_range& e)
    {
        return fail(2, e.what());
    }
    catch (const std::overflow_error& e)
    {
        return fail(5, e.what());
    }
    catch (const std::invalid_argument& e)
    {
        return fail(1, e.what());
    }
    catch (const std::logic_error& e)
    {
        return fail(4, e.what());
    }
    catch (const std::runtime_error& e)
    {
        return fail(3, e.what());
    }
    catch (const std::exception& e)
    {
        return fail(3, e.what());
    }
}

template <typename S>
int cooToCsrImpl(int64_t rows, int64_t cols, int64_t count, const int64_t* ri, const int64_t* ci,
                 const S* v, int64_t* row_offsets, int64_t* out_cols, S* out_vals, int64_t* out_nnz)
{
    return guarded([&] {
        std::vector<Index> r(ri, ri + count), c(ci, ci + count);
        std::vector<S> values(v, v + count);
        auto csr = plamatrix::cooToCsr<S>(rows, cols, r, c, values);
        std::memcpy(row_offsets, csr.rowOffsets(), sizeof(Index) * static_cast<size_t>(rows + 1));
        std::memcpy(out_cols, csr.colIndices(), sizeof(Index) * static_cast<size_t>(csr.nnz()));
        std::memcpy(out_vals, csr.values(), sizeof(S) * static_cast<size_t>(csr.nnz()));
        *out_nnz = csr.nnz();
    });
}

template <typename S>
plamatrix::CSRMatrix<S, plamatrix::Device::CPU> makeCsr(int64_t n, const int64_t* rp, const int64_t* ci,
                                                         const S* v, int64_t cols = -1)
{
    plamatrix::CSRMatrix<S, plamatrix::Device::CPU> csr(n, cols < 0 ? n : cols, rp[n]);
    std::memcpy(csr.rowOffsets(), rp, sizeof(Index) * static_cast<size_t>(n + 1));
    std::memcpy(csr.colIndices(), ci, sizeof(Index) * static_cast<size_t>(rp[n]));
    std::memcpy(csr.values(), v, sizeof(S) * static_cast<size_t>(rp[n]));
    return csr;
}

template <typename S>
int spmvImpl(int64_t n, int64_t cols, const int64_t* rp, const int64_t* ci, const S* v, const S* x, S* y)
{
    return guarded([&] {
        auto csr = makeCsr(n, rp, ci, v, cols);
        plamatrix::DenseMatrix<S, plamatrix::Device::CPU> xin(cols, 1), out(n, 1);
        std::memcpy(xin.data(), x, sizeof(S) * static_cast<size_t>(cols));
        plamatrix::spmv(csr, xin, out);
        std::memcpy(y, out.data(), sizeof(S) * static_cast<size_t>(n));
    });
}

template <typename S>
int spmmImpl(int64_t n, int64_t cols, const int64_t* rp, const int64_t* ci, const S* v, int64_t k, const S* in, S* out)
{
    return guarded([&] {
        auto csr = makeCsr(n, rp, ci, v, cols);
        plamatrix::DenseMatrix<S, plamatrix::Device::CPU> b(cols, k), c(n, k);
        std::memcpy(b.data(), in, sizeof(S) * static_cast<size_t>(cols * k));
        plamatrix::spmm(csr, b, c);
        std::memcpy(out, c.data(), sizeof(S) * static_cast<size_t>(n * k));
    });
}

struct SolverOptionsC
{
    int max_iterations;
    double relative_tolerance;
    double absolute_tolerance;
    int use_jacobi;
    int require_convergence;
};

struct SolverReportC
{
    int converged;
    int iterations;
    double initial_residual;
    double final_residual;
};

template <typename S>
int pcgImpl(int64_t n, const int64_t* rp, const int64_t* ci, const S* v, const S* rhs, S* solution,
            const SolverOptionsC* o, int preconditioned, SolverReportC* report)
{
    std::memset(report, 0, sizeof(*report));
    return guarded([&] {
        auto csr = makeCsr(n, rp, ci, v);
        plamatrix::DenseMatrix<S, plamatrix::Device::CPU> b(n, 1), x(n, 1);
        std::memcpy(b.data(), rhs, sizeof(S) * static_cast<size_t>(n));
        std::memcpy(x.data(), solution, sizeof(S) * static_cast<size_t>(n));
        plamatrix::IterativeSolverOptions options;
        options.maxIterations = o->max_iterations;
        options.relativeTolerance = o->relative_tolerance;
        options.absoluteTolerance = o->absolute_tolerance;
        options.useJacobiPreconditioner = o->use_jacobi != 0;
        options.requireConvergence = o->require_convergence != 0;
        const auto r = preconditioned ? plamatrix::pcg(csr, b, x, options) : plamatrix::cg(csr, b, x, options);
        std::memcpy(solution, x.data(), sizeof(S) * static_cast<size_t>(n));
        report->converged = r.converged;
        report->iterations = r.iterations;
        report->initial_residual = r.initialResidual;
        report->final_residual = r.finalResidual;
    });
}

template <typename S>
struct RefNe
{
    plamatrix::BlockNormalEquations<S> equations;
    plamatrix::SchurComplementSolverWorkspace<S> workspace;
    RefNe(Index P, Index L, Index bp, Index bl) : equations(P, L, bp, bl) {}
};

template <typename S>
int addResidualImpl(RefNe<S>* ne, int64_t np, const int64_t* primaries, const S* pj, int64_t eliminated,
                    const S* ej, const S* r, int64_t m, S w)
{
    return guarded([&] {
        auto& eq = ne->equations;
        if (np <= 0)
        {
            eq.addEliminatedResidualBlock(eliminated, ej, r, m, w);
            return;
        }
        std::vector<Index> blocks(primaries, primaries + np);
        std::vector<const S*> jacobians;
        for (int64_t k = 0; k < np; ++k)
        {
            jacobians.push_back(pj + k * m * eq.primaryBlockSize());
        }
        if (eliminated < 0)
        {
            eq.addPrimaryResidualBlocks(blocks, jacobians, r, m, w);
        }
        else
        {
            eq.addResidualBlocks(blocks, jacobians, eliminated, ej, r, m, w);
        }
    });
}

template <typename S>
int addObservationsImpl(RefNe<S>* ne, int64_t count, int64_t m, const int64_t* p, const int64_t* l,
                        const S* pj, const S* ej, const S* r, S delta)
{
    return guarded([&] {
        auto& eq = ne->equations;
        const Index bp = eq.primaryBlockSize(), bl = eq.eliminatedBlockSize();
        for (int64_t i = 0; i < count; ++i)
        {
            const S* residual = r + i * m;
            S squared = S(0);
            for (int64_t k = 0; k < m; ++k)
            {
                squared += residual[k] * residual[k];
            }
            const auto loss = plamatrix::evaluateHuberLoss(squared, delta);
            eq.addResidualBlock(p[i], l[i], pj + i * m * bp, ej + i * m * bl, residual, m, loss.weight);
        }
    });
}

template <typename S>
void exportImpl(const RefNe<S>* ne, S* hpp, S* hll, S* gp, S* gl, int64_t* adjacency_offsets,
                int64_t* cross_primary, S* cross_values, int64_t* pc_row, int64_t* pc_col, S* pc_values)
{
    const auto& eq = ne->equations;
    if (hpp)
        std::memcpy(hpp, eq._primaryDiagonal.data(), sizeof(S) * eq._primaryDiagonal.size());
    if (hll)
        std::memcpy(hll, eq._eliminatedDiagonal.data(), sizeof(S) * eq._eliminatedDiagonal.size());
    if (gp)
        std::memcpy(gp, eq._primaryGradient.data(), sizeof(S) * eq._primaryGradient.size());
    if (gl)
        std::memcpy(gl, eq._eliminatedGradient.data(), sizeof(S) * eq._eliminatedGradient.size());
    int64_t k = 0;
    const size_t cross_size = static_cast<size_t>(eq._primaryBlockSize * eq._eliminatedBlockSize);
    for (size_t l = 0; l < eq._eliminatedAdjacency.size(); ++l)
    {
        if (adjacency_offsets)
            adjacency_offsets[l] = k;
        for (const size_t c : eq._eliminatedAdjacency[l])
        {
            if (cross_primary)
                cross_primary[k] = eq._crossBlocks[c].primaryBlock;
            if (cross_values)
                std::memcpy(cross_values + k * cross_size, eq._crossBlocks[c].values.data(),
                            sizeof(S) * cross_size);
            ++k;
        }
    }
    if (adjacency_offsets)
        adjacency_offsets[eq._eliminatedAdjacency.size()] = k;
    const size_t pc_size = static_cast<size_t>(eq._primaryBlockSize * eq._primaryBlockSize);
    for (size_t i = 0; i < eq._primaryCrossBlocks.size(); ++i)
    {
        if (pc_row)
            pc_row[i] = eq._primaryCrossBlocks[i].rowBlock;
        if (pc_col)
            pc_col[i] = eq._primaryCrossBlocks[i].columnBlock;
        if (pc_values)
            std::memcpy(pc_values + i * pc_size, eq._primaryCrossBlocks[i].values.data(), sizeof(S) * pc_size);
    }
}

struct SchurOptionsC
{
    int backend;
    int max_iterations;
    double relative_tolerance;
    double absolute_tolerance;
    double minimum_diagonal;
    int use_initial_guess;
};

struct SchurReportC
{
    int converged;
    int iterations;
    double initial_residual_norm;
    double final_residual_norm;
    int pattern_reused;
    int64_t pattern_build_count;
    double linear_solve_seconds;
    double total_seconds;
    char message[128];
};

template <typename S>
int schurSolveImpl(RefNe<S>* ne, S damping, const SchurOptionsC* o, S* primary_step, S* eliminated_step,
                   SchurReportC* out)
{
    std::memset(out, 0, sizeof(*out));
    return guarded([&] {
        plamatrix::SchurComplementSolverOptions<S> options;
        options.linearBackend = o->backend == 1 ? plamatrix::SchurComplementLinearBackend::DenseCpu
                                                : plamatrix::SchurComplementLinearBackend::Cpu;
        options.maxIterations = o->max_iterations;
        options.relativeTolerance = static_cast<S>(o->relative_tolerance);
        options.absoluteTolerance = static_cast<S>(o->absolute_tolerance);
        options.minimumDiagonal = static_cast<S>(o->minimum_diagonal);
        options.useInitialGuess = o->use_initial_guess != 0;
        const auto& eq = ne->equations;
        const size_t n = static_cast<size_t>(eq.primaryBlockCount() * eq.primaryBlockSize());
        const size_t m = static_cast<size_t>(eq.eliminatedBlockCount() * eq.eliminatedBlockSize());
        std::vector<S> dp(primary_step, primary_step + n), dl;
        const auto start = std::chrono::steady_clock::now();
        const auto report =
            plamatrix::solveDampedSchurComplement(eq, damping, options, ne->workspace, &dp, &dl);
        out->total_seconds =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        out->converged = report.converged;
        out->iterations = report.iterations;
        out->initial_residual_norm = static_cast<double>(report.initialResidualNorm);
        out->final_residual_norm = static_cast<double>(report.finalResidualNorm);
        out->pattern_reused = report.schurPatternReused;
        out->pattern_build_count = static_cast<int64_t>(ne->workspace.patternBuildCount());
        out->linear_solve_seconds = report.linearSolveSeconds;
        std::snprintf(out->message, sizeof(out->message), "%s", report.message.c_str());
        if (dp.size() == n)
            std::memcpy(primary_step, dp.data(), sizeof(S) * n);
        if (dl.size() == m)
            std::memcpy(eliminated_step, dl.data(), sizeof(S) * m);
    });
}

// Reduced Schur CSR + RHS + block-Jacobi inverses, computed by the reference routines
// (block_schur.cpp:102-250 restated only for the small preliminaries it needs, then
// block_schur_detail::assembleReducedSchurCsr with the Cpu backend).
template <typename S>
int schurSystemImpl(RefNe<S>* ne, S damping, S minimum_diagonal, int64_t* nnz_out, int64_t* row_offsets,
                    int64_t* col_indices, S* values, S* rhs)
{
    return guarded([&] {
        const auto& eq = ne->equations;
        const Index P = eq._primaryBlockCount, L = eq._eliminatedBlockCount;
        const Index bp = eq._primaryBlockSize, bl = eq._eliminatedBlockSize;
        std::vector<S> primary = eq._primaryDiagonal, eliminated = eq._eliminatedDiagonal;
        auto damp = [&](std::vector<S>& blocks, Index count, Index size) {
            for (Index block = 0; block < count; ++block)
                for (Index d = 0; d < size; ++d)
                {
                    S& value = blocks[static_cast<size_t>(block * size * size + d * size + d)];
                    value += damping * std::max(std::abs(value), minimum_diagonal);
                }
        };
        damp(primary, P, bp);
        damp(eliminated, L, bl);
        std::vector<S> inverse(static_cast<size_t>(L * bl * bl));
        std::vector<S> scratch(static_cast<size_t>(bl * bl + 3 * bl));
        for (Index block = 0; block < L; ++block)
        {
            if (!plamatrix::block_schur_detail::invertPositiveDefiniteInto(
                    eliminated.data() + block * bl * bl, bl, inverse.data() + block * bl * bl, scratch.data(),
                    scratch.data() + bl * bl))
                throw std::runtime_error("eliminated block is not positive definite");
        }
        bool reused = false, on_device = false;
        auto csr = plamatrix::block_schur_detail::assembleReducedSchurCsr(
            P, L, bp, bl, primary, inverse, eq._primaryCrossBlocks, eq._crossBlocks, eq._eliminatedAdjacency,
            ne->workspace, &reused, plamatrix::SchurComplementLinearBackend::Cpu, &on_device);
        *nnz_out = csr.nnz();
        if (row_offsets)
            std::memcpy(row_offsets, csr.rowOffsets(), sizeof(Index) * static_cast<size_t>(csr.rows() + 1));
        if (col_indices)
            std::memcpy(col_indices, csr.colIndices(), sizeof(Index) * static_cast<size_t>(csr.nnz()));
        if (values)
            std::memcpy(values, csr.values(), sizeof(S) * static_cast<size_t>(csr.nnz()));
        if (rhs)
        {
            // block_schur.cpp:151-177
            for (Index i = 0; i < P * bp; ++i)
                rhs[i] = -eq._primaryGradient[static_cast<size_t>(i)];
            std::vector<S> product(static_cast<size_t>(bl));
            for (Index block = 0; block < L; ++block)
            {
                plamatrix::block_schur_detail::multiplyMatrixVector(
                    inverse.data() + block * bl * bl, bl, bl, eq._eliminatedGradient.data() + block * bl,
                    product.data());
                for (const size_t c : eq._eliminatedAdjacency[static_cast<size_t>(block)])
                {
                    const auto& cross = eq._crossBlocks[c];
                    plamatrix::block_schur_detail::addMatrixVector(cross.values.data(), bp, bl, product.data(),
                                                                  S(1), rhs + cross.primaryBlock * bp);
                }
            }
        }
    });
}

} // namespace

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

int ref_coo_to_csr_f32(int64_t rows, int64_t cols, int64_t count, const int64_t* ri, const int64_t* ci,
                       const float* v, int64_t* ro, int64_t* oc, float* ov, int64_t* nnz)
{
    return cooToCsrImpl(rows, cols, count, ri, ci, v, ro, oc, ov, nnz);
}
int ref_coo_to_csr_f64(int64_t rows, int64_t cols, int64_t count, const int64_t* ri, const int64_t* ci,
                       const double* v, int64_t* ro, int64_t* oc, double* ov, int64_t* nnz)
{
    return cooToCsrImpl(rows, cols, count, ri, ci, v, ro, oc, ov, nnz);
}
int ref_csr_spmv_f32(int64_t n, int64_t cols, const int64_t* rp, const int64_t* ci, const float* v,
                     const float* x, float* y)
{
    return spmvImpl(n, cols, rp, ci, v, x, y);
}
int ref_csr_spmv_f64(int64_t n, int64_t cols, const int64_t* rp, const int64_t* ci, const double* v,
                     const double* x, double* y)
{
    return spmvImpl(n, cols, rp, ci, v, x, y);
}
int ref_csr_spmm_f32(int64_t n, int64_t cols, const int64_t* rp, const int64_t* ci, const float* v, int64_t k,
                     const float* in, float* out)
{
    return spmmImpl(n, cols, rp, ci, v, k, in, out);
}
int ref_csr_spmm_f64(int64_t n, int64_t cols, const int64_t* rp, const int64_t* ci, const double* v, int64_t k,
                     const double* in, double* out)
{
    return spmmImpl(n, cols, rp, ci, v, k, in, out);
}
int ref_pcg_f32(int64_t n, const int64_t* rp, const int64_t* ci, const float* v, const float* rhs, float* x,
                const SolverOptionsC* o, int preconditioned, SolverReportC* r)
{
    return pcgImpl(n, rp, ci, v, rhs, x, o, preconditioned, r);
}
int ref_pcg_f64(int64_t n, const int64_t* rp, const int64_t* ci, const double* v, const double* rhs,
                double* x, const SolverOptionsC* o, int preconditioned, SolverReportC* r)
{
    return pcgImpl(n, rp, ci, v, rhs, x, o, preconditioned, r);
}
int ref_huber_f64(double s, double delta, double* cost, double* weight)
{
    return guarded([&] {
        const auto e = plamatrix::evaluateHuberLoss(s, delta);
        *cost = e.cost;
        *weight = e.weight;
    });
}
int ref_huber_f32(float s, float delta, float* cost, float* weight)
{
    return guarded([&] {
        const auto e = plamatrix::evaluateHuberLoss(s, delta);
        *cost = e.cost;
        *weight = e.weight;
    });
}

#define REF_NE_API(S, SFX)                                                                                  \
    void* ref_ne_create_##SFX(int64_t P, int64_t L, int64_t bp, int64_t bl)                                 \
    {                                                                                                       \
        try                                                                                                 \
        {                                                                                                   \
            return new RefNe<S>(P, L, bp, bl);                                                              \
        }                                                                                                   \
        catch (const std::exception& e)                                                                     \
        {                                                                                                   \
            g_error = e.what();                                                                             \
            return nullptr;                                                                                 \
        }                                                                                                   \
    }                                                                                                       \
    void ref_ne_destroy_##SFX(void* ne) { delete static_cast<RefNe<S>*>(ne); }                              \
    int ref_ne_add_residual_##SFX(void* ne, int64_t np, const int64_t* p, const S* pj, int64_t l,           \
                                  const S* lj, const S* r, int64_t m, S w)                                  \
    {                                                                                                       \
        return addResidualImpl(static_cast<RefNe<S>*>(ne), np, p, pj, l, lj, r, m, w);                      \
    }                                                                                                       \
    int ref_ne_add_observations_##SFX(void* ne, int64_t count, int64_t m, const int64_t* p,                 \
                                      const int64_t* l, const S* pj, const S* lj, const S* r, S delta)      \
    {                                                                                                       \
        return addObservationsImpl(static_cast<RefNe<S>*>(ne), count, m, p, l, pj, lj, r, delta);           \
    }                                                                                                       \
    int ref_ne_merge_##SFX(void* target, const void* source)                                                \
    {                                                                                                       \
        return guarded([&] {                                                                                \
            static_cast<RefNe<S>*>(target)->equations.mergeFrom(                                            \
                static_cast<const RefNe<S>*>(source)->equations);                                           \
        });                                                                                                 \
    }                                                                                                       \
    void ref_ne_counts_##SFX(const void* ne, int64_t* cross_count, int64_t* pc_count)                       \
    {                                                                                                       \
        const auto& eq = static_cast<const RefNe<S>*>(ne)->equations;                                       \
        *cross_count = static_cast<int64_t>(eq._crossBlocks.size());                                        \
        *pc_count = static_cast<int64_t>(eq._primaryCrossBlocks.size());                                    \
    }                                                                                                       \
    void ref_ne_export_##SFX(const void* ne, S* hpp, S* hll, S* gp, S* gl, int64_t* ao, int64_t* cp, S* cv, \
                             int64_t* pr, int64_t* pcn, S* pv)                                              \
    {                                                                                                       \
        exportImpl(static_cast<const RefNe<S>*>(ne), hpp, hll, gp, gl, ao, cp, cv, pr, pcn, pv);            \
    }                                                                                                       \
    int ref_schur_solve_##SFX(void* ne, S damping, const SchurOptionsC* o, S* dp, S* dl, SchurReportC* r)   \
    {                                                                                                       \
        return schurSolveImpl(static_cast<RefNe<S>*>(ne), damping, o, dp, dl, r);                           \
    }                                                                                                       \
    int ref_schur_system_##SFX(void* ne, S damping, S min_diag, int64_t* nnz, int64_t* ro, int64_t* ci,     \
                               S* v, S* rhs)                                                                \
    {                                                                                                       \
        return schurSystemImpl(static_cast<RefNe<S>*>(ne), damping, min_diag, nnz, ro, ci, v, rhs);         \
    }

REF_NE_API(float, f32)
REF_NE_API(double, f64)

} // extern "C"
