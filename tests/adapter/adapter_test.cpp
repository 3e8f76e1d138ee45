// The C++ drop-in (include/plamatrix_b200_adapter.hpp) against the reference library itself
// (TEST INFRASTRUCTURE: built by oracle/Makefile's `adapter` target with the reference's own CPU
// sources, run by tests/test_adapter_gpu.py on a GPU).
//
// Every case builds its input through the reference's own types and functions, runs the
// reference's CPU implementation and the adapter's device implementation, and compares:
//   - solveDampedSchurComplement on BlockNormalEquations<double / float> filled by the reference's
//     addResidualBlock with Huber weights from evaluateHuberLoss (P=20, L=2,000, 4 distinct
//     primaries per eliminated block): steps within 1e-6 (double) / 1e-4 (float) of the
//     reference's Cpu backend; pattern reuse on the second call; the report fields;
//   - cooToCsr of duplicated, shuffled triplets: bit for bit the reference's CPU conversion;
//     an out-of-range coordinate throws std::out_of_range in both;
//   - blockPcg on a 2-D Laplacian with Jacobi and 2x2 inverse blocks against the reference's CPU
//     Jacobi pcg.
// Prints one PASS / FAIL line per check and "ADAPTER OK" when all passed; exit status 0 / 1.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "plamatrix/optimization/block_schur.h"
#include "plamatrix/optimization/robust_loss.h"
#include "plamatrix/sparse/iterative_solver.h"
#include "plamatrix/sparse/sparse_ops.h"
#include "plamatrix_b200_adapter.hpp"

using plamatrix::Index;

namespace
{
int g_failures = 0;

void expect(bool ok, const std::string& what)
{
    std::printf("%s %s\n", ok ? "PASS" : "FAIL", what.c_str());
    if (!ok)
        ++g_failures;
}

template <typename S>
double rel_diff(const std::vector<S>& a, const std::vector<S>& b)
{
    double num = 0.0, den = 0.0;
    for (std::size_t i = 0; i < a.size() && i < b.size(); ++i)
    {
        num += (double(a[i]) - double(b[i])) * (double(a[i]) - double(b[i]));
        den += double(b[i]) * double(b[i]);
    }
    return a.size() == b.size() ? std::sqrt(num / (den > 0 ? den : 1.0)) : 1e300;
}

// P primaries, L eliminated blocks, 4 distinct uniform primaries each, 2-row residuals:
// Jacobians N(0,1), residuals N(0, 0.5^2) with 5% N(0, 20^2), Huber delta 1
template <typename S>
plamatrix::BlockNormalEquations<S> bundle(Index P, Index L, unsigned seed)
{
    plamatrix::BlockNormalEquations<S> eq(P, L, 6, 3);
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> normal(0.0, 1.0);
    std::uniform_real_distribution<double> unit(0.0, 1.0);
    std::uniform_int_distribution<Index> pick(0, P - 1);
    for (Index l = 0; l < L; ++l)
    {
        std::vector<Index> prim;
        while (prim.size() < 4)
        {
            const Index p = pick(rng);
            bool seen = false;
            for (Index q : prim)
                seen = seen || q == p;
            if (!seen)
                prim.push_back(p);
        }
        for (Index p : prim)
        {
            S jp[12], jl[6], r[2];
            for (S& v : jp)
                v = S(normal(rng));
            for (S& v : jl)
                v = S(normal(rng));
            const double scale = unit(rng) < 0.05 ? 20.0 : 0.5;
            r[0] = S(normal(rng) * scale);
            r[1] = S(normal(rng) * scale);
            const auto loss = plamatrix::evaluateHuberLoss<S>(r[0] * r[0] + r[1] * r[1], S(1));
            eq.addResidualBlock(p, l, jp, jl, r, 2, loss.weight);
        }
    }
    return eq;
}

template <typename S>
void check_schur(const char* name, double tol, S relative_tolerance)
{
    const auto eq = bundle<S>(20, 2000, 7);
    plamatrix::SchurComplementSolverOptions<S> ref_opts;
    ref_opts.linearBackend = plamatrix::SchurComplementLinearBackend::Cpu;
    ref_opts.maxIterations = 500;
    ref_opts.relativeTolerance = relative_tolerance;
    plamatrix::SchurComplementSolverWorkspace<S> ref_ws;
    std::vector<S> dp_ref, dl_ref;
    const auto ref = plamatrix::solveDampedSchurComplement(eq, S(1e-3), ref_opts, ref_ws, &dp_ref, &dl_ref);

    auto opts = ref_opts;
    opts.linearBackend = plamatrix::SchurComplementLinearBackend::Cuda;
    plamatrix_b200::SchurComplementSolverWorkspace ws;
    std::vector<S> dp, dl;
    const auto got = plamatrix_b200::solveDampedSchurComplement(eq, S(1e-3), opts, ws, &dp, &dl);
    const std::string n = name;
    expect(ref.converged && got.converged, n + ": both converged (" + got.message + ")");
    expect(got.message == "converged", n + ": report message");
    expect(std::abs(got.iterations - ref.iterations) <= 2,
           n + ": iterations " + std::to_string(got.iterations) + " vs " + std::to_string(ref.iterations));
    expect(rel_diff(dp, dp_ref) <= tol, n + ": primary step within tolerance of the reference");
    expect(rel_diff(dl, dl_ref) <= tol, n + ": eliminated step within tolerance of the reference");
    expect(got.schurAssemblyOnDevice && !got.schurPatternReused && !got.deviceName.empty(),
           n + ": first call builds the pattern on the device (" + got.deviceName + ")");
    std::vector<S> dp2, dl2;
    const auto again = plamatrix_b200::solveDampedSchurComplement(eq, S(1e-3), opts, ws, &dp2, &dl2);
    expect(again.converged && again.schurPatternReused && ws.patternBuildCount() == 1,
           n + ": second call reuses the pattern");
    expect(dp2 == dp && dl2 == dl, n + ": repeated solve is bitwise identical");
    // invalid options throw as the reference does
    auto bad = opts;
    bad.maxIterations = 0;
    bool threw = false;
    try
    {
        plamatrix_b200::solveDampedSchurComplement(eq, S(1e-3), bad, ws, &dp2, &dl2);
    }
    catch (const std::invalid_argument&)
    {
        threw = true;
    }
    expect(threw, n + ": invalid options throw std::invalid_argument");
}

template <typename S>
void check_coo(const char* name)
{
    std::mt19937_64 rng(11);
    const Index rows = 3000, cols = 500, count = 40000;
    std::uniform_int_distribution<Index> r_of(0, rows - 1), c_of(0, cols - 1), e_of(-4, 8);
    std::normal_distribution<double> normal(0.0, 1.0);
    std::vector<Index> r(count), c(count);
    std::vector<S> v(count);
    for (Index k = 0; k < count; ++k)
    {
        r[k] = k < count / 8 ? r_of(rng) % 3 : r_of(rng); // a few long rows, many duplicates
        c[k] = c_of(rng);
        v[k] = S(normal(rng) * std::pow(10.0, double(e_of(rng))));
    }
    const auto ref = plamatrix::cooToCsr<S>(rows, cols, r, c, v);
    const auto got = plamatrix_b200::cooToCsr<S>(rows, cols, r, c, v);
    const std::string n = name;
    bool same = ref.nnz() == got.nnz() && ref.rows() == got.rows();
    same = same && std::memcmp(ref.rowOffsets(), got.rowOffsets(), sizeof(Index) * (rows + 1)) == 0;
    same = same && std::memcmp(ref.colIndices(), got.colIndices(), sizeof(Index) * ref.nnz()) == 0;
    same = same && std::memcmp(ref.values(), got.values(), sizeof(S) * ref.nnz()) == 0;
    expect(same, n + ": cooToCsr bit for bit the reference (nnz " + std::to_string(got.nnz()) + ")");
    auto bad_r = r;
    bad_r[17] = rows; // out of range
    bool ref_threw = false, got_threw = false;
    try
    {
        plamatrix::cooToCsr<S>(rows, cols, bad_r, c, v);
    }
    catch (const std::out_of_range&)
    {
        ref_threw = true;
    }
    try
    {
        plamatrix_b200::cooToCsr<S>(rows, cols, bad_r, c, v);
    }
    catch (const std::out_of_range&)
    {
        got_threw = true;
    }
    expect(ref_threw && got_threw, n + ": out-of-range coordinate throws std::out_of_range in both");
}

template <typename S>
void check_block_pcg(const char* name, double tol)
{
    // 2-D 5-point Laplacian on a 64 x 64 grid plus a 1e-2 shift
    const Index g = 64, n = g * g;
    std::vector<Index> r, c;
    std::vector<S> v;
    for (Index i = 0; i < g; ++i)
        for (Index j = 0; j < g; ++j)
        {
            const Index row = i * g + j;
            r.push_back(row), c.push_back(row), v.push_back(S(4.01));
            if (i > 0)
                r.push_back(row), c.push_back(row - g), v.push_back(S(-1));
            if (i + 1 < g)
                r.push_back(row), c.push_back(row + g), v.push_back(S(-1));
            if (j > 0)
                r.push_back(row), c.push_back(row - 1), v.push_back(S(-1));
            if (j + 1 < g)
                r.push_back(row), c.push_back(row + 1), v.push_back(S(-1));
        }
    const auto A = plamatrix::cooToCsr<S>(n, n, r, c, v);
    plamatrix::DenseMatrix<S, plamatrix::Device::CPU> b(n, 1), x_ref(n, 1), x(n, 1);
    std::mt19937_64 rng(5);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    for (Index k = 0; k < n; ++k)
    {
        b.data()[k] = S(u(rng));
        x_ref.data()[k] = S(0);
    }
    plamatrix::IterativeSolverOptions opts;
    opts.relativeTolerance = 1e-8;
    opts.maxIterations = 2000;
    const auto ref = plamatrix::pcg(A, b, x_ref, opts);
    const std::string name_s = name;
    // block size 1: the Jacobi inverse diagonal
    plamatrix::DenseMatrix<S, plamatrix::Device::CPU> inv1(n, 1);
    for (Index k = 0; k < n; ++k)
        inv1.data()[k] = S(1) / S(4.01);
    for (Index k = 0; k < n; ++k)
        x.data()[k] = S(0);
    const auto got = plamatrix_b200::blockPcg(A, b, x, inv1, 1, opts);
    std::vector<S> xs(x.data(), x.data() + n), xr(x_ref.data(), x_ref.data() + n);
    expect(ref.converged && got.converged && std::abs(got.iterations - ref.iterations) <= 2,
           name_s + ": blockPcg (1x1 blocks) converged, iterations " + std::to_string(got.iterations) + " vs " +
               std::to_string(ref.iterations));
    expect(rel_diff(xs, xr) <= tol, name_s + ": blockPcg (1x1 blocks) solution within tolerance of pcg");
    // block size 2: exact inverses of the 2x2 diagonal blocks (rows 2k and 2k + 1 are horizontal
    // neighbours in one grid row, g being even: the block is [[4.01, -1], [-1, 4.01]])
    plamatrix::DenseMatrix<S, plamatrix::Device::CPU> inv2(n * 2, 1);
    for (Index blk = 0; blk < n / 2; ++blk)
    {
        const double a = 4.01, off = -1.0;
        const double det = a * a - off * off;
        S* m = inv2.data() + blk * 4;
        m[0] = S(a / det), m[1] = S(-off / det), m[2] = S(-off / det), m[3] = S(a / det);
    }
    for (Index k = 0; k < n; ++k)
        x.data()[k] = S(0);
    const auto got2 = plamatrix_b200::blockPcg(A, b, x, inv2, 2, opts);
    std::vector<S> xs2(x.data(), x.data() + n);
    expect(got2.converged, name_s + ": blockPcg (2x2 blocks) converged in " + std::to_string(got2.iterations));
    expect(rel_diff(xs2, xr) <= tol, name_s + ": blockPcg (2x2 blocks) solution within tolerance of pcg");
}
} // namespace

int main()
{
    try
    {
        check_schur<double>("schur<double>", 1e-6, 1e-10);
        check_schur<float>("schur<float>", 1e-4, 1e-5f);
        check_coo<double>("coo<double>");
        check_coo<float>("coo<float>");
        check_block_pcg<double>("pcg<double>", 1e-6);
        check_block_pcg<float>("pcg<float>", 1e-4);
    }
    catch (const std::exception& e)
    {
        std::printf("FAIL uncaught exception: %s\n", e.what());
        return 1;
    }
    if (g_failures == 0)
        std::printf("ADAPTER OK\n");
    return g_failures == 0 ? 0 : 1;
}
