/*
 * plamatrix_b200_adapter.hpp -- header-only C++ drop-in that puts the reference's own types on
 * the plamatrix_b200 C ABI (include/plamatrix_b200.h, libplamatrix_b200.so).
 *
 * Include it after (or instead of) the reference headers it needs:
 *   plamatrix/optimization/block_schur.h, plamatrix/sparse/sparse_ops.h,
 *   plamatrix/sparse/iterative_solver.h
 * It works with the reference built with or without CUDA: device memory and copies go through
 * the library (pm_device_malloc / pm_copy_*), so this header never includes the CUDA runtime.
 *
 * What it provides, in namespace plamatrix_b200 (same argument meaning, same exceptions as the
 * reference functions it stands in for):
 *   - solveDampedSchurComplement(equations, damping, options, workspace, primary_step,
 *     eliminated_step) for plamatrix::BlockNormalEquations<S>: the Cuda backend of the
 *     reference's include/plamatrix/optimization/block_schur.h:171-186 (src/optimization/
 *     block_schur.cpp:54-459), with plamatrix_b200::SchurComplementSolverWorkspace as the
 *     reusable pattern cache (block_schur.h:81-169, patternBuildCount()).
 *   - cooToCsr(rows, cols, row_indices, col_indices, values) -> plamatrix::CSRMatrix<S, CPU>
 *     (sparse_ops.h:80-99), converted on the device, bit for bit the reference's result.
 *   - SparseOpsWorkspace + cooToCsrAsync on device triplets + checkStatus(operation)
 *     (sparse_ops.h:17-77, 108-120): the deferred status contract of the reference.
 *   - blockPcg(matrix, rhs, solution, inverse_blocks, block_size, options) on CPU-resident
 *     reference matrices, solved on the device (iterative_solver.h:130-141).
 *
 * Status codes of the C ABI become the reference's exception classes (invalid_argument,
 * out_of_range, runtime_error, logic_error, overflow_error).
 */
#ifndef PLAMATRIX_B200_ADAPTER_HPP
#define PLAMATRIX_B200_ADAPTER_HPP

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "plamatrix/optimization/block_schur.h"
#include "plamatrix/sparse/iterative_solver.h"
#include "plamatrix/sparse/sparse_ops.h"
#include "plamatrix_b200.h"

namespace plamatrix_b200
{

using plamatrix::Index;

// ------------------------------------------------------------------ errors
[[noreturn]] inline void raise(int status)
{
    const std::string message = pm_last_error();
    switch (status)
    {
    case PM_INVALID_ARGUMENT:
        throw std::invalid_argument(message);
    case PM_OUT_OF_RANGE:
        throw std::out_of_range(message);
    case PM_LOGIC_ERROR:
        throw std::logic_error(message);
    case PM_OVERFLOW_ERROR:
        throw std::overflow_error(message);
    default:
        throw std::runtime_error(message);
    }
}

inline void check(int status)
{
    if (status != PM_OK)
        raise(status);
}

template <typename S>
constexpr char suffix_check()
{
    static_assert(std::is_same_v<S, float> || std::is_same_v<S, double>, "float or double scalars");
    return 0;
}

// ------------------------------------------------------------------ device memory (library-owned)
class DeviceBuffer
{
public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(std::size_t bytes) { resize(bytes); }
    ~DeviceBuffer() { pm_device_free(_ptr); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : _ptr(std::exchange(o._ptr, nullptr)), _bytes(std::exchange(o._bytes, 0)) {}
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept
    {
        std::swap(_ptr, o._ptr);
        std::swap(_bytes, o._bytes);
        return *this;
    }
    /// grow-only
    void resize(std::size_t bytes)
    {
        if (bytes <= _bytes)
            return;
        check(pm_device_free(_ptr));
        _ptr = nullptr;
        _bytes = 0;
        check(pm_device_malloc(bytes, &_ptr));
        _bytes = bytes;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(_ptr); }
    template <typename T>
    void upload(const T* host, std::size_t count, pm_stream_t stream = nullptr)
    {
        resize(count * sizeof(T));
        check(pm_copy_to_device(_ptr, host, count * sizeof(T), stream));
    }
    template <typename T>
    void download(T* host, std::size_t count, pm_stream_t stream = nullptr) const
    {
        check(pm_copy_to_host(host, _ptr, count * sizeof(T), stream));
    }

private:
    void* _ptr = nullptr;
    std::size_t _bytes = 0;
};

// ------------------------------------------------------------------ BlockNormalEquations state
/// The accumulated state of a plamatrix::BlockNormalEquations<S>, flattened for the device: the
/// cross blocks of every eliminated block in the reference's _eliminatedAdjacency order.
template <typename S>
struct NormalEquationsView
{
    Index primaryBlockCount = 0, eliminatedBlockCount = 0, primaryBlockSize = 0, eliminatedBlockSize = 0;
    const S* primaryDiagonal = nullptr;
    const S* eliminatedDiagonal = nullptr;
    const S* primaryGradient = nullptr;
    const S* eliminatedGradient = nullptr;
    std::vector<std::int64_t> crossOffsets; // L + 1
    std::vector<std::int64_t> crossPrimary; // C
    std::vector<S> crossValues;             // C x bp x bl
    std::vector<std::int64_t> primaryCrossRow, primaryCrossColumn;
    std::vector<S> primaryCrossValues;      // PC x bp x bp
};

namespace detail
{
// Inside the reference, solveDampedSchurComplement is a friend of BlockNormalEquations and reads
// its members directly; that is where a maintainer builds the view (INTEGRATION.md shows the two
// lines).  Callers outside the reference reach the same members through explicit instantiation
// with member-pointer arguments, where the standard does not apply access checks
// ([temp.spec]: "the usual access checking rules do not apply to names used to specify explicit
// instantiations"); each tag's friend returns the member pointer.
template <typename Tag, auto Member>
struct Expose
{
    friend constexpr auto member_of(Tag) { return Member; }
};

#define PLAMATRIX_B200_TAG(NAME, S, FIELD)                                                                         \
    struct NAME                                                                                                    \
    {                                                                                                              \
        friend constexpr auto member_of(NAME);                                                                     \
    };                                                                                                             \
    template struct Expose<NAME, &plamatrix::BlockNormalEquations<S>::FIELD>;

#define PLAMATRIX_B200_TAGS(S, SFX)                                                                                \
    PLAMATRIX_B200_TAG(PrimaryCount##SFX, S, _primaryBlockCount)                                                   \
    PLAMATRIX_B200_TAG(EliminatedCount##SFX, S, _eliminatedBlockCount)                                             \
    PLAMATRIX_B200_TAG(PrimarySize##SFX, S, _primaryBlockSize)                                                     \
    PLAMATRIX_B200_TAG(EliminatedSize##SFX, S, _eliminatedBlockSize)                                               \
    PLAMATRIX_B200_TAG(PrimaryDiagonal##SFX, S, _primaryDiagonal)                                                  \
    PLAMATRIX_B200_TAG(EliminatedDiagonal##SFX, S, _eliminatedDiagonal)                                            \
    PLAMATRIX_B200_TAG(PrimaryGradient##SFX, S, _primaryGradient)                                                  \
    PLAMATRIX_B200_TAG(EliminatedGradient##SFX, S, _eliminatedGradient)                                            \
    PLAMATRIX_B200_TAG(PrimaryCross##SFX, S, _primaryCrossBlocks)                                                  \
    PLAMATRIX_B200_TAG(Cross##SFX, S, _crossBlocks)                                                                \
    PLAMATRIX_B200_TAG(Adjacency##SFX, S, _eliminatedAdjacency)

PLAMATRIX_B200_TAGS(double, D)
PLAMATRIX_B200_TAGS(float, F)
#undef PLAMATRIX_B200_TAGS
#undef PLAMATRIX_B200_TAG

template <typename S, typename PC, typename EC, typename PS, typename ES, typename PD, typename ED, typename PG,
          typename EG, typename PX, typename CX, typename AD>
NormalEquationsView<S> build_view(const plamatrix::BlockNormalEquations<S>& eq)
{
    NormalEquationsView<S> v;
    v.primaryBlockCount = eq.*member_of(PC{});
    v.eliminatedBlockCount = eq.*member_of(EC{});
    v.primaryBlockSize = eq.*member_of(PS{});
    v.eliminatedBlockSize = eq.*member_of(ES{});
    v.primaryDiagonal = (eq.*member_of(PD{})).data();
    v.eliminatedDiagonal = (eq.*member_of(ED{})).data();
    v.primaryGradient = (eq.*member_of(PG{})).data();
    v.eliminatedGradient = (eq.*member_of(EG{})).data();
    const auto& crosses = eq.*member_of(CX{});
    const auto& adjacency = eq.*member_of(AD{});
    const std::size_t block = static_cast<std::size_t>(v.primaryBlockSize * v.eliminatedBlockSize);
    v.crossOffsets.assign(1, 0);
    v.crossPrimary.reserve(crosses.size());
    v.crossValues.reserve(crosses.size() * block);
    for (const auto& list : adjacency)
    {
        for (const std::size_t index : list)
        {
            const auto& cross = crosses[index];
            v.crossPrimary.push_back(static_cast<std::int64_t>(cross.primaryBlock));
            v.crossValues.insert(v.crossValues.end(), cross.values.begin(), cross.values.end());
        }
        v.crossOffsets.push_back(static_cast<std::int64_t>(v.crossPrimary.size()));
    }
    for (const auto& pc : eq.*member_of(PX{}))
    {
        v.primaryCrossRow.push_back(static_cast<std::int64_t>(pc.rowBlock));
        v.primaryCrossColumn.push_back(static_cast<std::int64_t>(pc.columnBlock));
        v.primaryCrossValues.insert(v.primaryCrossValues.end(), pc.values.begin(), pc.values.end());
    }
    return v;
}
} // namespace detail

/// The state of a reference BlockNormalEquations, viewed for the device (copies the cross
/// blocks into adjacency order; the diagonal blocks and gradients are referenced in place).
inline NormalEquationsView<double> view_of(const plamatrix::BlockNormalEquations<double>& eq)
{
    using namespace detail;
    return build_view<double, PrimaryCountD, EliminatedCountD, PrimarySizeD, EliminatedSizeD, PrimaryDiagonalD,
                      EliminatedDiagonalD, PrimaryGradientD, EliminatedGradientD, PrimaryCrossD, CrossD, AdjacencyD>(
        eq);
}
inline NormalEquationsView<float> view_of(const plamatrix::BlockNormalEquations<float>& eq)
{
    using namespace detail;
    return build_view<float, PrimaryCountF, EliminatedCountF, PrimarySizeF, EliminatedSizeF, PrimaryDiagonalF,
                      EliminatedDiagonalF, PrimaryGradientF, EliminatedGradientF, PrimaryCrossF, CrossF, AdjacencyF>(eq);
}

// ------------------------------------------------------------------ damped Schur solve
/// SchurComplementSolverWorkspace of the device path: the reduced-system pattern cache and the
/// device copies of the normal equations and steps, reused across calls (move-only).
class SchurComplementSolverWorkspace
{
public:
    SchurComplementSolverWorkspace() { check(pm_schur_workspace_create(&_ws)); }
    ~SchurComplementSolverWorkspace()
    {
        if (_ne)
            pm_ne_destroy(_ne);
        if (_ws)
            pm_schur_workspace_destroy(_ws);
    }
    SchurComplementSolverWorkspace(const SchurComplementSolverWorkspace&) = delete;
    SchurComplementSolverWorkspace& operator=(const SchurComplementSolverWorkspace&) = delete;
    SchurComplementSolverWorkspace(SchurComplementSolverWorkspace&& o) noexcept
        : _ws(std::exchange(o._ws, nullptr)), _ne(std::exchange(o._ne, nullptr)), _steps(std::move(o._steps))
    {
        std::memcpy(_shape, o._shape, sizeof(_shape));
    }
    std::size_t patternBuildCount() const noexcept
    {
        return static_cast<std::size_t>(pm_schur_pattern_build_count(_ws));
    }
    pm_schur_workspace* handle() const noexcept { return _ws; }

    /// the device normal equations of shape (P, L, bp, bl, value size), recreated when it changes
    pm_normal_equations* equations(Index P, Index L, Index bp, Index bl, int value_size)
    {
        const std::int64_t shape[5] = {P, L, bp, bl, value_size};
        if (!_ne || std::memcmp(shape, _shape, sizeof(shape)) != 0)
        {
            if (_ne)
                pm_ne_destroy(_ne);
            _ne = nullptr;
            check(pm_ne_create(P, L, bp, bl, value_size, &_ne));
            std::memcpy(_shape, shape, sizeof(shape));
        }
        return _ne;
    }
    DeviceBuffer& steps() { return _steps; }

private:
    pm_schur_workspace* _ws = nullptr;
    pm_normal_equations* _ne = nullptr;
    std::int64_t _shape[5] = {};
    DeviceBuffer _steps;
};

/// Device path of solveDampedSchurComplement for an already flattened state (the function a
/// maintainer calls from the reference's Cuda backend branch).
template <typename S>
plamatrix::SchurComplementSolverReport<S> solveDampedSchurComplement(const NormalEquationsView<S>& eq, S damping,
                                                                     const plamatrix::SchurComplementSolverOptions<S>& options,
                                                                     SchurComplementSolverWorkspace& workspace,
                                                                     std::vector<S>* primary_step,
                                                                     std::vector<S>* eliminated_step)
{
    suffix_check<S>();
    constexpr bool dbl = std::is_same_v<S, double>;
    if (!primary_step || !eliminated_step || primary_step == eliminated_step)
        throw std::invalid_argument("solveDampedSchurComplement: output vectors must be non-null and distinct");
    const Index n = eq.primaryBlockCount * eq.primaryBlockSize;
    const Index m = eq.eliminatedBlockCount * eq.eliminatedBlockSize;
    const bool guess = options.useInitialGuess && primary_step->size() == static_cast<std::size_t>(n);
    if (!guess)
        primary_step->assign(static_cast<std::size_t>(n), S(0));
    eliminated_step->assign(static_cast<std::size_t>(m), S(0));

    pm_normal_equations* ne = workspace.equations(eq.primaryBlockCount, eq.eliminatedBlockCount,
                                                  eq.primaryBlockSize, eq.eliminatedBlockSize, sizeof(S));
    const std::int64_t C = static_cast<std::int64_t>(eq.crossPrimary.size());
    const std::int64_t PC = static_cast<std::int64_t>(eq.primaryCrossRow.size());
    if constexpr (dbl)
        check(pm_ne_upload_f64(ne, nullptr, eq.primaryDiagonal, eq.eliminatedDiagonal, eq.primaryGradient,
                               eq.eliminatedGradient, C, eq.crossOffsets.data(), eq.crossPrimary.data(),
                               eq.crossValues.data(), PC, eq.primaryCrossRow.data(), eq.primaryCrossColumn.data(),
                               eq.primaryCrossValues.data()));
    else
        check(pm_ne_upload_f32(ne, nullptr, eq.primaryDiagonal, eq.eliminatedDiagonal, eq.primaryGradient,
                               eq.eliminatedGradient, C, eq.crossOffsets.data(), eq.crossPrimary.data(),
                               eq.crossValues.data(), PC, eq.primaryCrossRow.data(), eq.primaryCrossColumn.data(),
                               eq.primaryCrossValues.data()));

    pm_schur_options o{};
    o.max_iterations = options.maxIterations;
    o.relative_tolerance = static_cast<double>(options.relativeTolerance);
    o.absolute_tolerance = static_cast<double>(options.absoluteTolerance);
    o.minimum_diagonal = static_cast<double>(options.minimumDiagonal);
    o.use_initial_guess = guess ? 1 : 0;
    o.precision = options.useMixedPrecision && dbl ? PM_PRECISION_MIXED : PM_PRECISION_NATIVE;
    // the Cpu backend's PCG stops at abs + rel * ||r0||; the Cuda backend's blockPcg at
    // max(abs, rel * ||r0||) (block_schur_cpu_solver.h:14-82, iterative_solver.cu:262-349)
    o.tolerance_rule = options.linearBackend == plamatrix::SchurComplementLinearBackend::Cpu ? 0 : 1;
    o.check_true_residual = 1;
    o.inner_relative_tolerance = 1e-4;
    o.max_refinements = 8;
    o.learned = nullptr;
    o.stagnation_window = 25;
    o.linear_backend =
        options.linearBackend == plamatrix::SchurComplementLinearBackend::DenseCpu ? PM_LINEAR_DENSE : PM_LINEAR_PCG;

    DeviceBuffer& steps = workspace.steps();
    steps.resize(static_cast<std::size_t>(n + m + 2) * sizeof(S));
    S* dp = steps.as<S>();
    S* dl = dp + n + 1;
    if (guess && n > 0)
        check(pm_copy_to_device(dp, primary_step->data(), static_cast<std::size_t>(n) * sizeof(S), nullptr));
    pm_schur_report r{};
    if constexpr (dbl)
        check(pm_schur_solve_f64(workspace.handle(), nullptr, ne, damping, &o, dp, dl, &r));
    else
        check(pm_schur_solve_f32(workspace.handle(), nullptr, ne, damping, &o, dp, dl, &r));
    if (n > 0)
        check(pm_copy_to_host(primary_step->data(), dp, static_cast<std::size_t>(n) * sizeof(S), nullptr));
    if (m > 0 && r.converged)
        check(pm_copy_to_host(eliminated_step->data(), dl, static_cast<std::size_t>(m) * sizeof(S), nullptr));

    plamatrix::SchurComplementSolverReport<S> report;
    report.linearBackend = options.linearBackend;
    report.converged = r.converged != 0;
    report.iterations = r.iterations;
    report.initialResidualNorm = static_cast<S>(r.initial_residual_norm);
    report.finalResidualNorm = static_cast<S>(r.final_residual_norm);
    report.smallBlockInverseSeconds = r.eliminated_inverse_ms * 1e-3;
    report.schurAccumulationSeconds = r.assembly_ms * 1e-3;
    report.csrConversionSeconds = r.pattern_ms * 1e-3;
    report.schurAssemblySeconds = (r.pattern_ms + r.assembly_ms) * 1e-3;
    report.linearSolveSeconds = r.solve_ms * 1e-3;
    report.backSubstitutionSeconds = r.back_substitution_ms * 1e-3;
    report.schurPatternReused = r.pattern_reused != 0;
    report.schurAssemblyOnDevice = true;
    report.mixedPrecisionUsed = r.mixed_precision_used != 0;
    char name[128] = {};
    if (pm_device_name(name, sizeof(name)) == PM_OK)
        report.deviceName = name;
    report.message = r.message;
    return report;
}

/// solveDampedSchurComplement(equations, ...) for the reference's own BlockNormalEquations.
template <typename S>
plamatrix::SchurComplementSolverReport<S> solveDampedSchurComplement(const plamatrix::BlockNormalEquations<S>& equations,
                                                                     S damping,
                                                                     const plamatrix::SchurComplementSolverOptions<S>& options,
                                                                     SchurComplementSolverWorkspace& workspace,
                                                                     std::vector<S>* primary_step,
                                                                     std::vector<S>* eliminated_step)
{
    return solveDampedSchurComplement(view_of(equations), damping, options, workspace, primary_step,
                                      eliminated_step);
}

// ------------------------------------------------------------------ COO -> CSR
/// SparseOpsWorkspace of the device path (move-only, grow-only, bound to its first stream, with
/// the deferred status of cooToCsrAsync).
class SparseOpsWorkspace
{
public:
    SparseOpsWorkspace() { check(pm_sparse_workspace_create(&_ws)); }
    ~SparseOpsWorkspace()
    {
        if (_ws)
            pm_sparse_workspace_destroy(_ws);
    }
    SparseOpsWorkspace(const SparseOpsWorkspace&) = delete;
    SparseOpsWorkspace& operator=(const SparseOpsWorkspace&) = delete;
    SparseOpsWorkspace(SparseOpsWorkspace&& o) noexcept : _ws(std::exchange(o._ws, nullptr)) {}
    /// SparseOpsWorkspace::checkStatus (src/sparse/coo_to_csr.cu:531-534): throws the deferred error;
    /// the caller synchronises the stream first, as with the reference
    void checkStatus(const char* operation) { check(pm_coo_status(_ws, operation, nullptr)); }
    std::int64_t combinedNnz(const char* operation)
    {
        std::int64_t nnz = 0;
        check(pm_coo_status(_ws, operation, &nnz));
        return nnz;
    }
    void closeAsyncAllocation() { check(pm_sparse_workspace_close(_ws)); }
    std::size_t capacityBytes() const noexcept { return pm_sparse_workspace_capacity(_ws); }
    pm_sparse_workspace* handle() const noexcept { return _ws; }

private:
    pm_sparse_workspace* _ws = nullptr;
};

/// cooToCsrAsync on device triplets into a preallocated device CSR of exactly `nnz` entries.
/// Synchronize `stream`, then call workspace.checkStatus() before consuming the output.
template <typename S>
void cooToCsrAsync(Index rows, Index cols, Index count, const Index* row_indices_d, const Index* col_indices_d,
                   const S* values_d, Index nnz, Index* row_offsets_d, Index* col_indices_out_d, S* values_out_d,
                   SparseOpsWorkspace& workspace, pm_stream_t stream = nullptr)
{
    suffix_check<S>();
    if constexpr (std::is_same_v<S, double>)
        check(pm_coo_to_csr_async_f64(workspace.handle(), stream, rows, cols, count, row_indices_d, col_indices_d,
                                      values_d, nnz, row_offsets_d, col_indices_out_d, values_out_d));
    else
        check(pm_coo_to_csr_async_f32(workspace.handle(), stream, rows, cols, count, row_indices_d, col_indices_d,
                                      values_d, nnz, row_offsets_d, col_indices_out_d, values_out_d));
}

/// cooToCsr of host triplets (sparse_ops.h:80-86) converted on the device: sorted by (row, col),
/// duplicates combined in input order, bit for bit the reference's CPU conversion.
template <typename S>
plamatrix::CSRMatrix<S, plamatrix::Device::CPU> cooToCsr(Index rows, Index cols,
                                                         const std::vector<Index>& row_indices,
                                                         const std::vector<Index>& col_indices,
                                                         const std::vector<S>& values)
{
    suffix_check<S>();
    if (row_indices.size() != col_indices.size() || row_indices.size() != values.size())
        throw std::invalid_argument("cooToCsr: COO arrays must have the same length");
    const Index count = static_cast<Index>(values.size());
    DeviceBuffer r, c, v;
    r.upload(row_indices.data(), row_indices.size());
    c.upload(col_indices.data(), col_indices.size());
    v.upload(values.data(), values.size());
    SparseOpsWorkspace ws;
    if constexpr (std::is_same_v<S, double>)
        check(pm_coo_to_csr_count_f64(ws.handle(), nullptr, rows, cols, count, r.as<Index>(), c.as<Index>(),
                                      v.as<S>()));
    else
        check(pm_coo_to_csr_count_f32(ws.handle(), nullptr, rows, cols, count, r.as<Index>(), c.as<Index>(),
                                      v.as<S>()));
    check(pm_stream_synchronize(nullptr));
    const Index nnz = ws.combinedNnz("cooToCsr");
    DeviceBuffer ro(static_cast<std::size_t>(rows + 1) * sizeof(Index)),
        co(static_cast<std::size_t>(nnz + 1) * sizeof(Index)), vo(static_cast<std::size_t>(nnz + 1) * sizeof(S));
    if constexpr (std::is_same_v<S, double>)
        check(pm_coo_to_csr_fill_f64(ws.handle(), nullptr, nnz, ro.as<Index>(), co.as<Index>(), vo.as<S>()));
    else
        check(pm_coo_to_csr_fill_f32(ws.handle(), nullptr, nnz, ro.as<Index>(), co.as<Index>(), vo.as<S>()));
    check(pm_stream_synchronize(nullptr));
    ws.checkStatus("cooToCsr");
    plamatrix::CSRMatrix<S, plamatrix::Device::CPU> out(rows, cols, nnz);
    ro.download(out.rowOffsets(), static_cast<std::size_t>(rows + 1));
    if (nnz > 0)
    {
        co.download(out.colIndices(), static_cast<std::size_t>(nnz));
        vo.download(out.values(), static_cast<std::size_t>(nnz));
    }
    return out;
}

// ------------------------------------------------------------------ block-Jacobi PCG
/// blockPcg with caller-supplied row-major inverse diagonal blocks ((rows * block_size) x 1), for
/// a CPU-resident reference CSR matrix and vectors, solved on the device; `solution` is the
/// initial guess on entry (iterative_solver.h:130-141, src/sparse/iterative_solver.cu:386-402).
template <typename S>
plamatrix::IterativeSolverReport blockPcg(const plamatrix::CSRMatrix<S, plamatrix::Device::CPU>& matrix,
                                          const plamatrix::DenseMatrix<S, plamatrix::Device::CPU>& rhs,
                                          plamatrix::DenseMatrix<S, plamatrix::Device::CPU>& solution,
                                          const plamatrix::DenseMatrix<S, plamatrix::Device::CPU>& inverse_blocks,
                                          Index block_size, const plamatrix::IterativeSolverOptions& options = {})
{
    suffix_check<S>();
    constexpr bool dbl = std::is_same_v<S, double>;
    const Index n = matrix.rows(), nnz = matrix.nnz();
    if (rhs.size() != n || solution.size() != n)
        throw std::invalid_argument("blockPcg: vector sizes must match the matrix");
    DeviceBuffer ro, ci, v, b, x, inv;
    ro.upload(matrix.rowOffsets(), static_cast<std::size_t>(n + 1));
    ci.upload(matrix.colIndices(), static_cast<std::size_t>(nnz));
    v.upload(matrix.values(), static_cast<std::size_t>(nnz));
    b.upload(rhs.data(), static_cast<std::size_t>(n));
    x.upload(solution.data(), static_cast<std::size_t>(n));
    inv.upload(inverse_blocks.data(), static_cast<std::size_t>(inverse_blocks.size()));
    pm_csr* A = nullptr;
    if constexpr (dbl)
        check(pm_csr_create_f64(nullptr, n, matrix.cols(), nnz, ro.as<Index>(), ci.as<Index>(), v.as<S>(), &A));
    else
        check(pm_csr_create_f32(nullptr, n, matrix.cols(), nnz, ro.as<Index>(), ci.as<Index>(), v.as<S>(), &A));
    pm_solver_workspace* ws = nullptr;
    int status = pm_solver_workspace_create(&ws);
    pm_solver_report r{};
    if (status == PM_OK)
    {
        pm_solver_options o{options.maxIterations, options.relativeTolerance, options.absoluteTolerance,
                            options.useJacobiPreconditioner ? 1 : 0, options.requireConvergence ? 1 : 0};
        if constexpr (dbl)
            status = pm_block_pcg_f64(ws, nullptr, A, b.as<S>(), x.as<S>(), inv.as<S>(), block_size, &o, &r);
        else
            status = pm_block_pcg_f32(ws, nullptr, A, b.as<S>(), x.as<S>(), inv.as<S>(), block_size, &o, &r);
    }
    std::string message = status == PM_OK ? std::string() : std::string(pm_last_error());
    pm_solver_workspace_destroy(ws);
    pm_csr_destroy(A);
    if (status != PM_OK)
    {
        // rethrow with the solver's message (the frees above may have reset the last error)
        switch (status)
        {
        case PM_INVALID_ARGUMENT:
            throw std::invalid_argument(message);
        case PM_OUT_OF_RANGE:
            throw std::out_of_range(message);
        case PM_LOGIC_ERROR:
            throw std::logic_error(message);
        default:
            throw std::runtime_error(message);
        }
    }
    x.download(solution.data(), static_cast<std::size_t>(n));
    plamatrix::IterativeSolverReport report;
    report.converged = r.converged != 0;
    report.iterations = r.iterations;
    report.initialResidual = r.initial_residual;
    report.finalResidual = r.final_residual;
    return report;
}

} // namespace plamatrix_b200

#endif // PLAMATRIX_B200_ADAPTER_HPP
