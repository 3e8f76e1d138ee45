// Device-resident two-block normal equations (the state of the reference's
// BlockNormalEquations, include/plamatrix/optimization/block_schur.h:196-319) and the
// pieces shared by the accumulation and Schur-solver translation units.
#pragma once

#include "pm_common.cuh"

struct pm_normal_equations
{
    int64_t P = 0, L = 0, bp = 0, bl = 0;
    int value_size = 8;
    int64_t cross_count = 0;         // C: distinct (primary, eliminated) pairs
    int64_t primary_cross_count = 0; // PC: upper-triangular primary-primary blocks
    // numeric state (Scalar)
    pm::DeviceBuffer numeric;
    void* primary_diagonal = nullptr;    // P * bp * bp, row-major blocks
    void* eliminated_diagonal = nullptr; // L * bl * bl
    void* primary_gradient = nullptr;    // P * bp
    void* eliminated_gradient = nullptr; // L * bl
    void* cross_values = nullptr;        // C * bp * bl, grouped by eliminated block
    void* primary_cross_values = nullptr; // PC * bp * bp
    // topology (int32)
    pm::DeviceBuffer topology;
    int* cross_offsets = nullptr; // L + 1: crosses of eliminated l are [off[l], off[l+1])
    int* cross_primary = nullptr; // C
    int* cross_eliminated = nullptr; // C
    int* primary_cross_row = nullptr; // PC (row < col)
    int* primary_cross_col = nullptr; // PC
    int64_t topology_version = 0;     // bumped whenever the topology arrays change
    bool crosses_sorted = false;      // crosses of every eliminated block in ascending primary order
    // observation-path topology cache
    pm_sparse_workspace* by_eliminated = nullptr; // observations bucketed by eliminated block
    pm_sparse_workspace* by_primary = nullptr;    // observations bucketed by primary block
    pm_sparse_workspace* by_eliminated_order = nullptr; // observations bucketed by eliminated block, input order
    pm::DeviceBuffer cross_runs;                  // C + 1: first by_eliminated position of every cross
    pm::DeviceBuffer observation_slots;           // N: cross of every by_eliminated_order position (~c: not its first)
    pm::DeviceBuffer observation_copy;            // saved index arrays + zero column
    pm::DeviceBuffer weights;                     // Huber weight of every observation
    pm::DeviceBuffer observation_status;          // long long: first observation with a non-finite squared norm
    int64_t observation_count = -1;
    int64_t residual_size = 0;
    bool observation_topology = false;
    ~pm_normal_equations();
};

namespace pm
{

template <typename T>
__device__ __forceinline__ T mul_rn(T a, T b);
template <>
__device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <>
__device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }
template <typename T>
__device__ __forceinline__ T add_rn(T a, T b);
template <>
__device__ __forceinline__ float add_rn<float>(float a, float b) { return __fadd_rn(a, b); }
template <>
__device__ __forceinline__ double add_rn<double>(double a, double b) { return __dadd_rn(a, b); }

// Cholesky-based SPD inverse in FP64 (the arithmetic of invertPositiveDefiniteInto,
// src/optimization/block_schur_linear_algebra.h:91-147).  `lower` and `work` are scratch.
template <int N>
__device__ __forceinline__ bool spd_inverse(const double* m, int n, double* inv, double* lower, double* work)
{
    for (int i = 0; i < n * n; ++i)
        lower[i] = 0.0;
    for (int row = 0; row < n; ++row)
    {
        for (int col = 0; col <= row; ++col)
        {
            double value = m[row * n + col];
            for (int k = 0; k < col; ++k)
                value = __dadd_rn(value, -__dmul_rn(lower[row * n + k], lower[col * n + k]));
            if (row == col)
            {
                if (!(value > 0.0) || !isfinite(value))
                    return false;
                lower[row * n + col] = sqrt(value);
            }
            else
            {
                lower[row * n + col] = value / lower[col * n + col];
            }
        }
    }
    for (int i = 0; i < n * n; ++i)
        inv[i] = 0.0;
    for (int col = 0; col < n; ++col)
    {
        for (int row = 0; row < n; ++row)
        {
            double value = row == col ? 1.0 : 0.0;
            for (int k = 0; k < row; ++k)
                value = __dadd_rn(value, -__dmul_rn(lower[row * n + k], work[k]));
            work[row] = value / lower[row * n + row];
        }
        for (int off = 0; off < n; ++off)
        {
            const int row = n - 1 - off;
            double value = work[row];
            for (int k = row + 1; k < n; ++k)
                value = __dadd_rn(value, -__dmul_rn(lower[k * n + row], inv[k * n + col]));
            inv[row * n + col] = value / lower[row * n + row];
        }
    }
    return true;
}

// What the learned block-Jacobi correction reads from / writes into a Schur workspace.
struct SchurView
{
    int64_t P = 0, B = 0;
    int value_size = 0;
    bool mixed = false;             // minv32 must be refreshed too
    const int* block_row_ptr = nullptr;
    const int* block_col = nullptr;
    const int* diag_pos = nullptr;
    const void* S = nullptr;        // B x 36 values (value_size bytes each)
    double* minv = nullptr;         // P x 36 preconditioner blocks (FP64)
    float* minv32 = nullptr;        // P x 36, mixed precision only
};
SchurView schur_view(pm_schur_workspace* ws, bool mixed);
// dense FP64 Cholesky of the n = P bp reduced system in block CSR: A (n x n scratch) and x (the
// right-hand side in, the solution out); *status (device) = 0, or 1 + the column of the first
// pivot that is not positive and finite
template <typename T>
void dense_schur_factor_solve(cudaStream_t stream, int64_t P, int bp, const int* row_ptr, const int* block_col,
                              const T* S, double* A, double* x, int* status);
// features -> network -> (L'L'^T)^-1 of every diagonal block into v.minv (and v.minv32); when the
// network's blocks are unusable the device puts plain block Jacobi back.  flags_host (pinned,
// two ints, may be null) receives {block not positive definite, GEMM gave up} asynchronously.
void mlp_apply(const pm_mlp* mlp, const SchurView& v, cudaStream_t stream, int* flags_host);

} // namespace pm
