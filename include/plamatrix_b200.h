/*
 * plamatrix_b200 -- C ABI of the B200 (sm_100a) implementation of PlaMatrix's
 * Levenberg-Marquardt normal-equation hot path.
 *
 * Conventions (shared by every entry point):
 *   - Every function returns an int status: PM_OK or one of the PM_* codes below, which
 *     map one-to-one onto the reference's exception classes.  pm_last_error() returns the
 *     message of the last failure on the calling thread.
 *   - Pointers named *_d are device pointers; host arrays are named *_h.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Work is enqueued on it;
 *     functions documented as "synchronous" wait for it before returning.
 *   - Workspaces are caller-owned, move-only in spirit, not thread-safe, and bound to the
 *     first stream they are used with until *_close() (the reference's ownership rule).
 *   - Index arrays that cross this boundary are int64 (the reference's Index) unless
 *     a function says otherwise.
 *
 * Each declaration names the reference interface it replaces (paths inside the reference
 * project).
 */
#ifndef PLAMATRIX_B200_H
#define PLAMATRIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PM_API __attribute__((visibility("default")))
#else
#define PM_API
#endif

typedef struct CUstream_st* pm_stream_t; /* identical to cudaStream_t */

enum
{
    PM_OK = 0,
    PM_INVALID_ARGUMENT = 1, /* std::invalid_argument */
    PM_OUT_OF_RANGE = 2,     /* std::out_of_range */
    PM_RUNTIME_ERROR = 3,    /* std::runtime_error */
    PM_LOGIC_ERROR = 4,      /* std::logic_error */
    PM_OVERFLOW_ERROR = 5,   /* std::overflow_error */
    PM_CUDA_ERROR = 6        /* CUDA runtime failure (std::runtime_error in the reference) */
};

/* Message of the last non-zero status returned on this thread. */
PM_API const char* pm_last_error(void);
/* ABI version of this library. */
PM_API int pm_version(void);
/* Number of kernels this library has launched in the process so far. */
PM_API long long pm_kernel_launches(void);

/* Device memory and synchronous copies (on `stream`) for callers that do not link the CUDA
 * runtime themselves, e.g. C++ code built against the reference's CPU-only headers.  No
 * counterpart in the reference (its DenseMatrix<GPU> / GpuAllocator own device memory there). */
PM_API int pm_device_malloc(size_t bytes, void** out);
PM_API int pm_device_free(void* ptr);
PM_API int pm_copy_to_device(void* dst_d, const void* src_h, size_t bytes, pm_stream_t stream);
PM_API int pm_copy_to_host(void* dst_h, const void* src_d, size_t bytes, pm_stream_t stream);
/* Wait for the work queued on `stream` (what a caller does before pm_coo_status). */
PM_API int pm_stream_synchronize(pm_stream_t stream);
/* Name of the current CUDA device (SchurComplementSolverReport::deviceName). */
PM_API int pm_device_name(char* out, int capacity);

/* =========================================================================== workspaces
 * Replaces SparseOpsWorkspace (include/plamatrix/sparse/sparse_ops.h:13-77): grow-only,
 * stream-bound temporary storage plus the deferred COO status. */
typedef struct pm_sparse_workspace pm_sparse_workspace;
PM_API int pm_sparse_workspace_create(pm_sparse_workspace** out);
/* Frees the workspace (stream-ordered on its bound stream). */
PM_API void pm_sparse_workspace_destroy(pm_sparse_workspace* workspace);
/* closeAsyncAllocation (sparse_ops.h:26): release storage, unbind the stream. */
PM_API int pm_sparse_workspace_close(pm_sparse_workspace* workspace);
PM_API size_t pm_sparse_workspace_capacity(const pm_sparse_workspace* workspace);

/* =========================================================================== COO -> CSR
 * Deterministic, bit-exact with the reference CPU conversion
 * (src/sparse/sparse_ops_cpu.cpp:24-134): entries sorted by (row, col) with ties kept in
 * input order; duplicates combined by taking the first value and adding the rest in input
 * order.  Inputs: `count` triplets (int64 rows/cols, scalar values) on the device; limits
 * of the reference GPU path (src/sparse/coo_to_csr.cu:78-104): count and rows < 2^31,
 * cols <= 2^32-1.  Coordinate and value errors are deferred to pm_coo_status().
 */
/* First half of the synchronous cooToCsr (src/sparse/coo_to_csr.cu:536-561): enqueue the
 * sort and the duplicate-combined count; after a stream sync pm_coo_status() returns the
 * nnz to allocate, and pm_coo_to_csr_fill_*() writes the CSR from the same sorted state. */
PM_API int pm_coo_to_csr_count_f32(pm_sparse_workspace* workspace, pm_stream_t stream, int64_t rows, int64_t cols,
                            int64_t count, const int64_t* row_indices_d, const int64_t* col_indices_d,
                            const float* values_d);
PM_API int pm_coo_to_csr_count_f64(pm_sparse_workspace* workspace, pm_stream_t stream, int64_t rows, int64_t cols,
                            int64_t count, const int64_t* row_indices_d, const int64_t* col_indices_d,
                            const double* values_d);
PM_API int pm_coo_to_csr_fill_f32(pm_sparse_workspace* workspace, pm_stream_t stream, int64_t nnz,
                           int64_t* row_offsets_d, int64_t* col_indices_out_d, float* values_out_d);
PM_API int pm_coo_to_csr_fill_f64(pm_sparse_workspace* workspace, pm_stream_t stream, int64_t nnz,
                           int64_t* row_offsets_d, int64_t* col_indices_out_d, double* values_out_d);
/* cooToCsrAsync (include/plamatrix/sparse/sparse_ops.h:108-120, src/sparse/coo_to_csr.cu:563-576):
 * full conversion into preallocated output holding exactly `nnz` entries; no host sync.
 * Synchronize the stream, then call pm_coo_status() before consuming the output. */
PM_API int pm_coo_to_csr_async_f32(pm_sparse_workspace* workspace, pm_stream_t stream, int64_t rows, int64_t cols,
                            int64_t count, const int64_t* row_indices_d, const int64_t* col_indices_d,
                            const float* values_d, int64_t nnz, int64_t* row_offsets_d,
                            int64_t* col_indices_out_d, float* values_out_d);
PM_API int pm_coo_to_csr_async_f64(pm_sparse_workspace* workspace, pm_stream_t stream, int64_t rows, int64_t cols,
                            int64_t count, const int64_t* row_indices_d, const int64_t* col_indices_d,
                            const double* values_d, int64_t nnz, int64_t* row_offsets_d,
                            int64_t* col_indices_out_d, double* values_out_d);
/* SparseOpsWorkspace::checkStatus (src/sparse/coo_to_csr.cu:300-365, 531-534): reads the
 * deferred status of the last conversion.  Returns PM_LOGIC_ERROR if the stream has not
 * finished, PM_OUT_OF_RANGE for a coordinate outside the matrix (lowest offending offset),
 * PM_INVALID_ARGUMENT for a non-finite value or combined sum, PM_RUNTIME_ERROR for an
 * output nnz that differs from the duplicate-combined nnz.  `nnz_out` (may be NULL)
 * receives the duplicate-combined nnz. */
PM_API int pm_coo_status(pm_sparse_workspace* workspace, const char* operation, int64_t* nnz_out);
/* Allocation-free COO -> CSR (no counterpart in the reference).  For callers that cannot
 * allocate device memory while they run -- a host application that fixes the device-memory
 * budget at start-up and owns every allocation, or a latency-critical loop where cudaMalloc
 * could block or fail mid-run.  Same result as pm_coo_to_csr_async_*; the scratch is one
 * file-scope device array of 8 MiB that every GPU loading this library holds until exit, so
 * inputs are limited to 65,536 triplets and 65,536 rows (larger inputs: PM_INVALID_ARGUMENT).
 * No cudaMalloc / cudaFree or allocating library call is made.  Synchronous: enqueues on
 * `stream`, waits, and reports coordinate / value errors directly.  The output arrays hold
 * `capacity` entries (capacity = count always suffices); `nnz_out` (host) receives the
 * duplicate-combined nnz.  All calls share the scratch array: calls that overlap on one GPU,
 * from any stream or host thread, race, so serialise them (each device has its own copy).
 * Every call looks up the array's device address (cudaGetSymbolAddress, which allocates
 * nothing); the first call on a device loads the library's device code there, so make that
 * first call before any stream capture. */
PM_API int pm_coo_to_csr_static_f32(pm_stream_t stream, int64_t rows, int64_t cols, int64_t count,
                                    const int64_t* row_indices_d, const int64_t* col_indices_d,
                                    const float* values_d, int64_t capacity, int64_t* row_offsets_d,
                                    int64_t* col_indices_out_d, float* values_out_d, int64_t* nnz_out);
PM_API int pm_coo_to_csr_static_f64(pm_stream_t stream, int64_t rows, int64_t cols, int64_t count,
                                    const int64_t* row_indices_d, const int64_t* col_indices_d,
                                    const double* values_d, int64_t capacity, int64_t* row_offsets_d,
                                    int64_t* col_indices_out_d, double* values_out_d, int64_t* nnz_out);

/* =========================================================================== CSR matrices
 * A validated CSR operand for the device SpMV and solvers.  Replaces the structure checks
 * of CSRMatrix<GPU>::validateStructure (include/plamatrix/sparse/csr_matrix.h:197-240) and
 * the cached cuSPARSE descriptors of SparseOpsWorkspace (src/sparse/sparse_ops.cu:192-231):
 * the int64 structure is validated once and kept as a compact int32 copy; the values
 * stay in the caller's array, which must outlive the handle.  Synchronous. */
typedef struct pm_csr pm_csr;
PM_API int pm_csr_create_f32(pm_stream_t stream, int64_t rows, int64_t cols, int64_t nnz, const int64_t* row_offsets_d,
                      const int64_t* col_indices_d, const float* values_d, pm_csr** out);
PM_API int pm_csr_create_f64(pm_stream_t stream, int64_t rows, int64_t cols, int64_t nnz, const int64_t* row_offsets_d,
                      const int64_t* col_indices_d, const double* values_d, pm_csr** out);
PM_API void pm_csr_destroy(pm_csr* matrix);
/* Point the handle at new values with the same structure (e.g. the next LM iteration). */
PM_API int pm_csr_set_values(pm_csr* matrix, const void* values_d);

/* spmvAsync (include/plamatrix/sparse/sparse_ops.h:158-165, src/sparse/sparse_ops.cu:687-740):
 * y = A x on `stream`, hand-written kernel (no cuSPARSE). */
PM_API int pm_csr_spmv_f32(const pm_csr* matrix, pm_stream_t stream, const float* x_d, float* y_d);
PM_API int pm_csr_spmv_f64(const pm_csr* matrix, pm_stream_t stream, const double* x_d, double* y_d);

/* No counterpart in the reference (its SpMV is cuSPARSE's): the SpMV shape of an operand.
 * kernel -1 = heuristic (mean row length), 0 = row-group stream (a warp per 32 rows), 1..32 =
 * lanes per row.  pm_csr_autotune_* times every shape on this operand with the caller's vectors
 * and stream (synchronous; overwrites y_d) and keeps the fastest; CG / PCG on the operand use the
 * same shape.  Shapes order a row's additions differently, so the choice is part of a result's
 * rounding; pm_csr_set_kernel pins one for reproducibility across processes. */
PM_API int pm_csr_autotune_f32(pm_csr* matrix, pm_stream_t stream, const float* x_d, float* y_d, int* kernel_h);
PM_API int pm_csr_autotune_f64(pm_csr* matrix, pm_stream_t stream, const double* x_d, double* y_d, int* kernel_h);
PM_API int pm_csr_set_kernel(pm_csr* matrix, int kernel);
PM_API int pm_csr_kernel(const pm_csr* matrix, int* kernel_h, int* heuristic_lanes_h);

/* output = A input for dense matrices in column-major order (leading dimension = rows):
 * input is input_rows x input_cols (input_rows == A's columns), output is output_rows x
 * output_cols (A's rows x input_cols).  Replaces spmmAsync (sparse_ops.cu:762-818; the CPU order
 * of sparse_ops_cpu.cpp:244-270): PM_RUNTIME_ERROR on a dimension mismatch,
 * PM_INVALID_ARGUMENT when input and output alias; an empty A writes zeros. */
PM_API int pm_csr_spmm_f32(const pm_csr* matrix, pm_stream_t stream, int64_t input_rows, int64_t input_cols,
                           const float* input_d, int64_t output_rows, int64_t output_cols, float* output_d);
PM_API int pm_csr_spmm_f64(const pm_csr* matrix, pm_stream_t stream, int64_t input_rows, int64_t input_cols,
                           const double* input_d, int64_t output_rows, int64_t output_cols, double* output_d);

/* =========================================================================== CG / PCG
 * Replaces cg / pcg / blockPcg on the GPU (include/plamatrix/sparse/iterative_solver.h:297-329,
 * src/sparse/iterative_solver.cu:262-402).  Dots, alpha and beta are evaluated in FP64 for
 * both scalar types; convergence is tested on the device (no per-iteration host sync):
 * tolerance max(absolute, relative * ||r0||) on the recurrence residual, as in the
 * reference.  Synchronous: returns after the solve (one host read at the end). */
typedef struct
{
    int max_iterations;        /* IterativeSolverOptions::maxIterations (1000) */
    double relative_tolerance; /* 1e-6, in [0, 1] */
    double absolute_tolerance; /* 0 */
    int use_jacobi;            /* useJacobiPreconditioner (1); pcg only */
    int require_convergence;   /* requireConvergence (0): PM_RUNTIME_ERROR when not converged */
} pm_solver_options;

typedef struct
{
    int converged;
    int iterations;
    double initial_residual;
    double final_residual;
} pm_solver_report;

/* Replaces IterativeSolverWorkspace<Scalar> (include/plamatrix/sparse/iterative_solver.h:216-251). */
typedef struct pm_solver_workspace pm_solver_workspace;
PM_API int pm_solver_workspace_create(pm_solver_workspace** out);
PM_API void pm_solver_workspace_destroy(pm_solver_workspace* workspace);
PM_API int pm_solver_workspace_close(pm_solver_workspace* workspace);

PM_API int pm_cg_f32(pm_solver_workspace* workspace, pm_stream_t stream, const pm_csr* matrix, const float* rhs_d,
              float* solution_d, const pm_solver_options* options, pm_solver_report* report);
PM_API int pm_cg_f64(pm_solver_workspace* workspace, pm_stream_t stream, const pm_csr* matrix, const double* rhs_d,
              double* solution_d, const pm_solver_options* options, pm_solver_report* report);
PM_API int pm_pcg_f32(pm_solver_workspace* workspace, pm_stream_t stream, const pm_csr* matrix, const float* rhs_d,
               float* solution_d, const pm_solver_options* options, pm_solver_report* report);
PM_API int pm_pcg_f64(pm_solver_workspace* workspace, pm_stream_t stream, const pm_csr* matrix, const double* rhs_d,
               double* solution_d, const pm_solver_options* options, pm_solver_report* report);
/* blockPcg: caller-supplied row-major inverse diagonal blocks, (rows * block_size) entries. */
PM_API int pm_block_pcg_f32(pm_solver_workspace* workspace, pm_stream_t stream, const pm_csr* matrix,
                     const float* rhs_d, float* solution_d, const float* inverse_blocks_d, int64_t block_size,
                     const pm_solver_options* options, pm_solver_report* report);
PM_API int pm_block_pcg_f64(pm_solver_workspace* workspace, pm_stream_t stream, const pm_csr* matrix,
                     const double* rhs_d, double* solution_d, const double* inverse_blocks_d, int64_t block_size,
                     const pm_solver_options* options, pm_solver_report* report);

/* Fixed-iteration solves: cgFixedIterationsAsync / pcgFixedIterationsAsync and
 * finalizeIterativeSolverReport (include/plamatrix/sparse/iterative_solver.h:143-171,
 * src/sparse/iterative_solver.cu:166-233, 405-474).  Exactly `iterations` CG (Jacobi-PCG) steps
 * are enqueued on `stream` with no host check; the state records the initial and final
 * recurrence residuals and an event.  Finalize after the caller has synchronised the stream:
 * PM_LOGIC_ERROR while the work is still pending or on a destroyed state, PM_RUNTIME_ERROR
 * for a non-finite residual (breakdown) or, with require_convergence, for a residual above
 * max(absolute, relative * initial).  The workspace, matrix and vectors must stay alive until
 * the stream reaches the state's event. */
typedef struct pm_fixed_state pm_fixed_state;
PM_API int pm_cg_fixed_iterations_async_f32(pm_solver_workspace* workspace, pm_stream_t stream, const pm_csr* matrix,
                                            const float* rhs_d, float* solution_d, int iterations,
                                            pm_fixed_state** state);
PM_API int pm_cg_fixed_iterations_async_f64(pm_solver_workspace* workspace, pm_stream_t stream, const pm_csr* matrix,
                                            const double* rhs_d, double* solution_d, int iterations,
                                            pm_fixed_state** state);
PM_API int pm_pcg_fixed_iterations_async_f32(pm_solver_workspace* workspace, pm_stream_t stream,
                                             const pm_csr* matrix, const float* rhs_d, float* solution_d,
                                             int iterations, pm_fixed_state** state);
PM_API int pm_pcg_fixed_iterations_async_f64(pm_solver_workspace* workspace, pm_stream_t stream,
                                             const pm_csr* matrix, const double* rhs_d, double* solution_d,
                                             int iterations, pm_fixed_state** state);
PM_API int pm_fixed_state_finalize(const pm_fixed_state* state, const pm_solver_options* options,
                                   pm_solver_report* report);
PM_API void pm_fixed_state_destroy(pm_fixed_state* state);

/* =========================================================================== normal equations
 * Device-resident state of the reference's BlockNormalEquations<Scalar>
 * (include/plamatrix/optimization/block_schur.h:196-319, src/optimization/block_normal_equations.cpp):
 * primary diagonal blocks Hpp (P x bp x bp), eliminated diagonal blocks Hll (L x bl x bl),
 * gradients, cross blocks W (bp x bl) of every distinct (primary, eliminated) pair grouped by
 * eliminated block, and upper-triangular primary-primary cross blocks.  value_size selects the
 * Scalar: 4 (float) or 8 (double). */
typedef struct pm_normal_equations pm_normal_equations;
PM_API int pm_ne_create(int64_t primary_count, int64_t eliminated_count, int64_t primary_size,
                        int64_t eliminated_size, int value_size, pm_normal_equations** out);
PM_API void pm_ne_destroy(pm_normal_equations* equations);
/* Counts of the current structure; topology_version changes whenever the structure does. */
PM_API int pm_ne_counts(const pm_normal_equations* equations, int64_t* cross_count, int64_t* primary_cross_count,
                        int64_t* topology_version);
/* Load host state (the reference's accumulated members) onto the device.  Crosses are given
 * grouped by eliminated block: cross_offsets has L+1 entries, cross k belongs to the eliminated
 * block whose range holds k, cross_primary[k] is its primary block (the reference's
 * _eliminatedAdjacency order).  Synchronous. */
PM_API int pm_ne_upload_f32(pm_normal_equations* equations, pm_stream_t stream, const float* primary_diagonal_h,
                            const float* eliminated_diagonal_h, const float* primary_gradient_h,
                            const float* eliminated_gradient_h, int64_t cross_count, const int64_t* cross_offsets_h,
                            const int64_t* cross_primary_h, const float* cross_values_h, int64_t primary_cross_count,
                            const int64_t* primary_cross_row_h, const int64_t* primary_cross_col_h,
                            const float* primary_cross_values_h);
PM_API int pm_ne_upload_f64(pm_normal_equations* equations, pm_stream_t stream, const double* primary_diagonal_h,
                            const double* eliminated_diagonal_h, const double* primary_gradient_h,
                            const double* eliminated_gradient_h, int64_t cross_count, const int64_t* cross_offsets_h,
                            const int64_t* cross_primary_h, const double* cross_values_h, int64_t primary_cross_count,
                            const int64_t* primary_cross_row_h, const int64_t* primary_cross_col_h,
                            const double* primary_cross_values_h);
/* Copy the device state back to host arrays (any pointer may be NULL).  Synchronous. */
PM_API int pm_ne_download_f32(const pm_normal_equations* equations, pm_stream_t stream, float* primary_diagonal_h,
                              float* eliminated_diagonal_h, float* primary_gradient_h, float* eliminated_gradient_h,
                              int64_t* cross_offsets_h, int64_t* cross_primary_h, float* cross_values_h,
                              int64_t* primary_cross_row_h, int64_t* primary_cross_col_h,
                              float* primary_cross_values_h);
PM_API int pm_ne_download_f64(const pm_normal_equations* equations, pm_stream_t stream, double* primary_diagonal_h,
                              double* eliminated_diagonal_h, double* primary_gradient_h, double* eliminated_gradient_h,
                              int64_t* cross_offsets_h, int64_t* cross_primary_h, double* cross_values_h,
                              int64_t* primary_cross_row_h, int64_t* primary_cross_col_h,
                              double* primary_cross_values_h);
/* Huber-weighted accumulation of `count` device-resident observations, each one residual of
 * size m on one primary and one eliminated block: weight = evaluateHuberLoss(||r||^2, delta)
 * .weight (include/plamatrix/optimization/robust_loss.h:27-51), then addResidualBlock
 * (src/optimization/block_normal_equations.cpp:225-312) for every observation.  Jacobians are
 * row-major (count x m x bp) and (count x m x bl), residuals (count x m).  Replaces the
 * state: it equals a fresh BlockNormalEquations fed the observations in array order (cross
 * blocks of an eliminated block ordered by primary index).  The sorting topology is cached
 * while the index arrays are unchanged. */
PM_API int pm_ne_accumulate_observations_f32(pm_normal_equations* equations, pm_stream_t stream, int64_t count,
                                             int64_t residual_size, const int64_t* obs_primary_d,
                                             const int64_t* obs_eliminated_d, const float* primary_jacobians_d,
                                             const float* eliminated_jacobians_d, const float* residuals_d,
                                             float huber_delta);
PM_API int pm_ne_accumulate_observations_f64(pm_normal_equations* equations, pm_stream_t stream, int64_t count,
                                             int64_t residual_size, const int64_t* obs_primary_d,
                                             const int64_t* obs_eliminated_d, const double* primary_jacobians_d,
                                             const double* eliminated_jacobians_d, const double* residuals_d,
                                             double huber_delta);
/* Synchronous check of the last accumulation: PM_INVALID_ARGUMENT when an observation's squared
 * residual norm was not finite, which evaluateHuberLoss rejects (robust_loss.h:31-35);
 * *first_bad_h receives the first such observation index, or -1.  The accumulation itself
 * stays asynchronous; pm_schur_solve_* reports the same error from its own status read. */
PM_API int pm_ne_check_observations(const pm_normal_equations* equations, pm_stream_t stream, int64_t* first_bad_h);

/* =========================================================================== damped Schur solve
 * Replaces solveDampedSchurComplement (include/plamatrix/optimization/block_schur.h:171-186,
 * src/optimization/block_schur.cpp:54-459) with SchurComplementSolverWorkspace
 * (block_schur.h:81-169) as the reusable pattern cache. */
enum
{
    PM_PRECISION_NATIVE = 0, /* assembly, SpMV and PCG vectors in Scalar; dots in FP64 */
    PM_PRECISION_MIXED = 1,  /* double only: FP64 assembly, FP64 refinement around an FP32 inner PCG
                                (the reference's FP32 seed pass, block_schur_accelerated.cpp:131-196) */
    /* double normal equations with 6x6 / 3x3 blocks only (other shapes run PM_PRECISION_MIXED):
     * FP32 assembly products (V = W L^-T stored in FP32, off-diagonal Schur blocks formed and summed
     * in FP32), FP32 SpMV and preconditioner apply; FP64 dots / alpha / beta, FP64 Cholesky of the
     * eliminated and diagonal blocks (diagonal blocks and RHS summed in FP64), and an FP64 true
     * residual computed matrix-free from the FP64 normal equations for every refinement step.  A
     * refinement that fails hands the solve to FP64 PCG on an FP64 assembly.  After such a solve
     * the workspace holds the FP32 values: pm_schur_spmv_f32 and both exports read them. */
    PM_PRECISION_MIXED_FP32_ASSEMBLY = 2
};

typedef struct
{
    int max_iterations;          /* SchurComplementSolverOptions::maxIterations (100) */
    double relative_tolerance;   /* 1e-8 */
    double absolute_tolerance;   /* 1e-12 */
    double minimum_diagonal;     /* 1e-12 */
    int use_initial_guess;       /* 0 */
    int precision;               /* PM_PRECISION_* */
    int tolerance_rule;          /* 0: abs + rel*||r0|| (Cpu backend), 1: max(abs, rel*||r0||) (blockPcg) */
    int check_true_residual;     /* compute ||b - S x|| / ||b|| in FP64 after convergence */
    double inner_relative_tolerance; /* mixed: relative tolerance of each inner FP32 solve (1e-4) */
    int max_refinements;         /* mixed: outer FP64 refinement steps (8) */
    /* No counterpart in the reference: a learned correction of the block-Jacobi blocks
     * (pm_mlp_*), NULL for plain block Jacobi.  When its PCG has not reduced the residual by
     * half over `stagnation_window` iterations (or has not converged), the solve falls back to
     * plain block Jacobi from the iterate it reached. */
    const struct pm_mlp* learned;
    int stagnation_window;       /* 25 */
    /* SchurComplementLinearBackend (block_schur.h:21-27): PM_LINEAR_PCG (block-Jacobi PCG, the
     * Cpu / Cuda backends) or PM_LINEAR_DENSE (DenseCpu: a dense FP64 Cholesky of the reduced
     * system on the device, block_schur_dense_solver.h:236-318; up to PM_DENSE_MAX_UNKNOWNS
     * primary unknowns, single systems only; iterations = 1; messages as the reference's). */
    int linear_backend;
} pm_schur_options;

enum
{
    PM_LINEAR_PCG = 0,
    PM_LINEAR_DENSE = 1
};
#define PM_DENSE_MAX_UNKNOWNS 16384

typedef struct
{
    int converged;
    int iterations;                /* PCG iterations (inner iterations summed in mixed mode) */
    double initial_residual_norm;
    double final_residual_norm;
    double true_relative_residual; /* -1 when not computed */
    int pattern_reused;            /* SchurComplementSolverReport::schurPatternReused */
    int mixed_precision_used;
    int refinement_steps;
    double pattern_ms, eliminated_inverse_ms, assembly_ms, solve_ms, back_substitution_ms, total_ms;
    char message[128];             /* "converged" or the reference's failure message */
    int learned_used;              /* the learned correction preconditioned (part of) the solve */
    int learned_fallback;          /* it stagnated and plain block Jacobi finished the solve */
    int learned_iterations;        /* PCG iterations run with the learned correction */
} pm_schur_report;

typedef struct pm_schur_workspace pm_schur_workspace;
PM_API int pm_schur_workspace_create(pm_schur_workspace** out);
PM_API void pm_schur_workspace_destroy(pm_schur_workspace* workspace);
PM_API int pm_schur_workspace_close(pm_schur_workspace* workspace);
/* SchurComplementSolverWorkspace::patternBuildCount (block_schur.h:121-124). */
PM_API int64_t pm_schur_pattern_build_count(const pm_schur_workspace* workspace);
/* Scalar dimension, scalar nnz and 6x6 block count of the last assembled reduced system. */
PM_API int pm_schur_dims(const pm_schur_workspace* workspace, int64_t* dimension, int64_t* nnz, int64_t* blocks);
/* Solve for the primary step (P*bp, device) and the eliminated step (L*bl, device).
 * Synchronous.  Like the reference, SPD failures are returned in report->message with
 * converged = 0 and PM_OK; invalid arguments return PM_INVALID_ARGUMENT. */
PM_API int pm_schur_solve_f32(pm_schur_workspace* workspace, pm_stream_t stream, const pm_normal_equations* equations,
                              float damping, const pm_schur_options* options, float* primary_step_d,
                              float* eliminated_step_d, pm_schur_report* report);
PM_API int pm_schur_solve_f64(pm_schur_workspace* workspace, pm_stream_t stream, const pm_normal_equations* equations,
                              double damping, const pm_schur_options* options, double* primary_step_d,
                              double* eliminated_step_d, pm_schur_report* report);
/* Assembly launch shapes (no counterpart in the reference, whose assembly launch is fixed,
 * block_schur_device_assembly.cu:211-220).  The upper-block pass of the 6x3 assembly has
 * pm_schur_assembly_shape_count() lane layouts ({pair streams, lanes per pair}); each sums every
 * block in a fixed order of its own, so a shape gives repeatable values, and shapes differ from
 * one another only by rounding.  pm_schur_autotune_assembly times every shape `repeats` times on
 * the system `workspace` last solved (`equations` must be that system), keeps the fastest in the
 * workspace and reports its index, its mean ms and (shape_ms_h, may be NULL, one per shape)
 * every shape's mean ms.  It reassembles the system, so the workspace needs a new solve before
 * its values are exported or multiplied.  Synchronous.  Systems outside the 6x3 path have one
 * shape: *shape_h = 0, *best_ms_h = -1. */
PM_API int pm_schur_assembly_shape_count(void);
PM_API int pm_schur_assembly_shape_info(int shape, int* pair_streams_h, int* lanes_per_pair_h);
PM_API int pm_schur_set_assembly_shape(pm_schur_workspace* workspace, int shape);
PM_API int pm_schur_assembly_shape(const pm_schur_workspace* workspace, int* shape_h);
PM_API int pm_schur_autotune_assembly(pm_schur_workspace* workspace, pm_stream_t stream,
                                      const pm_normal_equations* equations, int repeats, int* shape_h,
                                      double* best_ms_h, double* shape_ms_h);
/* The last assembled reduced system in the reference's scalar-CSR layout
 * (block_schur_sparse_assembly.h:129-153, 262-272): row_offsets (n+1), col_indices and values
 * (nnz), reduced RHS (n, FP64) and block-Jacobi inverses (P*bp*bp, FP64).  Any may be NULL. */
PM_API int pm_schur_export_f32(pm_schur_workspace* workspace, pm_stream_t stream, int64_t* row_offsets_d,
                               int64_t* col_indices_d, float* values_d, double* rhs_d, double* preconditioner_d);
PM_API int pm_schur_export_f64(pm_schur_workspace* workspace, pm_stream_t stream, int64_t* row_offsets_d,
                               int64_t* col_indices_d, double* values_d, double* rhs_d, double* preconditioner_d);

/* y = S x on the last assembled reduced system of `workspace` (n = P * bp; x, y device, in the
 * system's scalar type).  The block-CSR SpMV of the PCG (replaces the spmvAsync call of
 * solveAcceleratedReducedSchur, block_schur_accelerated.cpp:261-263, iterative_solver.cu:54,99). */
PM_API int pm_schur_spmv_f32(pm_schur_workspace* workspace, pm_stream_t stream, const float* x_d, float* y_d);
PM_API int pm_schur_spmv_f64(pm_schur_workspace* workspace, pm_stream_t stream, const double* x_d, double* y_d);

/* =========================================================================== batched solves
 * No counterpart in the reference: many independent LM systems solved together.  The caller
 * accumulates them into one normal-equation object (system s owns the primary blocks
 * [offsets[s], offsets[s+1]) and its own eliminated blocks; no observation couples two
 * systems).  Pattern, assembly, eliminated inverses and back-substitution run once over the
 * union; the block-Jacobi (or learned, options->learned) PCG keeps per-system dots, alpha,
 * beta and convergence on the device; its iterations run as one CUDA graph whose 'while'
 * conditional node repeats a captured chunk of iterations until no system is active, decided
 * on the device (no host check between chunks).  Every system converges to its own tolerance
 * (options->relative_tolerance of its own initial residual).  A system whose learned PCG
 * stagnates restarts from its iterate with plain block Jacobi.  FP64 vectors and dots.  With
 * options->precision PM_PRECISION_MIXED (or MIXED_FP32_ASSEMBLY, treated the same here) the
 * values are assembled in FP64 and the iterations read FP32 copies of the values and of the
 * preconditioner blocks; every system that converges is checked against its FP64 true residual
 * and iterates on from it when the check misses (up to options->max_refinements checks, 8 when
 * 0); report->mixed_precision_used and report->refinement_steps (checks run) describe it. */
typedef struct
{
    int converged;
    int iterations;
    int learned_fallback;
    int breakdown;
    double initial_residual_norm;
    double final_residual_norm;
    double time_ms; /* device time from the start of the batched PCG to this system's convergence, -1 if not */
} pm_batched_system_report;
PM_API int pm_schur_batched_solve_f64(pm_schur_workspace* workspace, pm_stream_t stream,
                                      const pm_normal_equations* equations, double damping,
                                      const pm_schur_options* options, int64_t systems,
                                      const int64_t* system_primary_offsets, double* primary_step_d,
                                      double* eliminated_step_d, pm_schur_report* report,
                                      pm_batched_system_report* per_system);

/* =========================================================================== learned block Jacobi
 * No counterpart in the reference.  A per-block-row network (25 -> 128 -> 128 -> 21, GELU, BF16
 * operands and FP32 accumulation on the tensor cores) reads each 6x6 diagonal block of the
 * reduced system and statistics of its row's off-diagonal block norms, and corrects the
 * Cholesky factor L of the block:  L'_ii = L_ii softplus(o_ii) / ln 2,  L'_ij = L_ij + o_ij L_jj.
 * The preconditioner block is (L' L'^T)^-1, SPD by construction; a zero network is plain block
 * Jacobi.  Training minimises sum_p ||L'L'^T x_p - b_p||^2 / ||b||^2 over solved systems (x, b)
 * with Adam on FP32 master weights.  Parameters are one FP32 vector: W1 (25x128), b1 (128),
 * W2 (128x128), b2 (128), W3 (128x21), b3 (21), weights input-major. */
typedef struct pm_mlp pm_mlp;
PM_API int64_t pm_mlp_param_count(void);
/* Xavier-uniform hidden layers from `seed`, zero output layer (starts as block Jacobi). */
PM_API int pm_mlp_create(uint64_t seed, pm_mlp** out);
PM_API void pm_mlp_destroy(pm_mlp* mlp);
PM_API int pm_mlp_get_params(const pm_mlp* mlp, float* host_params);
PM_API int pm_mlp_set_params(pm_mlp* mlp, const float* host_params);
/* Forward pass on the system last assembled in `workspace` (6x6 blocks); keeps features and
 * outputs for pm_mlp_inspect.  Synchronous. */
PM_API int pm_mlp_forward(pm_mlp* mlp, pm_schur_workspace* workspace, pm_stream_t stream);
/* Loss and parameter gradients for that system with solution x and right-hand side b (device,
 * FP64, n = 6P); with `learning_rate` > 0 one Adam step follows.  Synchronous. */
PM_API int pm_mlp_train_step(pm_mlp* mlp, pm_schur_workspace* workspace, pm_stream_t stream, const double* x_d,
                             const double* b_d, double learning_rate, double* loss);
/* Loss and gradients of the preconditioned operator along a probe vector v (device, FP64, n = 6P)
 * for the system last assembled in `workspace`: ||(I - M S) v||^2 / ||v||^2, where M is the
 * corrected block preconditioner and sv = S v is supplied by the caller (pm_schur_spmv_f64, or the
 * float SpMV widened, of the same system); with `learning_rate` > 0 one Adam step follows.  It needs
 * no solved system, and it measures how well M inverts S along v -- the quantity PCG convergence
 * depends on.  Synchronous. */
PM_API int pm_mlp_train_probe_step(pm_mlp* mlp, pm_schur_workspace* workspace, pm_stream_t stream, const double* v_d,
                                   const double* sv_d, double learning_rate, double* loss);
/* Polls of an mbarrier wait between the network GEMM's operand stages before it gives up (default
 * 2^20; the final wait for the last MMA always uses 2^20).  A GEMM whose wait runs out stops
 * issuing MMAs, frees its tensor memory once its last MMA has completed, and the call that ran it
 * returns PM_RUNTIME_ERROR ("a tensor-core GEMM did not complete"); the network stays usable.
 * A limit of 0 makes every multi-step GEMM give up at its first stage wait (the error path). */
PM_API int pm_mlp_set_wait_limit(pm_mlp* mlp, int64_t polls);
/* Host copies of the last features (P x 25), outputs (P x 21) and gradients; any may be NULL. */
PM_API int pm_mlp_inspect(const pm_mlp* mlp, int64_t* rows, float* features, float* outputs, float* gradients);

/* =========================================================================== LM loop (caller side)
 * Replaces LevenbergMarquardtOptions / LevenbergMarquardtStrategy
 * (include/plamatrix/optimization/levenberg_marquardt.h:13-95): host state, the damping updated in
 * the strategy's scalar type (f32 / f64 as the template argument).  create returns
 * PM_INVALID_ARGUMENT ("LevenbergMarquardtStrategy: invalid damping options") for bounds or
 * factors the reference rejects; options == NULL takes the defaults. */
typedef struct
{
    double initial_damping; /* 1e-3 */
    double minimum_damping; /* 1e-12 */
    double maximum_damping; /* 1e12 */
    double decrease_factor; /* 0.3, after an accepted step */
    double increase_factor; /* 10, after a rejected or invalid step */
} pm_lm_options;
typedef struct pm_lm_strategy pm_lm_strategy;
PM_API void pm_lm_options_default(pm_lm_options* options);
PM_API int pm_lm_strategy_create_f32(const pm_lm_options* options, pm_lm_strategy** out);
PM_API int pm_lm_strategy_create_f64(const pm_lm_options* options, pm_lm_strategy** out);
PM_API void pm_lm_strategy_destroy(pm_lm_strategy* strategy);
PM_API int pm_lm_accept_step(pm_lm_strategy* strategy);
PM_API int pm_lm_reject_step(pm_lm_strategy* strategy);
PM_API int pm_lm_strategy_state(const pm_lm_strategy* strategy, double* damping_h, int* accepted_steps_h,
                                int* rejected_steps_h);

/* Total robust cost sum_i evaluateHuberLoss(|r_i|^2, delta).cost of `count` residuals of size m
 * (residual_d: count x m, row-major), written to *cost_d (device, FP64) -- the cost an LM loop
 * compares between trial steps (robust_loss.h:27-51 per residual, summed by the caller in the
 * reference).  Per-residual costs are exact in the residual's type; the FP64 sum uses a fixed
 * tree, so results repeat bit for bit.  A residual whose squared norm is not finite makes the
 * total non-finite (evaluateHuberLoss rejects it; an LM caller rejects the step).  scratch_d
 * holds PM_HUBER_COST_SCRATCH doubles of caller-owned device memory. */
#define PM_HUBER_COST_SCRATCH 1024
PM_API int pm_huber_cost_f32(pm_stream_t stream, int64_t count, int64_t m, const float* residual_d, float delta,
                             double* scratch_d, double* cost_d);
PM_API int pm_huber_cost_f64(pm_stream_t stream, int64_t count, int64_t m, const double* residual_d, double delta,
                             double* scratch_d, double* cost_d);

#ifdef __cplusplus
}
#endif

#endif /* PLAMATRIX_B200_H */
