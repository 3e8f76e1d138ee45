/*
 * CPU oracle for the PlaMatrix Levenberg-Marquardt normal-equation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithms, used by the test-suite, smoke() and bench.py's cpu_baseline leg
 * as the checker.  The product library (plamatrix_b200) never links, loads or
 * calls anything in this directory.
 *
 * Parity pinning: every function below is checked against (a) the golden
 * vectors of the reference's own unit tests (restated in tests/golden/) and
 * (b) the reference's CPU library itself, compiled from the reference sources
 * into oracle/_ref/ by oracle/Makefile and driven through oracle/ref_harness.cpp.
 *
 * Functions come in _f32 / _f64 pairs that follow the reference's float/double
 * instantiations.  Status codes mirror the reference's exception classes.
 */
#ifndef PLAMATRIX_ORACLE_H
#define PLAMATRIX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum
{
    ORC_OK = 0,
    ORC_INVALID_ARGUMENT = 1, /* std::invalid_argument */
    ORC_OUT_OF_RANGE = 2,     /* std::out_of_range */
    ORC_RUNTIME_ERROR = 3,    /* std::runtime_error */
    ORC_LOGIC_ERROR = 4,      /* std::logic_error */
    ORC_OVERFLOW = 5,         /* std::overflow_error */
    ORC_NO_MEMORY = 6
};

/* Message of the last non-zero status returned on this thread. */
const char* orc_last_error(void);

/* ---------------------------------------------------------------- COO -> CSR
 * Follows src/sparse/sparse_ops_cpu.cpp:24-134 (combineCoo + writeCombinedCoo):
 * stable sort of a permutation by (row, col); duplicates combined by pushing
 * the first value verbatim and then `+=` the rest in input order.  The output
 * arrays must hold `count` entries (an upper bound of the combined nnz). */
int orc_coo_to_csr_f32(int64_t rows, int64_t cols, int64_t count, const int64_t* row_indices,
                       const int64_t* col_indices, const float* values, int64_t* row_offsets,
                       int64_t* out_columns, float* out_values, int64_t* out_nnz);
int orc_coo_to_csr_f64(int64_t rows, int64_t cols, int64_t count, const int64_t* row_indices,
                       const int64_t* col_indices, const double* values, int64_t* row_offsets,
                       int64_t* out_columns, double* out_values, int64_t* out_nnz);

/* ---------------------------------------------------------------- CSR SpMV
 * Follows src/sparse/sparse_ops_cpu.cpp:214-233 (serial row loop in Scalar). */
int orc_csr_spmv_f32(int64_t rows, int64_t cols, const int64_t* row_offsets, const int64_t* columns,
                     const float* values, const float* x, float* y);
int orc_csr_spmv_f64(int64_t rows, int64_t cols, const int64_t* row_offsets, const int64_t* columns,
                     const double* values, const double* x, double* y);

/* ---------------------------------------------------------------- CSR SpMM
 * Follows src/sparse/sparse_ops_cpu.cpp:244-270: output (rows x k) = CSR x input (cols x k),
 * both dense matrices column-major. */
int orc_csr_spmm_f32(int64_t rows, int64_t cols, const int64_t* row_offsets, const int64_t* columns,
                     const float* values, int64_t k, const float* input, float* output);
int orc_csr_spmm_f64(int64_t rows, int64_t cols, const int64_t* row_offsets, const int64_t* columns,
                     const double* values, int64_t k, const double* input, double* output);

/* ---------------------------------------------------------------- CG / PCG */
typedef struct
{
    int max_iterations;        /* IterativeSolverOptions::maxIterations (1000) */
    double relative_tolerance; /* 1e-6 */
    double absolute_tolerance; /* 0 */
    int use_jacobi;            /* useJacobiPreconditioner (1) */
    int require_convergence;   /* requireConvergence (0) */
} orc_solver_options;

typedef struct
{
    int converged;
    int iterations;
    double initial_residual;
    double final_residual;
} orc_solver_report;

/* Follows src/sparse/iterative_solver_cpu.cpp:162-304: vectors and dots in FP64
 * regardless of Scalar, tolerance max(abs, rel*||r0||), scalar Jacobi with the
 * 16*eps*rowscale guard.  `preconditioned` selects pcg (1) or cg (0). */
int orc_pcg_f32(int64_t n, const int64_t* row_offsets, const int64_t* columns, const float* values,
                const float* rhs, float* solution, const orc_solver_options* options,
                int preconditioned, orc_solver_report* report);
int orc_pcg_f64(int64_t n, const int64_t* row_offsets, const int64_t* columns, const double* values,
                const double* rhs, double* solution, const orc_solver_options* options,
                int preconditioned, orc_solver_report* report);

/* ---------------------------------------------------------------- Huber
 * Follows include/plamatrix/optimization/robust_loss.h:27-51. */
int orc_huber_f32(float squared_norm, float delta, float* cost, float* weight);
int orc_huber_f64(double squared_norm, double delta, double* cost, double* weight);

/* ---------------------------------------------------------------- normal equations
 * Follows src/optimization/block_normal_equations.cpp (BlockNormalEquations). */
typedef struct orc_ne_f32 orc_ne_f32;
typedef struct orc_ne_f64 orc_ne_f64;

orc_ne_f32* orc_ne_create_f32(int64_t primary_count, int64_t eliminated_count, int64_t primary_size,
                              int64_t eliminated_size);
orc_ne_f64* orc_ne_create_f64(int64_t primary_count, int64_t eliminated_count, int64_t primary_size,
                              int64_t eliminated_size);
void orc_ne_destroy_f32(orc_ne_f32* ne);
void orc_ne_destroy_f64(orc_ne_f64* ne);

/* One residual: `primary_count_in_residual` primaries (jacobians packed back to
 * back, each residual_size x primary_size row-major) and an optional eliminated
 * block (eliminated < 0 means none; primary count 0 means eliminated-only).
 * Covers addResidualBlock(s), addPrimaryResidualBlock(s) and
 * addEliminatedResidualBlock (block_normal_equations.cpp:136-373). */
int orc_ne_add_residual_f32(orc_ne_f32* ne, int64_t primary_count_in_residual,
                            const int64_t* primaries, const float* primary_jacobians,
                            int64_t eliminated, const float* eliminated_jacobian,
                            const float* residual, int64_t residual_size, float weight);
int orc_ne_add_residual_f64(orc_ne_f64* ne, int64_t primary_count_in_residual,
                            const int64_t* primaries, const double* primary_jacobians,
                            int64_t eliminated, const double* eliminated_jacobian,
                            const double* residual, int64_t residual_size, double weight);

/* Huber-weighted observations (one primary + one eliminated block each), added
 * in array order with weight = evaluateHuberLoss(||r||^2, delta).weight -- the
 * caller-side loop of a reference LM iteration. */
int orc_ne_add_observations_f32(orc_ne_f32* ne, int64_t count, int64_t residual_size,
                                const int64_t* primaries, const int64_t* eliminated,
                                const float* primary_jacobians, const float* eliminated_jacobians,
                                const float* residuals, float huber_delta);
int orc_ne_add_observations_f64(orc_ne_f64* ne, int64_t count, int64_t residual_size,
                                const int64_t* primaries, const int64_t* eliminated,
                                const double* primary_jacobians, const double* eliminated_jacobians,
                                const double* residuals, double huber_delta);

/* mergeFrom (block_normal_equations.cpp:376-411). */
int orc_ne_merge_f32(orc_ne_f32* target, const orc_ne_f32* source);
int orc_ne_merge_f64(orc_ne_f64* target, const orc_ne_f64* source);

/* Sizes of the accumulated structure. */
void orc_ne_counts_f32(const orc_ne_f32* ne, int64_t* cross_count, int64_t* primary_cross_count);
void orc_ne_counts_f64(const orc_ne_f64* ne, int64_t* cross_count, int64_t* primary_cross_count);

/* Copies of the accumulated state.  Crosses are exported grouped by eliminated
 * block in adjacency (insertion) order: adjacency_offsets has L+1 entries and
 * cross k of the export is the k-th entry of that walk.  Any pointer may be NULL. */
void orc_ne_export_f32(const orc_ne_f32* ne, float* primary_diagonal, float* eliminated_diagonal,
                       float* primary_gradient, float* eliminated_gradient,
                       int64_t* adjacency_offsets, int64_t* cross_primary, float* cross_values,
                       int64_t* primary_cross_row, int64_t* primary_cross_col,
                       float* primary_cross_values);
void orc_ne_export_f64(const orc_ne_f64* ne, double* primary_diagonal, double* eliminated_diagonal,
                       double* primary_gradient, double* eliminated_gradient,
                       int64_t* adjacency_offsets, int64_t* cross_primary, double* cross_values,
                       int64_t* primary_cross_row, int64_t* primary_cross_col,
                       double* primary_cross_values);

/* ---------------------------------------------------------------- Schur solve */
enum
{
    ORC_BACKEND_CPU = 0,      /* matrix-free block-Jacobi PCG (block_schur_cpu_solver.h) */
    ORC_BACKEND_DENSE_CPU = 1 /* dense Cholesky of the assembled Schur (block_schur_dense_solver.h) */
};

typedef struct
{
    int backend;
    int max_iterations;        /* 100 */
    double relative_tolerance; /* 1e-8 */
    double absolute_tolerance; /* 1e-12 */
    double minimum_diagonal;   /* 1e-12 */
    int use_initial_guess;     /* 0 */
} orc_schur_options;

typedef struct
{
    int converged;
    int iterations;
    double initial_residual_norm;
    double final_residual_norm;
    char message[128];
} orc_schur_report;

/* solveDampedSchurComplement (src/optimization/block_schur.cpp:54-459).
 * primary_step has P*bp entries (read when use_initial_guess), eliminated_step
 * L*bl entries.  SPD failures are reported in report->message, not as status. */
int orc_schur_solve_f32(const orc_ne_f32* ne, float damping, const orc_schur_options* options,
                        float* primary_step, float* eliminated_step, orc_schur_report* report);
int orc_schur_solve_f64(const orc_ne_f64* ne, double damping, const orc_schur_options* options,
                        double* primary_step, double* eliminated_step, orc_schur_report* report);

/* Scalar-CSR nnz of the reduced Schur pattern (block_schur_sparse_assembly.h:41-260). */
int orc_schur_pattern_nnz_f32(const orc_ne_f32* ne, int64_t* nnz, int64_t* block_count);
int orc_schur_pattern_nnz_f64(const orc_ne_f64* ne, int64_t* nnz, int64_t* block_count);

/* Reduced Schur system: scalar CSR pattern + values (CPU branch of
 * assembleReducedSchurCsr, block_schur_sparse_assembly.h:679-911, on the damped
 * diagonals), reduced RHS (block_schur.cpp:151-177) and the block-Jacobi inverse
 * blocks (block_schur.cpp:180-250, P*bp*bp row-major).  Any output may be NULL.
 * Returns ORC_RUNTIME_ERROR when a block is not SPD. */
int orc_schur_system_f32(const orc_ne_f32* ne, float damping, float minimum_diagonal,
                         int64_t* row_offsets, int64_t* col_indices, float* values, float* rhs,
                         float* preconditioner_inverse);
int orc_schur_system_f64(const orc_ne_f64* ne, double damping, double minimum_diagonal,
                         int64_t* row_offsets, int64_t* col_indices, double* values, double* rhs,
                         double* preconditioner_inverse);

/* ---------------------------------------------------------------- learned correction
 * No counterpart in the reference: the FP64 restatement of the device MLP that corrects the
 * block-Jacobi preconditioner (definitions in oracle/mlp.c).  Parameters are one flat vector:
 * W1 (25x128) b1 (128) W2 (128x128) b2 (128) W3 (128x21) b3 (21), weights input-major. */
#define ORC_MLP_IN 25
#define ORC_MLP_HIDDEN 128
#define ORC_MLP_OUT 21
int64_t orc_mlp_param_count(void);
int orc_mlp_features(int64_t P, const int64_t* block_row_ptr, const int64_t* block_col, const double* blocks,
                     double* features);
int orc_mlp_forward(int64_t P, const double* features, const double* params, int bf16_operands, double* z1,
                    double* h1, double* z2, double* h2, double* out);
int orc_mlp_loss_grad(int64_t P, const double* diag_blocks, const double* out, const double* x, const double* b,
                      double* loss, double* dout);
int orc_mlp_probe_loss_grad(int64_t P, const double* diag_blocks, const double* out, const double* v, const double* sv,
                            double* loss, double* dout);
int orc_mlp_backward(int64_t P, const double* features, const double* params, int bf16_operands, const double* z1,
                     const double* h1, const double* z2, const double* h2, const double* dout, double* grads);
int orc_mlp_preconditioner(int64_t P, const double* diag_blocks, const double* out, double* minv);

#ifdef __cplusplus
}
#endif

#endif
