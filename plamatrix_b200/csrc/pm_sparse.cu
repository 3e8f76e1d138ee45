// CSR operands, CSR SpMV and CG / PCG / block-PCG for sm_100a.
//
// Replaces the reference's cuSPARSE SpMV (src/sparse/sparse_ops.cu:687-740) and its
// cuBLAS-driven adaptive solver loop (src/sparse/iterative_solver.cu:30-349), which
// synchronises with the host after every iteration.  Here:
//   * the int64 CSR structure is validated once and kept as int32 (4 B per index on the
//     HBM stream instead of 8 B);
//   * SpMV uses a sub-warp per row (width chosen from the mean row length) with shuffle
//     reductions;
//   * one PCG iteration is three kernels (direction update, SpMV fused with the p.q dot,
//     vector update fused with preconditioner apply and the r.z / r.r dots); every dot is
//     accumulated in FP64 per block and finished by the last block to arrive, in a fixed
//     order, which also evaluates alpha / beta, breakdown and convergence on the device;
//   * the iterations run as a CUDA graph whose 'while' node repeats a chunk of them until the
//     device state says done; the host reads the state once, after the solve.
#include "pm_common.cuh"

#include <cmath>
#include <limits>
#include <sstream>

struct pm_csr
{
    int value_size = 0;
    int64_t rows = 0, cols = 0, nnz = 0;
    int* row_ptr = nullptr; // int32 copy of the validated row offsets
    int* col_idx = nullptr; // int32 copy of the validated column indices
    const void* values = nullptr;
    int threads_per_row = 1; // lanes per row of the heuristic
    int kernel = -1;         // -1: heuristic; 0: row-group stream; 1..32: lanes per row (autotuned or set)
};

namespace pm
{

// the SpMV shape of an operand: the row-group stream kernel, or TPR lanes per row
inline bool use_stream(const pm_csr* A) { return A->kernel == 0; }
inline int lanes_per_row(const pm_csr* A) { return A->kernel > 0 ? A->kernel : A->threads_per_row; }

template <typename T>
struct Eps;
template <>
struct Eps<float>
{
    static constexpr double value = 1.1920928955078125e-7;
};
template <>
struct Eps<double>
{
    static constexpr double value = 2.2204460492503131e-16;
};

namespace
{

constexpr long long kNone = 0x7fffffffffffffffLL;
constexpr int kReduceBlock = 256;
constexpr int kMaxReduceBlocks = 1024;

struct CsrCheck
{
    long long bad_offsets_row;
    long long bad_column;
    long long bad_value;
    int endpoints_bad;
};

template <typename T>
__global__ void validate_csr_kernel(int64_t rows, int64_t cols, int64_t nnz, const int64_t* __restrict__ row_offsets,
                                    const int64_t* __restrict__ col_indices, const T* __restrict__ values,
                                    int* __restrict__ row_ptr32, int* __restrict__ col32, CsrCheck* check)
{
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t == 0 && (row_offsets[0] != 0 || row_offsets[rows] != nnz))
        check->endpoints_bad = 1;
    for (int64_t r = t; r < rows; r += stride)
    {
        const int64_t b = row_offsets[r], e = row_offsets[r + 1];
        if (b < 0 || e < b || e > nnz)
            atomicMin(&check->bad_offsets_row, static_cast<long long>(r));
        row_ptr32[r] = static_cast<int>(b);
    }
    if (t == 0)
        row_ptr32[rows] = static_cast<int>(nnz);
    for (int64_t p = t; p < nnz; p += stride)
    {
        const int64_t c = col_indices[p];
        if (c < 0 || c >= cols)
            atomicMin(&check->bad_column, static_cast<long long>(p));
        if (!isfinite(static_cast<double>(values[p])))
            atomicMin(&check->bad_value, static_cast<long long>(p));
        col32[p] = static_cast<int>(c);
    }
}

// y = A x with a TPR-wide sub-warp per row
template <typename T, int TPR>
__device__ __forceinline__ T csr_row_dot(const int* __restrict__ rp, const int* __restrict__ ci,
                                         const T* __restrict__ v, const T* __restrict__ x, int64_t row, bool valid,
                                         int lane)
{
    T sum = T(0);
    if (valid)
    {
        const int b = rp[row], e = rp[row + 1];
        if constexpr (TPR == 1)
        {
            // a thread per row: the row's columns and values in groups of eight, all loads of a
            // group issued before its products (streamed, no reuse), the sum in storage order
            constexpr int G = 8;
            for (int base = b; base < e; base += G)
            {
                int col[G];
                T val[G], xv[G];
#pragma unroll
                for (int k = 0; k < G; ++k)
                    if (base + k < e)
                    {
                        col[k] = __ldcs(ci + base + k);
                        val[k] = __ldcs(v + base + k);
                    }
#pragma unroll
                for (int k = 0; k < G; ++k)
                    if (base + k < e)
                        xv[k] = __ldg(x + col[k]);
#pragma unroll
                for (int k = 0; k < G; ++k)
                    if (base + k < e)
                        sum += val[k] * xv[k];
            }
        }
        else
        {
            for (int p = b + lane; p < e; p += TPR)
                sum += v[p] * __ldg(x + ci[p]);
        }
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1)
        sum += __shfl_xor_sync(0xffffffffu, sum, o, TPR);
    return sum;
}

// Row-group stream (chosen by pm_csr_set_kernel or the autotuner): a warp owns 32 consecutive rows.  Their nonzeros form one
// contiguous range, loaded coalesced in pieces of kStreamCap (values, columns, then the x
// gathers, all in flight together); products are staged in shared memory and lane i sums
// row i's products in column order.  The sum order is the row's storage order.
constexpr int kStreamCap = 256; // staged products per warp
constexpr int kStreamUnroll = kStreamCap / 32;

template <typename T>
__device__ __forceinline__ T csr_stream_rows(int64_t r0, int64_t rows, const int* __restrict__ rp,
                                             const int* __restrict__ ci, const T* __restrict__ v,
                                             const T* __restrict__ x, T* __restrict__ stage)
{
    const int lane = threadIdx.x & 31;
    const int64_t row = r0 + lane;
    const bool valid = row < rows;
    const int my_begin = valid ? rp[row] : 0;
    const int my_end = valid ? rp[row + 1] : 0;
    const int last = static_cast<int>(rows - 1 - r0 < 31 ? rows - 1 - r0 : 31);
    const int cb = __shfl_sync(0xffffffffu, my_begin, 0);
    const int ce = __shfl_sync(0xffffffffu, my_end, last);
    T sum = T(0);
    for (int base = cb; base < ce; base += kStreamCap)
    {
        const int n = ce - base < kStreamCap ? ce - base : kStreamCap;
        int col[kStreamUnroll];
        T val[kStreamUnroll];
#pragma unroll
        for (int u = 0; u < kStreamUnroll; ++u)
        {
            const int k = u * 32 + lane;
            if (k < n)
            {
                col[u] = __ldcs(ci + base + k);
                val[u] = __ldcs(v + base + k);
            }
        }
#pragma unroll
        for (int u = 0; u < kStreamUnroll; ++u)
        {
            const int k = u * 32 + lane;
            if (k < n)
                stage[k] = val[u] * __ldg(x + col[u]);
        }
        __syncwarp();
        const int lo = my_begin > base ? my_begin : base;
        const int hi = my_end < base + n ? my_end : base + n;
        for (int k = lo; k < hi; ++k)
            sum += stage[k - base];
        __syncwarp();
    }
    return sum;
}

template <typename T>
__global__ void __launch_bounds__(256) csr_stream_kernel(int64_t rows, const int* __restrict__ rp,
                                                         const int* __restrict__ ci, const T* __restrict__ v,
                                                         const T* __restrict__ x, T* __restrict__ y)
{
    __shared__ T stage[8][kStreamCap];
    const int warp = threadIdx.x >> 5;
    const int64_t warps = int64_t(gridDim.x) * 8;
    for (int64_t wrow = (int64_t(blockIdx.x) * 8 + warp) * 32; wrow < rows; wrow += warps * 32)
    {
        const T sum = csr_stream_rows<T>(wrow, rows, rp, ci, v, x, stage[warp]);
        if (wrow + (threadIdx.x & 31) < rows)
            y[wrow + (threadIdx.x & 31)] = sum;
    }
}

template <typename T, int TPR>
__global__ void __launch_bounds__(256) csr_spmv_kernel(int64_t rows, const int* __restrict__ rp,
                                                       const int* __restrict__ ci, const T* __restrict__ v,
                                                       const T* __restrict__ x, T* __restrict__ y)
{
    const int64_t gid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x / TPR;
    const int lane = threadIdx.x % TPR;
    const int64_t first = gid / TPR;
    const int64_t span = (rows + stride - 1) / stride; // uniform trip count keeps shuffles convergent
    for (int64_t k = 0; k < span; ++k)
    {
        const int64_t row = first + k * stride;
        const bool valid = row < rows;
        const T sum = csr_row_dot<T, TPR>(rp, ci, v, x, row, valid, lane);
        if (valid && lane == 0)
            y[row] = sum;
    }
}

// heuristic lanes per row: a thread per row up to 8 nonzeros per row on average (its grouped
// loads beat the row-group stream there: 49 vs 61 us on the 128^3 Laplacian), then the next
// power of two above the mean
int pick_tpr(int64_t rows, int64_t nnz)
{
    const double mean = rows > 0 ? double(nnz) / double(rows) : 1.0;
    if (mean <= 8.0)
        return 1;
    int tpr = 16;
    while (tpr < 32 && tpr < mean)
        tpr <<= 1;
    return tpr;
}

template <typename T>
void launch_spmv(const pm_csr* A, const T* x, T* y, cudaStream_t stream)
{
    if (A->rows == 0)
        return;
    const T* v = static_cast<const T*>(A->values);
    const int block = 256;
    if (use_stream(A))
    {
        csr_stream_kernel<T><<<grid_for(A->rows, 256, 1 << 20), 256, 0, stream>>>(A->rows, A->row_ptr, A->col_idx,
                                                                                    v, x, y);
        PM_LAUNCH_CHECK();
        return;
    }
    const unsigned grid = grid_for(A->rows * lanes_per_row(A), block, 65535);
    switch (lanes_per_row(A))
    {
    case 1: csr_spmv_kernel<T, 1><<<grid, block, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, x, y); break;
    case 2: csr_spmv_kernel<T, 2><<<grid, block, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, x, y); break;
    case 4: csr_spmv_kernel<T, 4><<<grid, block, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, x, y); break;
    case 8: csr_spmv_kernel<T, 8><<<grid, block, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, x, y); break;
    case 16: csr_spmv_kernel<T, 16><<<grid, block, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, x, y); break;
    default: csr_spmv_kernel<T, 32><<<grid, block, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, x, y); break;
    }
    PM_LAUNCH_CHECK();
}

// ------------------------------------------------------------------ PCG state
struct PcgState
{
    double rho;      // r.z of the current direction
    double alpha;
    double beta;
    double tolerance;
    double initial_squared;
    double residual_squared;
    int iterations;
    int max_iterations;
    int done;
    int converged;
    int breakdown;     // 1: not SPD / non-finite step
    int nonfinite_init;
    long long jacobi_bad_row;
    unsigned int ticket[3];
    int chunks; // bodies run by the iteration graph
};

// Last block to arrive sums the per-block partials (fixed order) and runs `finish`.
template <int K, typename Finish>
__device__ __forceinline__ void reduce_partials(double (&mine)[K], double* partials, unsigned int* ticket,
                                                Finish&& finish)
{
    __shared__ double smem[kReduceBlock / 32];
    __shared__ bool last;
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const double s = block_sum<double, kReduceBlock>(mine[k], smem);
        if (threadIdx.x == 0)
            partials[k * kMaxReduceBlocks + blockIdx.x] = s;
    }
    __threadfence();
    if (threadIdx.x == 0)
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last)
        return;
    __threadfence();
    double totals[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        double s = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
            s += __ldcg(partials + k * kMaxReduceBlocks + b);
        totals[k] = block_sum<double, kReduceBlock>(s, smem);
    }
    if (threadIdx.x == 0)
    {
        *ticket = 0;
        finish(totals);
    }
}

// preconditioned component i of the residual vector `r` (scalar Jacobi, caller blocks, none)
template <typename T, typename R>
__device__ __forceinline__ double apply_precond(int mode, int64_t i, R&& residual_at, const T* inv_diag,
                                                const T* blocks, int64_t bs)
{
    if (mode == 1)
        return static_cast<double>(inv_diag[i]) * residual_at(i);
    if (mode == 2)
    {
        const int64_t blk = i / bs, local = i - blk * bs;
        const T* row = blocks + blk * bs * bs + local * bs;
        double z = 0.0;
        for (int64_t c = 0; c < bs; ++c)
            z += static_cast<double>(row[c]) * residual_at(blk * bs + c);
        return z;
    }
    return residual_at(i);
}

// Jacobi inverse: iterative_solver_kernels.cuh:104-131 semantics (sum of diagonal duplicates,
// 16*eps*rowscale guard); invalid rows are reported (lowest row) instead of NaN markers.
template <typename T>
__global__ void jacobi_kernel(int64_t rows, const int* __restrict__ rp, const int* __restrict__ ci,
                              const T* __restrict__ v, T* __restrict__ inv, PcgState* st)
{
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += int64_t(gridDim.x) * blockDim.x)
    {
        double diag = 0.0, scale = 0.0;
        bool found = false;
        for (int p = rp[r]; p < rp[r + 1]; ++p)
        {
            const double value = static_cast<double>(v[p]);
            scale = fmax(scale, fabs(value));
            if (ci[p] == r)
            {
                diag += value;
                found = true;
            }
        }
        const double threshold = Eps<T>::value * scale * 16.0;
        const double reciprocal = 1.0 / diag;
        if (!found || !isfinite(diag) || diag <= threshold || !isfinite(reciprocal))
        {
            atomicMin(&st->jacobi_bad_row, static_cast<long long>(r));
            inv[r] = T(0);
        }
        else
        {
            inv[r] = static_cast<T>(reciprocal);
        }
    }
}

// r = b - Ax (Ax in q), z = M^-1 r, p = z; rho = r.z, initial ||r||^2
template <typename T>
__global__ void __launch_bounds__(kReduceBlock) pcg_init_kernel(int64_t n, const T* __restrict__ b,
                                                                const T* __restrict__ q, T* __restrict__ r,
                                                                T* __restrict__ z, T* __restrict__ p, int mode,
                                                                const T* __restrict__ inv, const T* __restrict__ blocks,
                                                                int64_t bs, double relative, double absolute,
                                                                double* partials, PcgState* st)
{
    double mine[2] = {0.0, 0.0};
    auto res = [&](int64_t k) { return static_cast<double>(static_cast<T>(static_cast<double>(b[k]) - static_cast<double>(q[k]))); };
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        const double ri = res(i);
        const T zi = static_cast<T>(apply_precond<T>(mode, i, res, inv, blocks, bs));
        r[i] = static_cast<T>(ri);
        z[i] = zi;
        p[i] = zi;
        mine[0] += ri * static_cast<double>(zi);
        mine[1] += ri * ri;
    }
    reduce_partials<2>(mine, partials, &st->ticket[0], [&](double (&tot)[2]) {
        st->rho = tot[0];
        st->initial_squared = tot[1];
        st->residual_squared = tot[1];
        const double initial = sqrt(tot[1]);
        st->tolerance = fmax(absolute, relative * initial);
        st->iterations = 0;
        st->beta = 0.0;
        if (!isfinite(tot[1]) || tot[1] < 0.0)
        {
            st->nonfinite_init = 1;
            st->done = 1;
        }
        else if (initial <= st->tolerance)
        {
            st->converged = 1;
            st->done = 1;
        }
        if (st->jacobi_bad_row != kNone)
            st->done = 1;
    });
}

// alpha = rho / p.q on the last block (alphaKernel semantics, iterative_solver_kernels.cuh:169-202)
template <typename T>
__device__ __forceinline__ void pcg_alpha(PcgState* st, double den, T)
{
    const double rho = st->rho;
    double alpha = 0.0;
    if (rho == 0.0 && den == 0.0)
        alpha = 0.0;
    else if (isfinite(rho) && isfinite(den) && rho > 0.0 && den > 0.0)
    {
        alpha = rho / den;
        // the step must also be representable in the vector type (the reference forms
        // alpha in Scalar precision and treats its overflow as breakdown)
        if (!isfinite(alpha) || !isfinite(static_cast<double>(static_cast<T>(alpha))))
        {
            st->breakdown = 1;
            alpha = 0.0;
        }
    }
    else
    {
        st->breakdown = 1;
    }
    st->alpha = alpha;
    if (st->breakdown)
        st->done = 1;
}

// q = A p, alpha = rho / p.q  (alphaKernel semantics, iterative_solver_kernels.cuh:169-202)
template <typename T, int TPR>
__global__ void __launch_bounds__(kReduceBlock) pcg_spmv_kernel(int64_t rows, const int* __restrict__ rp,
                                                                const int* __restrict__ ci, const T* __restrict__ v,
                                                                const T* __restrict__ p, T* __restrict__ q,
                                                                double* partials, PcgState* st)
{
    if (st->done)
        return;
    double mine[1] = {0.0};
    const int64_t stride = int64_t(gridDim.x) * blockDim.x / TPR;
    const int lane = threadIdx.x % TPR;
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / TPR;
    const int64_t span = (rows + stride - 1) / stride;
    for (int64_t k = 0; k < span; ++k)
    {
        const int64_t row = first + k * stride;
        const bool valid = row < rows;
        const T sum = csr_row_dot<T, TPR>(rp, ci, v, p, row, valid, lane);
        if (valid && lane == 0)
        {
            q[row] = sum;
            mine[0] += static_cast<double>(p[row]) * static_cast<double>(sum);
        }
    }
    reduce_partials<1>(mine, partials, &st->ticket[1], [&](double (&tot)[1]) { pcg_alpha(st, tot[0], T(0)); });
}

// q = A p with the short-row stream layout, alpha = rho / p.q
template <typename T>
__global__ void __launch_bounds__(kReduceBlock) pcg_stream_spmv_kernel(int64_t rows, const int* __restrict__ rp,
                                                                       const int* __restrict__ ci,
                                                                       const T* __restrict__ v,
                                                                       const T* __restrict__ p, T* __restrict__ q,
                                                                       double* partials, PcgState* st)
{
    if (st->done)
        return;
    __shared__ T stage[kReduceBlock / 32][kStreamCap];
    double mine[1] = {0.0};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (kReduceBlock / 32);
    for (int64_t wrow = (int64_t(blockIdx.x) * (kReduceBlock / 32) + warp) * 32; wrow < rows; wrow += warps * 32)
    {
        const T sum = csr_stream_rows<T>(wrow, rows, rp, ci, v, p, stage[warp]);
        const int64_t row = wrow + lane;
        if (row < rows)
        {
            q[row] = sum;
            mine[0] += static_cast<double>(p[row]) * static_cast<double>(sum);
        }
    }
    reduce_partials<1>(mine, partials, &st->ticket[1], [&](double (&tot)[1]) { pcg_alpha(st, tot[0], T(0)); });
}

// x += alpha p, r -= alpha q, z = M^-1 r; convergence on ||r||, beta = r.z / rho.
// r is ping-ponged (r_in -> r_out) so block preconditioners read only old values.
template <typename T>
__global__ void __launch_bounds__(kReduceBlock) pcg_update_kernel(int64_t n, T* __restrict__ x,
                                                                  const T* __restrict__ p, const T* __restrict__ q,
                                                                  const T* __restrict__ r_in, T* __restrict__ r_out,
                                                                  T* __restrict__ z, int mode,
                                                                  const T* __restrict__ inv,
                                                                  const T* __restrict__ blocks, int64_t bs,
                                                                  double* partials, PcgState* st)
{
    if (st->done)
        return;
    const double alpha = st->alpha;
    double mine[2] = {0.0, 0.0};
    auto res = [&](int64_t k) {
        return static_cast<double>(static_cast<T>(static_cast<double>(r_in[k]) - alpha * static_cast<double>(q[k])));
    };
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        x[i] = static_cast<T>(static_cast<double>(x[i]) + alpha * static_cast<double>(p[i]));
        const double ri = res(i);
        const T zi = static_cast<T>(apply_precond<T>(mode, i, res, inv, blocks, bs));
        r_out[i] = static_cast<T>(ri);
        z[i] = zi;
        mine[0] += ri * static_cast<double>(zi);
        mine[1] += ri * ri;
    }
    reduce_partials<2>(mine, partials, &st->ticket[2], [&](double (&tot)[2]) {
        st->iterations += 1;
        st->residual_squared = tot[1];
        if (!isfinite(tot[1]) || tot[1] < 0.0)
        {
            st->breakdown = 1;
            st->done = 1;
            return;
        }
        if (sqrt(tot[1]) <= st->tolerance)
        {
            st->converged = 1;
            st->done = 1;
            return;
        }
        if (st->iterations >= st->max_iterations)
        {
            st->done = 1;
            return;
        }
        // betaKernel semantics (iterative_solver_kernels.cuh:204-238)
        const double rho = st->rho, next = tot[0];
        double beta = 0.0;
        if (rho == 0.0 && next == 0.0)
            beta = 0.0;
        else if (isfinite(rho) && isfinite(next) && rho > 0.0 && next > 0.0)
        {
            beta = next / rho;
            if (!isfinite(beta) || !isfinite(static_cast<double>(static_cast<T>(beta))))
            {
                st->breakdown = 1;
                st->done = 1;
                beta = 0.0;
            }
        }
        else
        {
            st->breakdown = 1;
            st->done = 1;
        }
        st->beta = beta;
        st->rho = next;
    });
}

template <typename T>
__global__ void pcg_direction_kernel(int64_t n, const T* __restrict__ z, T* __restrict__ p, const PcgState* st)
{
    if (st->done || st->iterations == 0) // the first iteration's direction is z itself (set by the init)
        return;
    const double beta = st->beta;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        p[i] = static_cast<T>(static_cast<double>(z[i]) + beta * static_cast<double>(p[i]));
}

// Condition of the CG / PCG iteration graph: another chunk while the solve is not done, at most
// max_iterations / kCgChunk + 1 chunks (the update kernel also ends the solve at max_iterations).
constexpr int kCgChunk = 4; // iterations per graph body (even: the residual ping-pong returns to r0)
__global__ void cg_continue_kernel(cudaGraphConditionalHandle handle, PcgState* st)
{
    if (threadIdx.x == 0 && blockIdx.x == 0)
    {
        const int chunks = st->chunks + 1;
        st->chunks = chunks;
        cudaGraphSetConditional(handle, !st->done && chunks <= st->max_iterations / kCgChunk + 1 ? 1u : 0u);
    }
}

__global__ void pcg_reset_kernel(PcgState* st, int max_iterations)
{
    PcgState s{};
    s.max_iterations = max_iterations;
    s.jacobi_bad_row = kNone;
    *st = s;
}

// initial and final recurrence residuals of a fixed-iteration solve; NaN marks a breakdown
__global__ void fixed_finish_kernel(const PcgState* st, double* out)
{
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    const bool bad = st->breakdown || st->nonfinite_init || st->jacobi_bad_row != kNone;
    out[0] = st->nonfinite_init ? nan : st->initial_squared;
    out[1] = bad ? nan : st->residual_squared;
}

} // namespace
} // namespace pm

struct pm_fixed_state
{
    double* residuals = nullptr; // device: initial, final squared residual
    cudaEvent_t event = nullptr;
    cudaStream_t stream = nullptr;
    int submitted = 0;
    ~pm_fixed_state()
    {
        if (event)
            cudaEventDestroy(event);
        if (residuals)
            cudaFree(residuals);
    }
};

struct pm_solver_workspace
{
    pm::DeviceBuffer buffer;
    int* host_done = nullptr; // pinned
    cudaEvent_t event = nullptr;
    // CG / PCG iteration graphs ('while' node around a chunk of iterations), one per operand set
    struct IterationGraph
    {
        const void* key[5] = {};
        int64_t n = -1;
        int shape = 0, mode = -1, value_size = 0;
        int64_t block_size = 0;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
    };
    IterationGraph graphs[4];
    int graph_next = 0;
    cudaStream_t capture_stream = nullptr;
    void drop_graphs()
    {
        for (auto& g : graphs)
        {
            if (g.exec)
                cudaGraphExecDestroy(g.exec);
            if (g.graph)
                cudaGraphDestroy(g.graph);
            g = IterationGraph{};
        }
    }
    ~pm_solver_workspace()
    {
        drop_graphs();
        if (capture_stream)
            cudaStreamDestroy(capture_stream);
        buffer.release();
        if (host_done)
            cudaFreeHost(host_done);
        if (event)
            cudaEventDestroy(event);
    }
};

namespace pm
{
namespace
{

template <typename T>
void csr_create(cudaStream_t stream, int64_t rows, int64_t cols, int64_t nnz, const int64_t* ro, const int64_t* ci,
                const T* v, pm_csr** out)
{
    if (!out)
        fail(PM_INVALID_ARGUMENT, "CSR output handle pointer is null");
    if (rows < 0 || cols < 0 || nnz < 0)
        fail(PM_INVALID_ARGUMENT, "CSRMatrix dimensions must be non-negative");
    if (nnz > INT32_MAX - 1 || rows > INT32_MAX - 1 || cols > INT32_MAX)
        fail(PM_OVERFLOW_ERROR, "CSR operand exceeds the int32 index range of the device kernels");
    if (!ro || (nnz > 0 && (!ci || !v)))
        fail(PM_INVALID_ARGUMENT, "CSR arrays must be non-null");
    auto* A = new pm_csr();
    try
    {
        A->value_size = sizeof(T);
        A->rows = rows;
        A->cols = cols;
        A->nnz = nnz;
        A->values = v;
        A->threads_per_row = pick_tpr(rows, nnz);
        PM_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&A->row_ptr), (rows + 1) * sizeof(int), stream));
        PM_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&A->col_idx), (nnz > 0 ? nnz : 1) * sizeof(int), stream));
        CsrCheck* check = nullptr;
        PM_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&check), sizeof(CsrCheck), stream));
        CsrCheck init{kNone, kNone, kNone, 0};
        PM_CUDA(cudaMemcpyAsync(check, &init, sizeof(init), cudaMemcpyHostToDevice, stream));
        validate_csr_kernel<T><<<grid_for(std::max(rows, nnz), 256, 4096), 256, 0, stream>>>(
            rows, cols, nnz, ro, ci, v, A->row_ptr, A->col_idx, check);
        PM_LAUNCH_CHECK();
        CsrCheck result{};
        PM_CUDA(cudaMemcpyAsync(&result, check, sizeof(result), cudaMemcpyDeviceToHost, stream));
        PM_CUDA(cudaFreeAsync(check, stream));
        PM_CUDA(cudaStreamSynchronize(stream));
        if (result.endpoints_bad)
            fail(PM_INVALID_ARGUMENT, "CSRMatrix row offsets must start at zero and end at nnz");
        if (result.bad_offsets_row != kNone)
        {
            std::ostringstream m;
            m << "CSRMatrix invalid row offsets at row " << result.bad_offsets_row;
            fail(PM_INVALID_ARGUMENT, m.str());
        }
        if (result.bad_column != kNone)
        {
            std::ostringstream m;
            m << "CSRMatrix column index out of range at position " << result.bad_column;
            fail(PM_INVALID_ARGUMENT, m.str());
        }
        if (result.bad_value != kNone)
        {
            std::ostringstream m;
            m << "CSRMatrix value is not finite at position " << result.bad_value;
            fail(PM_INVALID_ARGUMENT, m.str());
        }
    }
    catch (...)
    {
        cudaStreamSynchronize(stream);
        cudaFree(A->row_ptr);
        cudaFree(A->col_idx);
        delete A;
        throw;
    }
    *out = A;
}

template <typename T>
void csr_spmv(const pm_csr* A, cudaStream_t stream, const T* x, T* y)
{
    if (!A)
        fail(PM_INVALID_ARGUMENT, "CSR handle is null");
    if (A->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "spmv scalar type differs from the CSR operand");
    if (A->rows > 0 && (!y || (A->cols > 0 && !x)))
        fail(PM_INVALID_ARGUMENT, "spmv vectors must be non-null");
    if (x && x == y)
        fail(PM_INVALID_ARGUMENT, "spmv input and output data must not alias");
    launch_spmv<T>(A, x, y, stream);
}

// ------------------------------------------------------------------ SpMV autotuning
// Times every SpMV shape (row-group stream; 1, 2, 4, 8, 16, 32 lanes per row) on the operand with
// the caller's vectors and stream (one warm-up, then `reps` launches each, CUDA events) and keeps
// the fastest in the handle; the CG / PCG solvers use the same shape.  Shapes differ in the order
// of a row's additions, so the choice is part of a result's rounding; pm_csr_set_kernel pins one.
template <typename T>
int csr_autotune(pm_csr* A, cudaStream_t stream, const T* x, T* y, int reps)
{
    if (!A)
        fail(PM_INVALID_ARGUMENT, "CSR handle is null");
    if (A->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "autotune scalar type differs from the CSR operand");
    if (A->rows > 0 && (!y || (A->cols > 0 && !x)))
        fail(PM_INVALID_ARGUMENT, "autotune vectors must be non-null");
    if (x && x == y)
        fail(PM_INVALID_ARGUMENT, "spmv input and output data must not alias");
    if (A->rows == 0 || A->nnz == 0)
        return A->kernel;
    const int candidates[] = {0, 1, 2, 4, 8, 16, 32};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PM_CUDA(cudaEventCreate(&e0));
    PM_CUDA(cudaEventCreate(&e1));
    int best = A->kernel;
    float best_ms = 0.f;
    try
    {
        for (const int c : candidates)
        {
            A->kernel = c;
            launch_spmv<T>(A, x, y, stream);
            PM_CUDA(cudaEventRecord(e0, stream));
            for (int r = 0; r < reps; ++r)
                launch_spmv<T>(A, x, y, stream);
            PM_CUDA(cudaEventRecord(e1, stream));
            PM_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            PM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (c == candidates[0] || ms < best_ms)
            {
                best = c;
                best_ms = ms;
            }
        }
    }
    catch (...)
    {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    A->kernel = best;
    return best;
}

// ------------------------------------------------------------------ SpMM
// output (rows x k) = A input (cols x k), dense matrices column-major (leading dimension = rows).
// A warp owns 32 consecutive rows; their nonzero range is staged in shared memory in pieces of
// kStreamCap (columns, values, coalesced) and lane i forms row i of up to kSpmmCols output
// columns at a time, each sum from zero in storage order with one rounded multiply and one
// rounded add per term (the reference CPU spmm, sparse_ops_cpu.cpp:244-270).
constexpr int kSpmmCols = 8;

template <typename T>
__device__ __forceinline__ T mul_round(T a, T b)
{
    if constexpr (sizeof(T) == 8)
        return __dmul_rn(a, b);
    else
        return __fmul_rn(a, b);
}
template <typename T>
__device__ __forceinline__ T add_round(T a, T b)
{
    if constexpr (sizeof(T) == 8)
        return __dadd_rn(a, b);
    else
        return __fadd_rn(a, b);
}

template <typename T>
__global__ void __launch_bounds__(256) csr_spmm_kernel(int64_t rows, int64_t cols, int64_t k,
                                                       const int* __restrict__ rp, const int* __restrict__ ci,
                                                       const T* __restrict__ v, const T* __restrict__ in,
                                                       T* __restrict__ out)
{
    __shared__ int scol[8][kStreamCap];
    __shared__ T sval[8][kStreamCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * 8;
    for (int64_t wrow = (int64_t(blockIdx.x) * 8 + warp) * 32; wrow < rows; wrow += warps * 32)
    {
        const int64_t row = wrow + lane;
        const bool valid = row < rows;
        const int my_begin = valid ? rp[row] : 0;
        const int my_end = valid ? rp[row + 1] : 0;
        const int last = static_cast<int>(rows - 1 - wrow < 31 ? rows - 1 - wrow : 31);
        const int cb = __shfl_sync(0xffffffffu, my_begin, 0);
        const int ce = __shfl_sync(0xffffffffu, my_end, last);
        for (int64_t j0 = 0; j0 < k; j0 += kSpmmCols)
        {
            const int nj = k - j0 < kSpmmCols ? static_cast<int>(k - j0) : kSpmmCols;
            T sum[kSpmmCols];
#pragma unroll
            for (int j = 0; j < kSpmmCols; ++j)
                sum[j] = T(0);
            for (int base = cb; base < ce; base += kStreamCap)
            {
                const int n = ce - base < kStreamCap ? ce - base : kStreamCap;
                for (int e = lane; e < n; e += 32)
                {
                    scol[warp][e] = __ldg(ci + base + e);
                    sval[warp][e] = __ldg(v + base + e);
                }
                __syncwarp();
                const int lo = my_begin > base ? my_begin : base;
                const int hi = my_end < base + n ? my_end : base + n;
                for (int e = lo; e < hi; ++e)
                {
                    const T a = sval[warp][e - base];
                    const T* b = in + scol[warp][e - base];
#pragma unroll
                    for (int j = 0; j < kSpmmCols; ++j)
                        if (j < nj)
                            sum[j] = add_round(sum[j], mul_round(a, __ldg(b + (j0 + j) * cols)));
                }
                __syncwarp();
            }
            if (valid)
            {
#pragma unroll
                for (int j = 0; j < kSpmmCols; ++j)
                    if (j < nj)
                        out[(j0 + j) * rows + row] = sum[j];
            }
        }
    }
}

template <typename T>
void csr_spmm(const pm_csr* A, cudaStream_t stream, int64_t in_rows, int64_t in_cols, const T* in, int64_t out_rows,
              int64_t out_cols, T* out)
{
    if (!A)
        fail(PM_INVALID_ARGUMENT, "CSR handle is null");
    if (A->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "spmm scalar type differs from the CSR operand");
    if (in_rows < 0 || in_cols < 0 || out_rows < 0 || out_cols < 0)
        fail(PM_INVALID_ARGUMENT, "spmm dimensions must be non-negative");
    if (in_rows != A->cols)
    {
        std::ostringstream m;
        m << "spmm GPU dimension mismatch: CSR is " << A->rows << "x" << A->cols << ", input is " << in_rows << "x"
          << in_cols;
        fail(PM_RUNTIME_ERROR, m.str());
    }
    if (out_rows != A->rows || out_cols != in_cols)
    {
        std::ostringstream m;
        m << "spmm GPU output dimension mismatch: output is " << out_rows << "x" << out_cols << ", expected "
          << A->rows << "x" << in_cols;
        fail(PM_RUNTIME_ERROR, m.str());
    }
    if (in && in == out)
        fail(PM_INVALID_ARGUMENT, "spmm GPU input and output data must not alias");
    if (out_rows * out_cols == 0)
        return;
    if (!out || (A->nnz > 0 && !in))
        fail(PM_INVALID_ARGUMENT, "spmm matrices must be non-null");
    if (A->nnz == 0)
    {
        PM_CUDA(cudaMemsetAsync(out, 0, size_t(out_rows * out_cols) * sizeof(T), stream));
        return;
    }
    csr_spmm_kernel<T><<<grid_for(A->rows, 256, 1 << 20), 256, 0, stream>>>(A->rows, A->cols, in_cols, A->row_ptr,
                                                                             A->col_idx, static_cast<const T*>(A->values),
                                                                             in, out);
    PM_LAUNCH_CHECK();
}

template <typename T>
void launch_pcg_spmv(const pm_csr* A, const T* p, T* q, double* partials, PcgState* st, unsigned grid,
                     cudaStream_t stream)
{
    const T* v = static_cast<const T*>(A->values);
    if (use_stream(A))
    {
        pcg_stream_spmv_kernel<T><<<grid, kReduceBlock, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, p, q,
                                                                     partials, st);
        PM_LAUNCH_CHECK();
        return;
    }
    switch (lanes_per_row(A))
    {
    case 1: pcg_spmv_kernel<T, 1><<<grid, kReduceBlock, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, p, q, partials, st); break;
    case 2: pcg_spmv_kernel<T, 2><<<grid, kReduceBlock, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, p, q, partials, st); break;
    case 4: pcg_spmv_kernel<T, 4><<<grid, kReduceBlock, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, p, q, partials, st); break;
    case 8: pcg_spmv_kernel<T, 8><<<grid, kReduceBlock, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, p, q, partials, st); break;
    case 16: pcg_spmv_kernel<T, 16><<<grid, kReduceBlock, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, p, q, partials, st); break;
    default: pcg_spmv_kernel<T, 32><<<grid, kReduceBlock, 0, stream>>>(A->rows, A->row_ptr, A->col_idx, v, p, q, partials, st); break;
    }
    PM_LAUNCH_CHECK();
}

// The iteration graph of one operand set (matrix and its SpMV shape, solution, preconditioner and
// the workspace's buffer), built on first use and kept in the workspace: a CUDA graph 'while' node
// whose body is kCgChunk iterations (direction, SpMV with p.q, update with the dots) and
// cg_continue_kernel, so the device decides when the solve is done.
template <typename T>
cudaGraphExec_t cg_iteration_graph(pm_solver_workspace* ws, const pm_csr* A, T* x, const T* blocks, int64_t bs,
                                   int mode)
{
    const int64_t n = A->rows;
    const int shape = use_stream(A) ? 0 : lanes_per_row(A);
    const void* key[5] = {A, A->values, x, blocks, ws->buffer.ptr};
    for (auto& g : ws->graphs)
        if (g.exec && g.n == n && g.shape == shape && g.mode == mode && g.block_size == bs &&
            g.value_size == int(sizeof(T)) && std::equal(key, key + 5, g.key))
            return g.exec;
    if (!ws->capture_stream)
        PM_CUDA(cudaStreamCreateWithFlags(&ws->capture_stream, cudaStreamNonBlocking));
    auto& slot = ws->graphs[ws->graph_next];
    ws->graph_next = (ws->graph_next + 1) % 4;
    if (slot.exec)
        cudaGraphExecDestroy(slot.exec);
    if (slot.graph)
        cudaGraphDestroy(slot.graph);
    slot = pm_solver_workspace::IterationGraph{};
    Carver c;
    c.base = static_cast<char*>(ws->buffer.ptr);
    PcgState* st = c.take<PcgState>(1);
    double* partials = c.take<double>(3 * kMaxReduceBlocks);
    T* r0 = c.take<T>(n);
    T* r1 = c.take<T>(n);
    T* z = c.take<T>(n);
    T* p = c.take<T>(n);
    T* q = c.take<T>(n);
    T* inv = c.take<T>(n);
    const unsigned vgrid = grid_for(n, kReduceBlock, kMaxReduceBlocks);
    const unsigned sgrid = use_stream(A) ? grid_for(n, kReduceBlock, kMaxReduceBlocks)
                                         : grid_for(n * lanes_per_row(A), kReduceBlock, kMaxReduceBlocks);
    cudaGraph_t graph = nullptr;
    PM_CUDA(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle handle = 0;
    cudaGraph_t body = nullptr;
    {
        const cudaError_t made = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        const cudaError_t added = made == cudaSuccess ? cudaGraphAddNode(&node, graph, nullptr, 0, &cp) : made;
        if (added != cudaSuccess)
        {
            cudaGraphDestroy(graph);
            fail(PM_CUDA_ERROR, std::string("CUDA iterative solver: conditional graph node: ") +
                                    cudaGetErrorString(added));
        }
        body = cp.conditional.phGraph_out[0];
    }
    const cudaStream_t cs = ws->capture_stream;
    PM_CUDA(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kCgChunk; ++k)
    {
        T* r_in = (k & 1) ? r1 : r0;
        T* r_out = (k & 1) ? r0 : r1;
        pcg_direction_kernel<T><<<vgrid, kReduceBlock, 0, cs>>>(n, z, p, st);
        launch_pcg_spmv<T>(A, p, q, partials, st, sgrid, cs);
        pcg_update_kernel<T><<<vgrid, kReduceBlock, 0, cs>>>(n, x, p, q, r_in, r_out, z, mode, inv, blocks, bs,
                                                              partials, st);
    }
    cg_continue_kernel<<<1, 32, 0, cs>>>(handle, st);
    cudaGraph_t captured = nullptr;
    const cudaError_t cap = cudaStreamEndCapture(cs, &captured);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t inst = cap == cudaSuccess ? cudaGraphInstantiate(&exec, graph, 0) : cap;
    if (inst != cudaSuccess)
    {
        cudaGraphDestroy(graph);
        fail(PM_CUDA_ERROR, std::string("CUDA iterative solver: iteration graph: ") + cudaGetErrorString(inst));
    }
    std::copy(key, key + 5, slot.key);
    slot.n = n;
    slot.shape = shape;
    slot.mode = mode;
    slot.block_size = bs;
    slot.value_size = int(sizeof(T));
    slot.graph = graph;
    slot.exec = exec;
    return exec;
}

// mode: 0 = CG, 1 = Jacobi PCG, 2 = caller block inverses
template <typename T>
void solve(pm_solver_workspace* ws, cudaStream_t stream, const pm_csr* A, const T* b, T* x, const T* blocks,
           int64_t bs, const pm_solver_options* o, pm_solver_report* report, int mode)
{
    if (!ws || !A || !o || !report)
        fail(PM_INVALID_ARGUMENT, "solver arguments must be non-null");
    *report = pm_solver_report{0, 0, 0.0, 0.0};
    if (o->max_iterations < 0 || !std::isfinite(o->relative_tolerance) || o->relative_tolerance < 0.0 ||
        o->relative_tolerance > 1.0 || !std::isfinite(o->absolute_tolerance) || o->absolute_tolerance < 0.0)
        fail(PM_INVALID_ARGUMENT, "invalid CUDA iterative solver options");
    if (A->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "solver scalar type differs from the CSR operand");
    if (A->rows != A->cols)
        fail(PM_INVALID_ARGUMENT, "CUDA iterative solver requires square A and Nx1 rhs/solution");
    const int64_t n = A->rows;
    if (n > 0 && (!b || !x))
        fail(PM_INVALID_ARGUMENT, "solver vectors must be non-null");
    if (b && b == x)
        fail(PM_INVALID_ARGUMENT, "CUDA iterative solver rhs and solution must not alias");
    if (mode == 2)
    {
        if (bs <= 0 || n % bs != 0 || !blocks)
            fail(PM_INVALID_ARGUMENT, "CUDA block PCG requires complete row-major inverse diagonal blocks");
        if (static_cast<const void*>(blocks) == static_cast<const void*>(b) ||
            static_cast<const void*>(blocks) == static_cast<const void*>(x))
            fail(PM_INVALID_ARGUMENT, "CUDA block PCG inverse blocks must not alias rhs or solution");
    }
    if (n == 0)
    {
        report->converged = 1;
        return;
    }
    Carver plan;
    plan.take<PcgState>(1);
    plan.take<double>(3 * kMaxReduceBlocks);
    for (int k = 0; k < 6; ++k)
        plan.take<T>(n);
    ws->buffer.ensure(plan.offset + 256, stream, "IterativeSolverWorkspace");
    if (!ws->host_done)
        PM_CUDA(cudaMallocHost(reinterpret_cast<void**>(&ws->host_done), 2 * sizeof(PcgState)));
    if (!ws->event)
        PM_CUDA(cudaEventCreateWithFlags(&ws->event, cudaEventDisableTiming));
    Carver c;
    c.base = static_cast<char*>(ws->buffer.ptr);
    PcgState* st = c.take<PcgState>(1);
    double* partials = c.take<double>(3 * kMaxReduceBlocks);
    T* r0 = c.take<T>(n);
    T* r1 = c.take<T>(n);
    T* z = c.take<T>(n);
    T* p = c.take<T>(n);
    T* q = c.take<T>(n);
    T* inv = c.take<T>(n);

    const unsigned vgrid = grid_for(n, kReduceBlock, kMaxReduceBlocks);
    const unsigned sgrid = use_stream(A) ? grid_for(n, kReduceBlock, kMaxReduceBlocks)
                                                   : grid_for(n * lanes_per_row(A), kReduceBlock, kMaxReduceBlocks);
    pcg_reset_kernel<<<1, 1, 0, stream>>>(st, o->max_iterations);
    PM_LAUNCH_CHECK();
    if (mode == 1)
    {
        jacobi_kernel<T><<<grid_for(n, 256, 4096), 256, 0, stream>>>(n, A->row_ptr, A->col_idx,
                                                                       static_cast<const T*>(A->values), inv, st);
        PM_LAUNCH_CHECK();
    }
    launch_spmv<T>(A, x, q, stream);
    pcg_init_kernel<T><<<vgrid, kReduceBlock, 0, stream>>>(n, b, q, r0, z, p, mode, inv, blocks, bs,
                                                            o->relative_tolerance, o->absolute_tolerance, partials, st);
    PM_LAUNCH_CHECK();
    // the iterations: one launch of the operand set's iteration graph, which stops on the device
    PcgState* host = reinterpret_cast<PcgState*>(ws->host_done);
    if (o->max_iterations > 0)
    {
        const cudaGraphExec_t exec = cg_iteration_graph<T>(ws, A, x, blocks, bs, mode);
        PM_CUDA(cudaMemsetAsync(&st->chunks, 0, sizeof(int), stream));
        PM_CUDA(cudaGraphLaunch(exec, stream));
    }
    PM_CUDA(cudaMemcpyAsync(host, st, sizeof(PcgState), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaEventRecord(ws->event, stream));
    PM_CUDA(cudaEventSynchronize(ws->event));
    if (o->max_iterations > 0) // the kernels the graph ran: three per iteration and the condition
        for (int k = 0; k < host->chunks * (3 * kCgChunk + 1); ++k)
            count_launch();
    const PcgState s = *host;
    if (s.jacobi_bad_row != kNone)
    {
        std::ostringstream m;
        m << "pcg Jacobi diagonal is missing, non-positive, or near zero at row " << s.jacobi_bad_row;
        fail(PM_RUNTIME_ERROR, m.str());
    }
    if (s.nonfinite_init)
        fail(PM_RUNTIME_ERROR, "CUDA iterative solver initial residual is not finite");
    report->initial_residual = std::sqrt(s.initial_squared);
    report->iterations = s.iterations;
    report->final_residual = std::sqrt(std::max(0.0, s.residual_squared));
    report->converged = s.converged;
    if (s.breakdown)
        fail(PM_RUNTIME_ERROR, "CUDA iterative solver breakdown: matrix is not numerically SPD");
    if (!s.converged && o->require_convergence)
    {
        std::ostringstream m;
        m << "CUDA iterative solver did not converge in " << s.iterations
          << " iterations; final residual=" << report->final_residual;
        fail(PM_RUNTIME_ERROR, m.str());
    }
}

// Exactly `iterations` CG (mode 0) or Jacobi-PCG (mode 1) steps with no host check
// (fixedSolve, src/sparse/iterative_solver.cu:166-233): tolerance 0, so the device state only
// stops early on an exact zero residual or a breakdown.
template <typename T>
pm_fixed_state* fixed_solve(pm_solver_workspace* ws, cudaStream_t stream, const pm_csr* A, const T* b, T* x,
                            int iterations, int mode)
{
    if (!ws || !A)
        fail(PM_INVALID_ARGUMENT, "solver arguments must be non-null");
    if (iterations < 0)
        fail(PM_INVALID_ARGUMENT, "fixed CUDA iterative solver iterations must be non-negative");
    if (A->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "solver scalar type differs from the CSR operand");
    if (A->rows != A->cols)
        fail(PM_INVALID_ARGUMENT, "CUDA iterative solver requires square A and Nx1 rhs/solution");
    const int64_t n = A->rows;
    if (n > 0 && (!b || !x))
        fail(PM_INVALID_ARGUMENT, "solver vectors must be non-null");
    if (b && b == x)
        fail(PM_INVALID_ARGUMENT, "CUDA iterative solver rhs and solution must not alias");
    auto* state = new pm_fixed_state();
    try
    {
        state->stream = stream;
        state->submitted = iterations;
        PM_CUDA(cudaMalloc(reinterpret_cast<void**>(&state->residuals), 2 * sizeof(double)));
        PM_CUDA(cudaEventCreateWithFlags(&state->event, cudaEventDisableTiming));
        if (n == 0)
        {
            PM_CUDA(cudaMemsetAsync(state->residuals, 0, 2 * sizeof(double), stream));
            PM_CUDA(cudaEventRecord(state->event, stream));
            return state;
        }
        Carver plan;
        plan.take<PcgState>(1);
        plan.take<double>(3 * kMaxReduceBlocks);
        for (int k = 0; k < 6; ++k)
            plan.take<T>(n);
        ws->buffer.ensure(plan.offset + 256, stream, "IterativeSolverWorkspace");
        Carver c;
        c.base = static_cast<char*>(ws->buffer.ptr);
        PcgState* st = c.take<PcgState>(1);
        double* partials = c.take<double>(3 * kMaxReduceBlocks);
        T* r0 = c.take<T>(n);
        T* r1 = c.take<T>(n);
        T* z = c.take<T>(n);
        T* p = c.take<T>(n);
        T* q = c.take<T>(n);
        T* inv = c.take<T>(n);
        const unsigned vgrid = grid_for(n, kReduceBlock, kMaxReduceBlocks);
        const unsigned sgrid = use_stream(A) ? grid_for(n, kReduceBlock, kMaxReduceBlocks)
                                                       : grid_for(n * lanes_per_row(A), kReduceBlock, kMaxReduceBlocks);
        pcg_reset_kernel<<<1, 1, 0, stream>>>(st, iterations);
        PM_LAUNCH_CHECK();
        if (mode == 1)
        {
            jacobi_kernel<T><<<grid_for(n, 256, 4096), 256, 0, stream>>>(n, A->row_ptr, A->col_idx,
                                                                           static_cast<const T*>(A->values), inv, st);
            PM_LAUNCH_CHECK();
        }
        launch_spmv<T>(A, x, q, stream);
        pcg_init_kernel<T><<<vgrid, kReduceBlock, 0, stream>>>(n, b, q, r0, z, p, mode, inv, static_cast<const T*>(nullptr),
                                                                0, 0.0, 0.0, partials, st);
        PM_LAUNCH_CHECK();
        T* r_in = r0;
        T* r_out = r1;
        for (int k = 0; k < iterations; ++k)
        {
            if (k > 0)
            {
                pcg_direction_kernel<T><<<vgrid, kReduceBlock, 0, stream>>>(n, z, p, st);
                PM_LAUNCH_CHECK();
            }
            launch_pcg_spmv<T>(A, p, q, partials, st, sgrid, stream);
            pcg_update_kernel<T><<<vgrid, kReduceBlock, 0, stream>>>(n, x, p, q, r_in, r_out, z, mode, inv,
                                                                      static_cast<const T*>(nullptr), 0, partials, st);
            PM_LAUNCH_CHECK();
            std::swap(r_in, r_out);
        }
        fixed_finish_kernel<<<1, 1, 0, stream>>>(st, state->residuals);
        PM_LAUNCH_CHECK();
        PM_CUDA(cudaEventRecord(state->event, stream));
    }
    catch (...)
    {
        delete state;
        throw;
    }
    return state;
}

void fixed_finalize(const pm_fixed_state* state, const pm_solver_options* o, pm_solver_report* report)
{
    if (!o || !report)
        fail(PM_INVALID_ARGUMENT, "finalize arguments must be non-null");
    if (!std::isfinite(o->relative_tolerance) || o->relative_tolerance < 0.0 || o->relative_tolerance > 1.0 ||
        !std::isfinite(o->absolute_tolerance) || o->absolute_tolerance < 0.0)
        fail(PM_INVALID_ARGUMENT, "invalid CUDA iterative solver options");
    if (!state || !state->event)
        fail(PM_LOGIC_ERROR, "fixed CUDA iterative solver state is empty or closed");
    const cudaError_t status = cudaEventQuery(state->event);
    if (status == cudaErrorNotReady)
        fail(PM_LOGIC_ERROR, "finalizeIterativeSolverReport requires caller stream synchronization");
    PM_CUDA(status);
    double host[2] = {0.0, 0.0};
    PM_CUDA(cudaMemcpy(host, state->residuals, sizeof(host), cudaMemcpyDeviceToHost));
    if (!std::isfinite(host[0]) || !std::isfinite(host[1]) || host[0] < 0.0 || host[1] < 0.0)
        fail(PM_RUNTIME_ERROR, "fixed CUDA iterative solver breakdown: residual is not finite");
    *report = pm_solver_report{0, 0, 0.0, 0.0};
    report->iterations = state->submitted;
    report->initial_residual = std::sqrt(host[0]);
    report->final_residual = std::sqrt(host[1]);
    const double tolerance = std::max(o->absolute_tolerance, o->relative_tolerance * report->initial_residual);
    report->converged = report->final_residual <= tolerance;
    if (!report->converged && o->require_convergence)
    {
        std::ostringstream m;
        m << "fixed CUDA iterative solver did not converge in " << report->iterations
          << " iterations; final residual=" << report->final_residual;
        fail(PM_RUNTIME_ERROR, m.str());
    }
}

} // namespace
} // namespace pm

extern "C" {

int pm_csr_create_f32(pm_stream_t stream, int64_t rows, int64_t cols, int64_t nnz, const int64_t* ro,
                      const int64_t* ci, const float* v, pm_csr** out)
{
    return pm::guarded([&] { pm::csr_create<float>(stream, rows, cols, nnz, ro, ci, v, out); });
}
int pm_csr_create_f64(pm_stream_t stream, int64_t rows, int64_t cols, int64_t nnz, const int64_t* ro,
                      const int64_t* ci, const double* v, pm_csr** out)
{
    return pm::guarded([&] { pm::csr_create<double>(stream, rows, cols, nnz, ro, ci, v, out); });
}
#define PM_FIXED(KIND, MODE, SFX, T)                                                                              \
    int pm_##KIND##_fixed_iterations_async_##SFX(pm_solver_workspace* ws, pm_stream_t s, const pm_csr* A, const T* b, \
                                                  T* x, int iterations, pm_fixed_state** state)                    \
    {                                                                                                              \
        return pm::guarded([&] {                                                                                   \
            if (!state)                                                                                            \
                pm::fail(PM_INVALID_ARGUMENT, "fixed solver state pointer is null");                               \
            *state = pm::fixed_solve<T>(ws, s, A, b, x, iterations, MODE);                                         \
        });                                                                                                        \
    }
PM_FIXED(cg, 0, f32, float)
PM_FIXED(cg, 0, f64, double)
PM_FIXED(pcg, 1, f32, float)
PM_FIXED(pcg, 1, f64, double)
#undef PM_FIXED

int pm_fixed_state_finalize(const pm_fixed_state* state, const pm_solver_options* o, pm_solver_report* report)
{
    return pm::guarded([&] { pm::fixed_finalize(state, o, report); });
}

void pm_fixed_state_destroy(pm_fixed_state* state)
{
    if (state)
    {
        if (state->event)
            cudaEventSynchronize(state->event);
        delete state;
    }
}

void pm_csr_destroy(pm_csr* A)
{
    if (A)
    {
        cudaFree(A->row_ptr);
        cudaFree(A->col_idx);
        delete A;
    }
}
int pm_csr_set_values(pm_csr* A, const void* values)
{
    return pm::guarded([&] {
        if (!A || (A->nnz > 0 && !values))
            pm::fail(PM_INVALID_ARGUMENT, "CSR handle and values must be non-null");
        A->values = values;
    });
}
int pm_csr_spmv_f32(const pm_csr* A, pm_stream_t stream, const float* x, float* y)
{
    return pm::guarded([&] { pm::csr_spmv<float>(A, stream, x, y); });
}
int pm_csr_spmv_f64(const pm_csr* A, pm_stream_t stream, const double* x, double* y)
{
    return pm::guarded([&] { pm::csr_spmv<double>(A, stream, x, y); });
}

int pm_csr_spmm_f32(const pm_csr* A, pm_stream_t stream, int64_t input_rows, int64_t input_cols, const float* input,
                    int64_t output_rows, int64_t output_cols, float* output)
{
    return pm::guarded(
        [&] { pm::csr_spmm<float>(A, stream, input_rows, input_cols, input, output_rows, output_cols, output); });
}
int pm_csr_spmm_f64(const pm_csr* A, pm_stream_t stream, int64_t input_rows, int64_t input_cols, const double* input,
                    int64_t output_rows, int64_t output_cols, double* output)
{
    return pm::guarded(
        [&] { pm::csr_spmm<double>(A, stream, input_rows, input_cols, input, output_rows, output_cols, output); });
}

int pm_csr_autotune_f32(pm_csr* A, pm_stream_t stream, const float* x, float* y, int* kernel)
{
    return pm::guarded([&] {
        const int k = pm::csr_autotune<float>(A, stream, x, y, 5);
        if (kernel)
            *kernel = k;
    });
}
int pm_csr_autotune_f64(pm_csr* A, pm_stream_t stream, const double* x, double* y, int* kernel)
{
    return pm::guarded([&] {
        const int k = pm::csr_autotune<double>(A, stream, x, y, 5);
        if (kernel)
            *kernel = k;
    });
}
int pm_csr_set_kernel(pm_csr* A, int kernel)
{
    return pm::guarded([&] {
        if (!A)
            pm::fail(PM_INVALID_ARGUMENT, "CSR handle is null");
        if (!(kernel == -1 || kernel == 0 || kernel == 1 || kernel == 2 || kernel == 4 || kernel == 8 ||
              kernel == 16 || kernel == 32))
            pm::fail(PM_INVALID_ARGUMENT, "SpMV kernel must be -1 (heuristic), 0 (row-group stream) or 1, 2, 4, "
                                          "8, 16, 32 lanes per row");
        A->kernel = kernel;
    });
}
int pm_csr_kernel(const pm_csr* A, int* kernel, int* heuristic_lanes)
{
    return pm::guarded([&] {
        if (!A)
            pm::fail(PM_INVALID_ARGUMENT, "CSR handle is null");
        if (kernel)
            *kernel = A->kernel;
        if (heuristic_lanes)
            *heuristic_lanes = A->threads_per_row;
    });
}

int pm_solver_workspace_create(pm_solver_workspace** out)
{
    return pm::guarded([&] {
        if (!out)
            pm::fail(PM_INVALID_ARGUMENT, "workspace output pointer is null");
        *out = new pm_solver_workspace();
    });
}
void pm_solver_workspace_destroy(pm_solver_workspace* ws) { delete ws; }
int pm_solver_workspace_close(pm_solver_workspace* ws)
{
    return pm::guarded([&] {
        if (!ws)
            pm::fail(PM_INVALID_ARGUMENT, "workspace is null");
        ws->drop_graphs(); // they hold pointers into the buffer released here
        ws->buffer.release();
    });
}

#define PM_SOLVER_API(SFX, T)                                                                                      \
    int pm_cg_##SFX(pm_solver_workspace* ws, pm_stream_t s, const pm_csr* A, const T* b, T* x,                      \
                    const pm_solver_options* o, pm_solver_report* r)                                                \
    {                                                                                                               \
        return pm::guarded([&] { pm::solve<T>(ws, s, A, b, x, nullptr, 0, o, r, 0); });                            \
    }                                                                                                               \
    int pm_pcg_##SFX(pm_solver_workspace* ws, pm_stream_t s, const pm_csr* A, const T* b, T* x,                     \
                     const pm_solver_options* o, pm_solver_report* r)                                               \
    {                                                                                                               \
        return pm::guarded([&] { pm::solve<T>(ws, s, A, b, x, nullptr, 0, o, r, o && o->use_jacobi ? 1 : 0); });  \
    }                                                                                                               \
    int pm_block_pcg_##SFX(pm_solver_workspace* ws, pm_stream_t s, const pm_csr* A, const T* b, T* x,               \
                           const T* blocks, int64_t bs, const pm_solver_options* o, pm_solver_report* r)            \
    {                                                                                                               \
        return pm::guarded([&] { pm::solve<T>(ws, s, A, b, x, blocks, bs, o, r, 2); });                            \
    }

PM_SOLVER_API(f32, float)
PM_SOLVER_API(f64, double)

} // extern "C"
