// Dense FP64 Cholesky solve of an assembled reduced Schur system: the device counterpart of the
// reference's DenseCpu backend (src/optimization/block_schur_dense_solver.h:88-262), for reduced
// systems small enough to hold densely (near-dense small systems, where a direct solve beats PCG).
//
// Layout: A is n x n row-major in FP64; only its lower triangle is read and overwritten by L.
// Factorisation is right-looking in column panels of kPanel:
//   potrf  -- one CTA factors the panel's diagonal block in shared memory;
//   trsm   -- a thread per row below it solves L21 = A21 L11^-T;
//   update -- 64 x 64 tiles of the trailing lower triangle subtract L21 L21^T (FP64 SIMT).
// A pivot that is not positive and finite stops the factorisation: status = 1 + its column.
// The triangular solves run in one CTA, blocked by kPanel rows.
#include "pm_schur.cuh"

namespace pm
{
namespace
{

constexpr int kPanel = 32;
constexpr int kTile = 64;
constexpr int kSolveThreads = 1024;

template <typename T>
__global__ void dense_from_blocks_kernel(int64_t P, int bp, const int* __restrict__ row_ptr,
                                         const int* __restrict__ block_col, const T* __restrict__ S, int64_t n,
                                         double* __restrict__ A)
{
    const int bpp = bp * bp;
    for (int64_t p = blockIdx.x; p < P; p += gridDim.x)
        for (int64_t k = int64_t(row_ptr[p]) * bpp + threadIdx.x; k < int64_t(row_ptr[p + 1]) * bpp; k += blockDim.x)
        {
            const int64_t b = k / bpp;
            const int e = static_cast<int>(k - b * bpp), r = e / bp, c = e % bp;
            A[(p * bp + r) * n + int64_t(block_col[b]) * bp + c] = static_cast<double>(S[k]);
        }
}

// diagonal block [k0, k0 + kb) of the panel, unblocked in shared memory
__global__ void __launch_bounds__(kPanel * kPanel) dense_potrf_kernel(int64_t n, int64_t k0, int kb, double* A,
                                                                      int* status)
{
    __shared__ double a[kPanel][kPanel + 1];
    __shared__ int bad;
    if (*status != 0)
        return;
    const int r = threadIdx.x / kPanel, c = threadIdx.x % kPanel;
    if (threadIdx.x == 0)
        bad = 0;
    if (r < kb && c <= r)
        a[r][c] = A[(k0 + r) * n + k0 + c];
    __syncthreads();
    for (int j = 0; j < kb; ++j)
    {
        if (threadIdx.x == 0)
        {
            const double pivot = a[j][j];
            if (!(pivot > 0.0) || !isfinite(pivot))
                bad = static_cast<int>(k0 + j) + 1;
            else
                a[j][j] = sqrt(pivot);
        }
        __syncthreads();
        if (bad)
            break;
        if (c == j && r > j && r < kb)
            a[r][j] = a[r][j] / a[j][j];
        __syncthreads();
        if (r > j && r < kb && c > j && c <= r)
            a[r][c] = __dadd_rn(a[r][c], -__dmul_rn(a[r][j], a[c][j]));
        __syncthreads();
    }
    if (bad)
    {
        if (threadIdx.x == 0)
            *status = bad;
        return;
    }
    if (r < kb && c <= r)
        A[(k0 + r) * n + k0 + c] = a[r][c];
}

// rows i >= k0 + kb of the panel: x L11^T = a, thread per row
__global__ void __launch_bounds__(256) dense_trsm_kernel(int64_t n, int64_t k0, int kb, double* A,
                                                         const int* status)
{
    __shared__ double l[kPanel][kPanel + 1];
    if (*status != 0)
        return;
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x)
    {
        const int r = e / kb, c = e % kb;
        l[r][c] = c <= r ? A[(k0 + r) * n + k0 + c] : 0.0;
    }
    __syncthreads();
    const int64_t i = k0 + kb + int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double x[kPanel];
    double* row = A + i * n + k0;
#pragma unroll
    for (int t = 0; t < kPanel; ++t)
        if (t < kb)
            x[t] = row[t];
#pragma unroll
    for (int t = 0; t < kPanel; ++t)
    {
        if (t >= kb)
            break;
        double v = x[t];
#pragma unroll
        for (int s = 0; s < t; ++s)
            v = __dadd_rn(v, -__dmul_rn(x[s], l[t][s]));
        x[t] = v / l[t][t];
    }
#pragma unroll
    for (int t = 0; t < kPanel; ++t)
        if (t < kb)
            row[t] = x[t];
}

// trailing lower triangle: A[i][j] -= sum_t L[i][k0 + t] L[j][k0 + t], 64 x 64 tiles (I >= J),
// 256 threads with 4 x 4 entries each
__global__ void __launch_bounds__(256) dense_update_kernel(int64_t n, int64_t k0, int kb, double* A,
                                                           const int* status)
{
    __shared__ double li[kTile][kPanel + 1];
    __shared__ double lj[kTile][kPanel + 1];
    if (*status != 0)
        return;
    const int64_t base = k0 + kb;
    // tile (I, J) with J <= I from the linear block index
    const int64_t t = blockIdx.x;
    int64_t I = static_cast<int64_t>((sqrt(8.0 * double(t) + 1.0) - 1.0) / 2.0);
    while ((I + 1) * (I + 2) / 2 <= t)
        ++I;
    while (I * (I + 1) / 2 > t)
        --I;
    const int64_t J = t - I * (I + 1) / 2;
    const int64_t i0 = base + I * kTile, j0 = base + J * kTile;
    for (int e = threadIdx.x; e < kTile * kPanel; e += blockDim.x)
    {
        const int r = e / kPanel, c = e % kPanel;
        li[r][c] = (i0 + r < n && c < kb) ? A[(i0 + r) * n + k0 + c] : 0.0;
        lj[r][c] = (j0 + r < n && c < kb) ? A[(j0 + r) * n + k0 + c] : 0.0;
    }
    __syncthreads();
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
            acc[a][b] = 0.0;
    for (int s = 0; s < kb; ++s)
    {
        double xi[4], xj[4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
        {
            xi[a] = li[tr + 16 * a][s];
            xj[a] = lj[tc + 16 * a][s];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
                acc[a][b] = fma(xi[a], xj[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
        {
            const int64_t i = i0 + tr + 16 * a, j = j0 + tc + 16 * b;
            if (i < n && j <= i)
                A[i * n + j] -= acc[a][b];
        }
}

// L y = b, then L^T x = y, in place in x; one CTA, blocked by kPanel rows
__global__ void __launch_bounds__(kSolveThreads) dense_solve_kernel(int64_t n, const double* __restrict__ A,
                                                                    double* __restrict__ x, const int* status)
{
    if (*status != 0)
        return;
    for (int64_t k0 = 0; k0 < n; k0 += kPanel)
    {
        const int kb = static_cast<int>(n - k0 < kPanel ? n - k0 : kPanel);
        if (threadIdx.x == 0)
            for (int t = 0; t < kb; ++t)
            {
                double v = x[k0 + t];
                for (int s = 0; s < t; ++s)
                    v = __dadd_rn(v, -__dmul_rn(A[(k0 + t) * n + k0 + s], x[k0 + s]));
                x[k0 + t] = v / A[(k0 + t) * n + k0 + t];
            }
        __syncthreads();
        for (int64_t i = k0 + kb + threadIdx.x; i < n; i += blockDim.x)
        {
            double v = x[i];
            for (int s = 0; s < kb; ++s)
                v = __dadd_rn(v, -__dmul_rn(A[i * n + k0 + s], x[k0 + s]));
            x[i] = v;
        }
        __syncthreads();
    }
    for (int64_t k1 = n; k1 > 0; k1 -= kPanel)
    {
        const int64_t k0 = k1 - kPanel > 0 ? k1 - kPanel : 0;
        const int kb = static_cast<int>(k1 - k0);
        if (threadIdx.x == 0)
            for (int t = kb - 1; t >= 0; --t)
            {
                double v = x[k0 + t];
                for (int s = t + 1; s < kb; ++s)
                    v = __dadd_rn(v, -__dmul_rn(A[(k0 + s) * n + k0 + t], x[k0 + s]));
                x[k0 + t] = v / A[(k0 + t) * n + k0 + t];
            }
        __syncthreads();
        for (int64_t i = threadIdx.x; i < k0; i += blockDim.x)
        {
            double v = x[i];
            for (int s = 0; s < kb; ++s)
                v = __dadd_rn(v, -__dmul_rn(A[(k0 + s) * n + i], x[k0 + s]));
            x[i] = v;
        }
        __syncthreads();
    }
}

} // namespace

template <typename T>
void dense_schur_factor_solve(cudaStream_t stream, int64_t P, int bp, const int* row_ptr, const int* block_col,
                              const T* S, double* A, double* x, int* status)
{
    const int64_t n = P * bp;
    PM_CUDA(cudaMemsetAsync(status, 0, sizeof(int), stream));
    PM_CUDA(cudaMemsetAsync(A, 0, size_t(n * n) * sizeof(double), stream));
    dense_from_blocks_kernel<T><<<grid_for(P, 1, 1 << 20), 256, 0, stream>>>(P, bp, row_ptr, block_col, S, n, A);
    PM_LAUNCH_CHECK();
    for (int64_t k0 = 0; k0 < n; k0 += kPanel)
    {
        const int kb = static_cast<int>(n - k0 < kPanel ? n - k0 : kPanel);
        dense_potrf_kernel<<<1, kPanel * kPanel, 0, stream>>>(n, k0, kb, A, status);
        PM_LAUNCH_CHECK();
        const int64_t rest = n - k0 - kb;
        if (rest <= 0)
            break;
        dense_trsm_kernel<<<grid_for(rest, 256), 256, 0, stream>>>(n, k0, kb, A, status);
        PM_LAUNCH_CHECK();
        const int64_t tiles = (rest + kTile - 1) / kTile;
        dense_update_kernel<<<static_cast<unsigned>(tiles * (tiles + 1) / 2), 256, 0, stream>>>(n, k0, kb, A, status);
        PM_LAUNCH_CHECK();
    }
    dense_solve_kernel<<<1, kSolveThreads, 0, stream>>>(n, A, x, status);
    PM_LAUNCH_CHECK();
}

template void dense_schur_factor_solve<float>(cudaStream_t, int64_t, int, const int*, const int*, const float*,
                                              double*, double*, int*);
template void dense_schur_factor_solve<double>(cudaStream_t, int64_t, int, const int*, const int*, const double*,
                                               double*, double*, int*);

} // namespace pm
