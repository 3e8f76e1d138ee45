// Dense FP64 Cholesky solve of an assembled reduced Schur system: the device counterpart of the
// reference's DenseCpu backend (src/optimization/block_schur_dense_solver.h:88-262), for reduced
// systems small enough to hold densely (near-dense small systems, where a direct solve beats PCG).
//
// Layout: A is n x n row-major in FP64; only its lower triangle is read and overwritten by L.
// Factorisation is right-looking in column panels of kPanel, two launches per panel:
//   trsm   -- a warp per row below the diagonal block solves L21 = A21 L11^-T;
//   update -- 64 x 64 tiles of the trailing lower triangle subtract L21 L21^T (FP64 SIMT); the
//             CTA of tile (0, 0), which finishes the next panel's diagonal block, then factors it
//             in shared memory (the first panel's block has a launch of its own).
// A pivot that is not positive and finite stops the factorisation: status = 1 + its column.
// The triangular solves are blocked by kSolvePanel unknowns: one CTA per diagonal block, then
// one wide launch per panel for the rows it updates.
#include "pm_schur.cuh"

namespace pm
{
namespace
{

constexpr int kPanel = 32;
constexpr int kTile = 64;
constexpr int kSolvePanel = 128;
constexpr int kSolveThreads = 256;
constexpr int kBlockLd = kSolvePanel + 1;
constexpr size_t kBlockSmem = size_t(kSolvePanel * kBlockLd + 2 * kSolvePanel) * sizeof(double);

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

// unblocked Cholesky of the kb x kb block a (lower triangle) by the CTA's threads; returns
// 1 + the global column of the first pivot that is not positive and finite, else 0
__device__ int factor_block(double (*a)[kPanel + 1], int kb, int64_t k0, int* bad)
{
    const int tid = threadIdx.x, threads = blockDim.x;
    if (tid == 0)
        *bad = 0;
    __syncthreads();
    for (int j = 0; j < kb; ++j)
    {
        if (tid == 0)
        {
            const double pivot = a[j][j];
            if (!(pivot > 0.0) || !isfinite(pivot))
                *bad = static_cast<int>(k0 + j) + 1;
            else
                a[j][j] = sqrt(pivot);
        }
        __syncthreads();
        if (*bad)
            break;
        for (int r = j + 1 + tid; r < kb; r += threads)
            a[r][j] = a[r][j] / a[j][j];
        __syncthreads();
        for (int e = tid; e < kPanel * kPanel; e += threads)
        {
            const int r = e / kPanel, c = e % kPanel;
            if (r > j && r < kb && c > j && c <= r)
                a[r][c] = __dadd_rn(a[r][c], -__dmul_rn(a[r][j], a[c][j]));
        }
        __syncthreads();
    }
    return *bad;
}

// factor the kb x kb diagonal block at (k0, k0) of A in place; a failed pivot sets *status
__device__ void factor_block_in_place(int64_t n, int64_t k0, int kb, double* A, int* status)
{
    __shared__ double a[kPanel][kPanel + 1];
    __shared__ int bad;
    for (int e = threadIdx.x; e < kPanel * kPanel; e += blockDim.x)
    {
        const int r = e / kPanel, c = e % kPanel;
        if (r < kb && c <= r)
            a[r][c] = A[(k0 + r) * n + k0 + c];
    }
    __syncthreads();
    if (factor_block(a, kb, k0, &bad))
    {
        if (threadIdx.x == 0)
            *status = bad;
        return;
    }
    for (int e = threadIdx.x; e < kPanel * kPanel; e += blockDim.x)
    {
        const int r = e / kPanel, c = e % kPanel;
        if (r < kb && c <= r)
            A[(k0 + r) * n + k0 + c] = a[r][c];
    }
}

// diagonal block [k0, k0 + kb) of the first panel (every later panel's block is factored by the
// update kernel that finishes it)
__global__ void __launch_bounds__(256) dense_potrf_kernel(int64_t n, int64_t k0, int kb, double* A, int* status)
{
    if (*status != 0)
        return;
    factor_block_in_place(n, k0, kb, A, status);
}

// rows i >= k0 + kb of the panel: x L11^T = a, a warp per row with lane t holding x_t; column
// sweep: step s scales x_s by 1 / L_ss on lane s, broadcasts it, and lanes t > s subtract
// x_s L_ts (so each x_t sees its terms in increasing s, then its scaling)
__global__ void __launch_bounds__(256) dense_trsm_kernel(int64_t n, int64_t k0, int kb, double* A,
                                                         const int* status)
{
    __shared__ double l[kPanel][kPanel + 1];
    __shared__ double rdiag[kPanel];
    if (*status != 0)
        return;
    const int lane = threadIdx.x % 32;
    const int64_t i = k0 + kb + (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    double* row = A + i * n + k0;
    double v = (i < n && lane < kb) ? row[lane] : 0.0;
    for (int e = threadIdx.x; e < kPanel * kPanel; e += blockDim.x)
    {
        const int r = e / kPanel, c = e % kPanel;
        l[r][c] = (r < kb && c <= r) ? A[(k0 + r) * n + k0 + c] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x < kb)
        rdiag[threadIdx.x] = 1.0 / l[threadIdx.x][threadIdx.x];
    __syncthreads();
    if (i >= n)
        return;
#pragma unroll
    for (int s = 0; s < kPanel; ++s)
    {
        if (s >= kb)
            break;
        if (lane == s)
            v = __dmul_rn(v, rdiag[s]);
        const double xs = __shfl_sync(0xffffffffu, v, s);
        if (lane > s && lane < kb)
            v = __dadd_rn(v, -__dmul_rn(xs, l[lane][s]));
    }
    if (lane < kb)
        row[lane] = v;
}

// trailing lower triangle: A[i][j] -= sum_t L[i][k0 + t] L[j][k0 + t], 64 x 64 tiles (I >= J),
// 256 threads with 4 x 4 entries each; tile (0, 0) then factors the next panel's diagonal block
__global__ void __launch_bounds__(256) dense_update_kernel(int64_t n, int64_t k0, int kb, double* A,
                                                           int* status)
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
    // the next panel's diagonal block lies in tile (0, 0), which no other CTA writes: factor it
    // here once the tile is final
    if (t == 0)
    {
        __syncthreads();
        factor_block_in_place(n, base, n - base < kPanel ? static_cast<int>(n - base) : kPanel, A, status);
    }
}

// fixed butterfly: every lane ends with the same, order-independent-of-lane sum
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int k = 16; k > 0; k >>= 1)
        v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, k));
    return v;
}

// Triangular solves L y = b, then L^T x = y, in place in x, blocked by kSolvePanel unknowns: one
// CTA stages a panel's diagonal block in shared memory and solves it (32-row column sweeps in a
// warp, the rest of the block updated between them; the sweeps multiply by the diagonal's
// reciprocals, computed in parallel beforehand, to keep divisions off the dependency chain), then
// a wide launch removes the panel from every remaining unknown.

// the panel's diagonal block, lower triangle, staged in shared memory with row stride kBlockLd
// (a warp per row, four rows per pass, so each thread keeps 16 loads in flight), and the
// reciprocals of its diagonal
__device__ __forceinline__ void stage_block(int64_t n, int64_t k0, int kb, const double* __restrict__ A,
                                            double* __restrict__ L, double* __restrict__ rdiag)
{
    constexpr int kWarps = kSolveThreads / 32;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int r0 = warp; r0 < kb; r0 += 4 * kWarps)
    {
        double v[4][kSolvePanel / 32];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < kSolvePanel / 32; ++b)
            {
                const int r = r0 + a * kWarps, c = b * 32 + lane;
                v[a][b] = (r < kb && c <= r) ? A[(k0 + r) * n + k0 + c] : 0.0;
            }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < kSolvePanel / 32; ++b)
            {
                const int r = r0 + a * kWarps, c = b * 32 + lane;
                if (r < kb && c <= r)
                    L[r * kBlockLd + c] = v[a][b];
            }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < kb; r += blockDim.x)
        rdiag[r] = 1.0 / L[r * kBlockLd + r];
}

// forward, diagonal block [k0, k0 + kb)
__global__ void __launch_bounds__(kSolveThreads) dense_forward_block_kernel(int64_t n, int64_t k0, int kb,
                                                                            const double* __restrict__ A,
                                                                            double* __restrict__ x, const int* status)
{
    extern __shared__ double staged[];
    double* L = staged;
    double* xs = staged + kSolvePanel * kBlockLd;
    double* rdiag = xs + kSolvePanel;
    if (*status != 0)
        return;
    stage_block(n, k0, kb, A, L, rdiag);
    for (int r = threadIdx.x; r < kb; r += blockDim.x)
        xs[r] = x[k0 + r];
    __syncthreads();
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int q = 0; q < kb; q += 32)
    {
        const int qb = kb - q < 32 ? kb - q : 32;
        if (warp == 0)
        {
            // lane t holds row q + t of the sub-block: lrow[s] = L[q + t][q + s], s <= t
            double lrow[32];
#pragma unroll
            for (int s = 0; s < 32; ++s)
                lrow[s] = (lane < qb && s <= lane) ? L[(q + lane) * kBlockLd + q + s] : 0.0;
            double v = lane < qb ? xs[q + lane] : 0.0;
#pragma unroll
            for (int s = 0; s < 32; ++s)
            {
                if (s >= qb)
                    break;
                if (lane == s)
                    v = __dmul_rn(v, rdiag[q + s]);
                const double ys = __shfl_sync(0xffffffffu, v, s);
                if (lane > s)
                    v = __dadd_rn(v, -__dmul_rn(lrow[s], ys));
            }
            if (lane < qb)
                xs[q + lane] = v;
        }
        __syncthreads();
        for (int r = q + qb + warp; r < kb; r += kSolveThreads / 32)
        {
            const double p = warp_sum(lane < qb ? __dmul_rn(L[r * kBlockLd + q + lane], xs[q + lane]) : 0.0);
            if (lane == 0)
                xs[r] = __dadd_rn(xs[r], -p);
        }
        __syncthreads();
    }
    for (int r = threadIdx.x; r < kb; r += blockDim.x)
        x[k0 + r] = xs[r];
}

// forward, rows i >= k0 + kb: x_i -= L[i][k0 : k0 + kb] . y[k0 : k0 + kb], a warp per row
__global__ void __launch_bounds__(kSolveThreads) dense_forward_rows_kernel(int64_t n, int64_t k0, int kb,
                                                                           const double* __restrict__ A,
                                                                           double* __restrict__ x, const int* status)
{
    __shared__ double ys[kSolvePanel];
    if (*status != 0)
        return;
    for (int r = threadIdx.x; r < kb; r += blockDim.x)
        ys[r] = x[k0 + r];
    __syncthreads();
    const int lane = threadIdx.x % 32;
    const int64_t warps = int64_t(gridDim.x) * (kSolveThreads / 32);
    for (int64_t i = k0 + kb + int64_t(blockIdx.x) * (kSolveThreads / 32) + threadIdx.x / 32; i < n; i += warps)
    {
        const double* row = A + i * n + k0;
        double p = 0.0;
#pragma unroll
        for (int c = 0; c < kSolvePanel / 32; ++c)
            if (c * 32 + lane < kb)
                p = __dadd_rn(p, __dmul_rn(row[c * 32 + lane], ys[c * 32 + lane]));
        p = warp_sum(p);
        if (lane == 0)
            x[i] = __dadd_rn(x[i], -p);
    }
}

// backward, diagonal block [k0, k0 + kb): L11^T z = x, 32-row sweeps from the bottom
__global__ void __launch_bounds__(kSolveThreads) dense_backward_block_kernel(int64_t n, int64_t k0, int kb,
                                                                             const double* __restrict__ A,
                                                                             double* __restrict__ x, const int* status)
{
    extern __shared__ double staged[];
    double* L = staged;
    double* xs = staged + kSolvePanel * kBlockLd;
    double* rdiag = xs + kSolvePanel;
    if (*status != 0)
        return;
    stage_block(n, k0, kb, A, L, rdiag);
    for (int r = threadIdx.x; r < kb; r += blockDim.x)
        xs[r] = x[k0 + r];
    __syncthreads();
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int q = ((kb - 1) / 32) * 32; q >= 0; q -= 32)
    {
        const int qb = kb - q < 32 ? kb - q : 32;
        if (warp == 0)
        {
            // lane t holds column q + t of the sub-block: lcol[s] = L[q + s][q + t], s >= t
            double lcol[32];
#pragma unroll
            for (int s = 0; s < 32; ++s)
                lcol[s] = (lane < qb && s < qb && s >= lane) ? L[(q + s) * kBlockLd + q + lane] : 0.0;
            double v = lane < qb ? xs[q + lane] : 0.0;
#pragma unroll
            for (int s = 31; s >= 0; --s)
            {
                if (s >= qb)
                    continue;
                if (lane == s)
                    v = __dmul_rn(v, rdiag[q + s]);
                const double zs = __shfl_sync(0xffffffffu, v, s);
                if (lane < s)
                    v = __dadd_rn(v, -__dmul_rn(lcol[s], zs));
            }
            if (lane < qb)
                xs[q + lane] = v;
        }
        __syncthreads();
        for (int r = threadIdx.x; r < q; r += blockDim.x)
        {
            double p = 0.0;
            for (int s = 0; s < qb; ++s)
                p = __dadd_rn(p, __dmul_rn(L[(q + s) * kBlockLd + r], xs[q + s]));
            xs[r] = __dadd_rn(xs[r], -p);
        }
        __syncthreads();
    }
    for (int r = threadIdx.x; r < kb; r += blockDim.x)
        x[k0 + r] = xs[r];
}

// backward, rows i < k0: x_i -= sum_s L[k0 + s][i] z_s; 32 consecutive i per CTA (coalesced
// reads of L's rows), the s range split over the CTA's warps and summed in warp order
__global__ void __launch_bounds__(kSolveThreads) dense_backward_rows_kernel(int64_t n, int64_t k0, int kb,
                                                                            const double* __restrict__ A,
                                                                            double* __restrict__ x, const int* status)
{
    constexpr int kGroups = kSolveThreads / 32;
    __shared__ double zs[kSolvePanel];
    __shared__ double part[kGroups][32];
    if (*status != 0)
        return;
    for (int r = threadIdx.x; r < kb; r += blockDim.x)
        zs[r] = x[k0 + r];
    __syncthreads();
    const int g = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int64_t i = int64_t(blockIdx.x) * 32 + lane;
    double p = 0.0;
    if (i < k0)
        for (int s = g; s < kb; s += kGroups)
            p = __dadd_rn(p, __dmul_rn(A[(k0 + s) * n + i], zs[s]));
    part[g][lane] = p;
    __syncthreads();
    if (g == 0 && i < k0)
    {
        double t = part[0][lane];
#pragma unroll
        for (int k = 1; k < kGroups; ++k)
            t = __dadd_rn(t, part[k][lane]);
        x[i] = __dadd_rn(x[i], -t);
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
        if (k0 == 0)
        {
            dense_potrf_kernel<<<1, 256, 0, stream>>>(n, k0, kb, A, status);
            PM_LAUNCH_CHECK();
        }
        const int64_t rest = n - k0 - kb;
        if (rest <= 0)
            break;
        dense_trsm_kernel<<<grid_for(rest, 256 / 32), 256, 0, stream>>>(n, k0, kb, A, status);
        PM_LAUNCH_CHECK();
        const int64_t tiles = (rest + kTile - 1) / kTile;
        dense_update_kernel<<<static_cast<unsigned>(tiles * (tiles + 1) / 2), 256, 0, stream>>>(n, k0, kb, A, status);
        PM_LAUNCH_CHECK();
    }
    PM_CUDA(cudaFuncSetAttribute(dense_forward_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kBlockSmem)));
    PM_CUDA(cudaFuncSetAttribute(dense_backward_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kBlockSmem)));
    for (int64_t k0 = 0; k0 < n; k0 += kSolvePanel)
    {
        const int kb = static_cast<int>(n - k0 < kSolvePanel ? n - k0 : kSolvePanel);
        dense_forward_block_kernel<<<1, kSolveThreads, kBlockSmem, stream>>>(n, k0, kb, A, x, status);
        PM_LAUNCH_CHECK();
        const int64_t rest = n - k0 - kb;
        if (rest > 0)
        {
            dense_forward_rows_kernel<<<grid_for(rest, kSolveThreads / 32, 8 * 148), kSolveThreads, 0, stream>>>(
                n, k0, kb, A, x, status);
            PM_LAUNCH_CHECK();
        }
    }
    for (int64_t k1 = n; k1 > 0; k1 -= kSolvePanel)
    {
        const int64_t k0 = k1 > kSolvePanel ? k1 - kSolvePanel : 0;
        const int kb = static_cast<int>(k1 - k0);
        dense_backward_block_kernel<<<1, kSolveThreads, kBlockSmem, stream>>>(n, k0, kb, A, x, status);
        PM_LAUNCH_CHECK();
        if (k0 > 0)
        {
            dense_backward_rows_kernel<<<grid_for(k0, 32), kSolveThreads, 0, stream>>>(n, k0, kb, A, x, status);
            PM_LAUNCH_CHECK();
        }
    }
}

template void dense_schur_factor_solve<float>(cudaStream_t, int64_t, int, const int*, const int*, const float*,
                                              double*, double*, int*);
template void dense_schur_factor_solve<double>(cudaStream_t, int64_t, int, const int*, const int*, const double*,
                                               double*, double*, int*);

} // namespace pm
