// Learned correction of the block-Jacobi preconditioner of the reduced Schur system (no
// counterpart in the reference; definitions in include/plamatrix_b200.h, pm_mlp_*).
//
//   features (25 per block row p, s = mean diag(S_pp) or 1 when not positive):
//     f[r(r+1)/2 + c] = sign(a) log1p(|a|),  a = S_pp[r][c] / s   (c <= r)
//     f[21..23] = log1p(mean / max / min of ||S_pq||_F / s over q != p), f[24] = log1p(count) / 4
//   network 25 -> 128 -> 128 -> 21 with GELU (x Phi(x)); every GEMM runs on the tensor cores
//   (mma.sync m16n8k16, BF16 operands rounded to nearest even, FP32 accumulation); master
//   weights, activations and gradients are FP32.
//   preconditioner: L = chol(S_pp) (FP64), L'_ii = L_ii softplus(o_ii) / ln 2,
//   L'_ij = L_ij + o_ij L_jj, block (L'L'^T)^-1 in FP64.
//   loss of a solved system (x, b): sum_p ||L'L'^T x_p - b_p||^2 / sum_p ||b_p||^2.
// Every reduction runs in a fixed order: results are bitwise reproducible.
#include "pm_schur.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace pm
{
namespace
{
constexpr int kIn = 25, kHid = 128, kOut = 21;
constexpr int kInPad = 32;   // feature row stride
constexpr int kOutPad = 24;  // output row stride
constexpr int64_t kOffW1 = 0, kOffB1 = kOffW1 + kIn * kHid, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
                  kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kOut, kParams = kOffB3 + kOut;
constexpr int kPartBlock = 256;
constexpr int kMaxPartBlocks = 512;
} // namespace
} // namespace pm

struct pm_mlp
{
    void* state = nullptr;   // params | adam m | adam v | grads | loss scratch | flag (cudaMalloc)
    float* params = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    float* grads = nullptr;
    double* scratch = nullptr; // 2 * kMaxPartBlocks partials, den, num
    int* bad = nullptr;
    void* act = nullptr;     // per-row activations (cudaMalloc, grown on demand)
    int64_t rows = 0;        // rows of the last forward pass
    int64_t capacity = 0;
    float *F = nullptr, *Z1 = nullptr, *H1 = nullptr, *Z2 = nullptr, *H2 = nullptr, *O = nullptr, *dO = nullptr,
          *dH = nullptr, *dZ = nullptr, *split = nullptr;
    int64_t step = 0;
};

namespace pm
{
namespace
{

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x)
{
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * expf(-0.5f * x * x) * 0.39894228040143268f;
}

// ---------------------------------------------------------------- features
// Warp per block row: lanes 0..20 the scaled lower-triangle entries of the diagonal block;
// lanes stride over the row's off-diagonal blocks (Frobenius norms), then fixed xor-tree
// reductions of the norm sum, maximum, minimum and count.
template <typename T>
__global__ void __launch_bounds__(128) features_kernel(int64_t P, const int* __restrict__ row_ptr,
                                                       const int* __restrict__ col, const int* __restrict__ diag_pos,
                                                       const T* __restrict__ S, float* __restrict__ F)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x / 32);
    for (int64_t p = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; p < P; p += warps)
    {
        const T* d = S + int64_t(diag_pos[p]) * 36;
        double s = 0.0;
        for (int i = 0; i < 6; ++i)
            s += static_cast<double>(d[i * 6 + i]);
        s /= 6.0;
        if (!(s > 0.0))
            s = 1.0;
        float* f = F + p * kInPad;
        if (lane < 21)
        {
            int r = 0;
            while (r * (r + 1) / 2 + r < lane)
                ++r;
            const int c = lane - r * (r + 1) / 2;
            const double a = static_cast<double>(d[r * 6 + c]) / s;
            f[lane] = static_cast<float>((a < 0.0 ? -1.0 : 1.0) * log1p(fabs(a)));
        }
        double sum = 0.0, mx = -1.0, mn = 1e300;
        int n = 0;
        for (int b = row_ptr[p] + lane; b < row_ptr[p + 1]; b += 32)
        {
            if (col[b] == p)
                continue;
            double fro = 0.0;
            for (int k = 0; k < 36; ++k)
            {
                const double e = static_cast<double>(S[int64_t(b) * 36 + k]);
                fro += e * e;
            }
            fro = sqrt(fro) / s;
            sum += fro;
            mx = fmax(mx, fro);
            mn = fmin(mn, fro);
            ++n;
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            sum += __shfl_xor_sync(0xffffffffu, sum, o);
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            n += __shfl_xor_sync(0xffffffffu, n, o);
        }
        if (lane == 0)
        {
            f[21] = n ? static_cast<float>(log1p(sum / n)) : 0.0f;
            f[22] = n ? static_cast<float>(log1p(mx)) : 0.0f;
            f[23] = n ? static_cast<float>(log1p(mn)) : 0.0f;
            f[24] = static_cast<float>(log1p(static_cast<double>(n)) / 4.0);
        }
        if (lane >= kIn && lane < kInPad)
            f[lane] = 0.0f;
    }
}

// ---------------------------------------------------------------- tensor-core GEMM
// C (M x N) = A (M x K) B (K x N) [+ bias], A(m, k) = A[m*sam + k*sak], B(k, n) = B[k*sbk + n*sbn];
// with H != nullptr also H = gelu(C).  CTA tile 64 x 64, four warps of 16 rows x 64 columns,
// K in steps of 32 staged in shared memory as BF16 (round to nearest even); mma.sync
// m16n8k16 with FP32 accumulators.  The K order is fixed: results are reproducible.
constexpr int kTileM = 64, kTileN = 64, kTileK = 32, kTilePad = 8;

__device__ __forceinline__ uint32_t pack2(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// With kchunk > 0 the K range is split over blockIdx.z (chunks of kchunk) and every split writes
// its partial tile to C + blockIdx.z * M * ldc (no bias / activation); reduce_splits_kernel
// adds the splits in order.
__global__ void __launch_bounds__(128) gemm_bf16_kernel(int M, int N, int K, const float* __restrict__ A, int64_t sam,
                                                        int64_t sak, const float* __restrict__ B, int64_t sbk,
                                                        int64_t sbn, const float* __restrict__ bias,
                                                        float* __restrict__ C, int64_t ldc, float* __restrict__ H,
                                                        int kchunk)
{
    __shared__ __align__(16) __nv_bfloat16 As[kTileM][kTileK + kTilePad]; // [m][k]
    __shared__ __align__(16) __nv_bfloat16 Bs[kTileN][kTileK + kTilePad]; // [n][k]
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int g = lane >> 2, tq = lane & 3;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * kTileN;
    const int kb = kchunk > 0 ? blockIdx.z * kchunk : 0;
    const int ke = kchunk > 0 ? min(K, kb + kchunk) : K;
    if (kchunk > 0)
        C += int64_t(blockIdx.z) * M * ldc;
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
            acc[j][e] = 0.0f;
    for (int k0 = kb; k0 < ke; k0 += kTileK)
    {
        for (int i = t; i < kTileM * kTileK; i += 128)
        {
            const int mm = i / kTileK, kk = i - mm * kTileK;
            const int gm = m0 + mm, gk = k0 + kk;
            const float a = gm < M && gk < ke ? A[int64_t(gm) * sam + int64_t(gk) * sak] : 0.0f;
            As[mm][kk] = __float2bfloat16_rn(a);
        }
        for (int i = t; i < kTileN * kTileK; i += 128)
        {
            const int nn = i / kTileK, kk = i - nn * kTileK;
            const int gn = n0 + nn, gk = k0 + kk;
            const float b = gn < N && gk < ke ? B[int64_t(gk) * sbk + int64_t(gn) * sbn] : 0.0f;
            Bs[nn][kk] = __float2bfloat16_rn(b);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kTileK; kk += 16)
        {
            const int r = warp * 16 + g;
            const uint32_t a0 = pack2(&As[r][kk + 2 * tq]);
            const uint32_t a1 = pack2(&As[r + 8][kk + 2 * tq]);
            const uint32_t a2 = pack2(&As[r][kk + 2 * tq + 8]);
            const uint32_t a3 = pack2(&As[r + 8][kk + 2 * tq + 8]);
#pragma unroll
            for (int j = 0; j < 8; ++j)
            {
                const uint32_t b0 = pack2(&Bs[j * 8 + g][kk + 2 * tq]);
                const uint32_t b1 = pack2(&Bs[j * 8 + g][kk + 2 * tq + 8]);
                asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, "
                             "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
                             : "+f"(acc[j][0]), "+f"(acc[j][1]), "+f"(acc[j][2]), "+f"(acc[j][3])
                             : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
        {
            const int gm = m0 + warp * 16 + g + (e >= 2 ? 8 : 0);
            const int gn = n0 + j * 8 + 2 * tq + (e & 1);
            if (gm < M && gn < N)
            {
                const float z = acc[j][e] + (bias ? bias[gn] : 0.0f);
                C[int64_t(gm) * ldc + gn] = z;
                if (H)
                    H[int64_t(gm) * ldc + gn] = gelu(z);
            }
        }
}

void gemm(cudaStream_t stream, int M, int N, int K, const float* A, int64_t sam, int64_t sak, const float* B,
          int64_t sbk, int64_t sbn, const float* bias, float* C, int64_t ldc, float* H = nullptr)
{
    if (M <= 0 || N <= 0)
        return;
    const dim3 grid((M + kTileM - 1) / kTileM, (N + kTileN - 1) / kTileN);
    gemm_bf16_kernel<<<grid, 128, 0, stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, C, ldc, H, 0);
    PM_LAUNCH_CHECK();
}

// sum of `splits` partial M x N tiles (compact, split-major) into C (row stride ldc), in order
__global__ void reduce_splits_kernel(int M, int N, int splits, const float* __restrict__ part, float* __restrict__ C,
                                     int64_t ldc)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < int64_t(M) * N;
         i += int64_t(gridDim.x) * blockDim.x)
    {
        float s = 0.0f;
        for (int z = 0; z < splits; ++z)
            s += part[int64_t(z) * M * N + i];
        C[(i / N) * ldc + i % N] = s;
    }
}

constexpr int kSplitRows = 512; // rows per split of the weight-gradient reductions

int split_count(int64_t K) { return static_cast<int>((K + kSplitRows - 1) / kSplitRows); }

// C = A B with the K (row) dimension split over CTAs; `part` holds split_count(K) * M * N floats
void gemm_split(cudaStream_t stream, int M, int N, int K, const float* A, int64_t sam, int64_t sak, const float* B,
                int64_t sbk, int64_t sbn, float* C, int64_t ldc, float* part)
{
    if (M <= 0 || N <= 0)
        return;
    const int splits = split_count(K);
    const dim3 grid((M + kTileM - 1) / kTileM, (N + kTileN - 1) / kTileN, splits);
    gemm_bf16_kernel<<<grid, 128, 0, stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, nullptr, part, N, nullptr,
                                               kSplitRows);
    PM_LAUNCH_CHECK();
    reduce_splits_kernel<<<grid_for(int64_t(M) * N, 256, 1024), 256, 0, stream>>>(M, N, splits, part, C, ldc);
    PM_LAUNCH_CHECK();
}

// ---------------------------------------------------------------- loss and output gradient
__device__ bool chol6(const double* d, double* L)
{
    for (int i = 0; i < 36; ++i)
        L[i] = 0.0;
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j <= i; ++j)
        {
            double v = d[i * 6 + j];
            for (int k = 0; k < j; ++k)
                v -= L[i * 6 + k] * L[j * 6 + k];
            if (i == j)
            {
                if (!(v > 0.0))
                    return false;
                L[i * 6 + i] = sqrt(v);
            }
            else
            {
                L[i * 6 + j] = v / L[j * 6 + j];
            }
        }
    return true;
}

__device__ __forceinline__ double softplus(double x) { return x > 30.0 ? x : log1p(exp(x)); }

__device__ void corrected(const double* L, const float* o, double* Lc)
{
    const double ln2 = 0.69314718055994531;
    for (int i = 0; i < 36; ++i)
        Lc[i] = 0.0;
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j <= i; ++j)
        {
            const double oo = static_cast<double>(o[i * (i + 1) / 2 + j]);
            Lc[i * 6 + j] = i == j ? L[i * 6 + i] * softplus(oo) / ln2 : L[i * 6 + j] + oo * L[j * 6 + j];
        }
}

template <typename T>
__device__ __forceinline__ void load_diag(const T* S, int pos, double* d)
{
    for (int k = 0; k < 36; ++k)
        d[k] = static_cast<double>(S[int64_t(pos) * 36 + k]);
}

// fixed-order block sums of v into part[blockIdx.x]
__device__ void block_partial(double v, double* part)
{
    __shared__ double s[kPartBlock / 32];
    v = block_sum<double, kPartBlock>(v, s);
    if (threadIdx.x == 0)
        part[blockIdx.x] = v;
}

__global__ void __launch_bounds__(kPartBlock) squares_kernel(int64_t n, const double* __restrict__ b, double* part)
{
    double mine = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        mine += b[i] * b[i];
    block_partial(mine, part);
}

__global__ void finish_sum_kernel(int parts, const double* __restrict__ part, double* out)
{
    double s = 0.0;
    for (int i = 0; i < parts; ++i)
        s += part[i];
    *out = s;
}

template <typename T>
__global__ void __launch_bounds__(kPartBlock) loss_kernel(int64_t P, const int* __restrict__ diag_pos,
                                                          const T* __restrict__ S, const float* __restrict__ O,
                                                          const double* __restrict__ x, const double* __restrict__ b,
                                                          const double* __restrict__ den, float* __restrict__ dO,
                                                          double* part, int* bad)
{
    const double ln2 = 0.69314718055994531;
    const double inv_den = 1.0 / *den;
    double mine = 0.0;
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
    {
        double d[36], L[36], Lc[36], u[6], r[6], v[6];
        load_diag<T>(S, diag_pos[p], d);
        float* g = dO + p * kOutPad;
        if (!chol6(d, L))
        {
            atomicExch(bad, 1);
            for (int k = 0; k < kOutPad; ++k)
                g[k] = 0.0f;
            continue;
        }
        const float* o = O + p * kOutPad;
        corrected(L, o, Lc);
        const double* xp = x + p * 6;
        const double* bp = b + p * 6;
        for (int j = 0; j < 6; ++j)
        {
            u[j] = 0.0;
            for (int i = j; i < 6; ++i)
                u[j] += Lc[i * 6 + j] * xp[i];
        }
        for (int i = 0; i < 6; ++i)
        {
            double s = 0.0;
            for (int j = 0; j <= i; ++j)
                s += Lc[i * 6 + j] * u[j];
            r[i] = s - bp[i];
            mine += r[i] * r[i];
        }
        for (int j = 0; j < 6; ++j)
        {
            v[j] = 0.0;
            for (int i = j; i < 6; ++i)
                v[j] += Lc[i * 6 + j] * r[i];
        }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j <= i; ++j)
            {
                const int k = i * (i + 1) / 2 + j;
                const double gg = 2.0 * (r[i] * u[j] + xp[i] * v[j]) * inv_den;
                const double ok = static_cast<double>(o[k]);
                g[k] = static_cast<float>(i == j ? gg * L[i * 6 + i] / (1.0 + exp(-ok)) / ln2 : gg * L[j * 6 + j]);
            }
        for (int k = kOut; k < kOutPad; ++k)
            g[k] = 0.0f;
    }
    block_partial(mine, part);
}

// dZ = dH * gelu'(Z)
__global__ void gelu_back_kernel(int64_t n, const float* __restrict__ dH, const float* __restrict__ Z,
                                 float* __restrict__ dZ)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        dZ[i] = dH[i] * gelu_grad(Z[i]);
}

// partial column sums of G over row chunks of kSplitRows (blockIdx.y), rows in order
__global__ void colsum_kernel(int64_t rows, int cols, int64_t ld, const float* __restrict__ G,
                              float* __restrict__ part)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols)
        return;
    const int64_t r0 = int64_t(blockIdx.y) * kSplitRows;
    const int64_t r1 = r0 + kSplitRows < rows ? r0 + kSplitRows : rows;
    float s = 0.0f;
    for (int64_t r = r0; r < r1; ++r)
        s += G[r * ld + c];
    part[int64_t(blockIdx.y) * cols + c] = s;
}

void colsum(cudaStream_t stream, int64_t rows, int cols, int64_t ld, const float* G, float* db, float* part)
{
    const int splits = split_count(rows);
    colsum_kernel<<<dim3((cols + 127) / 128, splits), 128, 0, stream>>>(rows, cols, ld, G, part);
    PM_LAUNCH_CHECK();
    reduce_splits_kernel<<<1, 128, 0, stream>>>(1, cols, splits, part, db, cols);
    PM_LAUNCH_CHECK();
}

__global__ void adam_kernel(int64_t n, float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, float lr, float c1, float c2)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        const float gi = g[i];
        const float mi = 0.9f * m[i] + 0.1f * gi;
        const float vi = 0.999f * v[i] + 0.001f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
    }
}

// ---------------------------------------------------------------- preconditioner blocks
template <typename T>
__global__ void precond_kernel(int64_t P, const int* __restrict__ diag_pos, const T* __restrict__ S,
                               const float* __restrict__ O, double* __restrict__ minv, float* __restrict__ minv32,
                               int* bad)
{
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
    {
        double d[36], L[36], Lc[36], M[36];
        load_diag<T>(S, diag_pos[p], d);
        if (!chol6(d, L))
        {
            atomicExch(bad, 1);
            continue;
        }
        corrected(L, O + p * kOutPad, Lc);
        bool ok = true;
        for (int i = 0; i < 6; ++i)
            ok = ok && Lc[i * 6 + i] > 0.0 && isfinite(Lc[i * 6 + i]);
        if (!ok)
        {
            atomicExch(bad, 1);
            continue;
        }
        for (int c = 0; c < 6; ++c)
        {
            double y[6];
            for (int i = 0; i < 6; ++i)
            {
                double val = i == c ? 1.0 : 0.0;
                for (int k = 0; k < i; ++k)
                    val -= Lc[i * 6 + k] * y[k];
                y[i] = val / Lc[i * 6 + i];
            }
            for (int i = 5; i >= 0; --i)
            {
                double val = y[i];
                for (int k = i + 1; k < 6; ++k)
                    val -= Lc[k * 6 + i] * M[k * 6 + c];
                M[i * 6 + c] = val / Lc[i * 6 + i];
            }
        }
        for (int k = 0; k < 36; ++k)
        {
            minv[p * 36 + k] = M[k];
            if (minv32)
                minv32[p * 36 + k] = static_cast<float>(M[k]);
        }
    }
}

// ---------------------------------------------------------------- host side
uint64_t splitmix(uint64_t& s)
{
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

void allocate_state(pm_mlp* mlp)
{
    Carver plan;
    for (int k = 0; k < 4; ++k)
        plan.take<float>(kParams);
    plan.take<double>(2 * kMaxPartBlocks + 4);
    plan.take<int>(4);
    PM_CUDA(cudaMalloc(&mlp->state, plan.offset + 256));
    Carver c;
    c.base = static_cast<char*>(mlp->state);
    mlp->params = c.take<float>(kParams);
    mlp->m = c.take<float>(kParams);
    mlp->v = c.take<float>(kParams);
    mlp->grads = c.take<float>(kParams);
    mlp->scratch = c.take<double>(2 * kMaxPartBlocks + 4);
    mlp->bad = c.take<int>(4);
}

int* bad_flag(pm_mlp* mlp) { return mlp->bad; }

void ensure_rows(pm_mlp* mlp, int64_t P, cudaStream_t stream)
{
    if (P <= mlp->capacity)
        return;
    PM_CUDA(cudaStreamSynchronize(stream));
    if (mlp->act)
    {
        PM_CUDA(cudaFree(mlp->act));
        mlp->act = nullptr;
        mlp->capacity = 0;
    }
    Carver plan;
    plan.take<float>(P * kInPad);
    for (int k = 0; k < 4; ++k)
        plan.take<float>(P * kHid);
    plan.take<float>(P * kOutPad);
    plan.take<float>(P * kOutPad);
    plan.take<float>(P * kHid);
    plan.take<float>(P * kHid);
    const int64_t splits = split_count(P);
    plan.take<float>(splits * kHid * kHid);
    PM_CUDA(cudaMalloc(&mlp->act, plan.offset + 256));
    Carver c;
    c.base = static_cast<char*>(mlp->act);
    mlp->F = c.take<float>(P * kInPad);
    mlp->Z1 = c.take<float>(P * kHid);
    mlp->H1 = c.take<float>(P * kHid);
    mlp->Z2 = c.take<float>(P * kHid);
    mlp->H2 = c.take<float>(P * kHid);
    mlp->O = c.take<float>(P * kOutPad);
    mlp->dO = c.take<float>(P * kOutPad);
    mlp->dH = c.take<float>(P * kHid);
    mlp->dZ = c.take<float>(P * kHid);
    mlp->split = c.take<float>(splits * kHid * kHid);
    mlp->capacity = P;
}

void forward(pm_mlp* mlp, const SchurView& v, cudaStream_t stream)
{
    const int64_t P = v.P;
    ensure_rows(mlp, std::max<int64_t>(P, 1), stream);
    mlp->rows = P;
    if (P == 0)
        return;
    const unsigned grid = grid_for(P * 32, 128, 1 << 16);
    if (v.value_size == 8)
        features_kernel<double><<<grid, 128, 0, stream>>>(P, v.block_row_ptr, v.block_col, v.diag_pos,
                                                          static_cast<const double*>(v.S), mlp->F);
    else
        features_kernel<float><<<grid, 128, 0, stream>>>(P, v.block_row_ptr, v.block_col, v.diag_pos,
                                                         static_cast<const float*>(v.S), mlp->F);
    PM_LAUNCH_CHECK();
    const int M = static_cast<int>(P);
    const float* W = mlp->params;
    gemm(stream, M, kHid, kIn, mlp->F, kInPad, 1, W + kOffW1, kHid, 1, W + kOffB1, mlp->Z1, kHid, mlp->H1);
    gemm(stream, M, kHid, kHid, mlp->H1, kHid, 1, W + kOffW2, kHid, 1, W + kOffB2, mlp->Z2, kHid, mlp->H2);
    PM_CUDA(cudaMemsetAsync(mlp->O, 0, size_t(P) * kOutPad * sizeof(float), stream));
    gemm(stream, M, kOut, kHid, mlp->H2, kHid, 1, W + kOffW3, kOut, 1, W + kOffB3, mlp->O, kOutPad);
}

void check_view(const SchurView& v)
{
    if (!v.S || (v.P > 0 && !v.diag_pos))
        fail(PM_LOGIC_ERROR, "learned preconditioner: the workspace holds no assembled 6x6 system");
    if (v.P > INT32_MAX)
        fail(PM_OVERFLOW_ERROR, "learned preconditioner: too many block rows");
}

} // namespace

void mlp_apply(const pm_mlp* cmlp, const SchurView& v, cudaStream_t stream)
{
    pm_mlp* mlp = const_cast<pm_mlp*>(cmlp); // parameters are read only; scratch is reused
    check_view(v);
    forward(mlp, v, stream);
    if (v.P == 0)
        return;
    PM_CUDA(cudaMemsetAsync(bad_flag(mlp), 0, sizeof(int), stream));
    const unsigned grid = grid_for(v.P, 64, 4096);
    if (v.value_size == 8)
        precond_kernel<double><<<grid, 64, 0, stream>>>(v.P, v.diag_pos, static_cast<const double*>(v.S), mlp->O,
                                                        v.minv, v.mixed ? v.minv32 : nullptr, bad_flag(mlp));
    else
        precond_kernel<float><<<grid, 64, 0, stream>>>(v.P, v.diag_pos, static_cast<const float*>(v.S), mlp->O,
                                                       v.minv, v.mixed ? v.minv32 : nullptr, bad_flag(mlp));
    PM_LAUNCH_CHECK();
    int bad = 0;
    PM_CUDA(cudaMemcpyAsync(&bad, bad_flag(mlp), sizeof(int), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaStreamSynchronize(stream));
    if (bad)
        fail(PM_RUNTIME_ERROR, "learned preconditioner: a corrected block is not positive definite");
}

namespace
{

double train(pm_mlp* mlp, const SchurView& v, cudaStream_t stream, const double* x, const double* b, double lr)
{
    check_view(v);
    if (v.P == 0)
        fail(PM_INVALID_ARGUMENT, "learned preconditioner: empty system");
    if (!x || !b)
        fail(PM_INVALID_ARGUMENT, "learned preconditioner: solution and right-hand side must be non-null");
    forward(mlp, v, stream);
    const int64_t P = v.P, n = 6 * P;
    const int M = static_cast<int>(P);
    double* part = mlp->scratch;
    double* den = mlp->scratch + 2 * kMaxPartBlocks;
    double* num = den + 1;
    int* bad = bad_flag(mlp);
    PM_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), stream));
    const unsigned sg = grid_for(n, kPartBlock, kMaxPartBlocks);
    squares_kernel<<<sg, kPartBlock, 0, stream>>>(n, b, part);
    PM_LAUNCH_CHECK();
    finish_sum_kernel<<<1, 1, 0, stream>>>(static_cast<int>(sg), part, den);
    PM_LAUNCH_CHECK();
    const unsigned lg = grid_for(P, kPartBlock, kMaxPartBlocks);
    if (v.value_size == 8)
        loss_kernel<double><<<lg, kPartBlock, 0, stream>>>(P, v.diag_pos, static_cast<const double*>(v.S), mlp->O, x,
                                                           b, den, mlp->dO, part + kMaxPartBlocks, bad);
    else
        loss_kernel<float><<<lg, kPartBlock, 0, stream>>>(P, v.diag_pos, static_cast<const float*>(v.S), mlp->O, x, b,
                                                          den, mlp->dO, part + kMaxPartBlocks, bad);
    PM_LAUNCH_CHECK();
    finish_sum_kernel<<<1, 1, 0, stream>>>(static_cast<int>(lg), part + kMaxPartBlocks, num);
    PM_LAUNCH_CHECK();
    // backward (tensor-core GEMMs; the row dimension is the reduction of the weight gradients)
    float* G = mlp->grads;
    const float* W = mlp->params;
    float* splits = mlp->split;
    gemm_split(stream, kHid, kOut, M, mlp->H2, 1, kHid, mlp->dO, kOutPad, 1, G + kOffW3, kOut, splits);
    colsum(stream, P, kOut, kOutPad, mlp->dO, G + kOffB3, splits);
    gemm(stream, M, kHid, kOut, mlp->dO, kOutPad, 1, W + kOffW3, 1, kOut, nullptr, mlp->dH, kHid);
    gelu_back_kernel<<<grid_for(P * kHid, 256, 4096), 256, 0, stream>>>(P * kHid, mlp->dH, mlp->Z2, mlp->dZ);
    PM_LAUNCH_CHECK();
    gemm_split(stream, kHid, kHid, M, mlp->H1, 1, kHid, mlp->dZ, kHid, 1, G + kOffW2, kHid, splits);
    colsum(stream, P, kHid, kHid, mlp->dZ, G + kOffB2, splits);
    gemm(stream, M, kHid, kHid, mlp->dZ, kHid, 1, W + kOffW2, 1, kHid, nullptr, mlp->dH, kHid);
    gelu_back_kernel<<<grid_for(P * kHid, 256, 4096), 256, 0, stream>>>(P * kHid, mlp->dH, mlp->Z1, mlp->dZ);
    PM_LAUNCH_CHECK();
    gemm_split(stream, kIn, kHid, M, mlp->F, 1, kInPad, mlp->dZ, kHid, 1, G + kOffW1, kHid, splits);
    colsum(stream, P, kHid, kHid, mlp->dZ, G + kOffB1, splits);
    if (lr > 0.0)
    {
        mlp->step += 1;
        const float c1 = static_cast<float>(1.0 - std::pow(0.9, double(mlp->step)));
        const float c2 = static_cast<float>(1.0 - std::pow(0.999, double(mlp->step)));
        adam_kernel<<<grid_for(kParams, 256, 1024), 256, 0, stream>>>(kParams, mlp->params, mlp->m, mlp->v, G,
                                                                      static_cast<float>(lr), c1, c2);
        PM_LAUNCH_CHECK();
    }
    double host[2] = {0.0, 0.0};
    int host_bad = 0;
    PM_CUDA(cudaMemcpyAsync(host, den, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaMemcpyAsync(&host_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaStreamSynchronize(stream));
    if (host_bad)
        fail(PM_RUNTIME_ERROR, "learned preconditioner: a diagonal block is not positive definite");
    if (!(host[0] > 0.0))
        fail(PM_INVALID_ARGUMENT, "learned preconditioner: the right-hand side is zero");
    return host[1] / host[0];
}

} // namespace
} // namespace pm

extern "C" {

int64_t pm_mlp_param_count(void) { return pm::kParams; }

int pm_mlp_create(uint64_t seed, pm_mlp** out)
{
    return pm::guarded([&] {
        if (!out)
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_create: output pointer is null");
        auto* mlp = new pm_mlp();
        try
        {
            std::vector<float> w(pm::kParams, 0.0f);
            uint64_t s = seed;
            auto fill = [&](int64_t off, int fan_in, int fan_out) {
                const double a = std::sqrt(6.0 / double(fan_in + fan_out));
                for (int64_t i = 0; i < int64_t(fan_in) * fan_out; ++i)
                {
                    const double u = double(pm::splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
                    w[off + i] = static_cast<float>((2.0 * u - 1.0) * a);
                }
            };
            fill(pm::kOffW1, pm::kIn, pm::kHid);
            fill(pm::kOffW2, pm::kHid, pm::kHid); // W3, biases: zero (the network starts as block Jacobi)
            pm::allocate_state(mlp);
            PM_CUDA(cudaMemcpy(mlp->params, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
            PM_CUDA(cudaMemset(mlp->m, 0, 3 * pm::kParams * sizeof(float)));
        }
        catch (...)
        {
            if (mlp->state)
                cudaFree(mlp->state);
            delete mlp;
            throw;
        }
        *out = mlp;
    });
}

void pm_mlp_destroy(pm_mlp* mlp)
{
    if (mlp)
    {
        cudaDeviceSynchronize();
        cudaFree(mlp->state);
        if (mlp->act)
            cudaFree(mlp->act);
        delete mlp;
    }
}

int pm_mlp_get_params(const pm_mlp* mlp, float* host)
{
    return pm::guarded([&] {
        if (!mlp || !host)
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_get_params: null argument");
        PM_CUDA(cudaDeviceSynchronize());
        PM_CUDA(cudaMemcpy(host, mlp->params, pm::kParams * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

int pm_mlp_set_params(pm_mlp* mlp, const float* host)
{
    return pm::guarded([&] {
        if (!mlp || !host)
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_set_params: null argument");
        PM_CUDA(cudaDeviceSynchronize());
        PM_CUDA(cudaMemcpy(mlp->params, host, pm::kParams * sizeof(float), cudaMemcpyHostToDevice));
        PM_CUDA(cudaMemset(mlp->m, 0, 2 * pm::kParams * sizeof(float)));
        mlp->step = 0;
    });
}

int pm_mlp_forward(pm_mlp* mlp, pm_schur_workspace* ws, pm_stream_t stream)
{
    return pm::guarded([&] {
        if (!mlp || !ws)
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_forward: null argument");
        const pm::SchurView v = pm::schur_view(ws, false);
        pm::check_view(v);
        pm::forward(mlp, v, stream);
        PM_CUDA(cudaStreamSynchronize(stream));
    });
}

int pm_mlp_train_step(pm_mlp* mlp, pm_schur_workspace* ws, pm_stream_t stream, const double* x, const double* b,
                      double learning_rate, double* loss)
{
    return pm::guarded([&] {
        if (!mlp || !ws)
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_train_step: null argument");
        if (!(learning_rate >= 0.0) || !std::isfinite(learning_rate))
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_train_step: learning rate must be finite and non-negative");
        const double l = pm::train(mlp, pm::schur_view(ws, false), stream, x, b, learning_rate);
        if (loss)
            *loss = l;
    });
}

int pm_mlp_inspect(const pm_mlp* mlp, int64_t* rows, float* features, float* outputs, float* gradients)
{
    return pm::guarded([&] {
        if (!mlp)
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_inspect: null argument");
        PM_CUDA(cudaDeviceSynchronize());
        const int64_t P = mlp->rows;
        if (rows)
            *rows = P;
        if (features && P > 0)
            PM_CUDA(cudaMemcpy2D(features, pm::kIn * sizeof(float), mlp->F, pm::kInPad * sizeof(float),
                                 pm::kIn * sizeof(float), P, cudaMemcpyDeviceToHost));
        if (outputs && P > 0)
            PM_CUDA(cudaMemcpy2D(outputs, pm::kOut * sizeof(float), mlp->O, pm::kOutPad * sizeof(float),
                                 pm::kOut * sizeof(float), P, cudaMemcpyDeviceToHost));
        if (gradients && mlp->grads)
            PM_CUDA(cudaMemcpy(gradients, mlp->grads, pm::kParams * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

} // extern "C"
