// Learned correction of the block-Jacobi preconditioner of the reduced Schur system (no
// counterpart in the reference; definitions in include/plamatrix_b200.h, pm_mlp_*).
//
//   features (25 per block row p, s = mean diag(S_pp) or 1 when not positive):
//     f[r(r+1)/2 + c] = sign(a) log1p(|a|),  a = S_pp[r][c] / s   (c <= r)
//     f[21..23] = log1p(mean / max / min of ||S_pq||_F / s over q != p), f[24] = log1p(count) / 4
//   network 25 -> 128 -> 128 -> 21 with GELU (x Phi(x)); every GEMM runs on the tensor cores
//   (tcgen05.mma kind::f16 into tensor memory, BF16 operands rounded to nearest even, FP32
//   accumulation); master weights, activations and gradients are FP32.
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
    long long wait_limit = 1ll << 20; // polls of a GEMM stage wait before it gives up
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

// ---------------------------------------------------------------- tensor-core GEMM (tcgen05)
// C (M x N) = A (M x K) B (K x N) [+ bias], A(m, k) = A[m*sam + k*sak], B(k, n) = B[k*sbk + n*sbn];
// with H != nullptr also H = gelu(C).  One CTA of 128 threads per 128 x 64 tile of C.  K runs in
// steps of 32 over two shared-memory stages: the threads fill one stage with both operands as
// BF16 (round to nearest even) in the K-major, unswizzled canonical layout (core matrices of 8
// rows x 16 bytes; K-adjacent core matrices kTcLbo bytes apart, 8-row groups kTcSbo apart) while
// the tensor core reads the other; thread 0 issues two tcgen05.mma kind::f16 per step (128 x 64
// x 16, FP32 accumulator in tensor memory) and commits them to the stage's mbarrier, which the
// threads wait on before they refill that stage.  The epilogue reads the accumulator with
// tcgen05.ld (warp w owns rows 32w..32w+31).  The K order is fixed, so results are
// reproducible.  Every wait is bounded.  A stage wait (before a step's MMAs are issued) gives up
// after `step_wait_limit` polls: the CTA then issues nothing more, sets *error and waits for
// its last commit with the full limit.  Tensor memory is freed only when that drain wait
// succeeded (or nothing was issued), so no MMA can still be writing the columns; if the drain
// itself runs out, the columns stay allocated and *error is set.  The host turns the flag into
// an error.
constexpr int kTcM = 128, kTcN = 64, kTcK = 32, kTcThreads = 128;
constexpr uint32_t kTcCols = 64;                     // tensor-memory columns of the accumulator
constexpr int kTcLbo = 128;                          // bytes between K-adjacent core matrices
constexpr int kTcSbo = kTcLbo * (kTcK / 8);          // bytes between 8-row groups
// dynamic shared memory reserved per CTA (beside 24.6 KB of static stages) so that at most 7
// CTAs share an SM: 7 x 64 columns fit the 512 columns of tensor memory, and no allocation waits
// for another CTA
constexpr size_t kTcSmemReserve = 4096;
constexpr long long kTcWaitLimit = 1ll << 20;
// kind::f16 instruction descriptor: FP32 accumulator (bits 4-5), BF16 A (7-9) and B (10-12),
// both K-major (15, 16), N >> 3 (17-22), M >> 4 (24-28)
constexpr uint32_t kTcIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kTcN >> 3) << 17) | (uint32_t(kTcM >> 4) << 24);

// element (r, k) of a staged operand tile -> its BF16 offset in the canonical layout
__device__ __forceinline__ int tc_offset(int r, int k)
{
    return (r >> 3) * (kTcSbo / 2) + (k >> 3) * (kTcLbo / 2) + (r & 7) * 8 + (k & 7);
}

// shared-memory matrix descriptor: start address, leading (K) and stride (8-row) byte offsets,
// all >> 4; version 1 (bit 46); no swizzle, base offset 0
__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t addr)
{
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((kTcLbo >> 4) & 0x3FFF) << 16) |
           (uint64_t((kTcSbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit)
{
    for (long long it = 0; it < limit; ++it)
    {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_load_32x32b_x64(uint32_t taddr, uint32_t (&r)[64])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
}

__global__ void __launch_bounds__(kTcThreads) gemm_tc_kernel(int M, int N, int K, const float* __restrict__ A,
                                                             int64_t sam, int64_t sak, const float* __restrict__ B,
                                                             int64_t sbk, int64_t sbn, const float* __restrict__ bias,
                                                             float* __restrict__ C, int64_t ldc,
                                                             float* __restrict__ H, int kchunk, int* __restrict__ error,
                                                             long long step_wait_limit)
{
    __shared__ __align__(128) __nv_bfloat16 As[2][kTcM * kTcK];
    __shared__ __align__(128) __nv_bfloat16 Bs[2][kTcN * kTcK];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_base;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int m0 = blockIdx.x * kTcM, n0 = blockIdx.y * kTcN;
    const int kb = kchunk > 0 ? blockIdx.z * kchunk : 0;
    const int ke = kchunk > 0 ? min(K, kb + kchunk) : K;
    if (kchunk > 0)
        C += int64_t(blockIdx.z) * M * ldc;
    const uint32_t bar_addr[2] = {static_cast<uint32_t>(__cvta_generic_to_shared(&bar[0])),
                                  static_cast<uint32_t>(__cvta_generic_to_shared(&bar[1]))};
    if (warp == 0)
    {
        const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(&tmem_base));
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst), "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (t == 32)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_addr[0]) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_addr[1]) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;
    const bool a_kfast = sak == 1, b_kfast = sbk == 1;
    // one step's operands in registers: every load of the step is issued before any is used, and
    // the next step's loads are issued while the tensor core works on the current one;
    // consecutive threads walk the operand's unit-stride index (k, or the row) so that the loads
    // of a warp are coalesced
    constexpr int kAPer = kTcM * kTcK / kTcThreads, kBPer = kTcN * kTcK / kTcThreads;
    float av[kAPer], bv[kBPer];
    auto load_step = [&](int k0) {
#pragma unroll
        for (int j = 0; j < kAPer; ++j)
        {
            const int i = t + j * kTcThreads;
            const int mm = a_kfast ? i / kTcK : i % kTcM, kk = a_kfast ? i % kTcK : i / kTcM;
            const int gm = m0 + mm, gk = k0 + kk;
            av[j] = gm < M && gk < ke ? A[int64_t(gm) * sam + int64_t(gk) * sak] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < kBPer; ++j)
        {
            const int i = t + j * kTcThreads;
            const int nn = b_kfast ? i / kTcK : i % kTcN, kk = b_kfast ? i % kTcK : i / kTcN;
            const int gn = n0 + nn, gk = k0 + kk;
            bv[j] = gn < N && gk < ke ? B[int64_t(gk) * sbk + int64_t(gn) * sbn] : 0.0f;
        }
    };
    // stage s is refilled at step i >= 2 once the commit of step i - 2 (completion (i >> 1) - 1 of
    // bar[s]) has arrived; the MMAs run in issue order, so the last commit covers every step
    int step = 0;
    bool ok = true;
    if (kb < ke)
        load_step(kb);
    for (int k0 = kb; k0 < ke; k0 += kTcK, ++step)
    {
        const int st = step & 1;
        if (step >= 2)
        {
            ok = __syncthreads_and(mbar_wait(bar_addr[st], uint32_t((step >> 1) - 1) & 1u, step_wait_limit)) != 0;
            if (!ok)
                break;
        }
        __nv_bfloat16* as = As[st];
        __nv_bfloat16* bs = Bs[st];
#pragma unroll
        for (int j = 0; j < kAPer; ++j)
        {
            const int i = t + j * kTcThreads;
            const int mm = a_kfast ? i / kTcK : i % kTcM, kk = a_kfast ? i % kTcK : i / kTcM;
            as[tc_offset(mm, kk)] = __float2bfloat16_rn(av[j]);
        }
#pragma unroll
        for (int j = 0; j < kBPer; ++j)
        {
            const int i = t + j * kTcThreads;
            const int nn = b_kfast ? i / kTcK : i % kTcN, kk = b_kfast ? i % kTcK : i / kTcN;
            bs[tc_offset(nn, kk)] = __float2bfloat16_rn(bv[j]);
        }
        // the generic-proxy stores must be visible to the tensor core's (async-proxy) reads
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (t == 0)
        {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t a_addr = static_cast<uint32_t>(__cvta_generic_to_shared(as));
            const uint32_t b_addr = static_cast<uint32_t>(__cvta_generic_to_shared(bs));
#pragma unroll
            for (int h = 0; h < kTcK / 16; ++h)
            {
                const uint64_t ad = tc_smem_desc(a_addr + h * 2 * kTcLbo);
                const uint64_t bd = tc_smem_desc(b_addr + h * 2 * kTcLbo);
                const uint32_t accumulate = (step > 0 || h > 0) ? 1u : 0u;
                asm volatile("{\n\t.reg .pred p;\n\t"
                             "setp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                             ::"r"(tmem), "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(accumulate), "r"(0u), "r"(0u),
                             "r"(0u), "r"(0u)
                             : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             bar_addr[st])
                         : "memory");
        }
        if (k0 + kTcK < ke)
            load_step(k0 + kTcK);
    }
    // commits issued: one per completed step (a failed wait breaks before its step issues); the
    // last one is step issued - 1, on bar[(issued - 1) & 1]
    const int issued = step;
    const bool waited = issued > 0 && __syncthreads_and(mbar_wait(bar_addr[(issued - 1) & 1],
                                                                  uint32_t((issued - 1) >> 1) & 1u, kTcWaitLimit)) != 0;
    const bool drained = issued == 0 || waited;
    ok = ok && drained;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (ok)
    {
        uint32_t r[64];
        if (issued > 0)
        {
            tmem_load_32x32b_x64(tmem + (uint32_t(warp * 32) << 16), r);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        }
        else
        {
#pragma unroll
            for (int j = 0; j < 64; ++j)
                r[j] = 0u;
        }
        const int gm = m0 + warp * 32 + lane;
        if (gm < M)
        {
#pragma unroll
            for (int j = 0; j < kTcN; ++j)
            {
                const int gn = n0 + j;
                if (gn < N)
                {
                    const float z = __uint_as_float(r[j]) + (bias ? bias[gn] : 0.0f);
                    C[int64_t(gm) * ldc + gn] = z;
                    if (H)
                        H[int64_t(gm) * ldc + gn] = gelu(z);
                }
            }
        }
    }
    else if (t == 0)
        atomicExch(error, 1);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0 && drained)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTcCols) : "memory");
}

void gemm(cudaStream_t stream, int M, int N, int K, const float* A, int64_t sam, int64_t sak, const float* B,
          int64_t sbk, int64_t sbn, const float* bias, float* C, int64_t ldc, int* error, long long wait_limit,
          float* H = nullptr)
{
    if (M <= 0 || N <= 0)
        return;
    const dim3 grid((M + kTcM - 1) / kTcM, (N + kTcN - 1) / kTcN);
    gemm_tc_kernel<<<grid, kTcThreads, kTcSmemReserve, stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, C, ldc, H,
                                                                 0, error, wait_limit);
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
                int64_t sbk, int64_t sbn, float* C, int64_t ldc, float* part, int* error, long long wait_limit)
{
    if (M <= 0 || N <= 0)
        return;
    const int splits = split_count(K);
    const dim3 grid((M + kTcM - 1) / kTcM, (N + kTcN - 1) / kTcN, splits);
    gemm_tc_kernel<<<grid, kTcThreads, kTcSmemReserve, stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, nullptr, part, N,
                                                                 nullptr, kSplitRows, error, wait_limit);
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

// x = L^-1 b and x = L^-T b for a lower-triangular 6x6 L (row-major)
__device__ __forceinline__ void lower_solve6(const double* L, const double* b, double* x)
{
    for (int i = 0; i < 6; ++i)
    {
        double s = b[i];
        for (int j = 0; j < i; ++j)
            s -= L[i * 6 + j] * x[j];
        x[i] = s / L[i * 6 + i];
    }
}

__device__ __forceinline__ void upper_solve6(const double* L, const double* b, double* x)
{
    for (int i = 5; i >= 0; --i)
    {
        double s = b[i];
        for (int j = i + 1; j < 6; ++j)
            s -= L[j * 6 + i] * x[j];
        x[i] = s / L[i * 6 + i];
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

// Per block row p, with A_p = L'_p L'_p^T (the corrected factor):
//   solution loss (probe = 0): sum_p ||A_p x_p - b_p||^2 / den, x a solution and b its right-hand side;
//   probe loss (probe = 1):    sum_p ||v_p - A_p^-1 u_p||^2 / den, v a probe vector and u = S v, i.e.
//                              ||(I - M S) v||^2 / ||v||^2 for the block preconditioner M = blockdiag(A_p^-1).
// The gradient with respect to the lower triangle of L' is, for the probe loss (y = L'^-1 u,
// w = L'^-T y = A^-1 u, e = v - w, z = L'^-1 e, q = L'^-T z):  2 (q_i y_j + w_i z_j) / den,
// and for the solution loss (u = L'^T x, r = A x - b, s = L'^T r):  2 (r_i u_j + x_i s_j) / den;
// both are then carried through the correction to the network outputs.
template <typename T>
__global__ void __launch_bounds__(kPartBlock) loss_kernel(int64_t P, const int* __restrict__ diag_pos,
                                                          const T* __restrict__ S, const float* __restrict__ O,
                                                          const double* __restrict__ x, const double* __restrict__ b,
                                                          const double* __restrict__ den, float* __restrict__ dO,
                                                          double* part, int* bad, int probe)
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
        // gradient factors: d loss / d L'_ij = 2 (fa_i fb_j + fc_i fd_j) / den
        double fa[6], fb[6], fc[6], fd[6];
        if (probe)
        {
            double y[6], w[6], e[6], z[6], q[6];
            lower_solve6(Lc, bp, y);  // y = L'^-1 u
            upper_solve6(Lc, y, w);   // w = L'^-T y = A^-1 u
            for (int i = 0; i < 6; ++i)
            {
                e[i] = xp[i] - w[i];
                mine += e[i] * e[i];
            }
            lower_solve6(Lc, e, z);   // z = L'^-1 e
            upper_solve6(Lc, z, q);   // q = A^-1 e
            for (int i = 0; i < 6; ++i)
            {
                fa[i] = q[i];
                fb[i] = y[i];
                fc[i] = w[i];
                fd[i] = z[i];
            }
        }
        else
        {
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
            {
                fa[i] = r[i];
                fb[i] = u[i];
                fc[i] = xp[i];
                fd[i] = v[i];
            }
        }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j <= i; ++j)
            {
                const int k = i * (i + 1) / 2 + j;
                const double gg = 2.0 * (fa[i] * fb[j] + fc[i] * fd[j]) * inv_den;
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
// set by a tensor-core GEMM whose bounded wait ran out (reset before every forward pass)
int* tc_error_flag(pm_mlp* mlp) { return mlp->bad + 1; }

void check_tc_error(pm_mlp* mlp, cudaStream_t stream)
{
    int flag = 0;
    PM_CUDA(cudaMemcpyAsync(&flag, tc_error_flag(mlp), sizeof(int), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaStreamSynchronize(stream));
    if (flag)
        fail(PM_RUNTIME_ERROR, "learned preconditioner: a tensor-core GEMM did not complete");
}

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
    PM_CUDA(cudaMemsetAsync(tc_error_flag(mlp), 0, sizeof(int), stream));
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
    int* error = tc_error_flag(mlp);
    gemm(stream, M, kHid, kIn, mlp->F, kInPad, 1, W + kOffW1, kHid, 1, W + kOffB1, mlp->Z1, kHid, error, mlp->wait_limit,
         mlp->H1);
    gemm(stream, M, kHid, kHid, mlp->H1, kHid, 1, W + kOffW2, kHid, 1, W + kOffB2, mlp->Z2, kHid, error, mlp->wait_limit,
         mlp->H2);
    PM_CUDA(cudaMemsetAsync(mlp->O, 0, size_t(P) * kOutPad * sizeof(float), stream));
    gemm(stream, M, kOut, kHid, mlp->H2, kHid, 1, W + kOffW3, kOut, 1, W + kOffB3, mlp->O, kOutPad, error, mlp->wait_limit);
}

void check_view(const SchurView& v)
{
    if (!v.S || (v.P > 0 && !v.diag_pos))
        fail(PM_LOGIC_ERROR, "learned preconditioner: the workspace holds no assembled 6x6 system");
    if (v.P > INT32_MAX)
        fail(PM_OVERFLOW_ERROR, "learned preconditioner: too many block rows");
}

} // namespace

// Plain block Jacobi again, on the device, when the network's blocks are unusable (a block not
// positive definite, or a tensor-core GEMM that gave up): every row's FP64 inverse of its own
// diagonal block.  Nothing is done when both flags are clear.
template <typename T>
__global__ void learned_guard_kernel(int64_t P, const int* __restrict__ diag_pos, const T* __restrict__ S,
                                     double* __restrict__ minv, float* __restrict__ minv32, const int* __restrict__ bad)
{
    if (!bad[0] && !bad[1])
        return;
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
    {
        double m[36], inv[36], lower[36], work[6];
        const T* d = S + int64_t(diag_pos[p]) * 36;
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c)
                m[r * 6 + c] = static_cast<double>(r >= c ? d[r * 6 + c] : d[c * 6 + r]);
        if (!spd_inverse<6>(m, 6, inv, lower, work))
            for (int k = 0; k < 36; ++k)
                inv[k] = 0.0;
        for (int k = 0; k < 36; ++k)
            minv[p * 36 + k] = inv[k];
        if (minv32)
            for (int k = 0; k < 36; ++k)
                minv32[p * 36 + k] = static_cast<float>(inv[k]);
    }
}

void mlp_apply(const pm_mlp* cmlp, const SchurView& v, cudaStream_t stream, int* flags_host)
{
    pm_mlp* mlp = const_cast<pm_mlp*>(cmlp); // parameters are read only; scratch is reused
    check_view(v);
    forward(mlp, v, stream);
    if (v.P == 0)
        return;
    PM_CUDA(cudaMemsetAsync(bad_flag(mlp), 0, sizeof(int), stream));
    const unsigned grid = grid_for(v.P, 64, 4096);
    float* const m32 = v.mixed ? v.minv32 : nullptr;
    if (v.value_size == 8)
    {
        precond_kernel<double><<<grid, 64, 0, stream>>>(v.P, v.diag_pos, static_cast<const double*>(v.S), mlp->O,
                                                        v.minv, m32, bad_flag(mlp));
        PM_LAUNCH_CHECK();
        learned_guard_kernel<double><<<grid, 64, 0, stream>>>(v.P, v.diag_pos, static_cast<const double*>(v.S),
                                                              v.minv, m32, bad_flag(mlp));
    }
    else
    {
        precond_kernel<float><<<grid, 64, 0, stream>>>(v.P, v.diag_pos, static_cast<const float*>(v.S), mlp->O,
                                                       v.minv, m32, bad_flag(mlp));
        PM_LAUNCH_CHECK();
        learned_guard_kernel<float><<<grid, 64, 0, stream>>>(v.P, v.diag_pos, static_cast<const float*>(v.S),
                                                             v.minv, m32, bad_flag(mlp));
    }
    PM_LAUNCH_CHECK();
    // [0]: a corrected block was not positive definite, [1]: a GEMM gave up; read by the caller
    // after its next synchronisation
    if (flags_host)
        PM_CUDA(cudaMemcpyAsync(flags_host, bad_flag(mlp), 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
}

namespace
{

double train(pm_mlp* mlp, const SchurView& v, cudaStream_t stream, const double* x, const double* b, double lr,
             int probe = 0)
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
    squares_kernel<<<sg, kPartBlock, 0, stream>>>(n, probe ? x : b, part); // ||v||^2 or ||b||^2
    PM_LAUNCH_CHECK();
    finish_sum_kernel<<<1, 1, 0, stream>>>(static_cast<int>(sg), part, den);
    PM_LAUNCH_CHECK();
    const unsigned lg = grid_for(P, kPartBlock, kMaxPartBlocks);
    if (v.value_size == 8)
        loss_kernel<double><<<lg, kPartBlock, 0, stream>>>(P, v.diag_pos, static_cast<const double*>(v.S), mlp->O, x,
                                                           b, den, mlp->dO, part + kMaxPartBlocks, bad, probe);
    else
        loss_kernel<float><<<lg, kPartBlock, 0, stream>>>(P, v.diag_pos, static_cast<const float*>(v.S), mlp->O, x, b,
                                                          den, mlp->dO, part + kMaxPartBlocks, bad, probe);
    PM_LAUNCH_CHECK();
    finish_sum_kernel<<<1, 1, 0, stream>>>(static_cast<int>(lg), part + kMaxPartBlocks, num);
    PM_LAUNCH_CHECK();
    // backward (tensor-core GEMMs; the row dimension is the reduction of the weight gradients)
    float* G = mlp->grads;
    const float* W = mlp->params;
    float* splits = mlp->split;
    int* error = tc_error_flag(mlp);
    gemm_split(stream, kHid, kOut, M, mlp->H2, 1, kHid, mlp->dO, kOutPad, 1, G + kOffW3, kOut, splits, error, mlp->wait_limit);
    colsum(stream, P, kOut, kOutPad, mlp->dO, G + kOffB3, splits);
    gemm(stream, M, kHid, kOut, mlp->dO, kOutPad, 1, W + kOffW3, 1, kOut, nullptr, mlp->dH, kHid, error, mlp->wait_limit);
    gelu_back_kernel<<<grid_for(P * kHid, 256, 4096), 256, 0, stream>>>(P * kHid, mlp->dH, mlp->Z2, mlp->dZ);
    PM_LAUNCH_CHECK();
    gemm_split(stream, kHid, kHid, M, mlp->H1, 1, kHid, mlp->dZ, kHid, 1, G + kOffW2, kHid, splits, error, mlp->wait_limit);
    colsum(stream, P, kHid, kHid, mlp->dZ, G + kOffB2, splits);
    gemm(stream, M, kHid, kHid, mlp->dZ, kHid, 1, W + kOffW2, 1, kHid, nullptr, mlp->dH, kHid, error, mlp->wait_limit);
    gelu_back_kernel<<<grid_for(P * kHid, 256, 4096), 256, 0, stream>>>(P * kHid, mlp->dH, mlp->Z1, mlp->dZ);
    PM_LAUNCH_CHECK();
    gemm_split(stream, kIn, kHid, M, mlp->F, 1, kInPad, mlp->dZ, kHid, 1, G + kOffW1, kHid, splits, error, mlp->wait_limit);
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
    check_tc_error(mlp, stream);
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

int pm_mlp_set_wait_limit(pm_mlp* mlp, int64_t polls)
{
    return pm::guarded([&] {
        if (!mlp)
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_set_wait_limit: null network");
        if (polls < 0)
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_set_wait_limit: the limit must be non-negative");
        mlp->wait_limit = polls;
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
        pm::check_tc_error(mlp, stream);
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

int pm_mlp_train_probe_step(pm_mlp* mlp, pm_schur_workspace* ws, pm_stream_t stream, const double* v,
                            const double* sv, double learning_rate, double* loss)
{
    return pm::guarded([&] {
        if (!mlp || !ws)
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_train_probe_step: null argument");
        if (!(learning_rate >= 0.0) || !std::isfinite(learning_rate))
            pm::fail(PM_INVALID_ARGUMENT, "pm_mlp_train_probe_step: learning rate must be finite and non-negative");
        const double l = pm::train(mlp, pm::schur_view(ws, false), stream, v, sv, learning_rate, 1);
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
