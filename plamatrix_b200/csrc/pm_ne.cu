// Device normal equations: upload/download of the reference's BlockNormalEquations state and
// the Huber-weighted accumulation of device-resident observations (the caller side of the
// reference's LM loop: evaluateHuberLoss + addResidualBlock, robust_loss.h:27-51 and
// block_normal_equations.cpp:136-312).
//
// Accumulation order.  For every eliminated block the observations are visited in input
// order, and so are the observations of every (primary, eliminated) pair; the products
// `weight * value * jacobian` are evaluated as two rounded multiplies and one rounded add
// (no fused multiply-add), so the eliminated diagonal blocks, eliminated gradients and cross
// blocks equal the reference's host accumulation bit for bit.  The primary diagonal blocks
// and gradients sum ~N/P observations per primary; they are reduced in a fixed
// (scheduling-independent) tree order instead of the reference's serial order.
#include "pm_schur.cuh"

#include <algorithm>
#include <cmath>
#include <sstream>
#include <vector>

pm_normal_equations::~pm_normal_equations()
{
    numeric.release();
    topology.release();
    observation_copy.release();
    weights.release();
    if (by_eliminated)
        pm_sparse_workspace_destroy(by_eliminated);
    if (by_primary)
        pm_sparse_workspace_destroy(by_primary);
    if (by_eliminated_order)
        pm_sparse_workspace_destroy(by_eliminated_order);
    cross_runs.release();
    observation_slots.release();
    observation_status.release();
}

namespace pm
{
namespace
{

void layout_numeric(pm_normal_equations* ne, cudaStream_t stream)
{
    const size_t s = ne->value_size;
    Carver plan;
    plan.take<char>(ne->P * ne->bp * ne->bp * s);
    plan.take<char>(ne->L * ne->bl * ne->bl * s);
    plan.take<char>(ne->P * ne->bp * s);
    plan.take<char>(ne->L * ne->bl * s);
    plan.take<char>(ne->cross_count * ne->bp * ne->bl * s);
    plan.take<char>(ne->primary_cross_count * ne->bp * ne->bp * s);
    ne->numeric.ensure(plan.offset + 256, stream, "normal equations");
    Carver c;
    c.base = static_cast<char*>(ne->numeric.ptr);
    ne->primary_diagonal = c.take<char>(ne->P * ne->bp * ne->bp * s);
    ne->eliminated_diagonal = c.take<char>(ne->L * ne->bl * ne->bl * s);
    ne->primary_gradient = c.take<char>(ne->P * ne->bp * s);
    ne->eliminated_gradient = c.take<char>(ne->L * ne->bl * s);
    ne->cross_values = c.take<char>(ne->cross_count * ne->bp * ne->bl * s);
    ne->primary_cross_values = c.take<char>(ne->primary_cross_count * ne->bp * ne->bp * s);
}

void layout_topology(pm_normal_equations* ne, cudaStream_t stream)
{
    Carver plan;
    plan.take<int>(ne->L + 1);
    plan.take<int>(ne->cross_count + 1);
    plan.take<int>(ne->cross_count + 1);
    plan.take<int>(ne->primary_cross_count + 1);
    plan.take<int>(ne->primary_cross_count + 1);
    ne->topology.ensure(plan.offset + 256, stream, "normal equations");
    Carver c;
    c.base = static_cast<char*>(ne->topology.ptr);
    ne->cross_offsets = c.take<int>(ne->L + 1);
    ne->cross_primary = c.take<int>(ne->cross_count + 1);
    ne->cross_eliminated = c.take<int>(ne->cross_count + 1);
    ne->primary_cross_row = c.take<int>(ne->primary_cross_count + 1);
    ne->primary_cross_col = c.take<int>(ne->primary_cross_count + 1);
}

__global__ void narrow_kernel(const int64_t* __restrict__ in, int* __restrict__ out, int64_t n)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = static_cast<int>(in[i]);
}

// cross_eliminated[c] = l for the crosses of every eliminated block
__global__ void cross_owner_kernel(const int* __restrict__ offsets, int64_t L, int* __restrict__ owner)
{
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < L; l += int64_t(gridDim.x) * blockDim.x)
        for (int c = offsets[l]; c < offsets[l + 1]; ++c)
            owner[c] = static_cast<int>(l);
}

// crosses of the observation path: one per distinct primary of each eliminated bucket, in
// ascending primary order; cross_run[c] is the bucket position of the cross's first observation
__global__ void observation_crosses_kernel(CooView v, const int* __restrict__ cross_offsets,
                                           int* __restrict__ cross_primary, int* __restrict__ cross_run)
{
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < v.rows; l += int64_t(gridDim.x) * blockDim.x)
    {
        int at = cross_offsets[l];
        const int b = v.bucket_start[l], e = v.bucket_start[l + 1];
        for (int q = b; q < e; ++q)
        {
            const uint32_t p = static_cast<uint32_t>(v.keys[q] >> 32);
            if (q == b || p != static_cast<uint32_t>(v.keys[q - 1] >> 32))
            {
                cross_run[at] = q;
                cross_primary[at++] = static_cast<int>(p);
            }
        }
        if (l == v.rows - 1)
            cross_run[at] = e;
    }
}

// position of every observation in the input-order buckets (indexed by observation)
__global__ void order_position_kernel(CooView vo, int* __restrict__ position)
{
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < vo.count; q += int64_t(gridDim.x) * blockDim.x)
        position[static_cast<uint32_t>(vo.keys[q])] = static_cast<int>(q);
}

// slot[q] for every input-order bucket position q: the cross c of that observation, stored as
// c when it is the cross's first observation in input order and as ~c otherwise
__global__ void observation_slots_kernel(int64_t C, const uint64_t* __restrict__ keys, const int* __restrict__ cross_run,
                                         const int* __restrict__ position, int* __restrict__ slot)
{
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < C; c += int64_t(gridDim.x) * blockDim.x)
        for (int q = cross_run[c]; q < cross_run[c + 1]; ++q)
            slot[position[static_cast<uint32_t>(keys[q])]] = q == cross_run[c] ? static_cast<int>(c) : ~static_cast<int>(c);
}

// *differs = 1 when either caller index array differs from the saved copy (int32: the saved
// arrays passed the topology build's range checks, so widening them back is exact)
__global__ void compare_kernel(const int64_t* __restrict__ a, const int* __restrict__ a_saved,
                               const int64_t* __restrict__ b, const int* __restrict__ b_saved, int64_t n,
                               int* differs)
{
    bool diff = false;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        diff |= (a[i] != static_cast<int64_t>(a_saved[i])) | (b[i] != static_cast<int64_t>(b_saved[i]));
    if (__any_sync(0xffffffffu, diff) && (threadIdx.x & 31) == 0)
        *differs = 1;
}

template <typename T>
__device__ __forceinline__ T squared_norm(const T* r, int m)
{
    T squared = T(0);
    for (int k = 0; k < m; ++k)
        squared = add_rn(squared, mul_rn(r[k], r[k]));
    return squared;
}

template <typename T>
__device__ __forceinline__ T huber_weight_of(T squared, T delta)
{
    if (delta == T(0) || squared <= mul_rn(delta, delta))
        return T(1);
    return delta / sqrt(squared);
}

template <typename T>
__device__ __forceinline__ T huber_weight(const T* r, int m, T delta)
{
    return huber_weight_of(squared_norm(r, m), delta);
}

// evaluateHuberLoss rejects a squared residual norm that is not finite (robust_loss.h:31-35):
// the device path records the first such observation for the host to report
template <typename T>
__device__ __forceinline__ void note_nonfinite(T squared, int64_t i, long long* first_bad)
{
    if (!isfinite(squared))
        atomicMin(first_bad, static_cast<long long>(i));
}

// One residual row's terms, each `weight * value * jacobian` as two rounded multiplies and a
// rounded add (the reference's host accumulation order).
template <typename T>
__device__ __forceinline__ void eliminated3_row(T* H, T* g, T weight, const T* jrow, T rr)
{
#pragma unroll
    for (int col = 0; col < 3; ++col)
    {
        const T wv = mul_rn(weight, jrow[col]);
        g[col] = add_rn(g[col], mul_rn(wv, rr));
#pragma unroll
        for (int other = 0; other < 3; ++other)
            H[col * 3 + other] = add_rn(H[col * 3 + other], mul_rn(wv, jrow[other]));
    }
}

template <typename T>
__device__ __forceinline__ void cross63_row(T* W, T weight, const T* prow, const T* lrow)
{
#pragma unroll
    for (int pc = 0; pc < 6; ++pc)
    {
        const T wv = mul_rn(weight, prow[pc]);
#pragma unroll
        for (int ec = 0; ec < 3; ++ec)
            W[pc * 3 + ec] = add_rn(W[pc * 3 + ec], mul_rn(wv, lrow[ec]));
    }
}

// position of entry (c, o), c <= o, of a symmetric 6x6 block in its packed upper triangle
__host__ __device__ constexpr int upper6(int c, int o) { return c * 6 - c * (c - 1) / 2 + (o - c); }

// One residual row's terms of the primary block: the upper triangle (w J_c) J_o, o >= c (21
// entries, packed), then the gradient (w J_c) r (6 entries).  The lower triangle is the mirror.
template <typename T>
__device__ __forceinline__ void primary6_row(T* sum, T weight, const T* jrow, T rr)
{
#pragma unroll
    for (int c = 0; c < 6; ++c)
    {
        const T wv = mul_rn(weight, jrow[c]);
        sum[21 + c] = add_rn(sum[21 + c], mul_rn(wv, rr));
#pragma unroll
        for (int o = c; o < 6; ++o)
            sum[upper6(c, o)] = add_rn(sum[upper6(c, o)], mul_rn(wv, jrow[o]));
    }
}

// N contiguous scalars in pairs (16-byte loads for double, 8-byte for float); p aligned to two
// scalars
template <typename T, int N>
__device__ __forceinline__ void load_vec(const T* __restrict__ p, T* out)
{
    static_assert(N % 2 == 0, "pairs of scalars");
    if constexpr (sizeof(T) == 8)
    {
#pragma unroll
        for (int e = 0; e < N / 2; ++e)
        {
            const double2 v = __ldg(reinterpret_cast<const double2*>(p) + e);
            out[2 * e] = v.x;
            out[2 * e + 1] = v.y;
        }
    }
    else
    {
#pragma unroll
        for (int e = 0; e < N / 2; ++e)
        {
            const float2 v = __ldg(reinterpret_cast<const float2*>(p) + e);
            out[2 * e] = v.x;
            out[2 * e + 1] = v.y;
        }
    }
}

template <typename T, int N>
__device__ __forceinline__ void store_vec(T* __restrict__ p, const T* in)
{
    static_assert(N % 2 == 0, "pairs of scalars");
#pragma unroll
    for (int e = 0; e < N / 2; ++e)
    {
        if constexpr (sizeof(T) == 8)
            reinterpret_cast<double2*>(p)[e] = make_double2(in[2 * e], in[2 * e + 1]);
        else
            reinterpret_cast<float2*>(p)[e] = make_float2(in[2 * e], in[2 * e + 1]);
    }
}

// Huber weight of every observation (one thread each, coalesced residual reads).
template <typename T>
__global__ void huber_weights_kernel(int64_t count, int m, const T* __restrict__ res, T delta, T* __restrict__ weight,
                                     long long* first_bad)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x)
    {
        const T squared = squared_norm(res + i * m, m);
        note_nonfinite(squared, i, first_bad);
        weight[i] = huber_weight_of(squared, delta);
    }
}

// Per eliminated block, any block sizes up to 16: the same sums as the fixed-size kernel below,
// accumulated in place in the output arrays.
template <typename T>
__global__ void __launch_bounds__(128) eliminated_accumulate_generic_kernel(
    CooView v, int m, int bp, int bl, const T* __restrict__ jp, const T* __restrict__ jl, const T* __restrict__ res,
    const T* __restrict__ weights, const int* __restrict__ cross_offsets, T* __restrict__ hll, T* __restrict__ gl,
    T* __restrict__ w)
{
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < v.rows; l += int64_t(gridDim.x) * blockDim.x)
    {
        const int b = v.bucket_start[l], e = v.bucket_start[l + 1];
        T* H = hll + l * bl * bl;
        T* g = gl + l * bl;
        for (int i = 0; i < bl * bl; ++i)
            H[i] = T(0);
        for (int i = 0; i < bl; ++i)
            g[i] = T(0);
        constexpr int kSelectMax = 64;
        const bool select = e - b <= kSelectMax;
        uint32_t last = 0;
        for (int visited = 0; visited < e - b; ++visited)
        {
            uint32_t best = 0xffffffffu;
            if (select)
            {
                for (int q = b; q < e; ++q)
                {
                    const uint32_t src = static_cast<uint32_t>(v.keys[q]);
                    if ((visited == 0 || src > last) && src < best)
                        best = src;
                }
            }
            else
            {
                best = static_cast<uint32_t>(v.keys[b + visited]);
            }
            last = best;
            const int64_t i = best;
            const T* r = res + i * m;
            const T weight = weights[i];
            const T* J = jl + i * m * bl;
            for (int row = 0; row < m; ++row)
                for (int col = 0; col < bl; ++col)
                {
                    const T wv = mul_rn(weight, J[row * bl + col]);
                    g[col] = add_rn(g[col], mul_rn(wv, r[row]));
                    for (int other = 0; other < bl; ++other)
                        H[col * bl + other] = add_rn(H[col * bl + other], mul_rn(wv, J[row * bl + other]));
                }
        }
        int cross = cross_offsets[l] - 1;
        for (int q = b; q < e; ++q)
        {
            const uint64_t key = v.keys[q];
            if (q == b || (key >> 32) != (v.keys[q - 1] >> 32))
            {
                ++cross;
                T* W = w + int64_t(cross) * bp * bl;
                for (int k = 0; k < bp * bl; ++k)
                    W[k] = T(0);
            }
            T* W = w + int64_t(cross) * bp * bl;
            const int64_t i = static_cast<uint32_t>(key);
            const T weight = weights[i];
            const T* Jp = jp + i * m * bp;
            const T* Jl = jl + i * m * bl;
            for (int row = 0; row < m; ++row)
                for (int pc = 0; pc < bp; ++pc)
                {
                    const T wv = mul_rn(weight, Jp[row * bp + pc]);
                    for (int ec = 0; ec < bl; ++ec)
                        W[pc * bl + ec] = add_rn(W[pc * bl + ec], mul_rn(wv, Jl[row * bl + ec]));
                }
        }
    }
}

// Eliminated block (3x3), thread per block: Hll and g_l over its observations in input order
// (addResidualBlocks accumulates per residual in call order, block_normal_equations.cpp:294-311).
// The bucket of l in `v` lists the observation indices in ascending order.
template <typename T>
__global__ void __launch_bounds__(128) eliminated_diagonal3_kernel(CooView v, int m, const T* __restrict__ jl,
                                                                   const T* __restrict__ res,
                                                                   const T* __restrict__ weights, T* __restrict__ hll,
                                                                   T* __restrict__ gl)
{
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < v.rows; l += int64_t(gridDim.x) * blockDim.x)
    {
        const int b = v.bucket_start[l], e = v.bucket_start[l + 1];
        T H[9], g[3];
#pragma unroll
        for (int k = 0; k < 9; ++k)
            H[k] = T(0);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            g[k] = T(0);
        for (int q = b; q < e; ++q)
        {
            const int64_t i = static_cast<uint32_t>(v.keys[q]);
            const T weight = weights[i];
            const T* J = jl + i * m * 3;
            const T* r = res + i * m;
            for (int row = 0; row < m; ++row)
                eliminated3_row(H, g, weight, J + row * 3, r[row]);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k)
            hll[l * 9 + k] = H[k];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            gl[l * 3 + k] = g[k];
    }
}

// Cross block (6x3), thread per cross: W = sum over the cross's observations (a run of equal
// primary in its eliminated bucket, input order) of w Jp^T Jl (block_normal_equations.cpp:268-292).
template <typename T>
__global__ void __launch_bounds__(128) cross_accumulate63_kernel(int64_t C, const uint64_t* __restrict__ keys,
                                                                 const int* __restrict__ cross_run, int m,
                                                                 const T* __restrict__ jp, const T* __restrict__ jl,
                                                                 const T* __restrict__ weights, T* __restrict__ w)
{
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < C; c += int64_t(gridDim.x) * blockDim.x)
    {
        T W[18];
#pragma unroll
        for (int k = 0; k < 18; ++k)
            W[k] = T(0);
        for (int q = cross_run[c]; q < cross_run[c + 1]; ++q)
        {
            const int64_t i = static_cast<uint32_t>(keys[q]);
            const T weight = weights[i];
            const T* Jp = jp + i * m * 6;
            const T* Jl = jl + i * m * 3;
            for (int row = 0; row < m; ++row)
                cross63_row(W, weight, Jp + row * 6, Jl + row * 3);
        }
        T* out = w + c * 18;
#pragma unroll
        for (int k = 0; k < 18; ++k)
            out[k] = W[k];
    }
}

// Two-row residuals, thread per eliminated block, one pass over the block's observations in
// input order: Hll and g_l (the sums of eliminated_diagonal3_kernel) and every cross block W
// (the sums of cross_accumulate63_kernel), the Huber weight evaluated once per observation and
// rows read in pairs of scalars.  slot[q] names the cross of input-order position q: its first
// observation starts the cross's W from zero, a later one (~c) adds to the row this thread
// stored before, so every W is its observations' sum in input order.  A thread's crosses are
// contiguous in W (crosses are grouped by eliminated block), so its row stores fill whole
// sectors.  The next observation's index and slot are loaded one step ahead.
template <typename T>
__global__ void __launch_bounds__(128) eliminated_cross3_m2_kernel(CooView vo, const int* __restrict__ slot,
                                                                   const T* __restrict__ jp, const T* __restrict__ jl,
                                                                   const T* __restrict__ res, T delta,
                                                                   T* __restrict__ hll, T* __restrict__ gl,
                                                                   T* __restrict__ w, long long* first_bad)
{
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < vo.rows; l += int64_t(gridDim.x) * blockDim.x)
    {
        T H[9], g[3];
#pragma unroll
        for (int k = 0; k < 9; ++k)
            H[k] = T(0);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            g[k] = T(0);
        const int e = vo.bucket_start[l + 1];
        int q = vo.bucket_start[l];
        // software pipeline: the next observation's rows are loaded before the current one is
        // summed (two observations in flight per thread), its index one step further ahead
        T r[2], Jl[6], Jp[12];
        int64_t i = 0;
        int s = 0;
        if (q < e)
        {
            i = static_cast<uint32_t>(vo.keys[q]);
            s = slot[q];
            load_vec<T, 2>(res + i * 2, r);
            load_vec<T, 6>(jl + i * 6, Jl);
            load_vec<T, 12>(jp + i * 12, Jp);
        }
        uint64_t next = q + 1 < e ? vo.keys[q + 1] : 0;
        int next_slot = q + 1 < e ? slot[q + 1] : 0;
        for (; q < e; ++q)
        {
            T rn[2], Jln[6], Jpn[12];
            const int64_t in = static_cast<uint32_t>(next);
            const int sn = next_slot;
            const bool more = q + 1 < e;
            if (more)
            {
                load_vec<T, 2>(res + in * 2, rn);
                load_vec<T, 6>(jl + in * 6, Jln);
                load_vec<T, 12>(jp + in * 12, Jpn);
                if (q + 2 < e)
                {
                    next = vo.keys[q + 2];
                    next_slot = slot[q + 2];
                }
            }
            const T squared = squared_norm(r, 2);
            note_nonfinite(squared, i, first_bad);
            const T weight = huber_weight_of(squared, delta);
            eliminated3_row(H, g, weight, Jl, r[0]);
            eliminated3_row(H, g, weight, Jl + 3, r[1]);
            const int64_t c = s >= 0 ? s : ~s;
            T W[18];
            if (s >= 0)
            {
#pragma unroll
                for (int k = 0; k < 18; ++k)
                    W[k] = T(0);
            }
            else
            {
                // a repeated (primary, eliminated) pair: this thread's own earlier store
#pragma unroll
                for (int k = 0; k < 18; ++k)
                    W[k] = w[c * 18 + k];
            }
            cross63_row(W, weight, Jp, Jl);
            cross63_row(W, weight, Jp + 6, Jl + 3);
            store_vec<T, 18>(w + c * 18, W);
            if (more)
            {
#pragma unroll
                for (int k = 0; k < 2; ++k)
                    r[k] = rn[k];
#pragma unroll
                for (int k = 0; k < 6; ++k)
                    Jl[k] = Jln[k];
#pragma unroll
                for (int k = 0; k < 12; ++k)
                    Jp[k] = Jpn[k];
                i = in;
                s = sn;
            }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k)
            hll[l * 9 + k] = H[k];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            gl[l * 3 + k] = g[k];
    }
}

// Per primary block (6x6): Hpp and g_p over its observations.  Warp w of the block owns a
// contiguous slice of the primary's observation list (a multiple of 32 long) and lane j of it the
// observations lo_w + j, lo_w + j + 32, ...; every lane sums its 27 terms serially (Hpp's upper
// triangle and g_p), the lanes of a warp are combined by a fixed xor-shuffle tree and the warps in
// warp order; Hpp's lower triangle is written as the mirror of the upper.  The reduction tree
// depends only on the list length, never on scheduling.  At most 128 registers: four CTAs per SM
// (a 4,000-primary system then runs 6.8 waves of 592 CTAs instead of 9.0 of 444).
// M == 2: two-row residuals read in pairs of scalars, Huber weight evaluated inline (weights
// unused); M == 0: any residual size m, weights precomputed.
template <typename T, int M>
__global__ void __launch_bounds__(128, 4) primary_accumulate6_kernel(CooView v, int m, const T* __restrict__ jp,
                                                                  const T* __restrict__ res, T delta,
                                                                  const T* __restrict__ weights, T* __restrict__ hpp,
                                                                  T* __restrict__ gp)
{
    constexpr int W = 27; // 21 upper Hpp entries + 6 gradient entries
    constexpr int kWarps = 4;
    __shared__ T part[kWarps][W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t p = blockIdx.x; p < v.rows; p += gridDim.x)
    {
        const int b = v.bucket_start[p], e = v.bucket_start[p + 1];
        const int len = e - b;
        const int per = ((len + kWarps * 32 - 1) / (kWarps * 32)) * 32;
        const int lo = b + min(len, warp * per), hi = b + min(len, (warp + 1) * per);
        T sum[W];
#pragma unroll
        for (int k = 0; k < W; ++k)
            sum[k] = T(0);
        // the next observation's index is loaded one step ahead
        uint64_t next = lo + lane < hi ? v.keys[lo + lane] : 0;
        for (int q = lo + lane; q < hi; q += 32)
        {
            const int64_t i = static_cast<uint32_t>(next);
            if (q + 32 < hi)
                next = v.keys[q + 32];
            if constexpr (M == 2)
            {
                T r[2], J[12];
                load_vec<T, 2>(res + i * 2, r);
                load_vec<T, 12>(jp + i * 12, J);
                const T weight = huber_weight(r, 2, delta);
                primary6_row(sum, weight, J, r[0]);
                primary6_row(sum, weight, J + 6, r[1]);
            }
            else
            {
                const T weight = weights[i];
                const T* r = res + i * m;
                const T* J = jp + i * m * 6;
                for (int row = 0; row < m; ++row)
                    primary6_row(sum, weight, J + row * 6, r[row]);
            }
        }
#pragma unroll
        for (int k = 0; k < W; ++k)
        {
            T x = sum[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                x = add_rn(x, __shfl_xor_sync(0xffffffffu, x, o));
            sum[k] = x;
        }
        if (lane == 0)
        {
#pragma unroll
            for (int k = 0; k < W; ++k)
                part[warp][k] = sum[k];
        }
        __syncthreads();
        if (threadIdx.x < 42)
        {
            const int t = threadIdx.x;
            const int k = t < 36 ? upper6(min(t / 6, t % 6), max(t / 6, t % 6)) : t - 15;
            T total = T(0);
            for (int wi = 0; wi < kWarps; ++wi)
                total = add_rn(total, part[wi][k]);
            if (t < 36)
                hpp[p * 36 + t] = total;
            else
                gp[p * 6 + (t - 36)] = total;
        }
        __syncthreads();
    }
}

// Generic block sizes: one thread per contiguous slice, slices combined in thread order.
template <typename T>
__global__ void __launch_bounds__(128) primary_accumulate_kernel(CooView v, int m, int bp, const T* __restrict__ jp,
                                                                 const T* __restrict__ res,
                                                                 const T* __restrict__ weights, T* __restrict__ hpp,
                                                                 T* __restrict__ gp)
{
    extern __shared__ unsigned char smem_raw[];
    T* part = reinterpret_cast<T*>(smem_raw); // [blockDim][bp*bp + bp]
    const int width = bp * bp + bp;
    for (int64_t p = blockIdx.x; p < v.rows; p += gridDim.x)
    {
        const int b = v.bucket_start[p], e = v.bucket_start[p + 1];
        const int len = e - b;
        const int per = (len + blockDim.x - 1) / blockDim.x;
        const int lo = b + min(len, int(threadIdx.x) * per), hi = b + min(len, int(threadIdx.x + 1) * per);
        T* acc = part + threadIdx.x * width;
        for (int k = 0; k < width; ++k)
            acc[k] = T(0);
        for (int q = lo; q < hi; ++q)
        {
            const int64_t i = static_cast<uint32_t>(v.keys[q]);
            const T* r = res + i * m;
            const T weight = weights[i];
            const T* J = jp + i * m * bp;
            for (int row = 0; row < m; ++row)
                for (int col = 0; col < bp; ++col)
                {
                    const T wv = mul_rn(weight, J[row * bp + col]);
                    acc[bp * bp + col] = add_rn(acc[bp * bp + col], mul_rn(wv, r[row]));
                    for (int other = 0; other < bp; ++other)
                        acc[col * bp + other] = add_rn(acc[col * bp + other], mul_rn(wv, J[row * bp + other]));
                }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < width; k += blockDim.x)
        {
            T total = T(0);
            for (int t = 0; t < blockDim.x; ++t)
                total = add_rn(total, part[t * width + k]);
            if (k < bp * bp)
                hpp[p * bp * bp + k] = total;
            else
                gp[p * bp + (k - bp * bp)] = total;
        }
        __syncthreads();
    }
}

template <typename T>
void ne_upload(pm_normal_equations* ne, cudaStream_t stream, const T* hpp, const T* hll, const T* gp, const T* gl,
               int64_t C, const int64_t* cross_offsets, const int64_t* cross_primary, const T* cross_values,
               int64_t PC, const int64_t* pc_row, const int64_t* pc_col, const T* pc_values)
{
    if (!ne)
        fail(PM_INVALID_ARGUMENT, "normal equations handle is null");
    if (ne->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "normal equations scalar type mismatch");
    if (C < 0 || PC < 0 || C > INT32_MAX - 1 || PC > INT32_MAX - 1)
        fail(PM_INVALID_ARGUMENT, "invalid cross block counts");
    if (ne->observation_status.ptr) // uploaded state carries no observations
        PM_CUDA(cudaMemsetAsync(ne->observation_status.ptr, 0x7f, sizeof(long long), stream));
    // host-side topology validation (the reference rejects these at accumulation time)
    if (ne->L > 0 && (!cross_offsets || cross_offsets[0] != 0 || cross_offsets[ne->L] != C))
        fail(PM_INVALID_ARGUMENT, "cross offsets must start at zero and end at the cross count");
    for (int64_t l = 0; l < ne->L; ++l)
        if (cross_offsets[l + 1] < cross_offsets[l])
            fail(PM_INVALID_ARGUMENT, "cross offsets must be non-decreasing");
    for (int64_t c = 0; c < C; ++c)
        if (cross_primary[c] < 0 || cross_primary[c] >= ne->P)
            fail(PM_OUT_OF_RANGE, "BlockNormalEquations: primary block index out of range");
    for (int64_t k = 0; k < PC; ++k)
        if (pc_row[k] < 0 || pc_col[k] >= ne->P || pc_row[k] >= pc_col[k])
            fail(PM_INVALID_ARGUMENT, "BlockNormalEquations: primary cross blocks must be upper triangular");
    ne->cross_count = C;
    ne->primary_cross_count = PC;
    layout_numeric(ne, stream);
    layout_topology(ne, stream);
    const size_t s = sizeof(T);
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (bytes)
            PM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
    };
    up(ne->primary_diagonal, hpp, ne->P * ne->bp * ne->bp * s);
    up(ne->eliminated_diagonal, hll, ne->L * ne->bl * ne->bl * s);
    up(ne->primary_gradient, gp, ne->P * ne->bp * s);
    up(ne->eliminated_gradient, gl, ne->L * ne->bl * s);
    up(ne->cross_values, cross_values, C * ne->bp * ne->bl * s);
    up(ne->primary_cross_values, pc_values, PC * ne->bp * ne->bp * s);
    // int64 -> int32 topology through a staging buffer
    std::vector<int> staging(static_cast<size_t>(std::max<int64_t>({ne->L + 1, C, PC, 1})));
    auto narrow = [&](int* dst, const int64_t* src, int64_t n) {
        for (int64_t i = 0; i < n; ++i)
            staging[i] = static_cast<int>(src[i]);
        if (n)
        {
            PM_CUDA(cudaMemcpyAsync(dst, staging.data(), n * sizeof(int), cudaMemcpyHostToDevice, stream));
            PM_CUDA(cudaStreamSynchronize(stream));
        }
    };
    if (ne->L > 0)
        narrow(ne->cross_offsets, cross_offsets, ne->L + 1);
    else
        PM_CUDA(cudaMemsetAsync(ne->cross_offsets, 0, sizeof(int), stream));
    narrow(ne->cross_primary, cross_primary, C);
    narrow(ne->primary_cross_row, pc_row, PC);
    narrow(ne->primary_cross_col, pc_col, PC);
    if (ne->L > 0)
    {
        cross_owner_kernel<<<grid_for(ne->L, 256, 4096), 256, 0, stream>>>(ne->cross_offsets, ne->L,
                                                                           ne->cross_eliminated);
        PM_LAUNCH_CHECK();
    }
    PM_CUDA(cudaStreamSynchronize(stream));
    ne->observation_topology = false;
    bool sorted = true;
    for (int64_t l = 0; l < ne->L && sorted; ++l)
        for (int64_t c = cross_offsets[l] + 1; c < cross_offsets[l + 1]; ++c)
            if (cross_primary[c] <= cross_primary[c - 1])
            {
                sorted = false;
                break;
            }
    ne->crosses_sorted = sorted;
    ne->topology_version += 1;
}

template <typename T>
void ne_download(const pm_normal_equations* ne, cudaStream_t stream, T* hpp, T* hll, T* gp, T* gl,
                 int64_t* cross_offsets, int64_t* cross_primary, T* cross_values, int64_t* pc_row, int64_t* pc_col,
                 T* pc_values)
{
    if (!ne)
        fail(PM_INVALID_ARGUMENT, "normal equations handle is null");
    if (ne->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "normal equations scalar type mismatch");
    const size_t s = sizeof(T);
    auto down = [&](void* dst, const void* src, size_t bytes) {
        if (dst && bytes)
            PM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream));
    };
    down(hpp, ne->primary_diagonal, ne->P * ne->bp * ne->bp * s);
    down(hll, ne->eliminated_diagonal, ne->L * ne->bl * ne->bl * s);
    down(gp, ne->primary_gradient, ne->P * ne->bp * s);
    down(gl, ne->eliminated_gradient, ne->L * ne->bl * s);
    down(cross_values, ne->cross_values, ne->cross_count * ne->bp * ne->bl * s);
    down(pc_values, ne->primary_cross_values, ne->primary_cross_count * ne->bp * ne->bp * s);
    std::vector<int> staging(static_cast<size_t>(std::max<int64_t>({ne->L + 1, ne->cross_count, ne->primary_cross_count, 1})));
    auto widen = [&](int64_t* dst, const int* src, int64_t n) {
        if (!dst || n == 0)
            return;
        PM_CUDA(cudaMemcpyAsync(staging.data(), src, n * sizeof(int), cudaMemcpyDeviceToHost, stream));
        PM_CUDA(cudaStreamSynchronize(stream));
        for (int64_t i = 0; i < n; ++i)
            dst[i] = staging[i];
    };
    if (ne->L > 0)
        widen(cross_offsets, ne->cross_offsets, ne->L + 1);
    else if (cross_offsets)
        cross_offsets[0] = 0;
    widen(cross_primary, ne->cross_primary, ne->cross_count);
    widen(pc_row, ne->primary_cross_row, ne->primary_cross_count);
    widen(pc_col, ne->primary_cross_col, ne->primary_cross_count);
    PM_CUDA(cudaStreamSynchronize(stream));
}

template <typename T>
void ne_accumulate(pm_normal_equations* ne, cudaStream_t stream, int64_t count, int64_t m, const int64_t* obs_primary,
                   const int64_t* obs_eliminated, const T* jp, const T* jl, const T* res, T delta)
{
    if (!ne)
        fail(PM_INVALID_ARGUMENT, "normal equations handle is null");
    if (ne->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "normal equations scalar type mismatch");
    if (count < 0 || m <= 0 || m > 64)
        fail(PM_INVALID_ARGUMENT, "observation count must be non-negative and residual size in [1, 64]");
    if (!(delta >= T(0)) || !std::isfinite(static_cast<double>(delta)))
        fail(PM_INVALID_ARGUMENT, "evaluateHuberLoss: delta must be finite and non-negative");
    if (count > INT32_MAX - 1)
        fail(PM_OVERFLOW_ERROR, "observation count exceeds the int32 range of the device path");
    if (ne->bp > 16 || ne->bl > 16)
        fail(PM_INVALID_ARGUMENT, "device observation path supports block sizes up to 16");
    if (count > 0 && (!obs_primary || !obs_eliminated || !jp || !jl || !res))
        fail(PM_INVALID_ARGUMENT, "observation arrays must be non-null");
    // ---- topology (cached while the index arrays are unchanged)
    bool rebuild = !ne->observation_topology || ne->observation_count != count || ne->residual_size != m;
    int* saved_primary = nullptr;
    int* saved_eliminated = nullptr;
    int64_t* zeros = nullptr;
    int* differs = nullptr;
    auto carve = [&]() {
        Carver c;
        c.base = static_cast<char*>(ne->observation_copy.ptr);
        zeros = c.take<int64_t>(count + 1);
        saved_primary = c.take<int>(count + 1);
        saved_eliminated = c.take<int>(count + 1);
        differs = c.take<int>(1);
    };
    if (!rebuild)
    {
        carve();
        PM_CUDA(cudaMemsetAsync(differs, 0, sizeof(int), stream));
        compare_kernel<<<grid_for(count, 256, 4096), 256, 0, stream>>>(obs_primary, saved_primary, obs_eliminated,
                                                                         saved_eliminated, count, differs);
        PM_LAUNCH_CHECK();
        int host_differs = 0;
        PM_CUDA(cudaMemcpyAsync(&host_differs, differs, sizeof(int), cudaMemcpyDeviceToHost, stream));
        PM_CUDA(cudaStreamSynchronize(stream));
        rebuild = host_differs != 0;
    }
    if (rebuild)
    {
        Carver plan;
        plan.take<int64_t>(count + 1);
        plan.take<int>(count + 1);
        plan.take<int>(count + 1);
        plan.take<int>(1);
        ne->observation_copy.ensure(plan.offset + 256, stream, "normal equations");
        carve();
        if (!ne->by_eliminated && pm_sparse_workspace_create(&ne->by_eliminated) != PM_OK)
            fail(PM_RUNTIME_ERROR, "could not create the observation sort workspace");
        if (!ne->by_primary && pm_sparse_workspace_create(&ne->by_primary) != PM_OK)
            fail(PM_RUNTIME_ERROR, "could not create the observation sort workspace");
        PM_CUDA(cudaMemsetAsync(zeros, 0, (count + 1) * sizeof(int64_t), stream));
        coo_prepare<float>(ne->by_eliminated, stream, ne->L, ne->P, count, obs_eliminated, obs_primary, nullptr);
        const int64_t crosses = coo_internal_status(ne->by_eliminated, stream, "accumulate observations");
        coo_prepare<float>(ne->by_primary, stream, ne->P, 1, count, obs_primary, zeros, nullptr);
        coo_internal_status(ne->by_primary, stream, "accumulate observations");
        if (!ne->by_eliminated_order && pm_sparse_workspace_create(&ne->by_eliminated_order) != PM_OK)
            fail(PM_RUNTIME_ERROR, "could not create the observation sort workspace");
        coo_prepare<float>(ne->by_eliminated_order, stream, ne->L, 1, count, obs_eliminated, zeros, nullptr);
        coo_internal_status(ne->by_eliminated_order, stream, "accumulate observations");
        ne->cross_count = crosses;
        ne->primary_cross_count = 0;
        layout_topology(ne, stream);
        ne->cross_runs.ensure(size_t(crosses + 1) * sizeof(int) + 256, stream, "normal equations");
        const CooView ve = coo_view(ne->by_eliminated);
        if (ne->L > 0)
        {
            narrow_kernel<<<grid_for(ne->L + 1, 256, 4096), 256, 0, stream>>>(ve.row_offsets, ne->cross_offsets,
                                                                              ne->L + 1);
            PM_LAUNCH_CHECK();
            observation_crosses_kernel<<<grid_for(ne->L, 128, 8192), 128, 0, stream>>>(
                ve, ne->cross_offsets, ne->cross_primary, static_cast<int*>(ne->cross_runs.ptr));
            PM_LAUNCH_CHECK();
            cross_owner_kernel<<<grid_for(ne->L, 256, 4096), 256, 0, stream>>>(ne->cross_offsets, ne->L,
                                                                               ne->cross_eliminated);
            PM_LAUNCH_CHECK();
            if (count > 0)
            {
                // slot map of the fused eliminated / cross pass (second half: scratch positions)
                ne->observation_slots.ensure(size_t(2 * (count + 1)) * sizeof(int) + 256, stream,
                                             "normal equations");
                int* slots = static_cast<int*>(ne->observation_slots.ptr);
                int* position = slots + (count + 1);
                const CooView vo = coo_view(ne->by_eliminated_order);
                order_position_kernel<<<grid_for(count, 256, 1 << 20), 256, 0, stream>>>(vo, position);
                PM_LAUNCH_CHECK();
                observation_slots_kernel<<<grid_for(crosses, 256, 1 << 20), 256, 0, stream>>>(
                    crosses, ve.keys, static_cast<const int*>(ne->cross_runs.ptr), position, slots);
                PM_LAUNCH_CHECK();
            }

        }
        else
        {
            PM_CUDA(cudaMemsetAsync(ne->cross_offsets, 0, sizeof(int), stream));
        }
        if (count > 0)
        {
            narrow_kernel<<<grid_for(count, 256, 4096), 256, 0, stream>>>(obs_primary, saved_primary, count);
            PM_LAUNCH_CHECK();
            narrow_kernel<<<grid_for(count, 256, 4096), 256, 0, stream>>>(obs_eliminated, saved_eliminated, count);
            PM_LAUNCH_CHECK();
        }
        ne->observation_count = count;
        ne->residual_size = m;
        ne->observation_topology = true;
        ne->crosses_sorted = true; // buckets are sorted by (primary, input offset)
        ne->topology_version += 1;
    }
    layout_numeric(ne, stream);
    // ---- numeric accumulation
    const CooView ve = coo_view(ne->by_eliminated);
    const CooView vp = coo_view(ne->by_primary);
    T* hll = static_cast<T*>(ne->eliminated_diagonal);
    T* gl = static_cast<T*>(ne->eliminated_gradient);
    T* w = static_cast<T*>(ne->cross_values);
    T* hpp = static_cast<T*>(ne->primary_diagonal);
    T* gp = static_cast<T*>(ne->primary_gradient);
    const int bp = static_cast<int>(ne->bp), bl = static_cast<int>(ne->bl), mm = static_cast<int>(m);
    // first observation with a non-finite squared residual norm (none: every byte 0x7f)
    ne->observation_status.ensure(256, stream, "normal equations");
    long long* first_bad = static_cast<long long*>(ne->observation_status.ptr);
    PM_CUDA(cudaMemsetAsync(first_bad, 0x7f, sizeof(long long), stream));
    // two-row residuals with pair-aligned rows: weights inline, rows read in pairs of scalars
    const auto paired = [](const void* ptr) { return reinterpret_cast<uintptr_t>(ptr) % (2 * sizeof(T)) == 0; };
    const bool rows2 = mm == 2 && bp == 6 && bl == 3 && paired(jp) && paired(jl) && paired(res) && paired(w);
    T* weights = nullptr;
    if (!rows2)
    {
        ne->weights.ensure(size_t(count + 1) * sizeof(T) + 256, stream, "normal equations");
        weights = static_cast<T*>(ne->weights.ptr);
        if (count > 0)
        {
            huber_weights_kernel<T><<<grid_for(count, 256, 1 << 20), 256, 0, stream>>>(count, mm, res, delta, weights,
                                                                                         first_bad);
            PM_LAUNCH_CHECK();
        }
    }
    if (ne->L > 0)
    {
        const unsigned grid = grid_for(ne->L, 128, 1 << 20);
        if (rows2)
        {
            eliminated_cross3_m2_kernel<T><<<grid, 128, 0, stream>>>(
                coo_view(ne->by_eliminated_order), static_cast<const int*>(ne->observation_slots.ptr), jp, jl, res,
                delta, hll, gl, w, first_bad);
            PM_LAUNCH_CHECK();
        }
        else if (bp == 6 && bl == 3)
        {
            const CooView vo = coo_view(ne->by_eliminated_order);
            eliminated_diagonal3_kernel<T><<<grid, 128, 0, stream>>>(vo, mm, jl, res, weights, hll, gl);
            PM_LAUNCH_CHECK();
            if (ne->cross_count > 0)
            {
                cross_accumulate63_kernel<T><<<grid_for(ne->cross_count, 128, 1 << 20), 128, 0, stream>>>(
                    ne->cross_count, ve.keys, static_cast<const int*>(ne->cross_runs.ptr), mm, jp, jl, weights, w);
                PM_LAUNCH_CHECK();
            }
        }
        else
        {
            eliminated_accumulate_generic_kernel<T><<<grid, 128, 0, stream>>>(ve, mm, bp, bl, jp, jl, res, weights,
                                                                             ne->cross_offsets, hll, gl, w);
            PM_LAUNCH_CHECK();
        }
    }
    if (ne->P > 0)
    {
        const unsigned grid = grid_for(ne->P, 1, 1 << 20);
        if (rows2)
            primary_accumulate6_kernel<T, 2><<<grid, 128, 0, stream>>>(vp, mm, jp, res, delta, nullptr, hpp, gp);
        else if (bp == 6)
        {
            primary_accumulate6_kernel<T, 0><<<grid, 128, 0, stream>>>(vp, mm, jp, res, delta, weights, hpp, gp);
        }
        else
        {
            // one slice per thread; the per-thread partials live in shared memory (<= 200 KB)
            const size_t width_bytes = size_t(bp * bp + bp) * sizeof(T);
            const int threads =
                static_cast<int>(std::max<size_t>(32, std::min<size_t>(128, (200u << 10) / width_bytes / 32 * 32)));
            const size_t smem = size_t(threads) * width_bytes;
            PM_CUDA(cudaFuncSetAttribute(primary_accumulate_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem)));
            primary_accumulate_kernel<T><<<grid, threads, smem, stream>>>(vp, mm, bp, jp, res, weights, hpp, gp);
        }
        PM_LAUNCH_CHECK();
    }
}

} // namespace
} // namespace pm

extern "C" {

int pm_ne_check_observations(const pm_normal_equations* ne, pm_stream_t stream, int64_t* first_bad)
{
    return pm::guarded([&] {
        if (!ne)
            pm::fail(PM_INVALID_ARGUMENT, "normal equations handle is null");
        long long bad = -1;
        if (ne->observation_status.ptr)
        {
            PM_CUDA(cudaMemcpyAsync(&bad, ne->observation_status.ptr, sizeof(long long), cudaMemcpyDeviceToHost, stream));
            PM_CUDA(cudaStreamSynchronize(stream));
            if (bad < 0 || bad >= ne->observation_count)
                bad = -1;
        }
        if (first_bad)
            *first_bad = bad;
        if (bad >= 0)
            pm::fail(PM_INVALID_ARGUMENT, "evaluateHuberLoss: squared residual norm must be finite and non-negative "
                                          "(observation " + std::to_string(bad) + ")");
    });
}

int pm_ne_create(int64_t P, int64_t L, int64_t bp, int64_t bl, int value_size, pm_normal_equations** out)
{
    return pm::guarded([&] {
        if (!out)
            pm::fail(PM_INVALID_ARGUMENT, "output handle pointer is null");
        if (P < 0 || L < 0 || bp <= 0 || bl <= 0)
            pm::fail(PM_INVALID_ARGUMENT,
                     "BlockNormalEquations: block counts must be non-negative and block sizes positive");
        if (value_size != 4 && value_size != 8)
            pm::fail(PM_INVALID_ARGUMENT, "value size must be 4 (float) or 8 (double)");
        if (P > INT32_MAX / 64 || L > INT32_MAX - 1)
            pm::fail(PM_OVERFLOW_ERROR, "block counts exceed the int32 range of the device path");
        auto* ne = new pm_normal_equations();
        ne->P = P;
        ne->L = L;
        ne->bp = bp;
        ne->bl = bl;
        ne->value_size = value_size;
        *out = ne;
    });
}

void pm_ne_destroy(pm_normal_equations* ne) { delete ne; }

int pm_ne_counts(const pm_normal_equations* ne, int64_t* cross_count, int64_t* primary_cross_count,
                 int64_t* topology_version)
{
    return pm::guarded([&] {
        if (!ne)
            pm::fail(PM_INVALID_ARGUMENT, "normal equations handle is null");
        if (cross_count)
            *cross_count = ne->cross_count;
        if (primary_cross_count)
            *primary_cross_count = ne->primary_cross_count;
        if (topology_version)
            *topology_version = ne->topology_version;
    });
}

#define PM_NE_API(SFX, T)                                                                                          \
    int pm_ne_upload_##SFX(pm_normal_equations* ne, pm_stream_t s, const T* hpp, const T* hll, const T* gp,          \
                           const T* gl, int64_t C, const int64_t* co, const int64_t* cp, const T* cv, int64_t PC,   \
                           const int64_t* pr, const int64_t* pcn, const T* pv)                                     \
    {                                                                                                               \
        return pm::guarded([&] { pm::ne_upload<T>(ne, s, hpp, hll, gp, gl, C, co, cp, cv, PC, pr, pcn, pv); });     \
    }                                                                                                               \
    int pm_ne_download_##SFX(const pm_normal_equations* ne, pm_stream_t s, T* hpp, T* hll, T* gp, T* gl,            \
                             int64_t* co, int64_t* cp, T* cv, int64_t* pr, int64_t* pcn, T* pv)                     \
    {                                                                                                               \
        return pm::guarded([&] { pm::ne_download<T>(ne, s, hpp, hll, gp, gl, co, cp, cv, pr, pcn, pv); });          \
    }                                                                                                               \
    int pm_ne_accumulate_observations_##SFX(pm_normal_equations* ne, pm_stream_t s, int64_t count, int64_t m,       \
                                            const int64_t* op, const int64_t* ol, const T* jp, const T* jl,         \
                                            const T* r, T delta)                                                    \
    {                                                                                                               \
        return pm::guarded([&] { pm::ne_accumulate<T>(ne, s, count, m, op, ol, jp, jl, r, delta); });               \
    }

PM_NE_API(f32, float)
PM_NE_API(f64, double)

} // extern "C"
