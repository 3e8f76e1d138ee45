// Damped Schur-complement solve on the device: the hot path of the reference's
// solveDampedSchurComplement (src/optimization/block_schur.cpp:54-459) with its reusable
// Schur pattern (src/optimization/block_schur_sparse_assembly.h:41-260, 472-520).
//
// Pipeline (all on one stream, no host round trip except the pattern-cache check and the
// convergence polls):
//   1. eliminated blocks: damping H_ii += lambda * max(|H_ii|, minDiag), FP64 Cholesky
//      inverse, y_l = Hll^-1 g_l                                (one thread per block)
//   2. pattern (only when the topology changed): per-primary cross lists, block-CSR rows
//      from shared-memory bitmaps over the block columns, transpose map
//   3. assembly, one CTA per block row p: S_pq = base_pq - sum_l W_pl Hll^-1 W_ql^T for the
//      upper blocks (q >= p), the diagonal block and its FP64 Cholesky inverse (block-Jacobi
//      preconditioner), and the reduced RHS b_p = -g_p + sum_l W_pl y_l.  Crosses are taken in
//      chunks of 64; each chunk cross marks the upper blocks it touches in per-block 64-bit
//      masks (integer atomicOr: order independent), then the thread owning a block walks its
//      mask in cross order and accumulates the 6x6 product in registers.  No float atomics:
//      the result is bitwise reproducible.  Lower blocks are mirrored afterwards.
//   4. block-Jacobi PCG on the 6x6 block-CSR (warp per block row SpMV with 128-bit loads,
//      FP64 dots finished by the last block, alpha/beta/convergence on the device); in mixed
//      mode an FP64 iterative-refinement loop around an FP32 inner PCG
//   5. back-substitution dl = Hll^-1 (-g_l - sum W^T dp)                (thread per block)
#include "pm_schur.cuh"

#include <algorithm>
#include <limits>
#include <cmath>
#include <cstring>
#include <sstream>
#include <vector>

namespace pm
{
namespace
{
constexpr long long kNone = 0x7fffffffffffffffLL;
constexpr int kRowThreads = 128;
constexpr int kVecBlock = 256;
constexpr int kMaxParts = 1024;
// the plain block-CSR SpMV keeps four CTAs of kVecBlock threads resident per SM (<= 64
// registers): a warp per block row then covers 4,736 rows in one wave (at the 66 registers it
// took unbounded only three fit, and a 4,000-row system ran 1.13 waves).  The PCG's and the
// batched SpMV take <= 64 registers unbounded; bounding them made ptxas spill.
constexpr int kSpmvCtasPerSm = 4;

struct SchurStatus
{
    long long eliminated_bad;
    long long preconditioner_bad;
    long long row_too_wide;
    int pad[2]; // pad[1]: scratch flag of the topology comparison
    long long observation_bad; // the normal equations' first observation with a non-finite residual norm
    int learned_bad[2];        // host copy only: the learned blocks were unusable / a GEMM gave up
};

struct SolveState // device-side PCG / refinement scalars
{
    double rho, alpha, beta, tolerance, initial_squared, residual_squared, rhs_squared;
    double true_squared;
    int iterations, max_iterations, done, converged, breakdown, chunks; // chunks: bodies run by the PCG graph
    unsigned int ticket[4];
    // stagnation watch: every `window` iterations the residual norm must have halved
    double window_squared;
    int window, window_start, stagnated, pad2;
};

} // namespace
} // namespace pm

struct pm_schur_workspace
{
    pm::DeviceBuffer pattern;
    pm::DeviceBuffer numeric;
    pm::DeviceBuffer scratch;
    pm::DeviceBuffer dense; // dense backend: n x n factor and status
    pm_sparse_workspace* prim_sort = nullptr;
    int64_t pattern_builds = 0;
    const pm_normal_equations* last_ne = nullptr;
    int64_t last_version = -1;
    int64_t P = -1, L = -1, bp = -1, bl = -1, C = -1, PC = -1, B = 0;
    int value_size = 0;
    bool assembled = false;
    // pattern (int32)
    int* prim_offsets = nullptr;
    int* prim_cross = nullptr;
    int* block_row_ptr = nullptr;
    int* block_col = nullptr;
    int* block_row = nullptr;
    int* diag_pos = nullptr;
    int* transpose = nullptr;
    int* block_pc = nullptr; // per block: primary-cross index k (forward), -(k+2) transposed, -1 none
    // 6x3 assembly cross pairs (pattern lifetime, own buffer)
    pm::DeviceBuffer pair_buffer;
    bool paired = false;           // the 6x3 factor-record path applies to this pattern
    int64_t E = 0;                 // cross pairs
    int2* row_entries = nullptr;   // C: {cross, eliminated} of every primary-list entry
    int64_t* pair_offset = nullptr; // B + 1: pairs of block b are [off[b], off[b+1]) (upper blocks only)
    int* upper_list = nullptr;     // U: the upper blocks (column > row), ascending
    int64_t U = 0;
    int2* pairs = nullptr;         // E: {row-list entry of cross (l, p), row-list entry of cross (l, q)}, per block in ascending l
    void* vfactor = nullptr;       // C x 18 (Scalar): V = W_lp L_l^-T of every row-list entry (written by the diagonal pass)
    int upper_shape = 0;           // launch shape of the upper-block pass (index into kUpperShapes)
    int* saved_offsets = nullptr;
    int* saved_primary = nullptr;
    int* saved_pc = nullptr;
    // numeric
    double* hinv = nullptr;
    double* y = nullptr;
    int hstride = 0, ystride = 0; // per eliminated block; 10 / 10 for the 6x3 pairs (record [L^-1 | z], see eliminated_factor3_kernel)
    void* S = nullptr;   // B * bp * bp, Scalar
    float* S32 = nullptr; // mixed-precision copy
    bool s32_only = false; // the last assembly formed FP32 products: S32 holds the system, S only its diagonal blocks
    double damping = 0.0, min_diag = 0.0; // of the last assembly
    double* mf_t = nullptr; // L x 4: matrix-free FP64 product scratch (t_l = Hll^-1 W_l^T x)
    double* rhs = nullptr;
    double* minv = nullptr;
    float* minv32 = nullptr;
    pm::SchurStatus* status = nullptr;
    pm::SolveState* state = nullptr;
    double* partials = nullptr;
    pm::SchurStatus* host_status = nullptr; // pinned
    pm::SolveState* host_state = nullptr;   // pinned
    cudaEvent_t events[8] = {};
    cudaEvent_t sync_event = nullptr;
    cudaStream_t graph_stream = nullptr; // batched PCG: graphs are captured and replayed here
    cudaEvent_t graph_events[2] = {};
    // block PCG iteration graphs ('while' node around a chunk of iterations), one per operand set
    struct PcgGraph
    {
        const void* key[6] = {};
        int64_t P = -1;
        int types = -1;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
    };
    PcgGraph pcg_graphs[4];
    int pcg_graph_next = 0;
    void drop_pcg_graphs()
    {
        for (auto& g : pcg_graphs)
        {
            if (g.exec)
                cudaGraphExecDestroy(g.exec);
            if (g.graph)
                cudaGraphDestroy(g.graph);
            g = PcgGraph{};
        }
    }
    ~pm_schur_workspace()
    {
        drop_pcg_graphs();
        pattern.release();
        numeric.release();
        scratch.release();
        dense.release();
        pair_buffer.release();
        if (prim_sort)
            pm_sparse_workspace_destroy(prim_sort);
        if (host_status)
            cudaFreeHost(host_status);
        if (host_state)
            cudaFreeHost(host_state);
        for (auto& e : events)
            if (e)
                cudaEventDestroy(e);
        if (sync_event)
            cudaEventDestroy(sync_event);
        for (auto& e : graph_events)
            if (e)
                cudaEventDestroy(e);
        if (graph_stream)
            cudaStreamDestroy(graph_stream);
    }
};

namespace pm
{
namespace
{

// ===================================================================== small kernels
__global__ void status_reset_kernel(SchurStatus* s)
{
    s->eliminated_bad = kNone;
    s->preconditioner_bad = kNone;
    s->row_too_wide = kNone;
    s->pad[0] = 0;
    s->observation_bad = kNone;
}

__global__ void widen_int_kernel(const int* __restrict__ in, int64_t* __restrict__ out, int64_t n)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = in[i];
}

__global__ void iota_kernel(int64_t* __restrict__ out, int64_t n)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = i;
}

__global__ void keys_to_cross_kernel(const uint64_t* __restrict__ keys, int64_t n, int* __restrict__ out)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = static_cast<int>(keys[i] >> 32);
}

__global__ void int_compare_kernel(const int* __restrict__ a, const int* __restrict__ b, int64_t n, int* differs)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        if (a[i] != b[i])
            *differs = 1;
}

// ===================================================================== 1. eliminated inverses
template <typename T, int BL>
__global__ void eliminated_inverse_kernel(int64_t L, int bl_rt, const T* __restrict__ hll, const T* __restrict__ gl,
                                          double lambda, double min_diag, double* __restrict__ hinv, int hstride,
                                          double* __restrict__ y, int ystride, SchurStatus* status)
{
    constexpr int MB = BL > 0 ? BL : 16;
    const int bl = BL > 0 ? BL : bl_rt;
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < L; l += int64_t(gridDim.x) * blockDim.x)
    {
        double m[MB * MB], inv[MB * MB], lower[MB * MB], work[MB];
        for (int i = 0; i < bl * bl; ++i)
            m[i] = static_cast<double>(hll[l * bl * bl + i]);
        for (int d = 0; d < bl; ++d)
        {
            double& v = m[d * bl + d];
            v = __dadd_rn(v, __dmul_rn(lambda, fmax(fabs(v), min_diag)));
        }
        if (!spd_inverse<MB>(m, bl, inv, lower, work))
        {
            atomicMin(&status->eliminated_bad, static_cast<long long>(l));
            for (int i = 0; i < bl * bl; ++i)
                inv[i] = 0.0;
        }
        double yl[MB];
        for (int r = 0; r < bl; ++r)
        {
            double s = 0.0;
            for (int c = 0; c < bl; ++c)
                s = __dadd_rn(s, __dmul_rn(inv[r * bl + c], static_cast<double>(gl[l * bl + c])));
            yl[r] = s;
        }
        if (BL == 3 && hstride == 12 && y == hinv + 9)
        {
            // packed [Hll^-1 | y] row of 96 bytes: six 16-byte stores
            double2* out = reinterpret_cast<double2*>(hinv + l * 12);
            out[0] = make_double2(inv[0], inv[1]);
            out[1] = make_double2(inv[2], inv[3]);
            out[2] = make_double2(inv[4], inv[5]);
            out[3] = make_double2(inv[6], inv[7]);
            out[4] = make_double2(inv[8], yl[0]);
            out[5] = make_double2(yl[1], yl[2]);
        }
        else
        {
            for (int i = 0; i < bl * bl; ++i)
                hinv[l * hstride + i] = inv[i];
            for (int r = 0; r < bl; ++r)
                y[l * ystride + r] = yl[r];
        }
    }
}

// 6x3 assembly: the damped block's Cholesky factor L (Hll + damping = L L^T, the same pivot
// test as spd_inverse) stored as L^-1 (lower, 6 values) and z = L^-1 g_l, one 80-byte record
// [L^-1 00, 10, 11, 20, 21, 22 | z 0, 1, 2 | 0] per eliminated block (five 16-byte stores).
// The assembly then forms V = W L^-T per cross, so W Hll^-1 W'^T = V V'^T and W Hll^-1 g = V z.
template <typename T>
__global__ void eliminated_factor3_kernel(int64_t L, const T* __restrict__ hll, const T* __restrict__ gl,
                                          double lambda, double min_diag, double* __restrict__ rec,
                                          SchurStatus* status)
{
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < L; l += int64_t(gridDim.x) * blockDim.x)
    {
        double m[9], inv[9], lo[9], work[3];
#pragma unroll
        for (int i = 0; i < 9; ++i)
            m[i] = static_cast<double>(hll[l * 9 + i]);
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            double& v = m[d * 3 + d];
            v = __dadd_rn(v, __dmul_rn(lambda, fmax(fabs(v), min_diag)));
        }
        double i00 = 0.0, i10 = 0.0, i11 = 0.0, i20 = 0.0, i21 = 0.0, i22 = 0.0;
        if (spd_inverse<3>(m, 3, inv, lo, work))
        {
            i00 = 1.0 / lo[0];
            i11 = 1.0 / lo[4];
            i22 = 1.0 / lo[8];
            i10 = -(lo[3] * i00) * i11;
            i21 = -(lo[7] * i11) * i22;
            i20 = -(lo[6] * i00 + lo[7] * i10) * i22;
        }
        else
        {
            atomicMin(&status->eliminated_bad, static_cast<long long>(l));
        }
        const double g0 = static_cast<double>(gl[l * 3]), g1 = static_cast<double>(gl[l * 3 + 1]),
                     g2 = static_cast<double>(gl[l * 3 + 2]);
        double2* out = reinterpret_cast<double2*>(rec + l * 10);
        out[0] = make_double2(i00, i10);
        out[1] = make_double2(i11, i20);
        out[2] = make_double2(i21, i22);
        out[3] = make_double2(i00 * g0, i10 * g0 + i11 * g1);
        out[4] = make_double2(i20 * g0 + i21 * g1 + i22 * g2, 0.0);
    }
}

// ===================================================================== 2. pattern
__device__ __forceinline__ void set_bit(unsigned* bits, int q) { atomicOr(&bits[q >> 5], 1u << (q & 31)); }

// mark every block column of row p in a shared bitmap of P bits
__device__ void mark_row(int p, const int* __restrict__ prim_offsets, const int* __restrict__ prim_cross,
                         const int* __restrict__ cross_eliminated, const int* __restrict__ cross_offsets,
                         const int* __restrict__ cross_primary, const int* __restrict__ pc_row,
                         const int* __restrict__ pc_col, int64_t PC, unsigned* bits, int words)
{
    for (int w = threadIdx.x; w < words; w += blockDim.x)
        bits[w] = 0u;
    __syncthreads();
    if (threadIdx.x == 0)
        set_bit(bits, p);
    const int cb = prim_offsets[p], ce = prim_offsets[p + 1];
    for (int j = cb + threadIdx.x; j < ce; j += blockDim.x)
    {
        const int l = cross_eliminated[prim_cross[j]];
        for (int c = cross_offsets[l]; c < cross_offsets[l + 1]; ++c)
            set_bit(bits, cross_primary[c]);
    }
    for (int64_t k = threadIdx.x; k < PC; k += blockDim.x)
    {
        if (pc_row[k] == p)
            set_bit(bits, pc_col[k]);
        if (pc_col[k] == p)
            set_bit(bits, pc_row[k]);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) row_count_kernel(int64_t P, const int* prim_offsets, const int* prim_cross,
                                                        const int* cross_eliminated, const int* cross_offsets,
                                                        const int* cross_primary, const int* pc_row, const int* pc_col,
                                                        int64_t PC, int* __restrict__ row_count)
{
    extern __shared__ unsigned bits[];
    __shared__ int red[256 / 32];
    const int words = static_cast<int>((P + 31) / 32);
    for (int64_t p = blockIdx.x; p < P; p += gridDim.x)
    {
        mark_row(static_cast<int>(p), prim_offsets, prim_cross, cross_eliminated, cross_offsets, cross_primary, pc_row,
                 pc_col, PC, bits, words);
        int local = 0;
        for (int w = threadIdx.x; w < words; w += blockDim.x)
            local += __popc(bits[w]);
        const int total = block_sum<int, 256>(local, red);
        if (threadIdx.x == 0)
            row_count[p] = total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) row_fill_kernel(int64_t P, const int* prim_offsets, const int* prim_cross,
                                                       const int* cross_eliminated, const int* cross_offsets,
                                                       const int* cross_primary, const int* pc_row, const int* pc_col,
                                                       int64_t PC, const int* __restrict__ row_ptr,
                                                       int* __restrict__ block_col, int* __restrict__ block_row,
                                                       int* __restrict__ diag_pos)
{
    extern __shared__ unsigned bits[];
    __shared__ int scan[256 / 32 + 1];
    const int words = static_cast<int>((P + 31) / 32);
    for (int64_t p = blockIdx.x; p < P; p += gridDim.x)
    {
        mark_row(static_cast<int>(p), prim_offsets, prim_cross, cross_eliminated, cross_offsets, cross_primary, pc_row,
                 pc_col, PC, bits, words);
        int carry = row_ptr[p];
        for (int w0 = 0; w0 < words; w0 += blockDim.x)
        {
            const int w = w0 + threadIdx.x;
            const unsigned word = w < words ? bits[w] : 0u;
            int total = 0;
            int at = carry + block_exclusive_scan<int, 256>(__popc(word), scan, total);
            unsigned rest = word;
            while (rest)
            {
                const int bit = __ffs(rest) - 1;
                rest &= rest - 1;
                const int q = w * 32 + bit;
                block_col[at] = q;
                block_row[at] = static_cast<int>(p);
                if (q == p)
                    diag_pos[p] = at;
                ++at;
            }
            carry += total;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int find_col(const int* __restrict__ cols, int lo, int hi, int q)
{
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if (cols[mid] < q)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void transpose_kernel(int64_t B, const int* __restrict__ row_ptr, const int* __restrict__ block_col,
                                 const int* __restrict__ block_row, int* __restrict__ transpose)
{
    for (int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; b < B; b += int64_t(gridDim.x) * blockDim.x)
    {
        const int p = block_row[b], q = block_col[b];
        transpose[b] = find_col(block_col, row_ptr[q], row_ptr[q + 1], p);
    }
}

__global__ void block_pc_kernel(int64_t PC, const int* __restrict__ pc_row, const int* __restrict__ pc_col,
                                const int* __restrict__ row_ptr, const int* __restrict__ block_col,
                                int* __restrict__ block_pc)
{
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < PC; k += int64_t(gridDim.x) * blockDim.x)
    {
        const int r = pc_row[k], c = pc_col[k];
        block_pc[find_col(block_col, row_ptr[r], row_ptr[r + 1], c)] = static_cast<int>(k);
        block_pc[find_col(block_col, row_ptr[c], row_ptr[c + 1], r)] = -static_cast<int>(k) - 2;
    }
}

// ===================================================================== 3. assembly
template <typename T>
struct AssembleArgs
{
    int64_t P;
    int bp, bl;
    const int* prim_offsets;
    const int* prim_cross;
    const int* cross_eliminated;
    const int* cross_offsets;
    const int* cross_primary;
    const int* block_row_ptr;
    const int* block_col;
    const int* diag_pos;
    const int* block_pc;
    const T* hpp;
    const T* gp;
    const T* w;
    const T* pcv;
    const double* hinv;
    const double* y;
    double lambda, min_diag;
    T* S;
    double* rhs;
    double* minv;
    SchurStatus* status;
};

template <typename T, int BP, int BL, int CH>
__global__ void __launch_bounds__(kRowThreads) assemble_kernel(AssembleArgs<T> a)
{
    using A = T; // accumulation type of the Schur products
    constexpr int MP = BP > 0 ? BP : 16;
    constexpr int ML = BL > 0 ? BL : 16;
    const int bp = BP > 0 ? BP : a.bp;
    const int bl = BL > 0 ? BL : a.bl;
    const int bpl = bp * bl, bpp = bp * bp;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    A* t_stage = reinterpret_cast<A*>(smem_raw);               // [CH][bp*bl]
    A* d_stage = t_stage + CH * bpl;                            // [CH][bp*bp]
    A* r_stage = d_stage + CH * bpp;                            // [CH][bp]
    double* diag = reinterpret_cast<double*>(r_stage + CH * bp); // [bp*bp] (FP64 copy of S_pp)
    unsigned long long* masks = reinterpret_cast<unsigned long long*>(diag + MP * MP); // [kRowThreads]
    int* c_off = reinterpret_cast<int*>(masks + kRowThreads);   // [CH]
    int* c_len = c_off + CH;                                    // [CH]
    const int t = threadIdx.x;

    for (int64_t pp = blockIdx.x; pp < a.P; pp += gridDim.x)
    {
        const int p = static_cast<int>(pp);
        const int row_end = a.block_row_ptr[p + 1];
        const int dpos = a.diag_pos[p];
        const int n_up = row_end - dpos; // upper blocks including the diagonal
        const int cb = a.prim_offsets[p], ce = a.prim_offsets[p + 1];
        const int groups = max(1, (n_up - 1 + kRowThreads - 1) / kRowThreads);
        A dacc = A(0), racc = A(0); // thread t < bp*bp: diagonal entry t; thread 64+t (t < bp): rhs entry
        for (int g = 0; g < groups; ++g)
        {
            const int my_u = 1 + g * kRowThreads + t;
            const bool owner = my_u < n_up;
            const int my_q = owner ? a.block_col[dpos + my_u] : -1;
            A acc[MP * MP];
#pragma unroll
            for (int k = 0; k < MP * MP; ++k)
                acc[k] = A(0);
            for (int c0 = cb; c0 < ce; c0 += CH)
            {
                const int nch = min(CH, ce - c0);
                masks[t] = 0ull;
                __syncthreads();
                if (t < nch)
                {
                    const int c = a.prim_cross[c0 + t];
                    const int l = a.cross_eliminated[c];
                    const int off = a.cross_offsets[l], len = a.cross_offsets[l + 1] - off;
                    c_off[t] = off;
                    c_len[t] = len;
                    const double* hi = a.hinv + int64_t(l) * bl * bl;
                    const T* W = a.w + int64_t(c) * bpl;
                    A* Ts = t_stage + t * bpl;
                    // T = W Hll^-1 (row r of T = Hll^-1 applied to row r of W; Hll^-1 symmetric)
                    for (int r = 0; r < bp; ++r)
                        for (int j = 0; j < bl; ++j)
                        {
                            A s = A(0);
                            for (int m = 0; m < bl; ++m)
                                s += static_cast<A>(hi[j * bl + m]) * static_cast<A>(W[r * bl + m]);
                            Ts[r * bl + j] = s;
                        }
                    if (g == 0)
                    {
                        A* Ds = d_stage + t * bpp;
                        for (int r = 0; r < bp; ++r)
                            for (int cc = 0; cc < bp; ++cc)
                            {
                                A s = A(0);
                                for (int m = 0; m < bl; ++m)
                                    s += Ts[r * bl + m] * static_cast<A>(W[cc * bl + m]);
                                Ds[r * bp + cc] = s;
                            }
                        A* Rs = r_stage + t * bp;
                        const double* yl = a.y + int64_t(l) * bl;
                        for (int r = 0; r < bp; ++r)
                        {
                            A s = A(0);
                            for (int m = 0; m < bl; ++m)
                                s += static_cast<A>(W[r * bl + m]) * static_cast<A>(yl[m]);
                            Rs[r] = s;
                        }
                    }
                    const int lo = dpos + 1 + g * kRowThreads;
                    const int hi_pos = min(row_end, lo + kRowThreads);
                    for (int k = 0; k < len; ++k)
                    {
                        const int q = a.cross_primary[off + k];
                        if (q <= p)
                            continue;
                        const int u = find_col(a.block_col, dpos + 1, row_end, q);
                        if (u >= lo && u < hi_pos)
                            atomicOr(&masks[u - lo], 1ull << t);
                    }
                }
                __syncthreads();
                if (g == 0)
                {
                    if (t < bpp)
                        for (int i = 0; i < nch; ++i)
                            dacc += d_stage[i * bpp + t];
                    if (t >= 64 && t < 64 + bp)
                        for (int i = 0; i < nch; ++i)
                            racc += r_stage[i * bp + (t - 64)];
                }
                if (owner)
                {
                    unsigned long long m = masks[t];
                    while (m)
                    {
                        const int i = __ffsll(static_cast<long long>(m)) - 1;
                        m &= m - 1;
                        const int off = c_off[i], len = c_len[i];
                        int c2 = off;
                        while (c2 < off + len && a.cross_primary[c2] != my_q)
                            ++c2;
                        if (c2 >= off + len)
                            continue;
                        const T* W2 = a.w + int64_t(c2) * bpl;
                        const A* Ts = t_stage + i * bpl;
                        A w2[MP * ML];
#pragma unroll
                        for (int k = 0; k < MP * ML; ++k)
                            if (k < bpl)
                                w2[k] = static_cast<A>(W2[k]);
#pragma unroll
                        for (int r = 0; r < MP; ++r)
                        {
                            if (r >= bp)
                                break;
#pragma unroll
                            for (int cc = 0; cc < MP; ++cc)
                            {
                                if (cc >= bp)
                                    break;
                                A s = A(0);
#pragma unroll
                                for (int mm = 0; mm < ML; ++mm)
                                {
                                    if (mm >= bl)
                                        break;
                                    s += Ts[r * bl + mm] * w2[cc * bl + mm];
                                }
                                acc[r * bp + cc] += s;
                            }
                        }
                    }
                }
                __syncthreads();
            }
            if (owner)
            {
                const int b = dpos + my_u;
                const int pc = a.block_pc[b];
                T* out = a.S + int64_t(b) * bpp;
                for (int r = 0; r < bp; ++r)
                    for (int cc = 0; cc < bp; ++cc)
                    {
                        A base = A(0);
                        if (pc >= 0)
                            base = static_cast<A>(a.pcv[int64_t(pc) * bpp + r * bp + cc]);
                        out[r * bp + cc] = static_cast<T>(base - acc[r * bp + cc]);
                    }
            }
        }
        // diagonal block, reduced RHS and block-Jacobi inverse
        if (t < bpp)
        {
            const int r = t / bp, cc = t % bp;
            double base = static_cast<double>(a.hpp[int64_t(p) * bpp + t]);
            if (r == cc)
                base = __dadd_rn(base, __dmul_rn(a.lambda, fmax(fabs(base), a.min_diag)));
            const A value = static_cast<A>(base) - dacc;
            a.S[int64_t(dpos) * bpp + t] = static_cast<T>(value);
            diag[t] = static_cast<double>(value);
        }
        if (t >= 64 && t < 64 + bp)
        {
            const int r = t - 64;
            a.rhs[int64_t(p) * bp + r] = -static_cast<double>(a.gp[int64_t(p) * bp + r]) + static_cast<double>(racc);
        }
        __syncthreads();
        if (t == 0)
        {
            double inv[MP * MP], lower[MP * MP], work[MP];
            // symmetrise from the lower triangle, as the reference's Cholesky reads it
            double m[MP * MP];
            for (int r = 0; r < bp; ++r)
                for (int cc = 0; cc < bp; ++cc)
                    m[r * bp + cc] = r >= cc ? diag[r * bp + cc] : diag[cc * bp + r];
            if (!spd_inverse<MP>(m, bp, inv, lower, work))
            {
                atomicMin(&a.status->preconditioner_bad, static_cast<long long>(p));
                for (int k = 0; k < bpp; ++k)
                    inv[k] = 0.0;
            }
            for (int k = 0; k < bpp; ++k)
                a.minv[int64_t(p) * bpp + k] = inv[k];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- 6x3 assembly over cross pairs
// Row p of the reduced system is
//   S_pp  = Hpp + damping - sum_l W_lp Hll_l^-1 W_lp^T
//   S_pq  = H_pq          - sum_l W_lp Hll_l^-1 W_lq^T      (q > p, l seeing both p and q)
//   rhs_p = -g_p          + sum_l W_lp y_l,   y_l = Hll_l^-1 g_l
// The pattern build lists, for every upper block (p, q), its cross pairs {cross (l, p),
// cross (l, q), l} in ascending l; the crosses {cross, l} of every row are its row list, also
// in ascending l.  Two numeric kernels: a CTA per row sums the diagonal block and RHS over the
// row's crosses, and a group of lanes per upper block sums its pairs.  Lanes stride over their
// crosses or pairs, keep their sums in registers (no float atomics) and combine them with fixed
// shuffle trees.  The upper-block lane layout is a launch shape (UpperShape): pair streams x
// lanes per pair, a lane holding three of the six rows (2 lanes per pair) or one 3x3 quadrant
// (4 lanes per pair).  Every sum runs in a fixed order for a given shape: scheduling never
// changes a result.

// items of row-list entry j: one per later primary of its eliminated block
__global__ void pair_count_kernel(int64_t P, const int* __restrict__ prim_offsets, const int* __restrict__ prim_cross,
                                  const int* __restrict__ cross_eliminated, const int* __restrict__ cross_offsets,
                                  const int* __restrict__ cross_primary, int sorted, int* __restrict__ count)
{
    for (int64_t pp = blockIdx.x; pp < P; pp += gridDim.x)
    {
        const int p = static_cast<int>(pp);
        for (int j = prim_offsets[p] + threadIdx.x; j < prim_offsets[p + 1]; j += blockDim.x)
        {
            const int c = prim_cross[j];
            const int l = cross_eliminated[c];
            const int e = cross_offsets[l + 1];
            int n = 0;
            if (sorted)
                n = e - c - 1; // crosses of l are in ascending primary order
            else
                for (int k = cross_offsets[l]; k < e; ++k)
                    n += cross_primary[k] > p;
            count[j] = n;
        }
    }
}

__global__ void row_entries_kernel(int64_t C, const int* __restrict__ prim_cross,
                                   const int* __restrict__ cross_eliminated, int2* __restrict__ row_entries)
{
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < C; j += int64_t(gridDim.x) * blockDim.x)
    {
        const int c = prim_cross[j];
        row_entries[j] = make_int2(c, cross_eliminated[c]);
    }
}

// upper blocks of every row (they follow its diagonal block): counts, then the list
__global__ void upper_count_kernel(int64_t P, const int* __restrict__ block_row_ptr, const int* __restrict__ diag_pos,
                                   int* __restrict__ count)
{
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
        count[p] = block_row_ptr[p + 1] - diag_pos[p] - 1;
}

__global__ void upper_list_kernel(int64_t P, const int* __restrict__ diag_pos, const int* __restrict__ offset,
                                  int* __restrict__ list)
{
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
        for (int j = offset[p]; j < offset[p + 1]; ++j)
            list[j] = diag_pos[p] + 1 + (j - offset[p]);
}

// row-list position of every cross: rowpos[prim_cross[j]] = j
__global__ void rowpos_kernel(int64_t C, const int* __restrict__ prim_cross, int* __restrict__ rowpos)
{
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < C; j += int64_t(gridDim.x) * blockDim.x)
        rowpos[prim_cross[j]] = static_cast<int>(j);
}

// items in row-list order: block index of (p, q) and the row-list entry of the cross (l, q);
// pairs per block counted with integer atomics (a count does not depend on the order)
__global__ void pair_emit_kernel(int64_t P, const int* __restrict__ prim_offsets, const int* __restrict__ prim_cross,
                                 const int* __restrict__ cross_eliminated, const int* __restrict__ cross_offsets,
                                 const int* __restrict__ cross_primary, int sorted, const int64_t* __restrict__ offset,
                                 const int* __restrict__ block_row_ptr, const int* __restrict__ block_col,
                                 const int* __restrict__ diag_pos, const int* __restrict__ rowpos,
                                 int* __restrict__ item_block, int* __restrict__ item_entry,
                                 int* __restrict__ block_pairs)
{
    for (int64_t pp = blockIdx.x; pp < P; pp += gridDim.x)
    {
        const int p = static_cast<int>(pp);
        const int lo0 = diag_pos[p] + 1, hi0 = block_row_ptr[p + 1];
        for (int j = prim_offsets[p] + threadIdx.x; j < prim_offsets[p + 1]; j += blockDim.x)
        {
            const int c = prim_cross[j];
            const int l = cross_eliminated[c];
            const int b = sorted ? c + 1 : cross_offsets[l], e = cross_offsets[l + 1];
            int64_t at = offset[j];
            for (int k = b; k < e; ++k)
            {
                const int q = cross_primary[k];
                if (q <= p)
                    continue;
                int lo = lo0, hi = hi0;
                while (lo < hi)
                {
                    const int mid = (lo + hi) >> 1;
                    if (block_col[mid] < q)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                item_block[at] = lo; // the pattern holds (p, q) by construction
                item_entry[at] = rowpos[k];
                atomicAdd(&block_pairs[lo], 1);
                ++at;
            }
        }
    }
}

// Stable placement of the items into per-block pair lists, warp per row.  A warp takes 32
// row-list entries at a time (ascending l); every entry has at most one item per block, so an
// item's rank in its block is the number of lower lanes with an item there (a lane bitmask per
// block), after which the block's cursor advances by the mask's population.
__global__ void pair_place_kernel(int64_t P, const int* __restrict__ prim_offsets, const int64_t* __restrict__ offset,
                                  const int* __restrict__ item_block, const int* __restrict__ item_entry,
                                  const int2* __restrict__ row_entries, unsigned* mask, int64_t* cursor,
                                  int2* __restrict__ pairs)
{
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    volatile unsigned* vmask = mask;
    volatile int64_t* vcursor = cursor;
    const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t pp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; pp < P; pp += warps)
    {
        const int J0 = prim_offsets[pp], J1 = prim_offsets[pp + 1];
        for (int j0 = J0; j0 < J1; j0 += 32)
        {
            const int j = j0 + lane;
            int64_t e0 = 0, e1 = 0;
            int2 re = make_int2(0, 0);
            if (j < J1)
            {
                e0 = offset[j];
                e1 = offset[j + 1];
                re = row_entries[j];
            }
            for (int64_t e = e0; e < e1; ++e)
                atomicOr(&mask[item_block[e]], 1u << lane);
            __syncwarp();
            for (int64_t e = e0; e < e1; ++e)
            {
                const int X = item_block[e];
                const int64_t at = vcursor[X] + __popc(vmask[X] & below);
                pairs[at] = make_int2(j, item_entry[e]);
            }
            __syncwarp();
            for (int64_t e = e0; e < e1; ++e)
            {
                const int X = item_block[e];
                const unsigned m = vmask[X];
                if (31 - __clz(m) == lane)
                {
                    vcursor[X] = vcursor[X] + __popc(m);
                    vmask[X] = 0u;
                }
            }
            __syncwarp();
        }
    }
}

// N consecutive scalars from global memory into doubles (16-byte loads for double, 8-byte for
// float; src aligned to two scalars)
template <typename T, int N>
__device__ __forceinline__ void load_pairs(const T* __restrict__ src, double* q)
{
    static_assert(N % 2 == 0, "pairs of scalars");
    if constexpr (sizeof(T) == 8)
    {
        const double2* s2 = reinterpret_cast<const double2*>(src);
#pragma unroll
        for (int e = 0; e < N / 2; ++e)
        {
            const double2 v = __ldg(s2 + e);
            q[2 * e] = v.x;
            q[2 * e + 1] = v.y;
        }
    }
    else
    {
        const float2* s2 = reinterpret_cast<const float2*>(src);
#pragma unroll
        for (int e = 0; e < N / 2; ++e)
        {
            const float2 v = __ldg(s2 + e);
            q[2 * e] = v.x;
            q[2 * e + 1] = v.y;
        }
    }
}

// N doubles to N consecutive scalars in global memory (16-byte stores for double, 8-byte for
// float; dst aligned to two scalars)
template <typename T, int N>
__device__ __forceinline__ void store_pairs(T* __restrict__ dst, const double* q)
{
    static_assert(N % 2 == 0, "pairs of scalars");
    if constexpr (sizeof(T) == 8)
    {
        double2* d2 = reinterpret_cast<double2*>(dst);
#pragma unroll
        for (int e = 0; e < N / 2; ++e)
            d2[e] = make_double2(q[2 * e], q[2 * e + 1]);
    }
    else
    {
        float2* d2 = reinterpret_cast<float2*>(dst);
#pragma unroll
        for (int e = 0; e < N / 2; ++e)
            d2[e] = make_float2(static_cast<float>(q[2 * e]), static_cast<float>(q[2 * e + 1]));
    }
}

// Diagonal block and RHS, CTA per row: thread t walks the row's entries t, t + 256, ... (one
// per cross (l, p), ascending l); per entry V = W_lp L_l^-T (6 x 3, from W and the 80-byte
// factor record of l) is stored at the entry's row-list position for the upper-block pass, and
// the 21 lower diagonal entries (V V^T) and 6 RHS terms (V z_l) accumulate in registers; then a
// fixed xor tree per warp and the warps' sums in warp order.
constexpr int kDiagThreads = 256;
template <typename T, typename VT>
__global__ void __launch_bounds__(kDiagThreads, 2) assemble_diag6_kernel(
    int64_t P, const int* __restrict__ prim_offsets, const int2* __restrict__ row_entries, const T* __restrict__ w,
    const double* __restrict__ rec, const T* __restrict__ hpp, const T* __restrict__ gp, double lambda,
    double min_diag, const int* __restrict__ diag_pos, T* __restrict__ S, double* __restrict__ rhs,
    VT* __restrict__ vfactor, float* __restrict__ S32)
{
    __shared__ double part[kDiagThreads / 32][27];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int64_t pp = blockIdx.x; pp < P; pp += gridDim.x)
    {
        const int p = static_cast<int>(pp);
        double d[27]; // 21 lower entries (r, c <= r), then the RHS terms
#pragma unroll
        for (int e = 0; e < 27; ++e)
            d[e] = 0.0;
        const int J1 = prim_offsets[p + 1];
        for (int j = prim_offsets[p] + t; j < J1; j += kDiagThreads)
        {
            const int2 re = row_entries[j];
            double f[10], wv[18];
            load_pairs<double, 10>(rec + int64_t(re.y) * 10, f);
            load_pairs<T, 18>(w + int64_t(re.x) * 18, wv);
            double v[18]; // V rows: (L^-1 w_r)^T
#pragma unroll
            for (int r = 0; r < 6; ++r)
            {
                const double w0 = wv[3 * r], w1 = wv[3 * r + 1], w2 = wv[3 * r + 2];
                v[3 * r] = f[0] * w0;
                v[3 * r + 1] = f[1] * w0 + f[2] * w1;
                v[3 * r + 2] = f[3] * w0 + f[4] * w1 + f[5] * w2;
            }
#pragma unroll
            for (int r = 0; r < 6; ++r)
            {
#pragma unroll
                for (int c = 0; c <= r; ++c)
                    d[r * (r + 1) / 2 + c] += v[3 * r] * v[3 * c] + v[3 * r + 1] * v[3 * c + 1] + v[3 * r + 2] * v[3 * c + 2];
                d[21 + r] += v[3 * r] * f[6] + v[3 * r + 1] * f[7] + v[3 * r + 2] * f[8];
            }
            store_pairs<VT, 18>(vfactor + int64_t(j) * 18, v);
        }
#pragma unroll
        for (int e = 0; e < 27; ++e)
        {
            const double v = warp_sum(d[e]);
            if (lane == 0)
                part[warp][e] = v;
        }
        __syncthreads();
        if (t < 42)
        {
            int e, r = 0, c = 0;
            if (t < 36)
            {
                r = t / 6;
                c = t % 6;
                const int lr = r >= c ? r : c, lc = r >= c ? c : r;
                e = lr * (lr + 1) / 2 + lc;
            }
            else
            {
                e = 21 + (t - 36);
            }
            double v = 0.0;
            for (int k = 0; k < kDiagThreads / 32; ++k)
                v = __dadd_rn(v, part[k][e]);
            if (t < 36)
            {
                double base = static_cast<double>(hpp[int64_t(p) * 36 + t]);
                if (r == c)
                    base = __dadd_rn(base, __dmul_rn(lambda, fmax(fabs(base), min_diag)));
                S[int64_t(diag_pos[p]) * 36 + t] = static_cast<T>(base - v);
                if (S32)
                    S32[int64_t(diag_pos[p]) * 36 + t] = static_cast<float>(base - v);
            }
            else
            {
                rhs[int64_t(p) * 6 + (t - 36)] = -static_cast<double>(gp[int64_t(p) * 6 + (t - 36)]) + v;
            }
        }
        __syncthreads(); // partial sums read before the next row writes them
    }
}

// Upper blocks, STREAMS x SPLIT lanes per block: lane g = SPLIT s + k walks the block's pairs
// s, s + STREAMS, ... (S_pq -= V_lp V_lq^T; both factors come from the row-ordered V array, and
// the lanes of a pair load the same rows, which the load unit merges).  SPLIT 2: lane k holds
// output rows 3k .. 3k + 2 against all six columns; SPLIT 4: lane k = 2 kr + kc holds the 3x3
// quadrant (rows 3 kr.., columns 3 kc..), fewer registers per lane for more resident warps.  A
// fixed xor tree over the streams ends it.
constexpr int kUpperThreads = 256;

template <typename AT, int LANES, int FIRST>
__device__ __forceinline__ AT stream_sum_as(AT v, unsigned gmask)
{
#pragma unroll
    for (int o = FIRST; o < LANES; o <<= 1)
        v += __shfl_xor_sync(gmask, v, o);
    return v;
}

// N consecutive scalars (two per load) into AT registers
template <typename VT, int N, typename AT>
__device__ __forceinline__ void load_as(const VT* __restrict__ src, AT* q)
{
    if constexpr (sizeof(VT) == 8)
    {
        const double2* s2 = reinterpret_cast<const double2*>(src);
#pragma unroll
        for (int e = 0; e < N / 2; ++e)
        {
            const double2 v = __ldg(s2 + e);
            q[2 * e] = static_cast<AT>(v.x);
            q[2 * e + 1] = static_cast<AT>(v.y);
        }
    }
    else
    {
        const float2* s2 = reinterpret_cast<const float2*>(src);
#pragma unroll
        for (int e = 0; e < N / 2; ++e)
        {
            const float2 v = __ldg(s2 + e);
            q[2 * e] = static_cast<AT>(v.x);
            q[2 * e + 1] = static_cast<AT>(v.y);
        }
    }
}

// three V rows (elements 9 h .. 9 h + 8 of an 18-element row) as t[3][3], read as the aligned
// run 8 h .. 8 h + 9
template <typename VT, typename AT>
__device__ __forceinline__ void load_v_half(const VT* __restrict__ row, int h, AT (&t)[3][3])
{
    AT a[10];
    load_as<VT, 10, AT>(row + 8 * h, a);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            t[r][k] = h ? a[3 * r + k + 1] : a[3 * r + k];
}

// TO: type of the assembled values, TP: type of the coupling blocks (the normal equations'),
// VT: type of the stored V factors, AT: type of the products and their sums
template <typename TO, typename TP, typename VT, typename AT, int STREAMS, int SPLIT>
__global__ void __launch_bounds__(kUpperThreads, SPLIT == 4 ? 3 : 2) assemble_upper6_kernel(
    int64_t U, const int* __restrict__ upper_list, const int64_t* __restrict__ pair_offset,
    const int2* __restrict__ pairs, const int* __restrict__ transpose, const int* __restrict__ block_pc,
    const VT* __restrict__ vfactor, const TP* __restrict__ pcv, TO* __restrict__ S)
{
    constexpr int LANES = STREAMS * SPLIT;
    constexpr int COLS = SPLIT == 2 ? 6 : 3; // output columns a lane holds
    static_assert(LANES <= 32 && (LANES & (LANES - 1)) == 0, "lanes per block: a power of two up to a warp");
    const int g = threadIdx.x & (LANES - 1);
    const int s = g / SPLIT, k = g % SPLIT;
    const int kr = SPLIT == 2 ? k : k >> 1, kc = SPLIT == 2 ? 0 : k & 1;
    const unsigned gmask = LANES == 32 ? 0xffffffffu : ((1u << LANES) - 1u) << (threadIdx.x & 31 & ~(LANES - 1));
    const int64_t groups = int64_t(gridDim.x) * (kUpperThreads / LANES);
    for (int64_t u = (int64_t(blockIdx.x) * kUpperThreads + threadIdx.x) / LANES; u < U; u += groups)
    {
        const int64_t b = upper_list[u];
        AT acc[3][COLS];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < COLS; ++c)
                acc[r][c] = AT(0);
        const int64_t k1 = pair_offset[b + 1];
        int64_t kk = pair_offset[b] + s;
        int2 next = kk < k1 ? pairs[kk] : make_int2(0, 0);
        while (kk < k1)
        {
            const int2 cur = next;
            kk += STREAMS;
            if (kk < k1)
                next = pairs[kk];
            AT tr[3][3];
            load_v_half<VT, AT>(vfactor + int64_t(cur.x) * 18, kr, tr);
            // V_lq three rows at a time (both halves for SPLIT 2) to keep fewer values live
#pragma unroll
            for (int half = 0; half < COLS / 3; ++half)
            {
                AT tq[3][3];
                load_v_half<VT, AT>(vfactor + int64_t(cur.y) * 18, SPLIT == 2 ? half : kc, tq);
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        acc[r][3 * half + c] += tr[r][0] * tq[c][0] + tr[r][1] * tq[c][1] + tr[r][2] * tq[c][2];
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < COLS; ++c)
                acc[r][c] = stream_sum_as<AT, LANES, SPLIT>(acc[r][c], gmask);
        const int pc = block_pc[b];
        TO* out = S + b * 36;
        TO* mirrored = S + int64_t(transpose[b]) * 36; // the lower block (q, p) holds the transpose
#pragma unroll
        for (int e = 0; e < 3 * COLS; ++e)
        {
            if ((e & (STREAMS - 1)) != s)
                continue;
            const int row = 3 * kr + e / COLS, col = 3 * kc + e % COLS;
            const AT base = pc >= 0 ? static_cast<AT>(pcv[int64_t(pc) * 36 + row * 6 + col]) : AT(0);
            const TO value = static_cast<TO>(base - acc[e / COLS][e % COLS]);
            out[row * 6 + col] = value;
            mirrored[col * 6 + row] = value;
        }
    }
}

// Block-Jacobi preconditioner of the assembled system: FP64 inverse of every diagonal block
// (symmetrised from its lower triangle), thread per block row.
template <typename T, int BP>
__global__ void diag_inverse_kernel(int64_t P, const int* __restrict__ diag_pos, const T* __restrict__ S,
                                    double* __restrict__ minv, SchurStatus* status)
{
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
    {
        const T* d = S + int64_t(diag_pos[p]) * BP * BP;
        double m[BP * BP], inv[BP * BP], lower[BP * BP], work[BP];
        for (int r = 0; r < BP; ++r)
            for (int c = 0; c < BP; ++c)
                m[r * BP + c] = static_cast<double>(r >= c ? d[r * BP + c] : d[c * BP + r]);
        if (!spd_inverse<BP>(m, BP, inv, lower, work))
        {
            atomicMin(&status->preconditioner_bad, static_cast<long long>(p));
            for (int k = 0; k < BP * BP; ++k)
                inv[k] = 0.0;
        }
        for (int k = 0; k < BP * BP; ++k)
            minv[p * BP * BP + k] = inv[k];
    }
}

// lower blocks: S[b] = S[transpose(b)]^T
template <typename T>
__global__ void mirror_kernel(int64_t B, int bp, const int* __restrict__ block_row, const int* __restrict__ block_col,
                              const int* __restrict__ transpose, T* __restrict__ S)
{
    const int bpp = bp * bp;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < B * bpp; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t b = i / bpp;
        if (block_col[b] >= block_row[b])
            continue;
        const int e = static_cast<int>(i - b * bpp), r = e / bp, c = e % bp;
        S[i] = S[int64_t(transpose[b]) * bpp + c * bp + r];
    }
}

template <typename Tin, typename Tout>
__global__ void convert_kernel(const Tin* __restrict__ in, Tout* __restrict__ out, int64_t n)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = static_cast<Tout>(in[i]);
}

// ===================================================================== 4. block PCG
template <int K, typename Finish>
__device__ __forceinline__ void finish_reduce(double (&mine)[K], double* partials, unsigned int* ticket, Finish&& fin)
{
    __shared__ double red[kVecBlock / 32];
    __shared__ bool last;
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const double s = block_sum<double, kVecBlock>(mine[k], red);
        if (threadIdx.x == 0)
            partials[k * kMaxParts + blockIdx.x] = s;
    }
    __threadfence();
    if (threadIdx.x == 0)
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last)
        return;
    __threadfence();
    double tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        double s = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
            s += __ldcg(partials + k * kMaxParts + b);
        tot[k] = block_sum<double, kVecBlock>(s, red);
    }
    if (threadIdx.x == 0)
    {
        *ticket = 0;
        fin(tot);
    }
}

// y_p = sum_b S_b x_col(b) for block row p; lane-strided over the row's blocks, warp reduce
template <typename V, typename M, int BP>
__device__ __forceinline__ void bsr_row(const int* __restrict__ row_ptr, const int* __restrict__ block_col,
                                        const M* __restrict__ S, const V* __restrict__ x, int bp_rt, int64_t p,
                                        bool valid, int lane, double* y /* [16] */)
{
    constexpr int MP = BP > 0 ? BP : 16;
    const int bp = BP > 0 ? BP : bp_rt;
    double acc[MP];
#pragma unroll
    for (int r = 0; r < MP; ++r)
        acc[r] = 0.0;
    if (valid)
    {
        const int b0 = row_ptr[p], b1 = row_ptr[p + 1];
        for (int b = b0 + lane; b < b1; b += 32)
        {
            const int q = block_col[b];
            const M* blk = S + int64_t(b) * bp * bp;
            V xv[MP];
#pragma unroll
            for (int c = 0; c < MP; ++c)
                if (c < bp)
                    xv[c] = x[int64_t(q) * bp + c];
            if constexpr (BP == 6 && sizeof(M) == 4)
            {
                const float4* v4 = reinterpret_cast<const float4*>(blk);
                float m[36];
#pragma unroll
                for (int k = 0; k < 9; ++k)
                {
                    const float4 f = __ldg(v4 + k);
                    m[4 * k] = f.x; m[4 * k + 1] = f.y; m[4 * k + 2] = f.z; m[4 * k + 3] = f.w;
                }
#pragma unroll
                for (int r = 0; r < 6; ++r)
                {
                    float s = 0.f;
#pragma unroll
                    for (int c = 0; c < 6; ++c)
                        s = fmaf(m[r * 6 + c], static_cast<float>(xv[c]), s);
                    acc[r] += s;
                }
            }
            else if constexpr (BP == 6 && sizeof(M) == 8)
            {
                const double2* v2 = reinterpret_cast<const double2*>(blk);
#pragma unroll
                for (int r = 0; r < 6; ++r)
                {
                    const double2 a0 = __ldg(v2 + 3 * r), a1 = __ldg(v2 + 3 * r + 1), a2 = __ldg(v2 + 3 * r + 2);
                    double s = a0.x * static_cast<double>(xv[0]);
                    s = fma(a0.y, static_cast<double>(xv[1]), s);
                    s = fma(a1.x, static_cast<double>(xv[2]), s);
                    s = fma(a1.y, static_cast<double>(xv[3]), s);
                    s = fma(a2.x, static_cast<double>(xv[4]), s);
                    s = fma(a2.y, static_cast<double>(xv[5]), s);
                    acc[r] += s;
                }
            }
            else
            {
                for (int r = 0; r < bp; ++r)
                {
                    double s = 0.0;
                    for (int c = 0; c < bp; ++c)
                        s += static_cast<double>(blk[r * bp + c]) * static_cast<double>(xv[c]);
                    acc[r] += s;
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < MP; ++r)
    {
        if (r >= bp)
            break;
        double v = acc[r];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, o);
        y[r] = v;
    }
}

// plain y = S x (vector type V)
template <typename V, typename M, int BP>
__global__ void __launch_bounds__(kVecBlock, kSpmvCtasPerSm) bsr_spmv_kernel(int64_t P, int bp, const int* __restrict__ row_ptr,
                                                             const int* __restrict__ block_col,
                                                             const M* __restrict__ S, const V* __restrict__ x,
                                                             V* __restrict__ y)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x / 32);
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const int64_t span = (P + warps - 1) / warps;
    for (int64_t k = 0; k < span; ++k)
    {
        const int64_t p = first + k * warps;
        double out[16];
        bsr_row<V, M, BP>(row_ptr, block_col, S, x, bp, p, p < P, lane, out);
        if (p < P && lane < bp)
        {
            double v = 0.0;
#pragma unroll
            for (int r = 0; r < (BP > 0 ? BP : 16); ++r)
                v = lane == r ? out[r] : v;
            y[p * bp + lane] = static_cast<V>(v);
        }
    }
}

// q = S p and the p.q partial; alpha = rho / p.q (CPU reduced-PCG semantics:
// block_schur_cpu_solver.h:41-51, non-positive curvature is reported, not thrown)
template <typename V, typename M, int BP>
__global__ void __launch_bounds__(kVecBlock) pcg_bsr_kernel(int64_t P, int bp, const int* __restrict__ row_ptr,
                                                            const int* __restrict__ block_col,
                                                            const M* __restrict__ S, const V* __restrict__ p_vec,
                                                            V* __restrict__ q, double* partials, SolveState* st)
{
    if (st->done)
        return;
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x / 32);
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const int64_t span = (P + warps - 1) / warps;
    double mine[1] = {0.0};
    for (int64_t k = 0; k < span; ++k)
    {
        const int64_t p = first + k * warps;
        double out[16];
        bsr_row<V, M, BP>(row_ptr, block_col, S, p_vec, bp, p, p < P, lane, out);
        if (p < P && lane < bp)
        {
            double v = 0.0;
#pragma unroll
            for (int r = 0; r < (BP > 0 ? BP : 16); ++r)
                v = lane == r ? out[r] : v;
            const V qv = static_cast<V>(v);
            q[p * bp + lane] = qv;
            mine[0] += static_cast<double>(p_vec[p * bp + lane]) * static_cast<double>(qv);
        }
    }
    finish_reduce<1>(mine, partials, &st->ticket[1], [&](double (&tot)[1]) {
        const double den = tot[0];
        if (!(den > 0.0) || !isfinite(den))
        {
            st->breakdown = 1;
            st->done = 1;
            st->alpha = 0.0;
            return;
        }
        st->alpha = st->rho / den;
    });
}

// the last block of an update: iteration count, residual norm, convergence / limit / stagnation,
// beta and rho (tot = {r.z, r.r})
__device__ __forceinline__ void update_finish(SolveState* st, const double (&tot)[2])
{
    st->iterations += 1;
    st->residual_squared = tot[1];
    const double norm = sqrt(fmax(0.0, tot[1]));
    if (!isfinite(tot[1]))
    {
        st->breakdown = 1;
        st->done = 1;
        return;
    }
    if (norm <= st->tolerance)
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
    if (st->window > 0 && st->iterations - st->window_start >= st->window)
    {
        if (tot[1] > 0.25 * st->window_squared) // the norm did not halve over the window
        {
            st->stagnated = 1;
            st->done = 1;
            return;
        }
        st->window_start = st->iterations;
        st->window_squared = tot[1];
    }
    st->beta = tot[0] / st->rho;
    st->rho = tot[0];
}

// x += alpha p; r_out = r_in - alpha q; z = Minv r_out; r.z, r.r; convergence; beta
template <typename V, typename PM, int BP>
__global__ void __launch_bounds__(kVecBlock) pcg_block_update_kernel(int64_t P, int bp_rt, V* __restrict__ x,
                                                                     const V* __restrict__ p_vec,
                                                                     const V* __restrict__ q, const V* __restrict__ r_in,
                                                                     V* __restrict__ r_out, V* __restrict__ z,
                                                                     const PM* __restrict__ minv, double* partials,
                                                                     SolveState* st)
{
    if (st->done)
        return;
    constexpr int MP = BP > 0 ? BP : 16;
    const int bp = BP > 0 ? BP : bp_rt;
    const double alpha = st->alpha;
    double mine[2] = {0.0, 0.0};
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
    {
        double r[MP];
#pragma unroll
        for (int k = 0; k < MP; ++k)
        {
            if (k >= bp)
                break;
            const int64_t i = p * bp + k;
            x[i] = static_cast<V>(static_cast<double>(x[i]) + alpha * static_cast<double>(p_vec[i]));
            r[k] = static_cast<double>(static_cast<V>(static_cast<double>(r_in[i]) - alpha * static_cast<double>(q[i])));
            r_out[i] = static_cast<V>(r[k]);
            mine[1] += r[k] * r[k];
        }
        const PM* m = minv + p * bp * bp;
#pragma unroll
        for (int k = 0; k < MP; ++k)
        {
            if (k >= bp)
                break;
            double s = 0.0;
#pragma unroll
            for (int c = 0; c < MP; ++c)
            {
                if (c >= bp)
                    break;
                s += static_cast<double>(m[k * bp + c]) * r[c];
            }
            const V zk = static_cast<V>(s);
            z[p * bp + k] = zk;
            mine[0] += r[k] * static_cast<double>(zk);
        }
    }
    finish_reduce<2>(mine, partials, &st->ticket[2], [&](double (&tot)[2]) { update_finish(st, tot); });
}

// x += alpha p; r_out = r_in - alpha q; z = Minv r_out; r.z, r.r for 6x6 blocks, eight lanes per
// block row (lane k < 6 owns entry k; the row's residual reaches every lane by shuffles), so a
// 4,000-row system spreads over 125 CTAs instead of 16.  Every entry takes the same arithmetic as
// pcg_block_update_kernel's; the dot partials are summed per lane.
template <typename V, typename PM>
__global__ void __launch_bounds__(kVecBlock) pcg_block_update6_kernel(int64_t P, V* __restrict__ x,
                                                                      const V* __restrict__ p_vec,
                                                                      const V* __restrict__ q, const V* __restrict__ r_in,
                                                                      V* __restrict__ r_out, V* __restrict__ z,
                                                                      const PM* __restrict__ minv, double* partials,
                                                                      SolveState* st)
{
    if (st->done)
        return;
    const double alpha = st->alpha;
    const int lane = threadIdx.x & 31, k = lane & 7, base = lane & ~7;
    const int64_t groups = int64_t(gridDim.x) * (blockDim.x / 8);
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 8;
    const int64_t span = (P + groups - 1) / groups; // warp-uniform trip count (the shuffles)
    double mine[2] = {0.0, 0.0};
    for (int64_t t = 0; t < span; ++t)
    {
        const int64_t row = first + t * groups;
        const bool own = row < P && k < 6;
        double rk = 0.0;
        if (own)
        {
            const int64_t i = row * 6 + k;
            x[i] = static_cast<V>(static_cast<double>(x[i]) + alpha * static_cast<double>(p_vec[i]));
            rk = static_cast<double>(static_cast<V>(static_cast<double>(r_in[i]) - alpha * static_cast<double>(q[i])));
            r_out[i] = static_cast<V>(rk);
            mine[1] += rk * rk;
        }
        double r[6];
#pragma unroll
        for (int c = 0; c < 6; ++c)
            r[c] = __shfl_sync(0xffffffffu, rk, base + c);
        if (own)
        {
            const PM* m = minv + row * 36 + k * 6;
            double sum = 0.0;
#pragma unroll
            for (int c = 0; c < 6; ++c)
                sum += static_cast<double>(m[c]) * r[c];
            const V zk = static_cast<V>(sum);
            z[row * 6 + k] = zk;
            mine[0] += rk * static_cast<double>(zk);
        }
    }
    finish_reduce<2>(mine, partials, &st->ticket[2], [&](double (&tot)[2]) { update_finish(st, tot); });
}

template <typename V>
__global__ void pcg_block_direction_kernel(int64_t n, const V* __restrict__ z, V* __restrict__ p,
                                           const SolveState* st)
{
    if (st->done || st->iterations == 0) // the first iteration's direction is z itself (set by the init)
        return;
    const double beta = st->beta;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        p[i] = static_cast<V>(static_cast<double>(z[i]) + beta * static_cast<double>(p[i]));
}

// r = b - q; z = Minv r; p = z; rho = r.z; ||r||^2.  tol = tolerance rule on ||r0||.
template <typename V, typename PM, typename B, int BP>
__global__ void __launch_bounds__(kVecBlock) pcg_block_init_kernel(int64_t P, int bp_rt, const B* __restrict__ b,
                                                                   const V* __restrict__ q, V* __restrict__ r,
                                                                   V* __restrict__ z, V* __restrict__ p_vec,
                                                                   const PM* __restrict__ minv, double rel, double abs_tol,
                                                                   int rule, int max_iterations, int window,
                                                                   double* partials, SolveState* st)
{
    constexpr int MP = BP > 0 ? BP : 16;
    const int bp = BP > 0 ? BP : bp_rt;
    double mine[2] = {0.0, 0.0};
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
    {
        double rr[MP];
#pragma unroll
        for (int k = 0; k < MP; ++k)
        {
            if (k >= bp)
                break;
            const int64_t i = p * bp + k;
            rr[k] = static_cast<double>(static_cast<V>(static_cast<double>(b[i]) - static_cast<double>(q[i])));
            r[i] = static_cast<V>(rr[k]);
            mine[1] += rr[k] * rr[k];
        }
        const PM* m = minv + p * bp * bp;
#pragma unroll
        for (int k = 0; k < MP; ++k)
        {
            if (k >= bp)
                break;
            double s = 0.0;
            for (int c = 0; c < bp; ++c)
                s += static_cast<double>(m[k * bp + c]) * rr[c];
            const V zk = static_cast<V>(s);
            z[p * bp + k] = zk;
            p_vec[p * bp + k] = zk;
            mine[0] += rr[k] * static_cast<double>(zk);
        }
    }
    finish_reduce<2>(mine, partials, &st->ticket[0], [&](double (&tot)[2]) {
        st->rho = tot[0];
        st->initial_squared = tot[1];
        st->residual_squared = tot[1];
        st->iterations = 0;
        st->max_iterations = max_iterations;
        st->done = 0;
        st->converged = 0;
        st->breakdown = 0;
        st->window = window;
        st->window_start = 0;
        st->window_squared = tot[1];
        st->stagnated = 0;
        const double r0 = sqrt(fmax(0.0, tot[1]));
        st->tolerance = rule == 0 ? abs_tol + rel * r0 : fmax(abs_tol, rel * r0);
        if (!isfinite(tot[1]))
        {
            st->breakdown = 1;
            st->done = 1;
        }
        else if (r0 <= st->tolerance)
        {
            st->converged = 1;
            st->done = 1;
        }
    });
}

// FP64 residual of the refinement loop: r = b - q (q = S64 x), ||r||^2, ||b||^2
__global__ void __launch_bounds__(kVecBlock) residual_kernel(int64_t n, const double* __restrict__ b,
                                                             const double* __restrict__ q, double* __restrict__ r,
                                                             double* partials, SolveState* st)
{
    double mine[2] = {0.0, 0.0};
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        const double v = b[i] - q[i];
        if (r)
            r[i] = v;
        mine[0] += v * v;
        mine[1] += b[i] * b[i];
    }
    finish_reduce<2>(mine, partials, &st->ticket[3], [&](double (&tot)[2]) {
        st->true_squared = tot[0];
        st->rhs_squared = tot[1];
    });
}

// FP64 matrix-free product q = S x of the damped 6x3 Schur complement, straight from the FP64
// normal equations (used when the assembled values are FP32 only):
//   q_p = (Hpp_p + damping) x_p + sum_q C_pq x_q - sum_{l in p} W_lp Hll^-1 sum_{q in l} W_lq^T x_q
// where C are the primary-primary coupling blocks.  Pass 1, thread per eliminated block:
// t_l = Hll^-1 (W_l^T x) = L^-T (L^-1 W_l^T x) from the factor record; pass 2, CTA per block row:
// the row's crosses in row-list order, then a fixed xor tree and the warps in order.  Both passes
// sum in fixed orders, so the product repeats bit for bit.
template <typename T, bool X16>
__global__ void mf_eliminated6_kernel(int64_t L, const int* __restrict__ cross_offsets,
                                      const int* __restrict__ cross_primary, const T* __restrict__ w,
                                      const double* __restrict__ rec, const double* __restrict__ x,
                                      double* __restrict__ t)
{
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < L; l += int64_t(gridDim.x) * blockDim.x)
    {
        double u0 = 0.0, u1 = 0.0, u2 = 0.0;
        for (int c = cross_offsets[l]; c < cross_offsets[l + 1]; ++c)
        {
            double wv[18], xv[6];
            load_pairs<T, 18>(w + int64_t(c) * 18, wv);
            // x is the caller's step vector: pairs when it starts on a 16-byte boundary (X16,
            // checked by the host), element by element otherwise
            const double* xp = x + int64_t(cross_primary[c]) * 6;
            if constexpr (X16)
                load_pairs<double, 6>(xp, xv);
            else
#pragma unroll
                for (int r = 0; r < 6; ++r)
                    xv[r] = xp[r];
#pragma unroll
            for (int r = 0; r < 6; ++r)
            {
                u0 += wv[3 * r] * xv[r];
                u1 += wv[3 * r + 1] * xv[r];
                u2 += wv[3 * r + 2] * xv[r];
            }
        }
        double f[10];
        load_pairs<double, 10>(rec + l * 10, f);
        const double v0 = f[0] * u0, v1 = f[1] * u0 + f[2] * u1, v2 = f[3] * u0 + f[4] * u1 + f[5] * u2;
        double2* out = reinterpret_cast<double2*>(t + l * 4);
        out[0] = make_double2(f[0] * v0 + f[1] * v1 + f[3] * v2, f[2] * v1 + f[4] * v2);
        out[1] = make_double2(f[5] * v2, 0.0);
    }
}

template <typename T>
__global__ void __launch_bounds__(kDiagThreads) mf_primary6_kernel(
    int64_t P, const int* __restrict__ prim_offsets, const int2* __restrict__ row_entries, const T* __restrict__ w,
    const double* __restrict__ t, const T* __restrict__ hpp, double lambda, double min_diag,
    const int* __restrict__ block_row_ptr, const int* __restrict__ block_col, const int* __restrict__ block_pc,
    const T* __restrict__ pcv, const double* __restrict__ x, double* __restrict__ q)
{
    __shared__ double part[kDiagThreads / 32][6];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int64_t pp = blockIdx.x; pp < P; pp += gridDim.x)
    {
        const int p = static_cast<int>(pp);
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        const int J1 = prim_offsets[p + 1];
        for (int j = prim_offsets[p] + tid; j < J1; j += kDiagThreads)
        {
            const int2 re = row_entries[j];
            double wv[18], tv[4];
            load_pairs<T, 18>(w + int64_t(re.x) * 18, wv);
            load_pairs<double, 4>(t + int64_t(re.y) * 4, tv);
#pragma unroll
            for (int r = 0; r < 6; ++r)
                acc[r] -= wv[3 * r] * tv[0] + wv[3 * r + 1] * tv[1] + wv[3 * r + 2] * tv[2];
        }
        // primary-primary coupling blocks: C_pq (upper, forward index k) or C_qp^T (lower)
        for (int b = block_row_ptr[p] + tid; b < block_row_ptr[p + 1]; b += kDiagThreads)
        {
            const int code = block_pc[b];
            if (code == -1)
                continue;
            const bool fwd = code >= 0;
            const T* C = pcv + int64_t(fwd ? code : -code - 2) * 36;
            const double* xq = x + int64_t(block_col[b]) * 6;
#pragma unroll
            for (int r = 0; r < 6; ++r)
            {
                double v = 0.0;
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    v += static_cast<double>(fwd ? C[r * 6 + c] : C[c * 6 + r]) * xq[c];
                acc[r] += v;
            }
        }
#pragma unroll
        for (int r = 0; r < 6; ++r)
        {
            const double v = warp_sum(acc[r]);
            if (lane == 0)
                part[warp][r] = v;
        }
        __syncthreads();
        if (tid < 6)
        {
            double v = 0.0;
            for (int k = 0; k < kDiagThreads / 32; ++k)
                v = __dadd_rn(v, part[k][tid]);
            // damped primary block times x_p (the block as stored, as the assembly uses it)
            double d = 0.0;
            for (int c = 0; c < 6; ++c)
            {
                double h = static_cast<double>(hpp[int64_t(p) * 36 + tid * 6 + c]);
                if (c == tid)
                    h = __dadd_rn(h, __dmul_rn(lambda, fmax(fabs(h), min_diag)));
                d += h * x[int64_t(p) * 6 + c];
            }
            q[int64_t(p) * 6 + tid] = d + v;
        }
        __syncthreads();
    }
}

template <typename V>
__global__ void axpy_to_double_kernel(int64_t n, const V* __restrict__ d, double* __restrict__ x)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        x[i] += static_cast<double>(d[i]);
}

// ===================================================================== 5. back-substitution
// dl_l = Hll^-1 (-g_l - W_l^T dp) = -L^-T z_l - t_l when the FP64 matrix-free pass that certified
// dp ran at dp itself: t_l = Hll^-1 W_l^T dp is what it stored, z_l = L^-1 g_l sits in the factor
// record [L^-1 00, 10, 11, 20, 21, 22 | z].  Reads 112 bytes per eliminated block instead of the
// block's cross blocks.
__global__ void backsub_from_t_kernel(int64_t L, const double* __restrict__ rec, const double* __restrict__ t,
                                      double* __restrict__ dl)
{
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < L; l += int64_t(gridDim.x) * blockDim.x)
    {
        double f[10], u[4];
        load_pairs<double, 10>(rec + l * 10, f);
        load_pairs<double, 4>(t + l * 4, u);
        dl[l * 3] = -(f[0] * f[6] + f[1] * f[7] + f[3] * f[8]) - u[0];
        dl[l * 3 + 1] = -(f[2] * f[7] + f[4] * f[8]) - u[1];
        dl[l * 3 + 2] = -(f[5] * f[8]) - u[2];
    }
}

template <typename T, int BP, int BL>
__global__ void backsub_kernel(int64_t L, int bp_rt, int bl_rt, const int* __restrict__ cross_offsets,
                               const int* __restrict__ cross_primary, const T* __restrict__ w,
                               const T* __restrict__ gl, const double* __restrict__ hinv, int hstride,
                               int factor, const T* __restrict__ dp, T* __restrict__ dl)
{
    constexpr int ML = BL > 0 ? BL : 16;
    const int bp = BP > 0 ? BP : bp_rt;
    const int bl = BL > 0 ? BL : bl_rt;
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l < L; l += int64_t(gridDim.x) * blockDim.x)
    {
        T point[ML];
        for (int i = 0; i < bl; ++i)
            point[i] = -gl[l * bl + i];
        for (int c = cross_offsets[l]; c < cross_offsets[l + 1]; ++c)
        {
            const T* W = w + int64_t(c) * bp * bl;
            const T* x = dp + int64_t(cross_primary[c]) * bp;
            if constexpr (BP == 6 && BL == 3 && sizeof(T) == 8)
            {
                // the cross block as 16-byte loads (the normal-equation buffers are 256-byte aligned
                // and a block is 144 bytes); the caller's step vector element by element
                double wv[18], xv[6];
                const double2* w2 = reinterpret_cast<const double2*>(W);
#pragma unroll
                for (int k = 0; k < 9; ++k)
                {
                    const double2 a = __ldg(w2 + k);
                    wv[2 * k] = a.x;
                    wv[2 * k + 1] = a.y;
                }
#pragma unroll
                for (int k = 0; k < 6; ++k)
                    xv[k] = static_cast<double>(x[k]);
#pragma unroll
                for (int col = 0; col < 3; ++col)
                {
                    double v = 0.0;
#pragma unroll
                    for (int row = 0; row < 6; ++row)
                        v = __dadd_rn(v, __dmul_rn(wv[row * 3 + col], xv[row]));
                    point[col] = add_rn(point[col], static_cast<T>(-v));
                }
            }
            else
            {
                for (int col = 0; col < bl; ++col)
                {
                    T v = T(0);
                    for (int row = 0; row < bp; ++row)
                        v = add_rn(v, mul_rn(W[row * bl + col], x[row]));
                    point[col] = add_rn(point[col], -v);
                }
            }
        }
        const double* H = hinv + l * hstride;
        if (BL == 3 && factor)
        {
            // Hll^-1 u = L^-T (L^-1 u) from the factor record [L^-1 00, 10, 11, 20, 21, 22 | z]
            const double u0 = static_cast<double>(point[0]), u1 = static_cast<double>(point[1]),
                         u2 = static_cast<double>(point[2]);
            const double v0 = H[0] * u0, v1 = H[1] * u0 + H[2] * u1, v2 = H[3] * u0 + H[4] * u1 + H[5] * u2;
            dl[l * 3] = static_cast<T>(H[0] * v0 + H[1] * v1 + H[3] * v2);
            dl[l * 3 + 1] = static_cast<T>(H[2] * v1 + H[4] * v2);
            dl[l * 3 + 2] = static_cast<T>(H[5] * v2);
        }
        else
        {
            for (int r = 0; r < bl; ++r)
            {
                double s = 0.0;
                for (int c = 0; c < bl; ++c)
                    s = __dadd_rn(s, __dmul_rn(H[r * bl + c], static_cast<double>(point[c])));
                dl[l * bl + r] = static_cast<T>(s);
            }
        }
    }
}

// scalar CSR in the reference layout (valuePosition, block_schur_sparse_assembly.h:262-272)
template <typename T, typename O>
__global__ void export_csr_kernel(int64_t B, int bp, int64_t P, const int* __restrict__ row_ptr,
                                  const int* __restrict__ block_col, const int* __restrict__ block_row,
                                  const T* __restrict__ S, int64_t* __restrict__ row_offsets,
                                  int64_t* __restrict__ col_indices, O* __restrict__ values)
{
    const int bpp = bp * bp;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < B * bpp; i += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t b = i / bpp;
        const int e = static_cast<int>(i - b * bpp), r = e / bp, c = e % bp;
        const int p = block_row[b];
        const int64_t first = row_ptr[p];
        const int64_t slots = row_ptr[p + 1] - first;
        const int64_t ordinal = b - first;
        const int64_t row_start = first * bpp + r * slots * bp;
        const int64_t pos = row_start + ordinal * bp + c;
        if (ordinal == 0 && c == 0 && row_offsets)
            row_offsets[int64_t(p) * bp + r] = row_start;
        if (col_indices)
            col_indices[pos] = int64_t(block_col[b]) * bp + c;
        if (values)
            values[pos] = static_cast<O>(S[i]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && row_offsets)
        row_offsets[P * bp] = B * bpp;
}

} // namespace
} // namespace pm

// ===================================================================== host orchestration
namespace pm
{
namespace
{

template <typename T>
void numeric_layout(pm_schur_workspace* ws, cudaStream_t stream, bool mixed, bool mixed32 = false)
{
    const int64_t n = ws->P * ws->bp;
    const int64_t bpp = ws->bp * ws->bp;
    // 6x3 cross-pair assembly: one 80-byte factor record [L^-1 | z] per eliminated block
    ws->hstride = ws->paired ? 10 : static_cast<int>(ws->bl * ws->bl);
    ws->ystride = ws->paired ? 10 : static_cast<int>(ws->bl);
    Carver plan;
    plan.take<double>(ws->L * ws->hstride + 1);
    plan.take<double>(ws->paired ? 1 : ws->L * ws->bl + 1);
    plan.take<T>(ws->B * bpp + 1);
    plan.take<float>(mixed ? ws->B * bpp + 1 : 1);
    plan.take<double>(n + 1);
    plan.take<double>(ws->P * bpp + 1);
    plan.take<float>(mixed ? ws->P * bpp + 1 : 1);
    plan.take<SchurStatus>(1);
    plan.take<SolveState>(1);
    plan.take<double>(4 * kMaxParts);
    plan.take<double>(8 * (n + 1)); // PCG / refinement vectors
    plan.take<double>(mixed32 ? ws->L * 4 + 4 : 1);
    ws->numeric.ensure(plan.offset + 256, stream, "SchurComplementSolverWorkspace");
    Carver c;
    c.base = static_cast<char*>(ws->numeric.ptr);
    ws->hinv = c.take<double>(ws->L * ws->hstride + 1);
    ws->y = c.take<double>(ws->paired ? 1 : ws->L * ws->bl + 1);
    if (ws->paired)
        ws->y = ws->hinv + 6;
    ws->S = c.take<T>(ws->B * bpp + 1);
    ws->S32 = c.take<float>(mixed ? ws->B * bpp + 1 : 1);
    ws->rhs = c.take<double>(n + 1);
    ws->minv = c.take<double>(ws->P * bpp + 1);
    ws->minv32 = c.take<float>(mixed ? ws->P * bpp + 1 : 1);
    ws->status = c.take<SchurStatus>(1);
    ws->state = c.take<SolveState>(1);
    ws->partials = c.take<double>(4 * kMaxParts);
    c.take<double>(8 * (n + 1));
    ws->mf_t = c.take<double>(mixed32 ? ws->L * 4 + 4 : 1);
}

double* vector_area(pm_schur_workspace* ws)
{
    Carver c;
    c.base = reinterpret_cast<char*>(ws->partials + 4 * kMaxParts);
    return c.take<double>(1); // aligned start of the 8 (n+1)-sized vector slots
}

void set_smem(const void* fn, size_t bytes)
{
    if (bytes > 48 * 1024)
        PM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
}

bool topology_matches(pm_schur_workspace* ws, const pm_normal_equations* ne, cudaStream_t stream)
{
    if (ws->P != ne->P || ws->L != ne->L || ws->bp != ne->bp || ws->bl != ne->bl || ws->C != ne->cross_count ||
        ws->PC != ne->primary_cross_count || !ws->saved_offsets)
        return false;
    if (ws->last_ne == ne && ws->last_version == ne->topology_version)
        return true;
    int* flag = reinterpret_cast<int*>(ws->status) + 7; // pad slot of the status block
    PM_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), stream));
    int_compare_kernel<<<grid_for(ne->L + 1, 256, 4096), 256, 0, stream>>>(ne->cross_offsets, ws->saved_offsets,
                                                                            ne->L + 1, flag);
    PM_LAUNCH_CHECK();
    int_compare_kernel<<<grid_for(ne->cross_count, 256, 4096), 256, 0, stream>>>(ne->cross_primary, ws->saved_primary,
                                                                                 ne->cross_count, flag);
    PM_LAUNCH_CHECK();
    int_compare_kernel<<<grid_for(ne->primary_cross_count, 256, 4096), 256, 0, stream>>>(
        ne->primary_cross_row, ws->saved_pc, ne->primary_cross_count, flag);
    PM_LAUNCH_CHECK();
    int_compare_kernel<<<grid_for(ne->primary_cross_count, 256, 4096), 256, 0, stream>>>(
        ne->primary_cross_col, ws->saved_pc + ne->primary_cross_count, ne->primary_cross_count, flag);
    PM_LAUNCH_CHECK();
    int differs = 0;
    PM_CUDA(cudaMemcpyAsync(&differs, flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaStreamSynchronize(stream));
    return differs == 0;
}

// Cross-pair lists of the 6x3 assembly (see assemble_upper6_kernel).
void build_pairs(pm_schur_workspace* ws, const pm_normal_equations* ne, cudaStream_t stream)
{
    const int64_t P = ne->P, C = ne->cross_count, B = ws->B;
    ws->paired = false;
    const int sorted = ne->crosses_sorted ? 1 : 0;
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(P, 8 * sm_count())));
    Carver s1;
    s1.take<int>(C + 1);
    s1.take<int64_t>(C + 2);
    s1.take<char>(scan_scratch_bytes(C + 1, sizeof(int64_t)));
    const size_t pass1 = ((s1.offset + 255) / 256) * 256;
    int64_t* offset = nullptr;
    int64_t E = 0;
    // pass 1: items per row-list entry (re-run when the scratch moves)
    auto run_pass1 = [&]() {
        Carver c1;
        c1.base = static_cast<char*>(ws->scratch.ptr);
        int* count = c1.take<int>(C + 1);
        offset = c1.take<int64_t>(C + 2);
        void* scan1 = c1.take<char>(scan_scratch_bytes(C + 1, sizeof(int64_t)));
        if (P > 0 && C > 0)
        {
            pair_count_kernel<<<grid, 128, 0, stream>>>(P, ws->prim_offsets, ws->prim_cross, ne->cross_eliminated,
                                                        ne->cross_offsets, ne->cross_primary, sorted, count);
            PM_LAUNCH_CHECK();
        }
        exclusive_scan<int, int64_t>(count, offset, C, scan1, stream);
        PM_CUDA(cudaMemcpyAsync(&E, offset + C, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
        PM_CUDA(cudaStreamSynchronize(stream));
    };
    ws->scratch.ensure(pass1 + 512, stream, "SchurComplementSolverWorkspace");
    run_pass1();
    // pass 2 scratch: items (block, row-list entry of (l, q)), row-list position of every cross,
    // upper-block counts, pairs per block, lane masks, cursors
    Carver s2;
    s2.take<int>(E + 1);
    s2.take<int>(E + 1);
    s2.take<int>(C + 1);
    s2.take<int>(P + 1);
    s2.take<int>(P + 2);
    s2.take<char>(scan_scratch_bytes(P + 1, sizeof(int)));
    s2.take<int>(B + 1);
    s2.take<unsigned>(B + 1);
    s2.take<int64_t>(B + 1);
    s2.take<char>(scan_scratch_bytes(B + 1, sizeof(int64_t)));
    void* before = ws->scratch.ptr;
    ws->scratch.ensure(pass1 + s2.offset + 512, stream, "SchurComplementSolverWorkspace");
    if (ws->scratch.ptr != before)
        run_pass1();
    Carver c2;
    c2.base = static_cast<char*>(ws->scratch.ptr) + pass1;
    int* item_block = c2.take<int>(E + 1);
    int* item_entry = c2.take<int>(E + 1);
    int* rowpos = c2.take<int>(C + 1);
    int* upper_count = c2.take<int>(P + 1);
    int* upper_offset = c2.take<int>(P + 2);
    void* upper_scan = c2.take<char>(scan_scratch_bytes(P + 1, sizeof(int)));
    int* block_pairs = c2.take<int>(B + 1);
    unsigned* mask = c2.take<unsigned>(B + 1);
    int64_t* cursor = c2.take<int64_t>(B + 1);
    void* scan2 = c2.take<char>(scan_scratch_bytes(B + 1, sizeof(int64_t)));
    // persistent: row entries (C) | pair offsets (B + 1) | pairs (E)
    Carver plan_b;
    plan_b.take<int2>(C + 1);
    plan_b.take<int64_t>(B + 2);
    plan_b.take<int2>(E + 1);
    plan_b.take<double>(C * 18 + 2); // V in the Scalar type (double at most)
    const int64_t U = (B - P) / 2;   // every row holds its diagonal block; the rest pair up by transpose
    plan_b.take<int>(U + 1);
    ws->pair_buffer.ensure(plan_b.offset + 512, stream, "SchurComplementSolverWorkspace");
    Carver bc;
    bc.base = static_cast<char*>(ws->pair_buffer.ptr);
    ws->row_entries = bc.take<int2>(C + 1);
    ws->pair_offset = bc.take<int64_t>(B + 2);
    ws->pairs = bc.take<int2>(E + 1);
    ws->vfactor = bc.take<double>(C * 18 + 2);
    ws->upper_list = bc.take<int>(U + 1);
    ws->U = U;
    ws->E = E;
    if (P > 0)
    {
        upper_count_kernel<<<grid_for(P, 256, 4096), 256, 0, stream>>>(P, ws->block_row_ptr, ws->diag_pos, upper_count);
        PM_LAUNCH_CHECK();
        exclusive_scan<int, int>(upper_count, upper_offset, P, upper_scan, stream);
        upper_list_kernel<<<grid_for(P, 128, 4096), 128, 0, stream>>>(P, ws->diag_pos, upper_offset, ws->upper_list);
        PM_LAUNCH_CHECK();
    }
    PM_CUDA(cudaMemsetAsync(block_pairs, 0, size_t(B + 1) * sizeof(int), stream));
    PM_CUDA(cudaMemsetAsync(mask, 0, size_t(B + 1) * sizeof(unsigned), stream));
    if (C > 0)
    {
        rowpos_kernel<<<grid_for(C, 256, 1 << 16), 256, 0, stream>>>(C, ws->prim_cross, rowpos);
        PM_LAUNCH_CHECK();
    }
    if (P > 0 && E > 0)
    {
        pair_emit_kernel<<<grid, 128, 0, stream>>>(P, ws->prim_offsets, ws->prim_cross, ne->cross_eliminated,
                                                   ne->cross_offsets, ne->cross_primary, sorted, offset,
                                                   ws->block_row_ptr, ws->block_col, ws->diag_pos, rowpos, item_block,
                                                   item_entry, block_pairs);
        PM_LAUNCH_CHECK();
    }
    exclusive_scan<int, int64_t>(block_pairs, ws->pair_offset, B, scan2, stream);
    if (B > 0)
        PM_CUDA(cudaMemcpyAsync(cursor, ws->pair_offset, size_t(B) * sizeof(int64_t), cudaMemcpyDeviceToDevice,
                                stream));
    if (C > 0)
    {
        row_entries_kernel<<<grid_for(C, 256, 1 << 16), 256, 0, stream>>>(C, ws->prim_cross, ne->cross_eliminated,
                                                                         ws->row_entries);
        PM_LAUNCH_CHECK();
    }
    if (P > 0 && E > 0)
    {
        pair_place_kernel<<<grid_for(P * 32, 256, 1 << 16), 256, 0, stream>>>(
            P, ws->prim_offsets, offset, item_block, item_entry, ws->row_entries, mask, cursor, ws->pairs);
        PM_LAUNCH_CHECK();
    }
    ws->paired = true;
}

void build_pattern(pm_schur_workspace* ws, const pm_normal_equations* ne, cudaStream_t stream)
{
    const int64_t P = ne->P, L = ne->L, C = ne->cross_count, PC = ne->primary_cross_count;
    const size_t bitmap = size_t((P + 31) / 32) * sizeof(unsigned);
    if (bitmap > 200 * 1024)
        fail(PM_OVERFLOW_ERROR, "Schur pattern build supports up to 1,638,400 primary blocks");
    // fixed-size pattern arrays and scratch
    Carver plan;
    plan.take<int>(P + 1);
    plan.take<int>(C + 1);
    plan.take<int>(P + 1);
    plan.take<int>(P + 1);
    plan.take<int>(P + 1);
    plan.take<int>(L + 1);
    plan.take<int>(C + 1);
    plan.take<int>(2 * PC + 1);
    plan.take<char>(scan_scratch_bytes(P + 1, sizeof(int)));
    ws->pattern.ensure(plan.offset + 256, stream, "SchurComplementSolverWorkspace");
    Carver c;
    c.base = static_cast<char*>(ws->pattern.ptr);
    ws->prim_offsets = c.take<int>(P + 1);
    ws->prim_cross = c.take<int>(C + 1);
    ws->block_row_ptr = c.take<int>(P + 1);
    int* row_count = c.take<int>(P + 1);
    ws->diag_pos = c.take<int>(P + 1);
    ws->saved_offsets = c.take<int>(L + 1);
    ws->saved_primary = c.take<int>(C + 1);
    ws->saved_pc = c.take<int>(2 * PC + 1);
    void* scan_scratch = c.take<char>(scan_scratch_bytes(P + 1, sizeof(int)));
    // per-primary cross lists, ascending eliminated index (crosses are eliminated-major)
    ws->scratch.ensure(size_t(2 * (C + 1)) * sizeof(int64_t) + 512, stream, "SchurComplementSolverWorkspace");
    int64_t* primary64 = static_cast<int64_t*>(ws->scratch.ptr);
    int64_t* ids64 = primary64 + (C + 1);
    if (!ws->prim_sort && pm_sparse_workspace_create(&ws->prim_sort) != PM_OK)
        fail(PM_RUNTIME_ERROR, "could not create the pattern sort workspace");
    if (C > 0)
    {
        widen_int_kernel<<<grid_for(C, 256, 4096), 256, 0, stream>>>(ne->cross_primary, primary64, C);
        PM_LAUNCH_CHECK();
        iota_kernel<<<grid_for(C, 256, 4096), 256, 0, stream>>>(ids64, C);
        PM_LAUNCH_CHECK();
    }
    coo_prepare<float>(ws->prim_sort, stream, P, C + 1, C, primary64, ids64, nullptr);
    coo_internal_status(ws->prim_sort, stream, "Schur pattern");
    const CooView v = coo_view(ws->prim_sort);
    PM_CUDA(cudaMemcpyAsync(ws->prim_offsets, v.bucket_start, (P + 1) * sizeof(int), cudaMemcpyDeviceToDevice, stream));
    if (C > 0)
    {
        keys_to_cross_kernel<<<grid_for(C, 256, 4096), 256, 0, stream>>>(v.keys, C, ws->prim_cross);
        PM_LAUNCH_CHECK();
    }
    // block-CSR rows
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(P, 8 * sm_count())));
    set_smem(reinterpret_cast<const void*>(row_count_kernel), bitmap);
    set_smem(reinterpret_cast<const void*>(row_fill_kernel), bitmap);
    if (P > 0)
    {
        row_count_kernel<<<grid, 256, bitmap, stream>>>(P, ws->prim_offsets, ws->prim_cross, ne->cross_eliminated,
                                                        ne->cross_offsets, ne->cross_primary, ne->primary_cross_row,
                                                        ne->primary_cross_col, PC, row_count);
        PM_LAUNCH_CHECK();
    }
    exclusive_scan<int, int>(row_count, ws->block_row_ptr, P, scan_scratch, stream);
    int B = 0;
    PM_CUDA(cudaMemcpyAsync(&B, ws->block_row_ptr + P, sizeof(int), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaStreamSynchronize(stream));
    ws->B = B;
    // block arrays live behind the fixed part of the scratch buffer's successor allocation
    Carver bplan;
    bplan.take<int>(B + 1);
    bplan.take<int>(B + 1);
    bplan.take<int>(B + 1);
    bplan.take<int>(B + 1);
    const size_t fixed = plan.offset;
    ws->pattern.ensure(fixed + bplan.offset + 512, stream, "SchurComplementSolverWorkspace");
    if (ws->pattern.ptr != c.base)
    {
        // the pattern buffer moved: re-carve the fixed part (contents are rebuilt below anyway,
        // except prim lists / row pointers, which are recomputed by re-running this function)
        return build_pattern(ws, ne, stream);
    }
    Carver bc;
    bc.base = static_cast<char*>(ws->pattern.ptr) + ((fixed + 255) / 256) * 256;
    ws->block_col = bc.take<int>(B + 1);
    ws->block_row = bc.take<int>(B + 1);
    ws->transpose = bc.take<int>(B + 1);
    ws->block_pc = bc.take<int>(B + 1);
    if (P > 0)
    {
        row_fill_kernel<<<grid, 256, bitmap, stream>>>(P, ws->prim_offsets, ws->prim_cross, ne->cross_eliminated,
                                                       ne->cross_offsets, ne->cross_primary, ne->primary_cross_row,
                                                       ne->primary_cross_col, PC, ws->block_row_ptr, ws->block_col,
                                                       ws->block_row, ws->diag_pos);
        PM_LAUNCH_CHECK();
        transpose_kernel<<<grid_for(B, 256, 8192), 256, 0, stream>>>(B, ws->block_row_ptr, ws->block_col, ws->block_row,
                                                                     ws->transpose);
        PM_LAUNCH_CHECK();
    }
    PM_CUDA(cudaMemsetAsync(ws->block_pc, 0xff, size_t(B + 1) * sizeof(int), stream));
    ws->paired = false;
    if (ne->bp == 6 && ne->bl == 3)
        build_pairs(ws, ne, stream);
    if (PC > 0)
    {
        block_pc_kernel<<<grid_for(PC, 256, 4096), 256, 0, stream>>>(PC, ne->primary_cross_row, ne->primary_cross_col,
                                                                     ws->block_row_ptr, ws->block_col, ws->block_pc);
        PM_LAUNCH_CHECK();
    }
    PM_CUDA(cudaMemcpyAsync(ws->saved_offsets, ne->cross_offsets, (L + 1) * sizeof(int), cudaMemcpyDeviceToDevice, stream));
    if (C > 0)
        PM_CUDA(cudaMemcpyAsync(ws->saved_primary, ne->cross_primary, C * sizeof(int), cudaMemcpyDeviceToDevice, stream));
    if (PC > 0)
    {
        PM_CUDA(cudaMemcpyAsync(ws->saved_pc, ne->primary_cross_row, PC * sizeof(int), cudaMemcpyDeviceToDevice, stream));
        PM_CUDA(cudaMemcpyAsync(ws->saved_pc + PC, ne->primary_cross_col, PC * sizeof(int), cudaMemcpyDeviceToDevice,
                                stream));
    }
    ws->P = P;
    ws->L = L;
    ws->bp = ne->bp;
    ws->bl = ne->bl;
    ws->C = C;
    ws->PC = PC;
    ws->pattern_builds += 1;
}

// Launch shapes of the upper-block pass: {pair streams, lanes per pair}.  Shape 0 is the default;
// pm_schur_autotune_assembly times them all on the caller's system and keeps the fastest.
struct UpperShape
{
    int streams, split;
};
constexpr UpperShape kUpperShapes[] = {{8, 2}, {4, 2}, {16, 2}, {4, 4}, {8, 4}, {2, 2}, {1, 2}};
constexpr int kUpperShapeCount = sizeof(kUpperShapes) / sizeof(kUpperShapes[0]);

template <typename TO, typename TP, typename VT, typename AT, int STREAMS, int SPLIT>
void launch_upper_shape(pm_schur_workspace* ws, const int* block_pc, const VT* vf, const TP* pcv, TO* S,
                        cudaStream_t stream)
{
    const unsigned grid = grid_for(std::max<int64_t>(ws->U, 1) * STREAMS * SPLIT, kUpperThreads);
    assemble_upper6_kernel<TO, TP, VT, AT, STREAMS, SPLIT><<<grid, kUpperThreads, 0, stream>>>(
        ws->U, ws->upper_list, ws->pair_offset, ws->pairs, ws->transpose, block_pc, vf, pcv, S);
    PM_LAUNCH_CHECK();
}

template <typename TO, typename TP, typename VT, typename AT>
void launch_upper(pm_schur_workspace* ws, const int* block_pc, const VT* vf, const TP* pcv, TO* S,
                  cudaStream_t stream)
{
    switch (ws->upper_shape)
    {
    case 1: launch_upper_shape<TO, TP, VT, AT, 4, 2>(ws, block_pc, vf, pcv, S, stream); break;
    case 2: launch_upper_shape<TO, TP, VT, AT, 16, 2>(ws, block_pc, vf, pcv, S, stream); break;
    case 3: launch_upper_shape<TO, TP, VT, AT, 4, 4>(ws, block_pc, vf, pcv, S, stream); break;
    case 4: launch_upper_shape<TO, TP, VT, AT, 8, 4>(ws, block_pc, vf, pcv, S, stream); break;
    case 5: launch_upper_shape<TO, TP, VT, AT, 2, 2>(ws, block_pc, vf, pcv, S, stream); break;
    case 6: launch_upper_shape<TO, TP, VT, AT, 1, 2>(ws, block_pc, vf, pcv, S, stream); break;
    default: launch_upper_shape<TO, TP, VT, AT, 8, 2>(ws, block_pc, vf, pcv, S, stream); break;
    }
}

template <typename T>
void launch_assembly(pm_schur_workspace* ws, const pm_normal_equations* ne, double lambda, double min_diag,
                     cudaStream_t stream, bool fp32_products = false)
{
    ws->s32_only = false;
    ws->damping = lambda;
    ws->min_diag = min_diag;
    AssembleArgs<T> a;
    a.P = ne->P;
    a.bp = static_cast<int>(ne->bp);
    a.bl = static_cast<int>(ne->bl);
    a.prim_offsets = ws->prim_offsets;
    a.prim_cross = ws->prim_cross;
    a.cross_eliminated = ne->cross_eliminated;
    a.cross_offsets = ne->cross_offsets;
    a.cross_primary = ne->cross_primary;
    a.block_row_ptr = ws->block_row_ptr;
    a.block_col = ws->block_col;
    a.diag_pos = ws->diag_pos;
    a.block_pc = ws->block_pc;
    a.hpp = static_cast<const T*>(ne->primary_diagonal);
    a.gp = static_cast<const T*>(ne->primary_gradient);
    a.w = static_cast<const T*>(ne->cross_values);
    a.pcv = static_cast<const T*>(ne->primary_cross_values);
    a.hinv = ws->hinv;
    a.y = ws->y;
    a.lambda = lambda;
    a.min_diag = min_diag;
    a.S = static_cast<T*>(ws->S);
    a.rhs = ws->rhs;
    a.minv = ws->minv;
    a.status = ws->status;
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, ne->P));
    auto smem_for = [&](int ch, int mp) {
        const int bpl = a.bp * a.bl, bpp = a.bp * a.bp;
        return size_t(ch) * (bpl + bpp + a.bp) * sizeof(T) + size_t(mp * mp) * sizeof(double) + 64 +
               kRowThreads * sizeof(unsigned long long) + 2 * ch * sizeof(int) + 64;
    };
    if (ws->paired)
    {
        if (fp32_products)
        {
            // FP32 products: V stored in FP32, upper blocks formed and summed in FP32 into S32;
            // the diagonal blocks and the RHS are still summed in FP64 (S keeps the FP64 diagonal
            // blocks for the FP64 block-Jacobi factorisation)
            float* vf = static_cast<float*>(ws->vfactor);
            assemble_diag6_kernel<T, float><<<grid_for(a.P, 1, 1 << 20), kDiagThreads, 0, stream>>>(
                a.P, ws->prim_offsets, ws->row_entries, a.w, ws->hinv, a.hpp, a.gp, a.lambda, a.min_diag,
                a.diag_pos, a.S, a.rhs, vf, ws->S32);
            PM_LAUNCH_CHECK();
            launch_upper<float, T, float, float>(ws, a.block_pc, vf, a.pcv, ws->S32, stream);
        }
        else
        {
            T* vf = static_cast<T*>(ws->vfactor);
            assemble_diag6_kernel<T, T><<<grid_for(a.P, 1, 1 << 20), kDiagThreads, 0, stream>>>(
                a.P, ws->prim_offsets, ws->row_entries, a.w, ws->hinv, a.hpp, a.gp, a.lambda, a.min_diag,
                a.diag_pos, a.S, a.rhs, vf, nullptr);
            PM_LAUNCH_CHECK();
            // every upper block, also those whose only terms are primary-primary couplings
            launch_upper<T, T, T, double>(ws, a.block_pc, vf, a.pcv, a.S, stream);
        }
        ws->s32_only = fp32_products;
        diag_inverse_kernel<T, 6><<<grid_for(a.P, 64, 1 << 16), 64, 0, stream>>>(a.P, a.diag_pos, a.S, a.minv,
                                                                                 a.status);
        PM_LAUNCH_CHECK();
    }
    else
    {
        if (ne->bp > 16 || ne->bl > 16)
            fail(PM_INVALID_ARGUMENT, "device Schur solver supports block sizes up to 16");
        const size_t smem = smem_for(16, 16);
        set_smem(reinterpret_cast<const void*>(assemble_kernel<T, 0, 0, 16>), smem);
        assemble_kernel<T, 0, 0, 16><<<grid, kRowThreads, smem, stream>>>(a);
        PM_LAUNCH_CHECK();
    }
    if (!ws->paired) // the pair kernel writes each upper block's transpose itself
    {
        mirror_kernel<T><<<grid_for(ws->B * ne->bp * ne->bp, 256, 65535), 256, 0, stream>>>(
            ws->B, static_cast<int>(ne->bp), ws->block_row, ws->block_col, ws->transpose, static_cast<T*>(ws->S));
        PM_LAUNCH_CHECK();
    }
}

} // namespace

SchurView schur_view(pm_schur_workspace* ws, bool mixed)
{
    SchurView v;
    if (!ws || !ws->assembled || ws->bp != 6)
        return v;
    v.P = ws->P;
    v.B = ws->B;
    v.value_size = ws->s32_only ? 4 : ws->value_size;
    v.mixed = mixed || ws->s32_only;
    v.block_row_ptr = ws->block_row_ptr;
    v.block_col = ws->block_col;
    v.diag_pos = ws->diag_pos;
    v.S = ws->s32_only ? static_cast<const void*>(ws->S32) : ws->S;
    v.minv = ws->minv;
    v.minv32 = ws->minv32;
    return v;
}

namespace
{

// ---------------------------------------------------------------- batched PCG
// Many independent systems assembled as one block-diagonal union (system s owns the block rows
// [row0[s], row0[s+1])).  One set of kernels serves every system: per-system dots are summed
// by one warp per system over its rows in a fixed order, alpha / beta / convergence are
// per-system device state, converged systems stop updating, and the iterations are captured
// once into the body of a CUDA graph 'while' node that repeats until no system is active.
struct BatchState
{
    double rho, alpha, beta, tol, rr, rr0, window_sq;
    long long t_start, t_done; // %globaltimer at (re)start and at convergence
    int active, iterations, converged, breakdown, stagnated, window_start, restart, pad;
};

__device__ __forceinline__ long long global_ns()
{
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// q = S v on the rows of systems selected by `want` (active, or restarting); row_dot = v.q
template <typename M, int Mode> // Mode 0: iteration (active systems), 1: (re)start (restart flag)
__global__ void __launch_bounds__(kVecBlock) batch_spmv_kernel(int64_t P, const int* __restrict__ row_ptr,
                                                               const int* __restrict__ block_col, const M* __restrict__ S,
                                                               const double* __restrict__ v, double* __restrict__ q,
                                                               double* __restrict__ row_dot,
                                                               const int* __restrict__ row_sys,
                                                               const BatchState* __restrict__ bs)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x / 32);
    for (int64_t p = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; p < P; p += warps)
    {
        const BatchState& st = bs[row_sys[p]];
        if (!(Mode == 0 ? st.active : st.restart))
            continue; // warp-uniform
        double out[16];
        bsr_row<double, M, 6>(row_ptr, block_col, S, v, 6, p, true, lane, out);
        double mine = 0.0;
        if (lane < 6)
        {
            double y = 0.0;
            for (int r = 0; r < 6; ++r)
                y = lane == r ? out[r] : y;
            q[p * 6 + lane] = y;
            mine = v[p * 6 + lane] * y;
        }
        for (int o = 4; o > 0; o >>= 1)
            mine += __shfl_xor_sync(0xffffffffu, mine, o);
        if (lane == 0)
            row_dot[p] = mine;
    }
}

// sum of a per-row array over a system's rows (warp, fixed order); valid in every lane
__device__ __forceinline__ double system_sum(const double* __restrict__ row_val, int r0, int r1, int lane)
{
    double s = 0.0;
    for (int p = r0 + lane; p < r1; p += 32)
        s += row_val[p];
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

__global__ void batch_alpha_kernel(int64_t systems, const int* __restrict__ sys_row, const double* __restrict__ row_dot,
                                   BatchState* __restrict__ bs)
{
    const int lane = threadIdx.x & 31;
    for (int64_t s = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; s < systems;
         s += int64_t(gridDim.x) * blockDim.x / 32)
    {
        BatchState& st = bs[s];
        if (!st.active)
            continue;
        const double pq = system_sum(row_dot, sys_row[s], sys_row[s + 1], lane);
        if (lane == 0)
        {
            if (!(pq > 0.0) || !isfinite(pq))
            {
                st.breakdown = 1;
                st.active = 0;
                st.alpha = 0.0;
            }
            else
            {
                st.alpha = st.rho / pq;
            }
        }
    }
}

// x += alpha p, r -= alpha q (Mode 0), or r = b - q, x kept (Mode 1, restarting systems);
// then z = Minv r and the row sums of r.z and r.r (p = z on restart)
template <int Mode, typename PM = double>
__global__ void batch_update_kernel(int64_t P, const int* __restrict__ row_sys, const BatchState* __restrict__ bs,
                                    double* __restrict__ x, double* __restrict__ p_vec, const double* __restrict__ q,
                                    const double* __restrict__ b, double* __restrict__ r, double* __restrict__ z,
                                    const PM* __restrict__ minv, double* __restrict__ row_rz,
                                    double* __restrict__ row_rr)
{
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
    {
        const BatchState& st = bs[row_sys[p]];
        if (!(Mode == 0 ? st.active : st.restart))
            continue;
        double rr[6];
        if (Mode == 0)
        {
            const double a = st.alpha;
            for (int k = 0; k < 6; ++k)
            {
                x[p * 6 + k] += a * p_vec[p * 6 + k];
                rr[k] = r[p * 6 + k] - a * q[p * 6 + k];
                r[p * 6 + k] = rr[k];
            }
        }
        else
        {
            for (int k = 0; k < 6; ++k)
            {
                rr[k] = b[p * 6 + k] - q[p * 6 + k];
                r[p * 6 + k] = rr[k];
            }
        }
        const PM* m = minv + p * 36;
        double rz = 0.0, r2 = 0.0;
        for (int k = 0; k < 6; ++k)
        {
            double zk = 0.0;
            for (int c = 0; c < 6; ++c)
                zk += static_cast<double>(m[k * 6 + c]) * rr[c];
            z[p * 6 + k] = zk;
            if (Mode == 1)
                p_vec[p * 6 + k] = zk;
            rz += rr[k] * zk;
            r2 += rr[k] * rr[k];
        }
        row_rz[p] = rz;
        row_rr[p] = r2;
    }
}

// Mode 0: one iteration's convergence / stagnation / beta; Mode 1: (re)start of flagged systems
template <int Mode>
__global__ void batch_beta_kernel(int64_t systems, const int* __restrict__ sys_row, const double* __restrict__ row_rz,
                                  const double* __restrict__ row_rr, BatchState* __restrict__ bs, int max_iterations,
                                  int window, double rel, double abs_tol, int rule, int* __restrict__ active_count)
{
    const int lane = threadIdx.x & 31;
    for (int64_t s = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; s < systems;
         s += int64_t(gridDim.x) * blockDim.x / 32)
    {
        BatchState& st = bs[s];
        if (!(Mode == 0 ? st.active : st.restart))
            continue;
        const double rz = system_sum(row_rz, sys_row[s], sys_row[s + 1], lane);
        const double r2 = system_sum(row_rr, sys_row[s], sys_row[s + 1], lane);
        if (lane != 0)
            continue;
        const long long now = global_ns();
        st.rr = r2;
        if (Mode == 1)
        {
            if (st.restart == 1) // first start: tolerance from this residual
            {
                st.rr0 = r2;
                const double r0 = sqrt(fmax(0.0, r2));
                st.tol = rule == 0 ? abs_tol + rel * r0 : fmax(abs_tol, rel * r0);
                st.t_start = now;
                st.iterations = 0;
            }
            st.restart = 0;
            st.rho = rz;
            st.window_start = st.iterations;
            st.window_sq = r2;
            st.stagnated = 0;
            st.breakdown = 0;
            const bool done = !(sqrt(fmax(0.0, r2)) > st.tol);
            st.converged = done && isfinite(r2);
            st.active = !done && isfinite(r2) && st.iterations < max_iterations;
            if (done)
                st.t_done = now;
            if (!isfinite(r2))
                st.breakdown = 1;
        }
        else
        {
            st.iterations += 1;
            if (!isfinite(r2))
            {
                st.breakdown = 1;
                st.active = 0;
            }
            else if (sqrt(r2) <= st.tol)
            {
                st.converged = 1;
                st.active = 0;
                st.t_done = now;
            }
            else if (st.iterations >= max_iterations)
            {
                st.active = 0;
            }
            else if (window > 0 && st.iterations - st.window_start >= window && r2 > 0.25 * st.window_sq)
            {
                st.stagnated = 1;
                st.active = 0;
            }
            else
            {
                if (window > 0 && st.iterations - st.window_start >= window)
                {
                    st.window_start = st.iterations;
                    st.window_sq = r2;
                }
                st.beta = rz / st.rho;
                st.rho = rz;
            }
        }
        if (st.active)
            atomicAdd(active_count, 1);
    }
}

__global__ void batch_direction_kernel(int64_t P, const int* __restrict__ row_sys, const BatchState* __restrict__ bs,
                                       const double* __restrict__ z, double* __restrict__ p_vec)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < P * 6; i += int64_t(gridDim.x) * blockDim.x)
    {
        const BatchState& st = bs[row_sys[i / 6]];
        if (st.active)
            p_vec[i] = z[i] + st.beta * p_vec[i];
    }
}

// Condition of the device-driven iteration loop (a CUDA graph 'while' node): another chunk of
// iterations while any system is active, at most max_chunks chunks per launch of the loop.
__global__ void batch_continue_kernel(cudaGraphConditionalHandle handle, const int* __restrict__ active,
                                      int* __restrict__ chunks, int max_chunks)
{
    if (threadIdx.x == 0 && blockIdx.x == 0)
    {
        const int done = *chunks + 1;
        *chunks = done;
        cudaGraphSetConditional(handle, *active > 0 && done < max_chunks ? 1u : 0u);
    }
}

__global__ void batch_rows_kernel(int64_t systems, const int* __restrict__ sys_row, int* __restrict__ row_sys)
{
    for (int64_t s = blockIdx.x; s < systems; s += gridDim.x)
        for (int p = sys_row[s] + threadIdx.x; p < sys_row[s + 1]; p += blockDim.x)
            row_sys[p] = static_cast<int>(s);
}

// every block must couple rows of one system
__global__ void batch_check_kernel(int64_t P, const int* __restrict__ row_ptr, const int* __restrict__ block_col,
                                   const int* __restrict__ row_sys, int* __restrict__ bad)
{
    for (int64_t p = blockIdx.x; p < P; p += gridDim.x)
        for (int b = row_ptr[p] + threadIdx.x; b < row_ptr[p + 1]; b += blockDim.x)
            if (row_sys[block_col[b]] != row_sys[p])
                atomicExch(bad, 1);
}

// restore block Jacobi on the rows of stagnated systems and flag them for a restart
// (a system that broke down restarts from zero)
template <typename T>
__global__ void batch_fallback_kernel(int64_t P, const int* __restrict__ row_sys, BatchState* __restrict__ bs,
                                      const int* __restrict__ diag_pos, const T* __restrict__ S,
                                      double* __restrict__ minv, float* __restrict__ minv32, double* __restrict__ x)
{
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x)
    {
        const BatchState& st = bs[row_sys[p]];
        if (!st.stagnated && !st.breakdown)
            continue;
        if (st.breakdown)
            for (int k = 0; k < 6; ++k)
                x[p * 6 + k] = 0.0;
        const T* d = S + int64_t(diag_pos[p]) * 36;
        double m[36], inv[36], lower[36], work[6];
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

// mixed precision: every system that converged on the FP32 operator restarts from its iterate
// for an FP64 check (true residual b - S x with the FP64 values, tolerance and iteration count
// kept); it stays converged only if that residual meets its tolerance
__global__ void batch_verify_kernel(int64_t systems, BatchState* __restrict__ bs)
{
    for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < systems; s += int64_t(gridDim.x) * blockDim.x)
        if (bs[s].converged)
        {
            bs[s].converged = 0;
            bs[s].restart = 2;
        }
}

__global__ void batch_flag_restart_kernel(int64_t systems, BatchState* __restrict__ bs, int* __restrict__ fallen)
{
    for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < systems; s += int64_t(gridDim.x) * blockDim.x)
        if (bs[s].stagnated || bs[s].breakdown)
        {
            bs[s].restart = 2; // keep the tolerance and the iteration count
            fallen[s] = 1;
        }
}

// Condition of the block PCG's iteration graph: another chunk while the solve is not done, at
// most max_iterations / kPcgChunk + 1 chunks (the update kernel also ends the solve at
// max_iterations).
constexpr int kPcgChunk = 4; // iterations per graph body (even: the residual ping-pong returns to r0)
__global__ void pcg_continue_kernel(cudaGraphConditionalHandle handle, SolveState* st)
{
    if (threadIdx.x == 0 && blockIdx.x == 0)
    {
        const int chunks = st->chunks + 1;
        st->chunks = chunks;
        cudaGraphSetConditional(handle, !st->done && chunks <= st->max_iterations / kPcgChunk + 1 ? 1u : 0u);
    }
}

// The iteration graph of one operand set (S, inverses, x, scratch vectors and the workspace's
// state), built on first use and kept in the workspace: a CUDA graph 'while' node whose body is
// kPcgChunk iterations (direction, block SpMV with p.q, update with r.z / r.r) and
// pcg_continue_kernel, so the device decides when the solve is done.
template <typename V, typename M, typename PM>
cudaGraphExec_t pcg_iteration_graph(pm_schur_workspace* ws, const M* S, const PM* minv, V* x, V* scratch)
{
    const void* key[6] = {S, minv, x, scratch, ws->block_row_ptr, ws->block_col};
    const int types = int(sizeof(V) == 8) | int(sizeof(M) == 8) << 1 | int(sizeof(PM) == 8) << 2 |
                      int(ws->bp == 6) << 3;
    for (auto& g : ws->pcg_graphs)
        if (g.exec && g.P == ws->P && g.types == types && std::equal(key, key + 6, g.key))
            return g.exec;
    if (!ws->graph_stream)
    {
        PM_CUDA(cudaStreamCreateWithFlags(&ws->graph_stream, cudaStreamNonBlocking));
        for (auto& e : ws->graph_events)
            PM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    auto& slot = ws->pcg_graphs[ws->pcg_graph_next];
    ws->pcg_graph_next = (ws->pcg_graph_next + 1) % 4;
    if (slot.exec)
        cudaGraphExecDestroy(slot.exec);
    if (slot.graph)
        cudaGraphDestroy(slot.graph);
    slot = pm_schur_workspace::PcgGraph{};
    const int64_t P = ws->P, n = ws->P * ws->bp;
    const int bp = static_cast<int>(ws->bp);
    V* r0 = scratch;
    V* r1 = r0 + (n + 1);
    V* z = r1 + (n + 1);
    V* p = z + (n + 1);
    V* q = p + (n + 1);
    const unsigned sgrid = grid_for(P * 32, kVecBlock, kMaxParts);
    const unsigned ugrid = grid_for(P, kVecBlock, kMaxParts);
    const unsigned u6grid = grid_for(P * 8, kVecBlock, kMaxParts);
    const unsigned dgrid = grid_for(n, kVecBlock, 4096);
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
            fail(PM_CUDA_ERROR, std::string("Schur PCG: conditional graph node: ") + cudaGetErrorString(added));
        }
        body = cp.conditional.phGraph_out[0];
    }
    const cudaStream_t gs = ws->graph_stream;
    PM_CUDA(cudaStreamBeginCaptureToGraph(gs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kPcgChunk; ++k)
    {
        V* r_in = (k & 1) ? r1 : r0;
        V* r_out = (k & 1) ? r0 : r1;
        pcg_block_direction_kernel<V><<<dgrid, kVecBlock, 0, gs>>>(n, z, p, ws->state);
        if (bp == 6)
        {
            pcg_bsr_kernel<V, M, 6><<<sgrid, kVecBlock, 0, gs>>>(P, bp, ws->block_row_ptr, ws->block_col, S, p, q,
                                                                 ws->partials, ws->state);
            pcg_block_update6_kernel<V, PM><<<u6grid, kVecBlock, 0, gs>>>(P, x, p, q, r_in, r_out, z, minv,
                                                                          ws->partials, ws->state);
        }
        else
        {
            pcg_bsr_kernel<V, M, 0><<<sgrid, kVecBlock, 0, gs>>>(P, bp, ws->block_row_ptr, ws->block_col, S, p, q,
                                                                 ws->partials, ws->state);
            pcg_block_update_kernel<V, PM, 0><<<ugrid, kVecBlock, 0, gs>>>(P, bp, x, p, q, r_in, r_out, z, minv,
                                                                           ws->partials, ws->state);
        }
    }
    pcg_continue_kernel<<<1, 32, 0, gs>>>(handle, ws->state);
    cudaGraph_t captured = nullptr;
    const cudaError_t cap = cudaStreamEndCapture(gs, &captured);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t inst = cap == cudaSuccess ? cudaGraphInstantiate(&exec, graph, 0) : cap;
    if (inst != cudaSuccess)
    {
        cudaGraphDestroy(graph);
        fail(PM_CUDA_ERROR, std::string("Schur PCG: iteration graph: ") + cudaGetErrorString(inst));
    }
    std::copy(key, key + 6, slot.key);
    slot.P = P;
    slot.types = types;
    slot.graph = graph;
    slot.exec = exec;
    return exec;
}

// One preconditioned CG solve on the block-CSR operand (matrix M, vectors V, inverses PM): the
// initial residual, then the iteration graph (the device ends it), then one read of the final
// state, which is returned.
template <typename V, typename M, typename PM>
SolveState block_pcg(pm_schur_workspace* ws, cudaStream_t stream, const M* S, const PM* minv, const double* rhs,
                     V* x, double rel, double abs_tol, int rule, int max_iterations, V* scratch, int window = 0)
{
    const int64_t P = ws->P, n = ws->P * ws->bp;
    const int bp = static_cast<int>(ws->bp);
    V* r0 = scratch;
    V* z = r0 + 2 * (n + 1);
    V* p = z + (n + 1);
    V* q = p + (n + 1);
    const unsigned sgrid = grid_for(P * 32, kVecBlock, kMaxParts);
    const unsigned ugrid = grid_for(P, kVecBlock, kMaxParts);
    const bool six = bp == 6;
    if (six)
        bsr_spmv_kernel<V, M, 6><<<sgrid, kVecBlock, 0, stream>>>(P, bp, ws->block_row_ptr, ws->block_col, S, x, q);
    else
        bsr_spmv_kernel<V, M, 0><<<sgrid, kVecBlock, 0, stream>>>(P, bp, ws->block_row_ptr, ws->block_col, S, x, q);
        PM_LAUNCH_CHECK();
    if (six)
        pcg_block_init_kernel<V, PM, double, 6><<<ugrid, kVecBlock, 0, stream>>>(P, bp, rhs, q, r0, z, p, minv, rel,
                                                                                abs_tol, rule, max_iterations, window,
                                                                                ws->partials, ws->state);
    else
        pcg_block_init_kernel<V, PM, double, 0><<<ugrid, kVecBlock, 0, stream>>>(P, bp, rhs, q, r0, z, p, minv, rel,
                                                                                abs_tol, rule, max_iterations, window,
                                                                                ws->partials, ws->state);
    PM_LAUNCH_CHECK();
    // the iterations: one launch of the operand set's iteration graph, which stops on the device
    if (max_iterations > 0)
    {
        const cudaGraphExec_t exec = pcg_iteration_graph<V, M, PM>(ws, S, minv, x, scratch);
        PM_CUDA(cudaMemsetAsync(&ws->state->chunks, 0, sizeof(int), stream));
        PM_CUDA(cudaGraphLaunch(exec, stream));
    }
    PM_CUDA(cudaMemcpyAsync(ws->host_state, ws->state, sizeof(SolveState), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaEventRecord(ws->sync_event, stream));
    PM_CUDA(cudaEventSynchronize(ws->sync_event));
    if (max_iterations > 0) // the kernels the graph ran: kPcgChunk x 3 + 1 per body
        for (int k = 0; k < ws->host_state->chunks * (3 * kPcgChunk + 1); ++k)
            count_launch();
    return *ws->host_state;
}

// FP64 true residual ||b - S x|| and ||b|| (S in Scalar precision, x FP64)
template <typename M>
void true_residual(pm_schur_workspace* ws, cudaStream_t stream, const M* S, const double* x, double* q, double* r,
                   double& norm, double& rhs_norm, bool x_is_zero = false)
{
    const int64_t P = ws->P, n = P * ws->bp;
    const int bp = static_cast<int>(ws->bp);
    const unsigned sgrid = grid_for(P * 32, kVecBlock, kMaxParts);
    if (x_is_zero)
    {
        // S 0 = 0: the residual is b itself (skips a matrix-free pass over W when values are FP32)
        PM_CUDA(cudaMemsetAsync(q, 0, n * sizeof(double), stream));
    }
    else if (ws->s32_only)
    {
        // the assembled values are FP32: the FP64 product comes from the FP64 normal equations
        const pm_normal_equations* ne = ws->last_ne;
        const unsigned egrid = grid_for(ws->L, 128, 1 << 20);
        if (reinterpret_cast<uintptr_t>(x) % 16 == 0)
            mf_eliminated6_kernel<double, true><<<egrid, 128, 0, stream>>>(
                ws->L, ne->cross_offsets, ne->cross_primary, static_cast<const double*>(ne->cross_values), ws->hinv,
                x, ws->mf_t);
        else
            mf_eliminated6_kernel<double, false><<<egrid, 128, 0, stream>>>(
                ws->L, ne->cross_offsets, ne->cross_primary, static_cast<const double*>(ne->cross_values), ws->hinv,
                x, ws->mf_t);
        PM_LAUNCH_CHECK();
        mf_primary6_kernel<double><<<grid_for(P, 1, 1 << 20), kDiagThreads, 0, stream>>>(
            P, ws->prim_offsets, ws->row_entries, static_cast<const double*>(ne->cross_values), ws->mf_t,
            static_cast<const double*>(ne->primary_diagonal), ws->damping, ws->min_diag, ws->block_row_ptr,
            ws->block_col, ws->block_pc, static_cast<const double*>(ne->primary_cross_values), x, q);
        PM_LAUNCH_CHECK();
    }
    else if (bp == 6)
        bsr_spmv_kernel<double, M, 6><<<sgrid, kVecBlock, 0, stream>>>(P, bp, ws->block_row_ptr, ws->block_col, S, x, q);
    else
        bsr_spmv_kernel<double, M, 0><<<sgrid, kVecBlock, 0, stream>>>(P, bp, ws->block_row_ptr, ws->block_col, S, x, q);
    PM_LAUNCH_CHECK();
    residual_kernel<<<grid_for(n, kVecBlock, kMaxParts), kVecBlock, 0, stream>>>(n, ws->rhs, q, r, ws->partials,
                                                                               ws->state);
    PM_LAUNCH_CHECK();
    PM_CUDA(cudaMemcpyAsync(ws->host_state, ws->state, sizeof(SolveState), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaEventRecord(ws->sync_event, stream));
    PM_CUDA(cudaEventSynchronize(ws->sync_event));
    norm = std::sqrt(std::max(0.0, ws->host_state->true_squared));
    rhs_norm = std::sqrt(std::max(0.0, ws->host_state->rhs_squared));
}

struct BatchSpec
{
    int64_t systems = 0;
    const int64_t* offsets = nullptr;          // host, systems + 1 block-row offsets
    pm_batched_system_report* out = nullptr;   // host, systems
};

// Batched block-Jacobi (or learned) PCG of independent systems; x (FP64, device) holds the
// initial guesses.  Fills the per-system reports and the summary in `rep`.
template <typename M>
void batched_pcg(pm_schur_workspace* ws, cudaStream_t stream, const BatchSpec& spec, const pm_schur_options* o,
                 bool learned, bool mixed, int window, double* x, pm_schur_report* rep)
{
    const int64_t P = ws->P, NS = spec.systems;
    const M* S = static_cast<const M*>(ws->S);
    Carver plan;
    plan.take<int>(NS + 1);
    plan.take<int>(P + 1);
    plan.take<BatchState>(NS + 1);
    for (int k = 0; k < 3; ++k)
        plan.take<double>(P + 1);
    for (int k = 0; k < 4; ++k)
        plan.take<double>(6 * P + 1);
    plan.take<int>(4);
    plan.take<int>(NS + 1);
    ws->scratch.ensure(plan.offset + 512, stream, "SchurComplementSolverWorkspace");
    Carver c;
    c.base = static_cast<char*>(ws->scratch.ptr);
    int* sys_row = c.take<int>(NS + 1);
    int* row_sys = c.take<int>(P + 1);
    BatchState* bs = c.take<BatchState>(NS + 1);
    double* row_dot = c.take<double>(P + 1);
    double* row_rz = c.take<double>(P + 1);
    double* row_rr = c.take<double>(P + 1);
    double* r = c.take<double>(6 * P + 1);
    double* z = c.take<double>(6 * P + 1);
    double* pv = c.take<double>(6 * P + 1);
    double* q = c.take<double>(6 * P + 1);
    int* flags = c.take<int>(4); // [0] active count, [1] coupling check, [2] chunks run by the loop
    int* fallen = c.take<int>(NS + 1);
    std::vector<int> rows32(NS + 1);
    for (int64_t s = 0; s <= NS; ++s)
        rows32[s] = static_cast<int>(spec.offsets[s]);
    std::vector<BatchState> init(NS);
    for (auto& st : init)
    {
        std::memset(&st, 0, sizeof(st));
        st.restart = 1;
    }
    PM_CUDA(cudaMemcpyAsync(sys_row, rows32.data(), (NS + 1) * sizeof(int), cudaMemcpyHostToDevice, stream));
    PM_CUDA(cudaMemcpyAsync(bs, init.data(), NS * sizeof(BatchState), cudaMemcpyHostToDevice, stream));
    PM_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(int), stream));
    PM_CUDA(cudaMemsetAsync(fallen, 0, (NS + 1) * sizeof(int), stream));
    batch_rows_kernel<<<grid_for(NS, 1, 4096), 128, 0, stream>>>(NS, sys_row, row_sys);
    PM_LAUNCH_CHECK();
    batch_check_kernel<<<grid_for(P, 1, 4096), 128, 0, stream>>>(P, ws->block_row_ptr, ws->block_col, row_sys,
                                                                  flags + 1);
    PM_LAUNCH_CHECK();
    int host_flags[4] = {0, 0, 0, 0};
    PM_CUDA(cudaMemcpyAsync(host_flags, flags, sizeof(host_flags), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaStreamSynchronize(stream));
    if (host_flags[1])
        fail(PM_INVALID_ARGUMENT, "batched Schur solve: a Schur block couples two systems");
    // the iterations run on the workspace's own stream (a caller's legacy default stream
    // cannot be captured), ordered after and before the caller's stream by events
    if (!ws->graph_stream)
    {
        PM_CUDA(cudaStreamCreateWithFlags(&ws->graph_stream, cudaStreamNonBlocking));
        for (auto& e : ws->graph_events)
            PM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const cudaStream_t caller = stream;
    PM_CUDA(cudaEventRecord(ws->graph_events[0], caller));
    stream = ws->graph_stream;
    PM_CUDA(cudaStreamWaitEvent(stream, ws->graph_events[0], 0));
    const unsigned rgrid = grid_for(P * 32, kVecBlock, 1 << 16);
    const unsigned pgrid = grid_for(P, 128, 1 << 16);
    const unsigned sgrid = grid_for(NS * 32, 128, 1 << 16);
    const double rel = o->relative_tolerance, abs_tol = o->absolute_tolerance;
    const int rule = o->tolerance_rule, maxit = o->max_iterations;
    auto start = [&]() {
        batch_spmv_kernel<M, 1><<<rgrid, kVecBlock, 0, stream>>>(P, ws->block_row_ptr, ws->block_col, S, x, q, row_dot,
                                                                 row_sys, bs);
        PM_LAUNCH_CHECK();
        batch_update_kernel<1><<<pgrid, 128, 0, stream>>>(P, row_sys, bs, x, pv, q, ws->rhs, r, z, ws->minv, row_rz,
                                                          row_rr);
        PM_LAUNCH_CHECK();
        PM_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), stream));
        batch_beta_kernel<1><<<sgrid, 128, 0, stream>>>(NS, sys_row, row_rz, row_rr, bs, maxit, learned ? window : 0,
                                                        rel, abs_tol, rule, flags);
        PM_LAUNCH_CHECK();
    };
    // The iterations run as one CUDA graph: a 'while' conditional node whose body holds kChunk
    // iterations of every active system and ends with batch_continue_kernel, which keeps the
    // loop going on the device while any system is active (no host check between chunks).
    constexpr int kChunk = 8;
    const int max_chunks = (maxit + kChunk - 1) / kChunk + 1;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
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
            fail(PM_CUDA_ERROR, std::string("batched Schur solve: conditional graph node: ") +
                                    cudaGetErrorString(added));
        }
        body = cp.conditional.phGraph_out[0];
    }
    PM_CUDA(cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kChunk; ++k)
    {
        // mixed precision: the iterations read the FP32 values and preconditioner blocks (FP64
        // vectors, dots, alpha and beta); every (re)start reads the FP64 ones
        if (mixed)
            batch_spmv_kernel<float, 0><<<rgrid, kVecBlock, 0, stream>>>(P, ws->block_row_ptr, ws->block_col, ws->S32,
                                                                         pv, q, row_dot, row_sys, bs);
        else
            batch_spmv_kernel<M, 0><<<rgrid, kVecBlock, 0, stream>>>(P, ws->block_row_ptr, ws->block_col, S, pv, q,
                                                                     row_dot, row_sys, bs);
        batch_alpha_kernel<<<sgrid, 128, 0, stream>>>(NS, sys_row, row_dot, bs);
        if (mixed)
            batch_update_kernel<0, float><<<pgrid, 128, 0, stream>>>(P, row_sys, bs, x, pv, q, ws->rhs, r, z,
                                                                     ws->minv32, row_rz, row_rr);
        else
            batch_update_kernel<0><<<pgrid, 128, 0, stream>>>(P, row_sys, bs, x, pv, q, ws->rhs, r, z, ws->minv, row_rz,
                                                              row_rr);
        cudaMemsetAsync(flags, 0, sizeof(int), stream);
        batch_beta_kernel<0><<<sgrid, 128, 0, stream>>>(NS, sys_row, row_rz, row_rr, bs, maxit,
                                                        learned ? window : 0, rel, abs_tol, rule, flags);
        batch_direction_kernel<<<grid_for(P * 6, 256, 1 << 16), 256, 0, stream>>>(P, row_sys, bs, z, pv);
        for (int l = 0; l < 5; ++l)
            count_launch();
    }
    batch_continue_kernel<<<1, 32, 0, stream>>>(handle, flags, flags + 2, max_chunks);
    count_launch();
    cudaGraph_t captured = nullptr;
    const cudaError_t cap = cudaStreamEndCapture(stream, &captured);
    if (cap != cudaSuccess)
    {
        cudaGraphDestroy(graph);
        fail(PM_CUDA_ERROR, std::string("batched Schur solve: graph capture failed: ") + cudaGetErrorString(cap));
    }
    {
        const cudaError_t inst = cudaGraphInstantiate(&exec, graph, 0);
        if (inst != cudaSuccess)
        {
            cudaGraphDestroy(graph);
            fail(PM_CUDA_ERROR, std::string("batched Schur solve: graph instantiation: ") + cudaGetErrorString(inst));
        }
    }
    int* host_count = reinterpret_cast<int*>(ws->host_state); // pinned; the state is not used here
    // one launch of the loop: it ends on the device once no system is active
    auto run = [&]() {
        PM_CUDA(cudaMemsetAsync(flags + 2, 0, sizeof(int), stream));
        PM_CUDA(cudaGraphLaunch(exec, stream));
    };
    int checks = 0;
    try
    {
        start();
        run();
        if (learned)
        {
            // systems whose learned PCG stagnated restart from their iterate with block Jacobi
            batch_fallback_kernel<M><<<pgrid, 128, 0, stream>>>(P, row_sys, bs, ws->diag_pos, S, ws->minv,
                                                                mixed ? ws->minv32 : nullptr, x);
            PM_LAUNCH_CHECK();
            batch_flag_restart_kernel<<<grid_for(NS, 128, 4096), 128, 0, stream>>>(NS, bs, fallen);
            PM_LAUNCH_CHECK();
            start();
            run();
        }
        // mixed precision: FP64 checks of the systems that converged on the FP32 operator; those
        // that miss their tolerance iterate on from the FP64 residual (iterative refinement)
        const int max_checks = o->max_refinements > 0 ? o->max_refinements : 8;
        while (mixed && checks < max_checks)
        {
            batch_verify_kernel<<<grid_for(NS, 128, 4096), 128, 0, stream>>>(NS, bs);
            PM_LAUNCH_CHECK();
            start();
            ++checks;
            PM_CUDA(cudaMemcpyAsync(host_count, flags, sizeof(int), cudaMemcpyDeviceToHost, stream));
            PM_CUDA(cudaEventRecord(ws->sync_event, stream));
            PM_CUDA(cudaEventSynchronize(ws->sync_event));
            if (*host_count == 0)
                break;
            run();
        }
    }
    catch (...)
    {
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        throw;
    }
    PM_CUDA(cudaGraphExecDestroy(exec));
    PM_CUDA(cudaGraphDestroy(graph));
    std::vector<BatchState> fin(NS);
    std::vector<int> fell(NS + 1);
    PM_CUDA(cudaMemcpyAsync(fin.data(), bs, NS * sizeof(BatchState), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaMemcpyAsync(fell.data(), fallen, (NS + 1) * sizeof(int), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaStreamSynchronize(stream));
    PM_CUDA(cudaEventRecord(ws->graph_events[1], stream));
    PM_CUDA(cudaStreamWaitEvent(caller, ws->graph_events[1], 0));
    double r0 = 0.0, r1 = 0.0;
    int all = 1, most = 0;
    for (int64_t s = 0; s < NS; ++s)
    {
        const BatchState& st = fin[s];
        pm_batched_system_report& out = spec.out[s];
        out.converged = st.converged;
        out.iterations = st.iterations;
        out.learned_fallback = fell[s];
        out.breakdown = st.breakdown;
        out.initial_residual_norm = std::sqrt(std::max(0.0, st.rr0));
        out.final_residual_norm = std::sqrt(std::max(0.0, st.rr));
        out.time_ms = st.converged ? double(st.t_done - st.t_start) * 1e-6 : -1.0;
        r0 += st.rr0;
        r1 += st.rr;
        all = all && st.converged;
        most = std::max(most, st.iterations);
    }
    rep->converged = all;
    rep->iterations = most;
    rep->mixed_precision_used = mixed ? 1 : 0;
    rep->refinement_steps = checks;
    rep->initial_residual_norm = std::sqrt(std::max(0.0, r0));
    rep->final_residual_norm = std::sqrt(std::max(0.0, r1));
    if (!all)
        std::snprintf(rep->message, sizeof(rep->message), "batched PCG: some systems did not converge");
}

// y = S x on the last assembled reduced system (6x6 block CSR, warp per block row)
template <typename T>
void schur_spmv(pm_schur_workspace* ws, cudaStream_t stream, const T* x, T* y)
{
    if (!ws || !ws->assembled || ws->P <= 0)
        fail(PM_LOGIC_ERROR, "Schur SpMV: the workspace holds no assembled system");
    const int vsize = ws->s32_only ? 4 : ws->value_size;
    if (vsize != static_cast<int>(sizeof(T)))
        fail(ws->s32_only ? PM_LOGIC_ERROR : PM_INVALID_ARGUMENT,
             ws->s32_only ? "Schur SpMV: the last solve assembled FP32 values; use the float SpMV"
                          : "Schur SpMV: scalar type differs from the assembled system");
    if (!x || !y || static_cast<const void*>(x) == static_cast<const void*>(y))
        fail(PM_INVALID_ARGUMENT, "Schur SpMV: vectors must be non-null and distinct");
    const void* values = ws->s32_only ? static_cast<const void*>(ws->S32) : ws->S;
    const int64_t P = ws->P;
    const int bp = static_cast<int>(ws->bp);
    const unsigned sgrid = grid_for(P * 32, kVecBlock, 1 << 16);
    if (bp == 6)
        bsr_spmv_kernel<T, T, 6><<<sgrid, kVecBlock, 0, stream>>>(P, bp, ws->block_row_ptr, ws->block_col,
                                                                  static_cast<const T*>(values), x, y);
    else
        bsr_spmv_kernel<T, T, 0><<<sgrid, kVecBlock, 0, stream>>>(P, bp, ws->block_row_ptr, ws->block_col,
                                                                  static_cast<const T*>(values), x, y);
    PM_LAUNCH_CHECK();
}

template <typename T>
void schur_solve(pm_schur_workspace* ws, cudaStream_t stream, const pm_normal_equations* ne, double damping,
                 const pm_schur_options* o, T* dp, T* dl, pm_schur_report* rep, const BatchSpec* batch = nullptr)
{
    if (!ws || !ne || !o || !rep)
        fail(PM_INVALID_ARGUMENT, "solveDampedSchurComplement: arguments must be non-null");
    std::memset(rep, 0, sizeof(*rep));
    rep->true_relative_residual = -1.0;
    const int64_t P = ne->P, L = ne->L, bp = ne->bp, bl = ne->bl;
    const int64_t n = P * bp, m = L * bl;
    if ((n > 0 && !dp) || (m > 0 && !dl) || (dp && static_cast<void*>(dp) == static_cast<void*>(dl)))
        fail(PM_INVALID_ARGUMENT, "solveDampedSchurComplement: output vectors must be non-null and distinct");
    if (!std::isfinite(damping) || damping < 0.0 || o->max_iterations <= 0 || !std::isfinite(o->relative_tolerance) ||
        o->relative_tolerance < 0.0 || !std::isfinite(o->absolute_tolerance) || o->absolute_tolerance < 0.0 ||
        !std::isfinite(o->minimum_diagonal) || o->minimum_diagonal <= 0.0)
        fail(PM_INVALID_ARGUMENT, "solveDampedSchurComplement: invalid solver options");
    if (ne->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "solveDampedSchurComplement: scalar type differs from the normal equations");
    if (bp > 16 || bl > 16)
        fail(PM_INVALID_ARGUMENT, "device Schur solver supports block sizes up to 16");
    if (o->linear_backend != PM_LINEAR_PCG && o->linear_backend != PM_LINEAR_DENSE)
        fail(PM_INVALID_ARGUMENT, "solveDampedSchurComplement: unknown linear backend");
    const bool dense = o->linear_backend == PM_LINEAR_DENSE;
    if (dense && batch)
        fail(PM_INVALID_ARGUMENT, "batched Schur solve: the dense backend solves single systems");
    if (dense && n > PM_DENSE_MAX_UNKNOWNS)
        fail(PM_INVALID_ARGUMENT, "dense Schur backend supports up to 16,384 primary unknowns");
    if (o->precision != PM_PRECISION_NATIVE && o->precision != PM_PRECISION_MIXED &&
        o->precision != PM_PRECISION_MIXED_FP32_ASSEMBLY)
        fail(PM_INVALID_ARGUMENT, "solveDampedSchurComplement: unknown precision mode");
    // FP32 assembly products (6x6 primary / 3x3 eliminated blocks, double normal equations)
    const bool mixed32 = o->precision == PM_PRECISION_MIXED_FP32_ASSEMBLY && sizeof(T) == 8 && !batch && !dense &&
                         bp == 6 && bl == 3;
    // batched solves: FP64 assembly with FP32 iterations for either mixed mode (their FP64 checks
    // read the assembled FP64 values)
    const bool mixed = (o->precision == PM_PRECISION_MIXED || mixed32 ||
                        (batch && o->precision == PM_PRECISION_MIXED_FP32_ASSEMBLY)) &&
                       sizeof(T) == 8 && !dense;
    if (batch)
    {
        if (sizeof(T) != 8 || bp != 6)
            fail(PM_INVALID_ARGUMENT, "batched Schur solve: double values and 6x6 primary blocks required");
        if (batch->systems <= 0 || !batch->offsets || !batch->out || batch->offsets[0] != 0 ||
            batch->offsets[batch->systems] != P)
            fail(PM_INVALID_ARGUMENT, "batched Schur solve: system offsets must run from 0 to the block-row count");
        for (int64_t s = 0; s < batch->systems; ++s)
            if (batch->offsets[s + 1] < batch->offsets[s])
                fail(PM_INVALID_ARGUMENT, "batched Schur solve: system offsets must be non-decreasing");
    }
    if (bp * bp > kRowThreads)
        fail(PM_INVALID_ARGUMENT, "device Schur solver supports primary block sizes up to 11");
    ws->numeric.bind(stream, "SchurComplementSolverWorkspace");
    if (!ws->host_state)
    {
        PM_CUDA(cudaMallocHost(reinterpret_cast<void**>(&ws->host_state), sizeof(SolveState)));
        PM_CUDA(cudaMallocHost(reinterpret_cast<void**>(&ws->host_status), sizeof(SchurStatus)));
        for (auto& e : ws->events)
            PM_CUDA(cudaEventCreate(&e));
        PM_CUDA(cudaEventCreateWithFlags(&ws->sync_event, cudaEventDisableTiming));
    }
    if (n > 0 && !o->use_initial_guess)
        PM_CUDA(cudaMemsetAsync(dp, 0, n * sizeof(T), stream));
    if (m > 0)
        PM_CUDA(cudaMemsetAsync(dl, 0, m * sizeof(T), stream));
    PM_CUDA(cudaEventRecord(ws->events[0], stream));
    // ---- pattern (checked first: the numeric layout depends on the block count)
    if (!ws->numeric.ptr || !ws->status)
    {
        ws->B = 0;
        ws->P = P;
        ws->L = L;
        ws->bp = bp;
        ws->bl = bl;
        numeric_layout<T>(ws, stream, mixed, mixed32);
    }
    const bool reused = ws->pattern_builds > 0 && topology_matches(ws, ne, stream);
    if (!reused)
        build_pattern(ws, ne, stream);
    ws->last_ne = ne;
    ws->last_version = ne->topology_version;
    ws->value_size = sizeof(T);
    rep->pattern_reused = reused;
    numeric_layout<T>(ws, stream, mixed, mixed32);
    PM_CUDA(cudaMemsetAsync(ws->state, 0, sizeof(SolveState), stream));
    PM_CUDA(cudaEventRecord(ws->events[1], stream));
    // ---- eliminated inverses
    status_reset_kernel<<<1, 1, 0, stream>>>(ws->status);
    PM_LAUNCH_CHECK();
    if (ne->observation_status.ptr)
        PM_CUDA(cudaMemcpyAsync(&ws->status->observation_bad, ne->observation_status.ptr, sizeof(long long),
                                cudaMemcpyDeviceToDevice, stream));
    if (L > 0 && ws->paired)
    {
        eliminated_factor3_kernel<T><<<grid_for(L, 128, 1 << 20), 128, 0, stream>>>(
            L, static_cast<const T*>(ne->eliminated_diagonal), static_cast<const T*>(ne->eliminated_gradient), damping,
            o->minimum_diagonal, ws->hinv, ws->status);
        PM_LAUNCH_CHECK();
    }
    else if (L > 0)
    {
        const unsigned grid = grid_for(L, 128, 1 << 20);
        if (bl == 3)
            eliminated_inverse_kernel<T, 3><<<grid, 128, 0, stream>>>(L, 3, static_cast<const T*>(ne->eliminated_diagonal),
                                                                      static_cast<const T*>(ne->eliminated_gradient),
                                                                      damping, o->minimum_diagonal, ws->hinv,
                                                                      ws->hstride, ws->y, ws->ystride, ws->status);
        else
            eliminated_inverse_kernel<T, 0><<<grid, 128, 0, stream>>>(L, static_cast<int>(bl),
                                                                      static_cast<const T*>(ne->eliminated_diagonal),
                                                                      static_cast<const T*>(ne->eliminated_gradient),
                                                                      damping, o->minimum_diagonal, ws->hinv,
                                                                      ws->hstride, ws->y, ws->ystride, ws->status);
        PM_LAUNCH_CHECK();
    }
    PM_CUDA(cudaEventRecord(ws->events[2], stream));
    // ---- assembly + preconditioner + RHS
    ws->s32_only = false;
    if (P > 0)
        launch_assembly<T>(ws, ne, damping, o->minimum_diagonal, stream, mixed32);
    if (mixed && P > 0)
    {
        if (!ws->s32_only)
        {
            convert_kernel<T, float><<<grid_for(ws->B * bp * bp, 256, 65535), 256, 0, stream>>>(
                static_cast<const T*>(ws->S), ws->S32, ws->B * bp * bp);
            PM_LAUNCH_CHECK();
        }
        convert_kernel<double, float><<<grid_for(P * bp * bp, 256, 4096), 256, 0, stream>>>(ws->minv, ws->minv32,
                                                                                            P * bp * bp);
        PM_LAUNCH_CHECK();
    }
    PM_CUDA(cudaEventRecord(ws->events[3], stream));
    // ---- status of the factorisations (one small read; the reference returns early here)
    PM_CUDA(cudaMemcpyAsync(ws->host_status, ws->status, sizeof(SchurStatus), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaEventRecord(ws->sync_event, stream));
    PM_CUDA(cudaEventSynchronize(ws->sync_event));
    ws->assembled = P > 0;
    auto timings = [&](int last) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ws->events[0], ws->events[1]);
        rep->pattern_ms = t;
        cudaEventElapsedTime(&t, ws->events[1], ws->events[2]);
        rep->eliminated_inverse_ms = t;
        cudaEventElapsedTime(&t, ws->events[2], ws->events[3]);
        rep->assembly_ms = t;
        if (last >= 4)
        {
            cudaEventElapsedTime(&t, ws->events[3], ws->events[4]);
            rep->solve_ms = t;
        }
        if (last >= 5)
        {
            cudaEventElapsedTime(&t, ws->events[4], ws->events[5]);
            rep->back_substitution_ms = t;
        }
        cudaEventElapsedTime(&t, ws->events[0], ws->events[last]);
        rep->total_ms = t;
    };
    {
        // the accumulation met a non-finite residual: evaluateHuberLoss throws on it before the
        // reference reaches the solve (robust_loss.h:31-35)
        const long long bad = ws->host_status->observation_bad;
        if (bad >= 0 && bad < ne->observation_count)
            fail(PM_INVALID_ARGUMENT, "evaluateHuberLoss: squared residual norm must be finite and non-negative "
                                      "(observation " + std::to_string(bad) + ")");
    }
    if (ws->host_status->eliminated_bad != kNone)
    {
        timings(3);
        std::snprintf(rep->message, sizeof(rep->message), "eliminated block is not positive definite");
        return;
    }
    if (ws->host_status->preconditioner_bad != kNone && !dense) // DenseCpu builds no preconditioner
    {
        timings(3);
        std::snprintf(rep->message, sizeof(rep->message), "Schur preconditioner block is not positive definite");
        return;
    }
    // ---- learned correction of the block-Jacobi blocks (6x6 only), with plain block Jacobi as
    // its fallback: when the network's blocks are unusable, or its PCG stagnates
    bool learned = o->learned && bp == 6 && n > 0;
    const int window = o->stagnation_window > 0 ? o->stagnation_window : 25;
    auto restore_block_jacobi = [&]() {
        diag_inverse_kernel<T, 6><<<grid_for(P, 64, 1 << 16), 64, 0, stream>>>(P, ws->diag_pos,
                                                                                static_cast<const T*>(ws->S),
                                                                                ws->minv, ws->status);
        PM_LAUNCH_CHECK();
        if (mixed)
        {
            convert_kernel<double, float><<<grid_for(P * 36, 256, 4096), 256, 0, stream>>>(ws->minv, ws->minv32,
                                                                                          P * 36);
            PM_LAUNCH_CHECK();
        }
    };
    // the network's outcome flags arrive in the pinned status with the next synchronisation; the
    // report takes them when the solve ends
    ws->host_status->learned_bad[0] = ws->host_status->learned_bad[1] = 0;
    bool learned_flags = false;
    if (learned)
    {
        try
        {
            mlp_apply(o->learned, schur_view(ws, mixed), stream, ws->host_status->learned_bad);
            rep->learned_used = 1;
            learned_flags = true;
        }
        catch (const Error&)
        {
            restore_block_jacobi();
            learned = false;
            rep->learned_fallback = 1;
        }
    }
    // after a synchronisation: a network whose blocks the device replaced by block Jacobi
    auto note_learned = [&]() {
        if (learned_flags && (ws->host_status->learned_bad[0] || ws->host_status->learned_bad[1]))
        {
            rep->learned_used = 0;
            rep->learned_fallback = 1;
        }
    };
    // ---- PCG
    double* area = vector_area(ws);
    // the FP64 matrix-free pass last run at the final step (mixed precision with FP32 values):
    // its t_l = Hll^-1 W_l^T dp is the back-substitution's product too
    bool t_at_step = false;
    SolveState st{};
    if (n == 0)
    {
        rep->converged = 1;
    }
    else if (dense)
    {
        // DenseCpu (block_schur_dense_solver.h:236-318): factor, solve, FP64 residual check
        Carver plan;
        plan.take<double>(n * n);
        plan.take<int>(1);
        ws->dense.ensure(plan.offset + 256, stream, "SchurComplementSolverWorkspace");
        Carver c;
        c.base = static_cast<char*>(ws->dense.ptr);
        double* A = c.take<double>(n * n);
        int* dstatus = c.take<int>(1);
        double* x64 = area;
        double* q64 = area + (n + 1);
        double* r64 = area + 2 * (n + 1);
        PM_CUDA(cudaMemcpyAsync(x64, ws->rhs, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        dense_schur_factor_solve<T>(stream, ws->P, static_cast<int>(bp), ws->block_row_ptr, ws->block_col,
                                    static_cast<const T*>(ws->S), A, x64, dstatus);
        int bad = 0;
        PM_CUDA(cudaMemcpyAsync(&bad, dstatus, sizeof(int), cudaMemcpyDeviceToHost, stream));
        PM_CUDA(cudaStreamSynchronize(stream));
        rep->iterations = 1;
        if (bad != 0)
        {
            std::snprintf(rep->message, sizeof(rep->message), "reduced Schur complement is not positive definite");
        }
        else
        {
            if constexpr (sizeof(T) == 8)
                PM_CUDA(cudaMemcpyAsync(dp, x64, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
            else
            {
                convert_kernel<double, float><<<grid_for(n, 256, 4096), 256, 0, stream>>>(x64, dp, n);
                PM_LAUNCH_CHECK();
            }
            double norm = 0.0, rhs_norm = 0.0;
            true_residual<T>(ws, stream, static_cast<const T*>(ws->S), x64, q64, r64, norm, rhs_norm);
            rep->initial_residual_norm = rhs_norm;
            rep->final_residual_norm = norm;
            rep->true_relative_residual = rhs_norm > 0 ? norm / rhs_norm : 0.0;
            const double eps = std::numeric_limits<T>::epsilon();
            const double tol = std::max(o->absolute_tolerance + o->relative_tolerance * rhs_norm,
                                        100.0 * eps * std::max(1.0, rhs_norm));
            rep->converged = std::isfinite(norm) && norm <= tol;
            if (!rep->converged)
                std::snprintf(rep->message, sizeof(rep->message), "dense Cholesky residual exceeds tolerance");
        }
    }
    else if (batch)
    {
        batched_pcg<T>(ws, stream, *batch, o, learned, mixed, window, reinterpret_cast<double*>(dp), rep);
        for (int64_t s = 0; s < batch->systems; ++s)
            rep->learned_fallback = rep->learned_fallback || batch->out[s].learned_fallback;
    }
    else if (!mixed)
    {
        st = block_pcg<T, T, double>(ws, stream, static_cast<const T*>(ws->S), ws->minv, ws->rhs, dp,
                                     o->relative_tolerance, o->absolute_tolerance, o->tolerance_rule, o->max_iterations,
                                     reinterpret_cast<T*>(area), learned ? window : 0);
        rep->initial_residual_norm = std::sqrt(std::max(0.0, st.initial_squared));
        if (learned)
        {
            rep->learned_iterations = st.iterations;
            if (!st.converged)
            {
                // plain block Jacobi from the iterate reached (from the start after a breakdown),
                // to the original tolerance
                restore_block_jacobi();
                rep->learned_fallback = 1;
                if (st.breakdown)
                    PM_CUDA(cudaMemsetAsync(dp, 0, n * sizeof(T), stream));
                const int used = st.iterations;
                const double tol = st.tolerance;
                st = block_pcg<T, T, double>(ws, stream, static_cast<const T*>(ws->S), ws->minv, ws->rhs, dp, 0.0,
                                             tol, 1, std::max(0, o->max_iterations - used), reinterpret_cast<T*>(area));
                st.iterations += used;
            }
        }
        rep->converged = st.converged;
        rep->iterations = st.iterations;
        rep->final_residual_norm = std::sqrt(std::max(0.0, st.residual_squared));
        if (st.breakdown)
            std::snprintf(rep->message, sizeof(rep->message), "reduced Schur complement is not positive definite");
    }
    else
    {
        // FP64 iterative refinement around FP32 inner PCG solves (FP64 dots / alpha / beta)
        double* x64 = reinterpret_cast<double*>(dp);
        double* q64 = area;
        double* r64 = area + (n + 1);
        float* d32 = reinterpret_cast<float*>(area + 2 * (n + 1));
        float* inner = d32 + 2 * (n + 1);
        double norm = 0.0, rhs_norm = 0.0;
        true_residual<T>(ws, stream, static_cast<const T*>(ws->S), x64, q64, r64, norm, rhs_norm,
                         !o->use_initial_guess);
        rep->initial_residual_norm = norm;
        const double target = o->tolerance_rule == 0 ? o->absolute_tolerance + o->relative_tolerance * norm
                                                     : std::max(o->absolute_tolerance, o->relative_tolerance * norm);
        const double inner_rel = o->inner_relative_tolerance > 0.0 ? o->inner_relative_tolerance : 1e-4;
        int total = 0;
        const int max_refinements = o->max_refinements > 0 ? o->max_refinements : 8;
        // the FP32 pass is guarded (block_schur_accelerated.cpp:160-195): a step that breaks
        // down or does not reduce the FP64 residual hands the solve to FP64 PCG from the iterate
        // reached, and mixed precision counts as used only when some FP32 step was kept
        bool kept_fp32 = false, fp64_fallback = false;
        for (int k = 0; k <= max_refinements; ++k)
        {
            rep->final_residual_norm = norm;
            if (norm <= target)
            {
                rep->converged = 1;
                break;
            }
            if (k == max_refinements || total >= o->max_iterations)
            {
                fp64_fallback = total < o->max_iterations;
                break;
            }
            // r64 holds b - S x; solve S32 d = r64 to inner_rel (or to the outer target)
            PM_CUDA(cudaMemsetAsync(d32, 0, n * sizeof(float), stream));
            st = block_pcg<float, float, float>(ws, stream, ws->S32, ws->minv32, r64, d32, inner_rel, 0.5 * target, 1,
                                                o->max_iterations - total, inner, learned ? window : 0);
            total += st.iterations;
            rep->refinement_steps += 1;
            if (learned)
            {
                rep->learned_iterations += st.iterations;
                if (!st.converged)
                {
                    // plain block Jacobi for the rest of the refinement; a step that broke down
                    // or stagnated is discarded
                    restore_block_jacobi();
                    rep->learned_fallback = 1;
                    learned = false;
                    if (st.breakdown || st.stagnated)
                        continue;
                }
            }
            if (st.breakdown)
            {
                fp64_fallback = true;
                break;
            }
            axpy_to_double_kernel<float><<<grid_for(n, 256, 4096), 256, 0, stream>>>(n, d32, x64);
            PM_LAUNCH_CHECK();
            const double before = norm;
            true_residual<T>(ws, stream, static_cast<const T*>(ws->S), x64, q64, r64, norm, rhs_norm);
            t_at_step = ws->s32_only && ws->paired && ws->hstride == 10;
            if (!(norm < before))
            {
                fp64_fallback = true;
                break;
            }
            kept_fp32 = true;
        }
        if (!rep->converged && fp64_fallback)
        {
            t_at_step = false; // the FP64 PCG below moves the step
            if (ws->s32_only)
            {
                // the FP64 PCG needs the FP64 values: assemble them now (the rare path)
                launch_assembly<T>(ws, ne, damping, o->minimum_diagonal, stream, false);
                if (learned)
                    restore_block_jacobi();
            }
            // FP64 block-Jacobi PCG from the iterate reached (from zero when it is not finite)
            if (!std::isfinite(norm))
                PM_CUDA(cudaMemsetAsync(x64, 0, n * sizeof(double), stream));
            const SolveState fs = block_pcg<T, T, double>(ws, stream, static_cast<const T*>(ws->S), ws->minv, ws->rhs,
                                                          dp, 0.0, target, 1, std::max(0, o->max_iterations - total),
                                                          reinterpret_cast<T*>(area));
            total += fs.iterations;
            if (fs.breakdown)
                std::snprintf(rep->message, sizeof(rep->message), "reduced Schur complement is not positive definite");
            true_residual<T>(ws, stream, static_cast<const T*>(ws->S), x64, area, area + (n + 1), norm, rhs_norm);
            rep->final_residual_norm = norm;
            rep->converged = fs.converged;
        }
        rep->iterations = total;
        rep->mixed_precision_used = kept_fp32 ? 1 : 0;
        rep->true_relative_residual = rhs_norm > 0 ? rep->final_residual_norm / rhs_norm : 0.0;
    }
    PM_CUDA(cudaEventRecord(ws->events[4], stream));
    if (rep->converged && o->check_true_residual && !mixed && n > 0 && sizeof(T) == 8)
    {
        double* q64 = area + 2 * (n + 1);
        double norm = 0.0, rhs_norm = 0.0;
        true_residual<T>(ws, stream, static_cast<const T*>(ws->S), reinterpret_cast<const double*>(dp), q64, nullptr,
                         norm, rhs_norm);
        rep->true_relative_residual = rhs_norm > 0 ? norm / rhs_norm : 0.0;
    }
    if (!rep->converged)
    {
        PM_CUDA(cudaEventRecord(ws->events[5], stream));
        PM_CUDA(cudaEventSynchronize(ws->events[5]));
        timings(5);
        note_learned();
        if (rep->message[0] == '\0')
            std::snprintf(rep->message, sizeof(rep->message), "PCG iteration limit reached");
        return;
    }
    // ---- back-substitution
    if (L > 0)
    {
        const unsigned grid = grid_for(L, 128, 1 << 20);
        if (t_at_step && bp == 6 && bl == 3 && sizeof(T) == 8)
            backsub_from_t_kernel<<<grid, 128, 0, stream>>>(L, ws->hinv, ws->mf_t, reinterpret_cast<double*>(dl));
        else if (bp == 6 && bl == 3)
            backsub_kernel<T, 6, 3><<<grid, 128, 0, stream>>>(L, 6, 3, ne->cross_offsets, ne->cross_primary,
                                                              static_cast<const T*>(ne->cross_values),
                                                              static_cast<const T*>(ne->eliminated_gradient), ws->hinv,
                                                              ws->hstride, ws->paired ? 1 : 0, dp, dl);
        else
            backsub_kernel<T, 0, 0><<<grid, 128, 0, stream>>>(L, static_cast<int>(bp), static_cast<int>(bl),
                                                              ne->cross_offsets, ne->cross_primary,
                                                              static_cast<const T*>(ne->cross_values),
                                                              static_cast<const T*>(ne->eliminated_gradient), ws->hinv,
                                                              ws->hstride, 0, dp, dl);
        PM_LAUNCH_CHECK();
    }
    PM_CUDA(cudaEventRecord(ws->events[5], stream));
    PM_CUDA(cudaEventSynchronize(ws->events[5]));
    timings(5);
    note_learned();
    std::snprintf(rep->message, sizeof(rep->message), "converged");
}

template <typename T, typename O>
void export_system(pm_schur_workspace* ws, cudaStream_t stream, int64_t* ro, int64_t* ci, O* values, double* rhs,
                   double* minv)
{
    if (!ws || !ws->assembled)
        fail(PM_LOGIC_ERROR, "CUDA Schur values have not been assembled");
    const int64_t bpp = ws->bp * ws->bp;
    if (ws->s32_only)
    {
        // FP32-assembled values (mixed precision with FP32 products), widened for a double export
        export_csr_kernel<float, O><<<grid_for(ws->B * bpp, 256, 65535), 256, 0, stream>>>(
            ws->B, static_cast<int>(ws->bp), ws->P, ws->block_row_ptr, ws->block_col, ws->block_row, ws->S32, ro, ci,
            values);
    }
    else
    {
        if (ws->value_size != static_cast<int>(sizeof(T)))
            fail(PM_INVALID_ARGUMENT, "export scalar type differs from the assembled system");
        export_csr_kernel<T, O><<<grid_for(ws->B * bpp, 256, 65535), 256, 0, stream>>>(
            ws->B, static_cast<int>(ws->bp), ws->P, ws->block_row_ptr, ws->block_col, ws->block_row,
            static_cast<const T*>(ws->S), ro, ci, values);
    }
    PM_LAUNCH_CHECK();
    if (rhs)
        PM_CUDA(cudaMemcpyAsync(rhs, ws->rhs, ws->P * ws->bp * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    if (minv)
        PM_CUDA(cudaMemcpyAsync(minv, ws->minv, ws->P * bpp * sizeof(double), cudaMemcpyDeviceToDevice, stream));
}

template <typename T>
void autotune_assembly(pm_schur_workspace* ws, cudaStream_t stream, const pm_normal_equations* ne, int repeats,
                       int* shape, double* best_ms, double* shape_ms)
{
    if (!ws || !ne || !shape || !best_ms)
        fail(PM_INVALID_ARGUMENT, "assembly autotune arguments must be non-null");
    if (repeats <= 0)
        fail(PM_INVALID_ARGUMENT, "assembly autotune needs at least one repeat");
    if (!ws->assembled || ws->last_ne != ne || ws->last_version != ne->topology_version)
        fail(PM_LOGIC_ERROR, "assembly autotune needs the workspace to have solved these normal equations");
    if (!ws->paired)
    {
        *shape = 0;
        *best_ms = -1.0;
        if (shape_ms)
            shape_ms[0] = -1.0;
        return;
    }
    const bool fp32 = ws->s32_only;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PM_CUDA(cudaEventCreate(&e0));
    PM_CUDA(cudaEventCreate(&e1));
    double best = 0.0;
    int chosen = -1;
    for (int k = 0; k < kUpperShapeCount; ++k)
    {
        ws->upper_shape = k;
        launch_assembly<T>(ws, ne, ws->damping, ws->min_diag, stream, fp32); // warm-up
        PM_CUDA(cudaEventRecord(e0, stream));
        for (int r = 0; r < repeats; ++r)
            launch_assembly<T>(ws, ne, ws->damping, ws->min_diag, stream, fp32);
        PM_CUDA(cudaEventRecord(e1, stream));
        PM_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        PM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const double mean = double(ms) / repeats;
        if (shape_ms)
            shape_ms[k] = mean;
        if (chosen < 0 || mean < best)
        {
            best = mean;
            chosen = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ws->upper_shape = chosen;
    ws->assembled = false; // values and their FP32 copies now belong to the last shape timed
    *shape = chosen;
    *best_ms = best;
}

} // namespace
} // namespace pm

extern "C" {

int pm_schur_workspace_create(pm_schur_workspace** out)
{
    return pm::guarded([&] {
        if (!out)
            pm::fail(PM_INVALID_ARGUMENT, "workspace output pointer is null");
        *out = new pm_schur_workspace();
    });
}

void pm_schur_workspace_destroy(pm_schur_workspace* ws) { delete ws; }

int pm_schur_workspace_close(pm_schur_workspace* ws)
{
    return pm::guarded([&] {
        if (!ws)
            pm::fail(PM_INVALID_ARGUMENT, "workspace is null");
        ws->drop_pcg_graphs(); // they hold pointers into the buffers released here
        ws->pattern.release();
        ws->numeric.release();
        ws->scratch.release();
        ws->pattern_builds = ws->pattern_builds; // the count survives, the cache does not
        ws->saved_offsets = nullptr;
        ws->status = nullptr;
        ws->assembled = false;
        ws->last_ne = nullptr;
        ws->P = -1;
    });
}

int64_t pm_schur_pattern_build_count(const pm_schur_workspace* ws) { return ws ? ws->pattern_builds : 0; }

int pm_schur_assembly_shape_count(void) { return pm::kUpperShapeCount; }

int pm_schur_assembly_shape_info(int shape, int* streams, int* split)
{
    return pm::guarded([&] {
        if (!streams || !split)
            pm::fail(PM_INVALID_ARGUMENT, "shape outputs must be non-null");
        if (shape < 0 || shape >= pm::kUpperShapeCount)
            pm::fail(PM_INVALID_ARGUMENT, "assembly shape out of range");
        *streams = pm::kUpperShapes[shape].streams;
        *split = pm::kUpperShapes[shape].split;
    });
}

int pm_schur_set_assembly_shape(pm_schur_workspace* ws, int shape)
{
    return pm::guarded([&] {
        if (!ws)
            pm::fail(PM_INVALID_ARGUMENT, "workspace is null");
        if (shape < 0 || shape >= pm::kUpperShapeCount)
            pm::fail(PM_INVALID_ARGUMENT, "assembly shape out of range");
        ws->upper_shape = shape;
    });
}

int pm_schur_assembly_shape(const pm_schur_workspace* ws, int* shape)
{
    return pm::guarded([&] {
        if (!ws || !shape)
            pm::fail(PM_INVALID_ARGUMENT, "workspace and shape output must be non-null");
        *shape = ws->upper_shape;
    });
}

int pm_schur_autotune_assembly(pm_schur_workspace* ws, pm_stream_t stream, const pm_normal_equations* ne, int repeats,
                               int* shape, double* best_ms, double* shape_ms)
{
    return pm::guarded([&] {
        if (!ws)
            pm::fail(PM_INVALID_ARGUMENT, "workspace is null");
        if (ws->value_size == 4)
            pm::autotune_assembly<float>(ws, static_cast<cudaStream_t>(stream), ne, repeats, shape, best_ms, shape_ms);
        else
            pm::autotune_assembly<double>(ws, static_cast<cudaStream_t>(stream), ne, repeats, shape, best_ms, shape_ms);
    });
}

int pm_schur_dims(const pm_schur_workspace* ws, int64_t* dimension, int64_t* nnz, int64_t* blocks)
{
    return pm::guarded([&] {
        if (!ws || !ws->assembled)
            pm::fail(PM_LOGIC_ERROR, "CUDA Schur values have not been assembled");
        if (dimension)
            *dimension = ws->P * ws->bp;
        if (nnz)
            *nnz = ws->B * ws->bp * ws->bp;
        if (blocks)
            *blocks = ws->B;
    });
}

int pm_schur_solve_f32(pm_schur_workspace* ws, pm_stream_t stream, const pm_normal_equations* ne, float damping,
                       const pm_schur_options* o, float* dp, float* dl, pm_schur_report* rep)
{
    return pm::guarded([&] { pm::schur_solve<float>(ws, stream, ne, damping, o, dp, dl, rep); });
}
int pm_schur_spmv_f32(pm_schur_workspace* ws, pm_stream_t stream, const float* x, float* y)
{
    return pm::guarded([&] { pm::schur_spmv<float>(ws, stream, x, y); });
}
int pm_schur_spmv_f64(pm_schur_workspace* ws, pm_stream_t stream, const double* x, double* y)
{
    return pm::guarded([&] { pm::schur_spmv<double>(ws, stream, x, y); });
}
int pm_schur_batched_solve_f64(pm_schur_workspace* ws, pm_stream_t stream, const pm_normal_equations* ne,
                               double damping, const pm_schur_options* o, int64_t systems,
                               const int64_t* system_primary_offsets, double* dp, double* dl, pm_schur_report* rep,
                               pm_batched_system_report* per_system)
{
    return pm::guarded([&] {
        pm::BatchSpec spec;
        spec.systems = systems;
        spec.offsets = system_primary_offsets;
        spec.out = per_system;
        pm::schur_solve<double>(ws, stream, ne, damping, o, dp, dl, rep, &spec);
    });
}
int pm_schur_solve_f64(pm_schur_workspace* ws, pm_stream_t stream, const pm_normal_equations* ne, double damping,
                       const pm_schur_options* o, double* dp, double* dl, pm_schur_report* rep)
{
    return pm::guarded([&] { pm::schur_solve<double>(ws, stream, ne, damping, o, dp, dl, rep); });
}

int pm_schur_export_f32(pm_schur_workspace* ws, pm_stream_t stream, int64_t* ro, int64_t* ci, float* v, double* rhs,
                        double* minv)
{
    return pm::guarded([&] { pm::export_system<float, float>(ws, stream, ro, ci, v, rhs, minv); });
}
int pm_schur_export_f64(pm_schur_workspace* ws, pm_stream_t stream, int64_t* ro, int64_t* ci, double* v, double* rhs,
                        double* minv)
{
    return pm::guarded([&] { pm::export_system<double, double>(ws, stream, ro, ci, v, rhs, minv); });
}

} // extern "C"
