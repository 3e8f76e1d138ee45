// Deterministic COO -> CSR for sm_100a.
//
// Contract (src/sparse/sparse_ops_cpu.cpp:24-134): the output equals a stable sort of the
// triplets by (row, col) followed by an in-order combination of duplicates (first value
// taken as is, the rest added one by one in input order).
//
// Design: instead of a device-wide radix sort of packed (row, col) keys, the triplets are
// bucketed by row with integer atomics (positions inside a row bucket are arbitrary), and
// every row segment is then sorted by the unique 64-bit key (col << 32 | source offset).
// Because the key contains the source offset, any correct sort yields the one order that
// the stable sort defines -- the result does not depend on scheduling.  Segments are sorted
// where they fit: <= 16 entries in registers (one thread per row), <= 2048 in shared memory
// (one CTA per row), longer rows by CTA-local merge passes in global memory.  Runs are then
// combined serially in key order, which reproduces the reference's left-to-right sums bit for
// bit.  Errors are recorded in a device status (lowest offending offset, as the reference's
// CooStatus, src/sparse/coo_to_csr.cu:22-29) and read by pm_coo_status().
#include "pm_common.cuh"

#include <climits>
#include <cmath>
#include <sstream>

namespace pm
{
namespace
{

constexpr unsigned long long kNoOffset = 0x7fffffffffffffffULL;
constexpr uint64_t kPadKey = ~uint64_t(0);
constexpr int kShortMax = 16;       // register-sorted segment length
constexpr int kLongCap = 2048;      // shared-memory segment length
constexpr int kLongThreads = 256;
constexpr int kMergeItems = kLongCap / kLongThreads;

struct CooStatus
{
    unsigned long long invalid_source;
    unsigned long long invalid_value;
    unsigned long long mismatch_actual;
    unsigned long long mismatch_expected;
    long long actual_nnz;
    int long_count;
    int pad;
};

// (key, value) of one scattered triplet: a single 16-byte store into its row bucket
template <typename T>
struct alignas(16) CooRec
{
    uint64_t key;
    T value;
};

__device__ __forceinline__ uint32_t key_col(uint64_t key) { return static_cast<uint32_t>(key >> 32); }
__device__ __forceinline__ unsigned source_of(uint64_t key) { return static_cast<unsigned>(key & 0xffffffffu); }

template <typename T>
__device__ __forceinline__ bool finite_value(T v)
{
    return isfinite(static_cast<double>(v));
}

__global__ void init_status_kernel(CooStatus* status)
{
    status->invalid_source = kNoOffset;
    status->invalid_value = kNoOffset;
    status->mismatch_actual = kNoOffset;
    status->mismatch_expected = kNoOffset;
    status->actual_nnz = 0;
    status->long_count = 0;
    status->pad = 0;
}

// 1) validate the indices and reserve a slot inside the row bucket (values are checked by the
// scatter, which reads them anyway)
template <typename T>
__global__ void __launch_bounds__(256) count_kernel(const int64_t* __restrict__ rows, const int64_t* __restrict__ cols,
                                                    int64_t count, int64_t row_count,
                                                    int64_t col_count, int* __restrict__ bucket_sizes,
                                                    int* __restrict__ slots, CooStatus* status)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const int64_t row = rows[i];
    const int64_t col = cols[i];
    if (row < 0 || row >= row_count || col < 0 || col >= col_count)
    {
        atomicMin(&status->invalid_source, static_cast<unsigned long long>(i));
        slots[i] = -1;
        return;
    }
    slots[i] = atomicAdd(&bucket_sizes[row], 1);
}

// 2) scatter (key, value) into the row buckets as one 16-byte record per triplet (the sorts
// below read the records and write the sorted keys and values)
template <typename T>
__global__ void __launch_bounds__(256) scatter_kernel(const int64_t* __restrict__ rows, const int64_t* __restrict__ cols,
                                                      const T* __restrict__ values, int64_t count,
                                                      const int* __restrict__ slots, const int* __restrict__ bucket_start,
                                                      CooRec<T>* __restrict__ recs, CooStatus* status)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    // every value is checked here, also those of triplets whose indices the count rejected
    const T value = values ? values[i] : T(0);
    if (!finite_value(value))
        atomicMin(&status->invalid_value, static_cast<unsigned long long>(i));
    const int slot = slots[i];
    if (slot < 0)
        return;
    const int pos = bucket_start[rows[i]] + slot;
    CooRec<T> r;
    r.key = (static_cast<uint64_t>(cols[i]) << 32) | static_cast<uint64_t>(i);
    r.value = value;
    recs[pos] = r;
}

// bitonic network over N register-resident (key, value) pairs; indices are compile-time
template <int N, typename T>
__device__ __forceinline__ void register_sort(uint64_t (&k)[N], T (&v)[N])
{
#pragma unroll
    for (int size = 2; size <= N; size <<= 1)
    {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1)
        {
#pragma unroll
            for (int i = 0; i < N; ++i)
            {
                const int j = i ^ stride;
                if (j > i)
                {
                    const bool ascending = (i & size) == 0;
                    const uint64_t a = k[i], b = k[j];
                    const bool swap = ascending ? (a > b) : (a < b);
                    const T va = v[i], vb = v[j];
                    k[i] = swap ? b : a;
                    k[j] = swap ? a : b;
                    v[i] = swap ? vb : va;
                    v[j] = swap ? va : vb;
                }
            }
        }
    }
}

// 3) short rows: one thread per row, sorted in registers; long rows are queued
// store == 0: only the unique count of every short row (the fill re-sorts them; keys and values
// of short rows are not written)
template <typename T>
__global__ void __launch_bounds__(128) sort_short_kernel(const int* __restrict__ bucket_start, int64_t row_count,
                                                         const CooRec<T>* __restrict__ recs,
                                                         uint64_t* __restrict__ keys, T* __restrict__ values,
                                                         int* __restrict__ unique_count, int* __restrict__ long_rows,
                                                         CooStatus* status, int store)
{
    const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= row_count)
        return;
    const int start = bucket_start[r];
    const int len = bucket_start[r + 1] - start;
    if (len > kShortMax)
    {
        long_rows[atomicAdd(&status->long_count, 1)] = static_cast<int>(r);
        return;
    }
    if (len <= 1)
    {
        if (len == 1 && store)
        {
            const CooRec<T> one = recs[start];
            keys[start] = one.key;
            values[start] = one.value;
        }
        unique_count[r] = len;
        return;
    }
    uint64_t k[kShortMax];
    T v[kShortMax];
#pragma unroll
    for (int q = 0; q < kShortMax; ++q)
    {
        if (q < len)
        {
            const CooRec<T> one = recs[start + q];
            k[q] = one.key;
            v[q] = one.value;
        }
        else
        {
            k[q] = kPadKey;
            v[q] = T(0);
        }
    }
    register_sort<kShortMax, T>(k, v);
    int unique = 0;
    uint32_t previous = 0;
#pragma unroll
    for (int q = 0; q < kShortMax; ++q)
    {
        if (q < len)
        {
            if (store)
            {
                keys[start + q] = k[q];
                values[start + q] = v[q];
            }
            const uint32_t col = key_col(k[q]);
            unique += (q == 0 || col != previous) ? 1 : 0;
            previous = col;
        }
    }
    unique_count[r] = unique;
}

// bitonic sort of m (power of two, <= kLongCap) staged pairs in shared memory
template <typename T>
__device__ void smem_bitonic(uint64_t* sk, T* sv, int m)
{
    for (int size = 2; size <= m; size <<= 1)
    {
        for (int stride = size >> 1; stride > 0; stride >>= 1)
        {
            for (int i = threadIdx.x; i < m; i += blockDim.x)
            {
                const int j = i ^ stride;
                if (j > i)
                {
                    const bool ascending = (i & size) == 0;
                    const uint64_t a = sk[i], b = sk[j];
                    if ((a > b) == ascending)
                    {
                        sk[i] = b;
                        sk[j] = a;
                        const T t = sv[i];
                        sv[i] = sv[j];
                        sv[j] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// merge-path split of diagonal d between sorted runs a[0..na) and b[0..nb) (unique keys)
__device__ __forceinline__ int merge_split(const uint64_t* a, int na, const uint64_t* b, int nb, int d)
{
    int lo = d > nb ? d - nb : 0;
    int hi = d < na ? d : na;
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < b[d - mid - 1])
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// 4) long rows: one CTA per row.  <= kLongCap entries are sorted in shared memory; longer
// rows are sorted chunk by chunk and merged pairwise in global memory (ping-pong with
// `spare`), all inside the CTA.  Also counts the distinct columns of the row.
template <typename T>
__global__ void __launch_bounds__(kLongThreads) sort_long_kernel(const int* __restrict__ bucket_start,
                                                                 const CooRec<T>* __restrict__ recs,
                                                                 uint64_t* __restrict__ keys, T* __restrict__ values,
                                                                 uint64_t* __restrict__ spare_keys,
                                                                 T* __restrict__ spare_values,
                                                                 int* __restrict__ unique_count,
                                                                 const int* __restrict__ long_rows,
                                                                 const CooStatus* __restrict__ status)
{
    __shared__ uint64_t sk[kLongCap];
    __shared__ T sv[kLongCap];
    __shared__ int reduce[kLongThreads / 32];
    const int long_count = status->long_count;
    for (int li = blockIdx.x; li < long_count; li += gridDim.x)
    {
        const int r = long_rows[li];
        const int start = bucket_start[r];
        const int len = bucket_start[r + 1] - start;
        uint64_t* rk = keys + start;
        T* rv = values + start;
        // chunk sorts
        for (int c0 = 0; c0 < len; c0 += kLongCap)
        {
            const int n = min(kLongCap, len - c0);
            int m = 1;
            while (m < n)
                m <<= 1;
            for (int i = threadIdx.x; i < m; i += blockDim.x)
            {
                if (i < n)
                {
                    const CooRec<T> one = recs[start + c0 + i];
                    sk[i] = one.key;
                    sv[i] = one.value;
                }
                else
                {
                    sk[i] = kPadKey;
                    sv[i] = T(0);
                }
            }
            __syncthreads();
            smem_bitonic<T>(sk, sv, m);
            for (int i = threadIdx.x; i < n; i += blockDim.x)
            {
                rk[c0 + i] = sk[i];
                rv[c0 + i] = sv[i];
            }
            __syncthreads();
        }
        // merge passes (only rows longer than one chunk)
        uint64_t* src_k = rk;
        T* src_v = rv;
        uint64_t* dst_k = spare_keys + start;
        T* dst_v = spare_values + start;
        for (int width = kLongCap; width < len; width <<= 1)
        {
            for (int tile = 0; tile < len; tile += kLongCap)
            {
                const int pair = tile / (2 * width) * (2 * width);
                const int na = min(width, len - pair);
                const int nb = max(0, min(width, len - pair - width));
                const uint64_t* a = src_k + pair;
                const uint64_t* b = a + na;
                const T* av = src_v + pair;
                const T* bv = av + na;
                int d = tile - pair + threadIdx.x * kMergeItems;
                if (d < na + nb)
                {
                    int i = merge_split(a, na, b, nb, d);
                    int j = d - i;
                    for (int q = 0; q < kMergeItems && d + q < na + nb; ++q)
                    {
                        const bool take_a = i < na && (j >= nb || a[i] < b[j]);
                        dst_k[pair + d + q] = take_a ? a[i] : b[j];
                        dst_v[pair + d + q] = take_a ? av[i] : bv[j];
                        i += take_a ? 1 : 0;
                        j += take_a ? 0 : 1;
                    }
                }
            }
            __syncthreads();
            uint64_t* tk = src_k;
            src_k = dst_k;
            dst_k = tk;
            T* tv = src_v;
            src_v = dst_v;
            dst_v = tv;
        }
        if (src_k != rk)
        {
            for (int i = threadIdx.x; i < len; i += blockDim.x)
            {
                rk[i] = src_k[i];
                rv[i] = src_v[i];
            }
            __syncthreads();
        }
        // distinct columns
        int local = 0;
        for (int i = threadIdx.x; i < len; i += blockDim.x)
            local += (i == 0 || key_col(rk[i]) != key_col(rk[i - 1])) ? 1 : 0;
        const int unique = block_sum<int, kLongThreads>(local, reduce);
        if (threadIdx.x == 0)
            unique_count[r] = unique;
        __syncthreads();
    }
}

__global__ void finish_status_kernel(const int64_t* __restrict__ row_offsets, int64_t row_count, int64_t expected,
                                     CooStatus* status)
{
    const long long actual = row_offsets[row_count];
    status->actual_nnz = actual;
    if (expected >= 0 && actual != expected)
    {
        status->mismatch_actual = static_cast<unsigned long long>(actual);
        status->mismatch_expected = static_cast<unsigned long long>(expected);
    }
}

template <typename T>
__device__ __forceinline__ void emit(int64_t at, int64_t capacity, uint32_t col, T sum, int64_t* col_out, T* val_out)
{
    if (at < capacity)
    {
        col_out[at] = col;
        val_out[at] = sum;
    }
}

// 5) combine runs of short rows: one thread per row, serial left-to-right sums
template <typename T>
__global__ void __launch_bounds__(128) write_short_kernel(const int* __restrict__ bucket_start, int64_t row_count,
                                                          const uint64_t* __restrict__ keys,
                                                          const T* __restrict__ values,
                                                          const int64_t* __restrict__ row_offsets, int64_t capacity,
                                                          int64_t* __restrict__ col_out, T* __restrict__ val_out,
                                                          CooStatus* status)
{
    const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= row_count)
        return;
    const int start = bucket_start[r];
    const int len = bucket_start[r + 1] - start;
    if (len > kShortMax || len == 0)
        return;
    int64_t at = row_offsets[r];
    uint32_t col = key_col(keys[start]);
    T sum = values[start];
    for (int q = 1; q < len; ++q)
    {
        const uint64_t key = keys[start + q];
        const uint32_t c = key_col(key);
        if (c != col)
        {
            emit(at++, capacity, col, sum, col_out, val_out);
            col = c;
            sum = values[start + q];
        }
        else
        {
            sum += values[start + q];
            if (!finite_value(sum))
                atomicMin(&status->invalid_value, static_cast<unsigned long long>(source_of(key)));
        }
    }
    emit(at, capacity, col, sum, col_out, val_out);
}

// 5') the same from the scattered records: every short row is sorted in registers again (the
// count phase kept only its unique count) and its runs combined serially in key order
template <typename T>
__global__ void __launch_bounds__(128) write_short_resort_kernel(const int* __restrict__ bucket_start,
                                                                 int64_t row_count, const CooRec<T>* __restrict__ recs,
                                                                 const int64_t* __restrict__ row_offsets,
                                                                 int64_t capacity, int64_t* __restrict__ col_out,
                                                                 T* __restrict__ val_out, CooStatus* status)
{
    const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= row_count)
        return;
    const int start = bucket_start[r];
    const int len = bucket_start[r + 1] - start;
    if (len > kShortMax || len == 0)
        return;
    int64_t at = row_offsets[r];
    if (len == 1)
    {
        const CooRec<T> one = recs[start];
        emit(at, capacity, key_col(one.key), one.value, col_out, val_out);
        return;
    }
    uint64_t k[kShortMax];
    T v[kShortMax];
#pragma unroll
    for (int q = 0; q < kShortMax; ++q)
    {
        if (q < len)
        {
            const CooRec<T> one = recs[start + q];
            k[q] = one.key;
            v[q] = one.value;
        }
        else
        {
            k[q] = kPadKey;
            v[q] = T(0);
        }
    }
    register_sort<kShortMax, T>(k, v);
    uint32_t col = key_col(k[0]);
    T sum = v[0];
#pragma unroll
    for (int q = 1; q < kShortMax; ++q)
    {
        if (q < len)
        {
            const uint32_t c = key_col(k[q]);
            if (c != col)
            {
                emit(at++, capacity, col, sum, col_out, val_out);
                col = c;
                sum = v[q];
            }
            else
            {
                sum += v[q];
                if (!finite_value(sum))
                    atomicMin(&status->invalid_value, static_cast<unsigned long long>(source_of(k[q])));
            }
        }
    }
    emit(at, capacity, col, sum, col_out, val_out);
}

// 6) combine runs of long rows: one CTA per row; run heads found by a block scan, each
// head thread sums its run serially in key order
template <typename T>
__global__ void __launch_bounds__(kLongThreads) write_long_kernel(const int* __restrict__ bucket_start,
                                                                  const uint64_t* __restrict__ keys,
                                                                  const T* __restrict__ values,
                                                                  const int64_t* __restrict__ row_offsets,
                                                                  int64_t capacity, int64_t* __restrict__ col_out,
                                                                  T* __restrict__ val_out,
                                                                  const int* __restrict__ long_rows,
                                                                  CooStatus* status)
{
    __shared__ int scan[kLongThreads / 32 + 1];
    const int long_count = status->long_count;
    for (int li = blockIdx.x; li < long_count; li += gridDim.x)
    {
        const int r = long_rows[li];
        const int start = bucket_start[r];
        const int len = bucket_start[r + 1] - start;
        const uint64_t* rk = keys + start;
        const T* rv = values + start;
        int64_t carry = row_offsets[r];
        for (int c0 = 0; c0 < len; c0 += kLongThreads)
        {
            const int i = c0 + threadIdx.x;
            const bool head = i < len && (i == 0 || key_col(rk[i]) != key_col(rk[i - 1]));
            int chunk_heads = 0;
            const int ordinal = block_exclusive_scan<int, kLongThreads>(head ? 1 : 0, scan, chunk_heads);
            if (head)
            {
                const uint32_t col = key_col(rk[i]);
                T sum = rv[i];
                for (int q = i + 1; q < len && key_col(rk[q]) == col; ++q)
                {
                    sum += rv[q];
                    if (!finite_value(sum))
                        atomicMin(&status->invalid_value, static_cast<unsigned long long>(source_of(rk[q])));
                }
                emit(carry + ordinal, capacity, col, sum, col_out, val_out);
            }
            carry += chunk_heads;
        }
    }
}

} // namespace
} // namespace pm

// =========================================================================== workspace
struct pm_sparse_workspace
{
    pm::DeviceBuffer buffer;
    bool status_pending = false; // a conversion was enqueued and not yet checked
    bool prepared = false;       // count phase enqueued; fill may follow
    int value_size = 0;
    int64_t rows = 0, cols = 0, count = 0;
    // carved device arrays of the last prepared conversion
    pm::CooStatus* status = nullptr;
    int* bucket_sizes = nullptr;
    int* bucket_start = nullptr;
    int* slots = nullptr;
    uint64_t* keys = nullptr;
    void* values = nullptr;
    uint64_t* spare_keys = nullptr;
    void* spare_values = nullptr;
    int* unique_count = nullptr;
    int* long_rows = nullptr;
    int64_t* row_offsets = nullptr;
    void* scan_scratch = nullptr;
    void* recs = nullptr;             // the scattered (key, value) records of the last conversion
    bool short_rows_kept = true;      // short rows' sorted keys / values are stored (else re-sorted at fill)
};

namespace pm
{

void require_values(int64_t count, const void* values)
{
    if (count > 0 && !values)
        fail(PM_INVALID_ARGUMENT, "cooToCsr GPU triplet pointers must be non-null");
}

void check_metadata(int64_t rows, int64_t cols, int64_t count)
{
    if (rows < 0 || cols < 0 || count < 0)
        fail(PM_INVALID_ARGUMENT, "cooToCsr GPU dimensions must be non-negative");
    if (count > INT_MAX || rows >= INT_MAX || cols > int64_t(UINT32_MAX))
        fail(PM_OVERFLOW_ERROR, "cooToCsr GPU dimensions exceed the supported packed-key range");
}

template <typename T>
void coo_prepare(pm_sparse_workspace* ws, cudaStream_t stream, int64_t rows, int64_t cols, int64_t count,
                 const int64_t* row_indices, const int64_t* col_indices, const T* values, bool keep_sorted)
{
    if (!ws)
        fail(PM_INVALID_ARGUMENT, "cooToCsr GPU workspace is null");
    check_metadata(rows, cols, count);
    if (ws->status_pending)
        fail(PM_LOGIC_ERROR, "SparseOpsWorkspace status must be checked before another COO conversion");
    if (count > 0 && (!row_indices || !col_indices))
        fail(PM_INVALID_ARGUMENT, "cooToCsr GPU triplet pointers must be non-null");
    const size_t scan_bytes = scan_scratch_bytes(rows + 1, sizeof(int64_t)) + scan_scratch_bytes(rows + 1, sizeof(int));
    const size_t n = static_cast<size_t>(count > 0 ? count : 1);
    const size_t R = static_cast<size_t>(rows + 1);
    Carver plan;
    plan.take<CooStatus>(1);
    plan.take<int>(R);
    plan.take<int>(R + 1);
    plan.take<int>(n);
    plan.take<uint64_t>(n);
    plan.take<T>(n);
    plan.take<uint64_t>(n);
    plan.take<T>(n);
    plan.take<int>(R);
    plan.take<int>(R);
    plan.take<int64_t>(R + 1);
    plan.take<char>(scan_bytes);
    plan.take<CooRec<T>>(n);
    ws->buffer.ensure(plan.offset + 256, stream, "SparseOpsWorkspace");
    Carver carve;
    carve.base = static_cast<char*>(ws->buffer.ptr);
    ws->status = carve.take<CooStatus>(1);
    ws->bucket_sizes = carve.take<int>(R);
    ws->bucket_start = carve.take<int>(R + 1);
    ws->slots = carve.take<int>(n);
    ws->keys = carve.take<uint64_t>(n);
    ws->values = carve.take<T>(n);
    ws->spare_keys = carve.take<uint64_t>(n);
    ws->spare_values = carve.take<T>(n);
    ws->unique_count = carve.take<int>(R);
    ws->long_rows = carve.take<int>(R);
    ws->row_offsets = carve.take<int64_t>(R + 1);
    ws->scan_scratch = carve.take<char>(scan_bytes);
    CooRec<T>* recs = carve.take<CooRec<T>>(n);
    ws->recs = recs;
    ws->short_rows_kept = keep_sorted;
    ws->rows = rows;
    ws->cols = cols;
    ws->count = count;
    ws->value_size = sizeof(T);

    init_status_kernel<<<1, 1, 0, stream>>>(ws->status);
    PM_LAUNCH_CHECK();
    ws->status_pending = true;
    ws->prepared = true;
    if (count == 0)
    {
        // empty input: every bucket is empty (callers read bucket_start / unique_count)
        PM_CUDA(cudaMemsetAsync(ws->bucket_start, 0, (rows + 1) * sizeof(int), stream));
        PM_CUDA(cudaMemsetAsync(ws->unique_count, 0, (rows > 0 ? rows : 1) * sizeof(int), stream));
        PM_CUDA(cudaMemsetAsync(ws->row_offsets, 0, (rows + 1) * sizeof(int64_t), stream));
        finish_status_kernel<<<1, 1, 0, stream>>>(ws->row_offsets, rows, -1, ws->status);
        PM_LAUNCH_CHECK();
        return;
    }
    T* sorted_values = static_cast<T*>(ws->values);
    PM_CUDA(cudaMemsetAsync(ws->bucket_sizes, 0, rows * sizeof(int), stream));
    count_kernel<T><<<grid_for(count, 256), 256, 0, stream>>>(row_indices, col_indices, count, rows, cols,
                                                              ws->bucket_sizes, ws->slots, ws->status);
    PM_LAUNCH_CHECK();
    exclusive_scan<int, int>(ws->bucket_sizes, ws->bucket_start, rows, ws->scan_scratch, stream);
    scatter_kernel<T><<<grid_for(count, 256), 256, 0, stream>>>(row_indices, col_indices, values, count, ws->slots,
                                                                ws->bucket_start, recs, ws->status);
    PM_LAUNCH_CHECK();
    if (rows > 0)
    {
        sort_short_kernel<T><<<grid_for(rows, 128), 128, 0, stream>>>(ws->bucket_start, rows, recs, ws->keys,
                                                                      sorted_values, ws->unique_count, ws->long_rows,
                                                                      ws->status, keep_sorted ? 1 : 0);
        PM_LAUNCH_CHECK();
        sort_long_kernel<T><<<2 * sm_count(), kLongThreads, 0, stream>>>(
            ws->bucket_start, recs, ws->keys, sorted_values, ws->spare_keys, static_cast<T*>(ws->spare_values),
            ws->unique_count, ws->long_rows, ws->status);
        PM_LAUNCH_CHECK();
    }
    exclusive_scan<int, int64_t>(ws->unique_count, ws->row_offsets, rows, ws->scan_scratch, stream);
    finish_status_kernel<<<1, 1, 0, stream>>>(ws->row_offsets, rows, -1, ws->status);
    PM_LAUNCH_CHECK();
}

template void coo_prepare<float>(pm_sparse_workspace*, cudaStream_t, int64_t, int64_t, int64_t, const int64_t*,
                                  const int64_t*, const float*, bool);
template void coo_prepare<double>(pm_sparse_workspace*, cudaStream_t, int64_t, int64_t, int64_t, const int64_t*,
                                   const int64_t*, const double*, bool);

CooView coo_view(const pm_sparse_workspace* ws)
{
    return CooView{ws->rows, ws->count, ws->bucket_start, ws->keys, ws->unique_count, ws->row_offsets};
}

// Host read of the status of an internal (sort-only) use of the workspace.
int64_t coo_internal_status(pm_sparse_workspace* ws, cudaStream_t stream, const char* operation)
{
    CooStatus status{};
    PM_CUDA(cudaMemcpyAsync(&status, ws->status, sizeof(status), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaStreamSynchronize(stream));
    ws->status_pending = false;
    if (status.invalid_source != kNoOffset)
    {
        std::ostringstream m;
        m << operation << ": block index out of range at entry " << status.invalid_source;
        fail(PM_OUT_OF_RANGE, m.str());
    }
    return status.actual_nnz;
}

namespace
{

template <typename T>
void coo_fill(pm_sparse_workspace* ws, cudaStream_t stream, int64_t nnz, int64_t* row_offsets, int64_t* col_out,
              T* val_out, bool async_api)
{
    if (!ws || !ws->prepared)
        fail(PM_LOGIC_ERROR, "cooToCsr fill requires a preceding count on the same workspace");
    if (ws->value_size != static_cast<int>(sizeof(T)))
        fail(PM_INVALID_ARGUMENT, "cooToCsr fill scalar type differs from the counted triplets");
    ws->buffer.bind(stream, "SparseOpsWorkspace");
    if (nnz < 0)
        fail(PM_INVALID_ARGUMENT, "cooToCsr output nnz must be non-negative");
    if (ws->count == 0 && nnz != 0)
        fail(PM_RUNTIME_ERROR, "cooToCsrAsync empty input requires output nnz=0");
    if (!row_offsets || (nnz > 0 && (!col_out || !val_out)))
        fail(PM_INVALID_ARGUMENT, "cooToCsr output pointers must be non-null");
    finish_status_kernel<<<1, 1, 0, stream>>>(ws->row_offsets, ws->rows, nnz, ws->status);
    PM_LAUNCH_CHECK();
    PM_CUDA(cudaMemcpyAsync(row_offsets, ws->row_offsets, (ws->rows + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice,
                            stream));
    if (ws->count == 0 || ws->rows == 0)
        return;
    const T* sorted_values = static_cast<const T*>(ws->values);
    if (ws->short_rows_kept)
        write_short_kernel<T><<<grid_for(ws->rows, 128), 128, 0, stream>>>(ws->bucket_start, ws->rows, ws->keys,
                                                                           sorted_values, ws->row_offsets, nnz,
                                                                           col_out, val_out, ws->status);
    else
        write_short_resort_kernel<T><<<grid_for(ws->rows, 128), 128, 0, stream>>>(
            ws->bucket_start, ws->rows, static_cast<const CooRec<T>*>(ws->recs), ws->row_offsets, nnz, col_out,
            val_out, ws->status);
    PM_LAUNCH_CHECK();
    write_long_kernel<T><<<2 * sm_count(), kLongThreads, 0, stream>>>(ws->bucket_start, ws->keys, sorted_values,
                                                                      ws->row_offsets, nnz, col_out, val_out,
                                                                      ws->long_rows, ws->status);
    PM_LAUNCH_CHECK();
    (void)async_api;
}

template <typename T>
int coo_async(pm_sparse_workspace* ws, cudaStream_t stream, int64_t rows, int64_t cols, int64_t count,
              const int64_t* ri, const int64_t* ci, const T* v, int64_t nnz, int64_t* ro, int64_t* co, T* vo)
{
    return guarded([&] {
        if (v && vo && static_cast<const void*>(v) == static_cast<const void*>(vo))
            fail(PM_INVALID_ARGUMENT, "cooToCsrAsync values and output must not alias");
        if (count == 0 && nnz != 0)
        {
            check_metadata(rows, cols, count);
            fail(PM_RUNTIME_ERROR, "cooToCsrAsync empty input requires output nnz=0");
        }
        require_values(count, v);
        coo_prepare<T>(ws, stream, rows, cols, count, ri, ci, v, false);
        coo_fill<T>(ws, stream, nnz, ro, co, vo, true);
    });
}

} // namespace
} // namespace pm

extern "C" {

int pm_sparse_workspace_create(pm_sparse_workspace** out)
{
    return pm::guarded([&] {
        if (!out)
            pm::fail(PM_INVALID_ARGUMENT, "workspace output pointer is null");
        *out = new pm_sparse_workspace();
    });
}

void pm_sparse_workspace_destroy(pm_sparse_workspace* ws)
{
    if (ws)
    {
        ws->buffer.release();
        delete ws;
    }
}

int pm_sparse_workspace_close(pm_sparse_workspace* ws)
{
    return pm::guarded([&] {
        if (!ws)
            pm::fail(PM_INVALID_ARGUMENT, "workspace is null");
        ws->buffer.release();
        ws->status_pending = false;
        ws->prepared = false;
    });
}

size_t pm_sparse_workspace_capacity(const pm_sparse_workspace* ws) { return ws ? ws->buffer.bytes : 0; }

int pm_coo_to_csr_count_f32(pm_sparse_workspace* ws, pm_stream_t stream, int64_t rows, int64_t cols, int64_t count,
                            const int64_t* ri, const int64_t* ci, const float* v)
{
    return pm::guarded([&] {
        pm::require_values(count, v);
        pm::coo_prepare<float>(ws, stream, rows, cols, count, ri, ci, v, false);
    });
}
int pm_coo_to_csr_count_f64(pm_sparse_workspace* ws, pm_stream_t stream, int64_t rows, int64_t cols, int64_t count,
                            const int64_t* ri, const int64_t* ci, const double* v)
{
    return pm::guarded([&] {
        pm::require_values(count, v);
        pm::coo_prepare<double>(ws, stream, rows, cols, count, ri, ci, v, false);
    });
}
int pm_coo_to_csr_fill_f32(pm_sparse_workspace* ws, pm_stream_t stream, int64_t nnz, int64_t* ro, int64_t* co,
                           float* vo)
{
    return pm::guarded([&] {
        if (ws)
            ws->status_pending = true;
        pm::coo_fill<float>(ws, stream, nnz, ro, co, vo, false);
    });
}
int pm_coo_to_csr_fill_f64(pm_sparse_workspace* ws, pm_stream_t stream, int64_t nnz, int64_t* ro, int64_t* co,
                           double* vo)
{
    return pm::guarded([&] {
        if (ws)
            ws->status_pending = true;
        pm::coo_fill<double>(ws, stream, nnz, ro, co, vo, false);
    });
}
int pm_coo_to_csr_async_f32(pm_sparse_workspace* ws, pm_stream_t stream, int64_t rows, int64_t cols, int64_t count,
                            const int64_t* ri, const int64_t* ci, const float* v, int64_t nnz, int64_t* ro,
                            int64_t* co, float* vo)
{
    return pm::coo_async<float>(ws, stream, rows, cols, count, ri, ci, v, nnz, ro, co, vo);
}
int pm_coo_to_csr_async_f64(pm_sparse_workspace* ws, pm_stream_t stream, int64_t rows, int64_t cols, int64_t count,
                            const int64_t* ri, const int64_t* ci, const double* v, int64_t nnz, int64_t* ro,
                            int64_t* co, double* vo)
{
    return pm::coo_async<double>(ws, stream, rows, cols, count, ri, ci, v, nnz, ro, co, vo);
}

int pm_coo_status(pm_sparse_workspace* ws, const char* operation, int64_t* nnz_out)
{
    return pm::guarded([&] {
        if (!ws)
            pm::fail(PM_INVALID_ARGUMENT, "workspace is null");
        const char* name = operation ? operation : "cooToCsrAsync";
        if (nnz_out)
            *nnz_out = 0;
        if (!ws->buffer.bound || !ws->status)
            return;
        const cudaError_t query = cudaStreamQuery(ws->buffer.stream);
        if (query == cudaErrorNotReady)
            pm::fail(PM_LOGIC_ERROR, "SparseOpsWorkspace::checkStatus requires stream synchronization first");
        PM_CUDA(query);
        pm::CooStatus status{};
        PM_CUDA(cudaMemcpy(&status, ws->status, sizeof(status), cudaMemcpyDeviceToHost));
        ws->status_pending = false;
        if (nnz_out)
            *nnz_out = status.actual_nnz;
        if (status.invalid_source != pm::kNoOffset)
        {
            std::ostringstream m;
            m << name << ": coordinate out of range at source offset " << status.invalid_source;
            ws->prepared = false;
            pm::fail(PM_OUT_OF_RANGE, m.str());
        }
        if (status.invalid_value != pm::kNoOffset)
        {
            std::ostringstream m;
            m << name << ": non-finite value at source offset " << status.invalid_value;
            ws->prepared = false;
            pm::fail(PM_INVALID_ARGUMENT, m.str());
        }
        if (status.mismatch_actual != pm::kNoOffset)
        {
            std::ostringstream m;
            m << name << ": output nnz is " << status.mismatch_expected << ", but duplicate-combined nnz is "
              << status.mismatch_actual;
            pm::fail(PM_RUNTIME_ERROR, m.str());
        }
    });
}

} // extern "C"

// =========================================================================== allocation-free variant
// COO -> CSR for callers that must not allocate device memory at call time: for example a
// host application that hands the library a fixed device-memory budget at start-up and owns
// every allocation after that, or a latency-critical loop where a cudaMalloc could block or
// fail in the middle of a run.  The scratch of the conversion (row buckets, sort keys, scan
// partials, status) lives in one file-scope device array of kStaticScratchBytes, created when
// the library's device code is loaded on a GPU and held by every GPU that loads the library
// until the process exits.  Inputs are limited to kStaticMaxTriplets triplets and
// kStaticMaxRows rows so that the scratch always fits.  All calls share the array: calls
// that overlap on one GPU, from any stream or host thread, race on it, so serialise them;
// each device has its own copy.  Each call clears what must start at zero.
namespace pm
{
namespace
{
constexpr int64_t kStaticMaxTriplets = 65536;
constexpr int64_t kStaticMaxRows = 65536;
constexpr size_t kStaticScratchBytes = size_t(8) << 20;
} // namespace
} // namespace pm

static __device__ __align__(256) unsigned char g_static_coo_scratch[pm::kStaticScratchBytes];

namespace pm
{
namespace
{

// Device address of g_static_coo_scratch in the current device's context.  The host-side name
// of the array is only a stand-in, so the address is looked up with that device current.  It
// is looked up on every call (cudaGetSymbolAddress allocates nothing): a cached address would
// outlive a cudaDeviceReset, after which the module is loaded again and the array may move.
// The first call on a device loads the library's device code there; issue that first call
// before any stream capture.
void* static_scratch_address()
{
    void* address = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&address, g_static_coo_scratch);
    if (rc != cudaSuccess || !address)
        fail(PM_CUDA_ERROR, std::string("cudaGetSymbolAddress(static COO scratch): ") + cudaGetErrorString(rc));
    return address;
}

// Bytes coo_prepare carves for (rows, count) triplets of type T (same layout, same order).
template <typename T>
size_t static_plan_bytes(int64_t rows, int64_t count)
{
    const size_t scan_bytes = scan_scratch_bytes(rows + 1, sizeof(int64_t)) + scan_scratch_bytes(rows + 1, sizeof(int));
    const size_t n = static_cast<size_t>(count > 0 ? count : 1);
    const size_t R = static_cast<size_t>(rows + 1);
    Carver plan;
    plan.take<CooStatus>(1);
    plan.take<int>(R);
    plan.take<int>(R + 1);
    plan.take<int>(n);
    plan.take<uint64_t>(n);
    plan.take<T>(n);
    plan.take<uint64_t>(n);
    plan.take<T>(n);
    plan.take<int>(R);
    plan.take<int>(R);
    plan.take<int64_t>(R + 1);
    plan.take<char>(scan_bytes);
    plan.take<CooRec<T>>(n);
    return plan.offset + 256;
}

template <typename T>
void coo_static(cudaStream_t stream, int64_t rows, int64_t cols, int64_t count, const int64_t* ri, const int64_t* ci,
                const T* v, int64_t capacity, int64_t* ro, int64_t* co, T* vo, int64_t* nnz_out)
{
    check_metadata(rows, cols, count);
    if (count > kStaticMaxTriplets || rows > kStaticMaxRows)
    {
        std::ostringstream m;
        m << "cooToCsr (static scratch): at most " << kStaticMaxTriplets << " triplets and " << kStaticMaxRows
          << " rows are supported, got " << count << " triplets and " << rows << " rows";
        fail(PM_INVALID_ARGUMENT, m.str());
    }
    require_values(count, v);
    if (capacity < 0 || !ro || (capacity > 0 && (!co || !vo)))
        fail(PM_INVALID_ARGUMENT, "cooToCsr (static scratch): output pointers must be non-null");
    if (v && vo && static_cast<const void*>(v) == static_cast<const void*>(vo))
        fail(PM_INVALID_ARGUMENT, "cooToCsrAsync values and output must not alias");
    const size_t need = static_plan_bytes<T>(rows, count);
    if (need > kStaticScratchBytes)
        fail(PM_INVALID_ARGUMENT, "cooToCsr (static scratch): scratch plan exceeds the static array");
    // a workspace whose storage is the static array: it never grows, so nothing is allocated
    void* const base = static_scratch_address();
    pm_sparse_workspace ws;
    ws.buffer.ptr = base;
    ws.buffer.bytes = kStaticScratchBytes;
    coo_prepare<T>(&ws, stream, rows, cols, count, ri, ci, v, false);
    PM_CUDA(cudaStreamSynchronize(stream));
    int64_t nnz = 0;
    int status = pm_coo_status(&ws, "cooToCsr", &nnz);
    if (status != PM_OK)
        throw Error(status, pm_last_error());
    if (nnz > capacity)
    {
        std::ostringstream m;
        m << "cooToCsr (static scratch): output capacity " << capacity << " is below the duplicate-combined nnz "
          << nnz;
        fail(PM_RUNTIME_ERROR, m.str());
    }
    ws.status_pending = true;
    coo_fill<T>(&ws, stream, nnz, ro, co, vo, false);
    PM_CUDA(cudaStreamSynchronize(stream));
    if (ws.buffer.ptr != base)
        fail(PM_RUNTIME_ERROR, "cooToCsr (static scratch): scratch storage changed unexpectedly");
    status = pm_coo_status(&ws, "cooToCsr", nullptr);
    if (status != PM_OK)
        throw Error(status, pm_last_error());
    if (nnz_out)
        *nnz_out = nnz;
}

} // namespace
} // namespace pm

extern "C" {

int pm_coo_to_csr_static_f32(pm_stream_t stream, int64_t rows, int64_t cols, int64_t count, const int64_t* ri,
                             const int64_t* ci, const float* v, int64_t capacity, int64_t* ro, int64_t* co, float* vo,
                             int64_t* nnz_out)
{
    return pm::guarded([&] { pm::coo_static<float>(stream, rows, cols, count, ri, ci, v, capacity, ro, co, vo, nnz_out); });
}

int pm_coo_to_csr_static_f64(pm_stream_t stream, int64_t rows, int64_t cols, int64_t count, const int64_t* ri,
                             const int64_t* ci, const double* v, int64_t capacity, int64_t* ro, int64_t* co, double* vo,
                             int64_t* nnz_out)
{
    return pm::guarded([&] { pm::coo_static<double>(stream, rows, cols, count, ri, ci, v, capacity, ro, co, vo, nnz_out); });
}

} // extern "C"
