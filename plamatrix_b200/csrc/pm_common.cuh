// Shared host/device plumbing for the plamatrix_b200 kernels: status codes that mirror the
// reference's exception classes, CUDA error checks, a stream-ordered growable device
// buffer, block/warp reductions and a device-wide exclusive scan.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>

#include "plamatrix_b200.h"

namespace pm
{

struct Error : std::exception
{
    int status;
    std::string message;
    Error(int s, std::string m) : status(s), message(std::move(m)) {}
    const char* what() const noexcept override { return message.c_str(); }
};

[[noreturn]] inline void fail(int status, const std::string& message) { throw Error(status, message); }

void set_last_error(const std::string& message);

inline void check_cuda(cudaError_t error, const char* what)
{
    if (error != cudaSuccess)
    {
        fail(PM_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(error));
    }
}

// Every kernel launch is followed by PM_LAUNCH_CHECK(), which also counts it
// (pm_kernel_launches(): the number of kernels this library has launched).
void count_launch();

#define PM_CUDA(call) ::pm::check_cuda((call), #call)
#define PM_LAUNCH_CHECK() (::pm::count_launch(), ::pm::check_cuda(cudaGetLastError(), "kernel launch"))

// Runs `fn`, converting exceptions into PM_* status codes and the thread's last-error text.
template <typename Fn>
int guarded(Fn&& fn) noexcept
{
    try
    {
        fn();
        return PM_OK;
    }
    catch (const Error& e)
    {
        set_last_error(e.message);
        return e.status;
    }
    catch (const std::bad_alloc&)
    {
        set_last_error("host allocation failed");
        return PM_RUNTIME_ERROR;
    }
    catch (const std::exception& e)
    {
        set_last_error(e.what());
        return PM_RUNTIME_ERROR;
    }
    catch (...)
    {
        set_last_error("unknown error");
        return PM_RUNTIME_ERROR;
    }
}

// Stream-ordered, grow-only device allocation bound to the stream that first used it
// (the ownership rule of the reference's SparseOpsWorkspace / IterativeSolverWorkspace).
struct DeviceBuffer
{
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    bool bound = false;

    void bind(cudaStream_t s, const char* owner)
    {
        if (bound && stream != s)
        {
            fail(PM_LOGIC_ERROR, std::string(owner) + " cannot be reused on a different stream; close it first");
        }
        stream = s;
        bound = true;
    }

    void ensure(size_t required, cudaStream_t s, const char* owner)
    {
        bind(s, owner);
        if (required <= bytes)
        {
            return;
        }
        void* replacement = nullptr;
        PM_CUDA(cudaMallocAsync(&replacement, required, s));
        if (ptr)
        {
            PM_CUDA(cudaFreeAsync(ptr, s));
        }
        ptr = replacement;
        bytes = required;
    }

    void release() noexcept
    {
        if (ptr)
        {
            cudaFreeAsync(ptr, stream);
        }
        ptr = nullptr;
        bytes = 0;
        bound = false;
    }
};

// Carves aligned sub-arrays out of one allocation.
struct Carver
{
    size_t offset = 0;
    char* base = nullptr;
    template <typename T>
    T* take(size_t count, size_t align = 256)
    {
        offset = (offset + align - 1) / align * align;
        T* out = reinterpret_cast<T*>(base + offset);
        offset += count * sizeof(T);
        return out;
    }
};

inline unsigned grid_for(int64_t items, int per_block, int64_t cap = 1 << 30)
{
    int64_t blocks = (items + per_block - 1) / per_block;
    if (blocks < 1)
        blocks = 1;
    if (blocks > cap)
        blocks = cap;
    return static_cast<unsigned>(blocks);
}

int sm_count();

// ------------------------------------------------------------------ device helpers
template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum (fixed shuffle tree, warps combined in index order).
template <typename T, int BLOCK>
__device__ __forceinline__ T block_sum(T v, T* smem /* BLOCK/32 */)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        smem[warp] = v;
    __syncthreads();
    T total = T(0);
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int w = 0; w < BLOCK / 32; ++w)
            total += smem[w];
        smem[0] = total;
    }
    __syncthreads();
    total = smem[0];
    __syncthreads();
    return total;
}

// Exclusive block scan of one value per thread; returns the block total in `total`.
template <typename T, int BLOCK>
__device__ __forceinline__ T block_exclusive_scan(T v, T* smem /* BLOCK/32 + 1 */, T& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inclusive = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        T n = __shfl_up_sync(0xffffffffu, inclusive, o);
        if (lane >= o)
            inclusive += n;
    }
    if (lane == 31)
        smem[warp] = inclusive;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        T running = T(0);
#pragma unroll
        for (int w = 0; w < BLOCK / 32; ++w)
        {
            T t = smem[w];
            smem[w] = running;
            running += t;
        }
        smem[BLOCK / 32] = running;
    }
    __syncthreads();
    T result = smem[warp] + inclusive - v;
    total = smem[BLOCK / 32];
    __syncthreads();
    return result;
}

// ------------------------------------------------------------------ device-wide scan
// Exclusive scan of n inputs into n+1 outputs (out[n] = total), reduce-then-scan over
// tiles; deterministic; no inter-block waiting.
size_t scan_scratch_bytes(int64_t n, size_t out_size);

template <typename Tin, typename Tout>
void exclusive_scan(const Tin* in, Tout* out, int64_t n, void* scratch, cudaStream_t stream);

// ------------------------------------------------------------------ bucket sort (COO machinery)
// Entries (rows[i], cols[i]) are bucketed by row and each bucket is sorted by the unique key
// (col << 32 | i); `unique_count[row]` counts distinct cols and `row_offsets` is its scan.
struct CooView
{
    int64_t rows;
    int64_t count;
    const int* bucket_start;   // rows + 1
    const uint64_t* keys;      // count, bucket-major, ascending inside a bucket
    const int* unique_count;   // rows
    const int64_t* row_offsets; // rows + 1 (scan of unique_count)
};

// keep_sorted: store every row's sorted keys and values (coo_view readers need them); a
// conversion that only fills a CSR passes false, and its fill re-sorts the short rows
template <typename T>
void coo_prepare(pm_sparse_workspace* ws, cudaStream_t stream, int64_t rows, int64_t cols, int64_t count,
                 const int64_t* row_indices, const int64_t* col_indices, const T* values, bool keep_sorted = true);
CooView coo_view(const pm_sparse_workspace* ws);
int64_t coo_internal_status(pm_sparse_workspace* ws, cudaStream_t stream, const char* operation);

// ---------------------------------------------------------------- async copies
__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// cp.async (LSU path) of 16 / 8 bytes global -> shared; completion tracked per thread in
// commit groups
__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

} // namespace pm
