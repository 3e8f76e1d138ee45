// Last-error storage, device queries and the device-wide exclusive scan.
#include "pm_common.cuh"

#include <atomic>
#include <mutex>
#include <vector>
#include <cstdio>

namespace pm
{

namespace
{
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
}

void set_last_error(const std::string& message) { g_last_error = message; }

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int sm_count()
{
    static int counts[64] = {0};
    int device = 0;
    PM_CUDA(cudaGetDevice(&device));
    if (device < 64 && counts[device] > 0)
        return counts[device];
    int value = 0;
    PM_CUDA(cudaDeviceGetAttribute(&value, cudaDevAttrMultiProcessorCount, device));
    if (device < 64)
        counts[device] = value;
    return value;
}

// ------------------------------------------------------------------ scan
// Tile = 256 threads x 8 items.  Level k reduces its tiles into the (k+1)-th level input;
// the top level fits one tile.  Every tile sum is formed in a fixed order, so the result
// does not depend on scheduling.
namespace
{
constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int64_t kScanTile = int64_t(kScanBlock) * kScanItems;

template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kScanBlock) scan_reduce_kernel(const Tin* in, int64_t n, Tout* tile_sums)
{
    __shared__ Tout smem[kScanBlock / 32];
    const int64_t base = int64_t(blockIdx.x) * kScanTile;
    Tout sum = Tout(0);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        const int64_t i = base + int64_t(k) * kScanBlock + threadIdx.x;
        if (i < n)
            sum += static_cast<Tout>(in[i]);
    }
    sum = block_sum<Tout, kScanBlock>(sum, smem);
    if (threadIdx.x == 0)
        tile_sums[blockIdx.x] = sum;
}

// out has n+1 entries: out[i] = offset + sum(in[0..i)), out[n] = grand total.
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kScanBlock) scan_apply_kernel(const Tin* in, int64_t n, const Tout* tile_offsets,
                                                                Tout* out)
{
    __shared__ Tout staged[kScanTile];
    __shared__ Tout smem[kScanBlock / 32 + 1];
    const int64_t base = int64_t(blockIdx.x) * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        const int64_t i = base + int64_t(k) * kScanBlock + threadIdx.x;
        staged[k * kScanBlock + threadIdx.x] = i < n ? static_cast<Tout>(in[i]) : Tout(0);
    }
    __syncthreads();
    Tout local[kScanItems];
    Tout thread_sum = Tout(0);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        local[k] = staged[threadIdx.x * kScanItems + k];
        thread_sum += local[k];
    }
    Tout total;
    Tout running = block_exclusive_scan<Tout, kScanBlock>(thread_sum, smem, total);
    running += tile_offsets ? tile_offsets[blockIdx.x] : Tout(0);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        staged[threadIdx.x * kScanItems + k] = running;
        running += local[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        const int64_t i = base + int64_t(k) * kScanBlock + threadIdx.x;
        if (i < n)
            out[i] = staged[k * kScanBlock + threadIdx.x];
    }
    // the last tile writes the grand total into out[n]
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanBlock - 1)
        out[n] = running;
}

int64_t tiles_of(int64_t n) { return n <= 0 ? 1 : (n + kScanTile - 1) / kScanTile; }

} // namespace

size_t scan_scratch_bytes(int64_t n, size_t out_size)
{
    size_t bytes = 0;
    int64_t level = n;
    while (true)
    {
        const int64_t tiles = tiles_of(level);
        if (tiles <= 1)
            break;
        bytes += size_t(2 * tiles + 1) * out_size + 256;
        level = tiles;
    }
    return bytes + 256;
}

template <typename Tin, typename Tout>
void exclusive_scan(const Tin* in, Tout* out, int64_t n, void* scratch, cudaStream_t stream)
{
    const int64_t tiles = tiles_of(n);
    if (tiles <= 1)
    {
        scan_apply_kernel<Tin, Tout><<<1, kScanBlock, 0, stream>>>(in, n, nullptr, out);
        PM_LAUNCH_CHECK();
        return;
    }
    Tout* sums = static_cast<Tout*>(scratch);
    Tout* offsets = sums + tiles;
    char* rest = reinterpret_cast<char*>(offsets + tiles + 1);
    rest = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(rest) + 255) & ~uintptr_t(255));
    scan_reduce_kernel<Tin, Tout><<<static_cast<unsigned>(tiles), kScanBlock, 0, stream>>>(in, n, sums);
    PM_LAUNCH_CHECK();
    exclusive_scan<Tout, Tout>(sums, offsets, tiles, rest, stream);
    scan_apply_kernel<Tin, Tout><<<static_cast<unsigned>(tiles), kScanBlock, 0, stream>>>(in, n, offsets, out);
    PM_LAUNCH_CHECK();
}

template void exclusive_scan<int32_t, int32_t>(const int32_t*, int32_t*, int64_t, void*, cudaStream_t);
template void exclusive_scan<int32_t, int64_t>(const int32_t*, int64_t*, int64_t, void*, cudaStream_t);
template void exclusive_scan<int64_t, int64_t>(const int64_t*, int64_t*, int64_t, void*, cudaStream_t);

} // namespace pm

extern "C" const char* pm_last_error(void) { return pm::g_last_error.c_str(); }
extern "C" int pm_version(void) { return 1; }
extern "C" long long pm_kernel_launches(void) { return pm::g_launches.load(std::memory_order_relaxed); }

// Device memory and copies for callers that do not link the CUDA runtime themselves.
extern "C" int pm_device_malloc(size_t bytes, void** out)
{
    return pm::guarded([&] {
        if (!out)
            pm::fail(PM_INVALID_ARGUMENT, "pm_device_malloc: null output");
        *out = nullptr;
        if (bytes > 0)
            PM_CUDA(cudaMalloc(out, bytes));
    });
}

extern "C" int pm_device_free(void* ptr)
{
    return pm::guarded([&] {
        if (ptr)
            PM_CUDA(cudaFree(ptr));
    });
}

extern "C" int pm_copy_to_device(void* dst_d, const void* src_h, size_t bytes, pm_stream_t stream)
{
    return pm::guarded([&] {
        if (bytes == 0)
            return;
        if (!dst_d || !src_h)
            pm::fail(PM_INVALID_ARGUMENT, "pm_copy_to_device: null pointer");
        PM_CUDA(cudaMemcpyAsync(dst_d, src_h, bytes, cudaMemcpyHostToDevice, stream));
        PM_CUDA(cudaStreamSynchronize(stream));
    });
}

extern "C" int pm_copy_to_host(void* dst_h, const void* src_d, size_t bytes, pm_stream_t stream)
{
    return pm::guarded([&] {
        if (bytes == 0)
            return;
        if (!dst_h || !src_d)
            pm::fail(PM_INVALID_ARGUMENT, "pm_copy_to_host: null pointer");
        PM_CUDA(cudaMemcpyAsync(dst_h, src_d, bytes, cudaMemcpyDeviceToHost, stream));
        PM_CUDA(cudaStreamSynchronize(stream));
    });
}

extern "C" int pm_stream_synchronize(pm_stream_t stream)
{
    return pm::guarded([&] { PM_CUDA(cudaStreamSynchronize(stream)); });
}

extern "C" int pm_device_name(char* out, int capacity)
{
    return pm::guarded([&] {
        if (!out || capacity <= 0)
            pm::fail(PM_INVALID_ARGUMENT, "pm_device_name: null or empty output");
        int device = 0;
        PM_CUDA(cudaGetDevice(&device));
        cudaDeviceProp prop{};
        PM_CUDA(cudaGetDeviceProperties(&prop, device));
        std::snprintf(out, static_cast<size_t>(capacity), "%s", prop.name);
    });
}
