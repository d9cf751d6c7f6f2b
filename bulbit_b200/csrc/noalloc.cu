// bbg_intersect_static: closest-hit queries that allocate no memory.
//
// Some callers cannot allocate device memory at the point where they trace
// rays: a plugin host that forbids allocation after start-up, a real-time
// loop that must not block in the allocator, or a process whose device memory
// is already claimed by another framework's caching allocator (a cudaMalloc
// there fails or stalls). bbg_intersect with host buffers stages rays and hits
// through buffers the library allocates on first use, so it cannot serve them.
// This entry point stages through one fixed array instead, defined below at
// file scope in device memory; it exists for the lifetime of the process on
// every device that loads the library, so it is kept small (kStaticMaxRays
// rays per call, about 12 MiB).

#include "accel.cuh"

#include <algorithm>
#include <mutex>

namespace bbg
{
namespace
{

constexpr int64_t kStaticMaxRays = int64_t(1) << 18; // 262,144 rays per call
constexpr size_t kCounterBytes = 256;                 // work counter, padded to keep the rays aligned
constexpr size_t kRayBytes = size_t(kStaticMaxRays) * sizeof(bbg_ray);
constexpr size_t kHitBytes = size_t(kStaticMaxRays) * sizeof(bbg_hit);
constexpr size_t kScratchBytes = kCounterBytes + kRayBytes + kHitBytes;

// Shared by every call of bbg_intersect_static in the process: the work
// counter, the staged rays, then the staged hits.
static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

constexpr int kBlock = 128;

struct StaticSrc
{
    const float4* rays;
    float4* hits;

    __device__ __forceinline__ void Load(int32_t i, RayQ* q, float* t_min, float* t_max) const
    {
        float4 r0 = rays[2 * i];
        float4 r1 = rays[2 * i + 1];
        *q = MakeRayQ(V3{ r0.x, r0.y, r0.z }, V3{ r0.w, r1.x, r1.y });
        *t_min = r1.z;
        *t_max = r1.w;
    }
    __device__ __forceinline__ void Store(int32_t i, const TraceResult& r) const
    {
        hits[i] = make_float4(__int_as_float(r.prim), r.t, r.u, r.v);
    }
};

template <bool WIDE>
__global__ void __launch_bounds__(kBlock) StaticTraceKernel(AccelView a, const float4* rays, int32_t n, float4* hits,
                                                            int32_t* next)
{
    StaticSrc src{ rays, hits };
    if constexpr (WIDE)
    {
        TracePersistentWide<false>(a, n, next, src);
    }
    else
    {
        TracePersistent<false>(a, n, next, src);
    }
}

__global__ void __launch_bounds__(kBlock) StaticTraceReferenceKernel(AccelView a, const float4* rays, int32_t n,
                                                                     float4* hits)
{
    StaticSrc src{ rays, hits };
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        RayQ q;
        float t_min, t_max;
        src.Load(i, &q, &t_min, &t_max);
        src.Store(i, TraceReference<false, false>(a, q, t_min, t_max));
    }
}

// Device address of g_static_scratch per device ordinal. The host-side name
// of a __device__ array is not a device address: it is looked up with
// cudaGetSymbolAddress, with that device current, once per device at set-up
// (ReserveStaticScratch, called when an accel is created), and cached. The
// library does not support cudaDeviceReset while any of its handles exist:
// their device memory, and this cached address, do not survive it.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

} // namespace

bbg_status ReserveStaticScratch()
{
    int dev = 0;
    BBG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_ptr[dev])
    {
        return BBG_OK;
    }
    // Kernel modules load lazily: looking the symbol up loads this file's
    // module on the current device and so creates the array now.
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
    {
        return Fail(BBG_ERR_CUDA, "bbg_intersect_static set-up: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(e));
    }
    unsigned char* base = static_cast<unsigned char*>(p);
    // Load the query's kernels too, and launch each once over zero rays, so
    // that the device's code and per-thread local-memory reservations for
    // them are made here rather than in the query's first call.
    cudaFuncAttributes attr;
    BBG_CUDA(cudaFuncGetAttributes(&attr, StaticTraceKernel<true>));
    BBG_CUDA(cudaFuncGetAttributes(&attr, StaticTraceKernel<false>));
    BBG_CUDA(cudaFuncGetAttributes(&attr, StaticTraceReferenceKernel));
    int32_t* counter = reinterpret_cast<int32_t*>(base);
    const AccelView none{};
    StaticTraceKernel<true><<<1, kBlock>>>(none, nullptr, 0, nullptr, counter);
    StaticTraceKernel<false><<<1, kBlock>>>(none, nullptr, 0, nullptr, counter);
    StaticTraceReferenceKernel<<<1, kBlock>>>(none, nullptr, 0, nullptr);
    BBG_CUDA(cudaGetLastError());
    BBG_CUDA(cudaDeviceSynchronize());
    g_scratch_ptr[dev] = base;
    return BBG_OK;
}

namespace
{

// The cached address for the current device; set-up on a device that has
// none yet (an accel created there always has made it).
bbg_status ScratchAddress(unsigned char** out)
{
    int dev = 0;
    BBG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "bbg_intersect_static: device ordinal %d out of range", dev);
    }
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (g_scratch_ptr[dev])
        {
            *out = g_scratch_ptr[dev];
            return BBG_OK;
        }
    }
    BBG_TRY(ReserveStaticScratch());
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    *out = g_scratch_ptr[dev];
    return BBG_OK;
}

} // namespace
} // namespace bbg

using namespace bbg;

extern "C" bbg_status bbg_intersect_static(bbg_accel* accel, const bbg_ray* rays, int64_t n, bbg_hit* hits)
{
    if (!accel || n < 0 || (n > 0 && (!rays || !hits)))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_intersect_static: bad argument");
    }
    if (n > kStaticMaxRays)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_intersect_static: %lld rays exceed the fixed limit of %lld per call",
                    (long long)n, (long long)kStaticMaxRays);
    }
    if (n == 0)
    {
        return BBG_OK;
    }
    if (accel->n_prims == 0)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "closest-hit query on an accel with no primitives");
    }
    // The accel's device, whatever device the caller has current (restored
    // on return).
    DeviceScope ds(accel->device);
    unsigned char* base = nullptr;
    BBG_TRY(ScratchAddress(&base));
    int32_t* counter = reinterpret_cast<int32_t*>(base);
    float4* d_rays = reinterpret_cast<float4*>(base + kCounterBytes);
    float4* d_hits = reinterpret_cast<float4*>(base + kCounterBytes + kRayBytes);

    cudaStream_t st = accel->stream;
    BBG_CUDA(cudaMemcpyAsync(d_rays, rays, size_t(n) * sizeof(bbg_ray), cudaMemcpyHostToDevice, st));
    const int32_t m = int32_t(n);
    // A counting accel traverses in the reference's node order in
    // bbg_intersect; so does this query (so results agree on exact ties too),
    // but it records no counts.
    if (accel->ordered && !accel->counting)
    {
        // The array keeps the previous call's contents: the counter must start at 0.
        BBG_CUDA(cudaMemsetAsync(counter, 0, sizeof(int32_t), st));
        auto k = accel->wide8_active() ? StaticTraceKernel<true> : StaticTraceKernel<false>;
        int grid = PersistentGrid(reinterpret_cast<const void*>(k), kBlock);
        grid = int(std::min<int64_t>(grid, (n + kBlock - 1) / kBlock));
        k<<<grid, kBlock, 0, st>>>(accel->view(), d_rays, m, d_hits, counter);
    }
    else
    {
        int grid = PersistentGrid(reinterpret_cast<const void*>(StaticTraceReferenceKernel), kBlock);
        grid = int(std::min<int64_t>(grid, (n + kBlock - 1) / kBlock));
        StaticTraceReferenceKernel<<<grid, kBlock, 0, st>>>(accel->view(), d_rays, m, d_hits);
    }
    BBG_CUDA(cudaGetLastError());
    BBG_CUDA(cudaMemcpyAsync(hits, d_hits, size_t(n) * sizeof(bbg_hit), cudaMemcpyDeviceToHost, st));
    BBG_CUDA(cudaStreamSynchronize(st));
    return BBG_OK;
}
