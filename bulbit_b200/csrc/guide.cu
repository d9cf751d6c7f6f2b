// Neural path guiding on the device: the guide handle, the fused forward
// (inference) kernel, the fused training kernel (forward, the vMF-mixture
// negative log-likelihood gradient, and the backward pass through all layers
// on the tensor cores) and Adam. No counterpart in the reference renderer.

#include "guide.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

namespace bbg
{

namespace
{

constexpr int kTrainWarps = 6;

// ------------------------------------------------------- tensor-core helpers

constexpr uint32_t kTcMaxPolls = 1u << 22; // bound on each wait for a commit of MMAs

__device__ __forceinline__ uint32_t SmemAddr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, leading (K direction) and
// stride (M/N direction) byte offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t TcDesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return uint64_t((addr >> 4) & 0x3fffu) | (uint64_t((lbo >> 4) & 0x3fffu) << 16) |
           (uint64_t((sbo >> 4) & 0x3fffu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 and M >> 4.
__device__ __forceinline__ uint32_t TcInstr(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

// One tcgen05.mma.cta_group::1.kind::f16 into tensor memory at d; accumulate
// selects D += A B over D = A B.
__device__ __forceinline__ void TcMma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
                 "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// Arrives on the mbarrier once every MMA this thread issued has completed.
__device__ __forceinline__ void TcCommit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Waits, at most kTcMaxPolls polls, for the mbarrier phase of the given
// parity to complete; true if it did.
__device__ __forceinline__ bool TcWait(uint32_t bar, uint32_t parity)
{
    uint32_t done = 0;
    for (uint32_t poll = 0; poll < kTcMaxPolls && !done; ++poll)
    {
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (!done && poll >= 16)
        {
            __nanosleep(32);
        }
    }
    return done != 0;
}

// 16 consecutive FP32 accumulator columns of the calling thread's tensor-
// memory lane (32x32b shape: warp w reads lanes 32w..32w+31); the values are
// valid after TcWaitLoads.
__device__ __forceinline__ void TcLoad16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                 "%12, %13, %14, %15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                   "=r"(v[15])
                 : "r"(taddr));
}

__device__ __forceinline__ void TcLoad8(uint32_t taddr, uint32_t (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}

__device__ __forceinline__ void TcWaitLoads()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// A barrier across the CTA that also orders tensor-core operations (issued
// MMAs, tensor-memory loads) and generic shared-memory writes, which the
// MMAs read through the async proxy, with the threads' program order.
__device__ __forceinline__ void TcSyncThreads()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// ---------------------------------------------------------------- forward

// Inference on the fifth-generation tensor cores: a tile is 128 queries and
// a CTA has two threads per query. Threads t and t + 128 (warps w and w + 4,
// which share tensor-memory lanes 32 (w % 4) .. + 31) take query t % 128 and
// one half of its columns each. They write the query's 80 features (BF16)
// into the A tile in shared memory (canonical K-major layout: 8-row x 16-byte
// core matrices, 8-row groups 128 bytes apart, 8-column groups kFtLboA bytes
// apart, so a warp's 16-byte stores of one column group are contiguous);
// thread 0 issues the layer's MMAs (128 x N x 16, BF16 in, FP32 accumulator in
// tensor memory, weights staged once per CTA in the same layout) and commits
// them to an mbarrier; each thread then reads its half of the accumulator row
// with tcgen05.ld, adds the bias, applies the ReLU and writes it back as BF16
// into the A tile as the next layer's input (the MMAs that read it have
// completed). The output layer's 40 values go to the query's output record.
// The next tile's raw inputs are loaded while the current tile's layers run.
constexpr int kFtRows = 128;                                  // queries per tile (MMA M)
constexpr int kFtThreads = 2 * kFtRows;                       // two threads per query
constexpr uint32_t kFtSbo = 128;                              // bytes between 8-row groups
constexpr uint32_t kFtLboA = (kFtRows / 8) * 128;             // bytes between 8-column groups of A
constexpr size_t kFtSmemW = size_t(kTcImage) * 2;             // 32 KB
constexpr size_t kFtSmemBias = 1024;                          // 232 floats, padded
constexpr size_t kFtSmemA = size_t(kGuideIn / 8) * kFtLboA;   // 20 KB (80 columns; the hidden layers use 64)
constexpr size_t kFtOffBias = kFtSmemW;
constexpr size_t kFtOffA = kFtOffBias + kFtSmemBias;
constexpr size_t kFtOffBar = kFtOffA + kFtSmemA;
constexpr size_t kFtSmem = kFtOffBar + 16;                    // + mbarrier and tensor-memory address
constexpr uint32_t kFtCols = 64;                              // tensor-memory columns (widest layer: N = 64)
static_assert(kBfTc % 8 == 0, "the tensor-core image starts on a 16-byte boundary");
static_assert(kFtSmemBias >= size_t(kCBias) * 4, "bias staging");
static_assert(kGuideGroupChunk == kFtRows, "a grouped-forward chunk is one tile");

// Loads a guide's tensor-core weight image and packed biases into shared
// memory.
__device__ __forceinline__ void StageTcWeights(const __nv_bfloat16* wg, const float* pg, uint8_t* smem)
{
    const uint4* src = reinterpret_cast<const uint4*>(wg + kBfTc);
    uint4* dst = reinterpret_cast<uint4*>(smem);
    for (int i = threadIdx.x; i < kTcImage / 8; i += blockDim.x)
    {
        dst[i] = src[i];
    }
    float* bs = reinterpret_cast<float*>(smem + kFtOffBias);
    for (int i = threadIdx.x; i < kCBias; i += blockDim.x)
    {
        int src_at = i < kCB1 ? kB0 + i : i < kCB2 ? kB1 + (i - kCB1) : i < kCB3 ? kB2 + (i - kCB2) : kB3 + (i - kCB3);
        bs[i] = pg[src_at];
    }
}

// Issues one layer's MMAs (K / 16 of them) and commits them to the barrier.
__device__ __forceinline__ void IssueTcLayer(uint32_t tmem, uint32_t a, uint32_t w, int n, int k, uint32_t bar)
{
    const uint32_t idesc = TcInstr(kFtRows, n);
    const uint32_t lbo_w = uint32_t(n / 8) * 128;
    for (int ks = 0; ks < k / 16; ++ks)
    {
        TcMma(tmem, TcDesc(a + 2 * ks * kFtLboA, kFtLboA, kFtSbo), TcDesc(w + 2 * ks * lbo_w, lbo_w, kFtSbo), idesc,
              ks > 0 ? 1u : 0u);
    }
    TcCommit(bar);
}

// One half (32 columns) of the calling thread's hidden-layer row: accumulators
// + bias, ReLU, BF16, stored into the A row as the next layer's input.
__device__ __forceinline__ void HiddenHalfToA(uint32_t tmem_row, const float* bias, int half, uint8_t* a_row)
{
    uint32_t v[2][16];
    TcLoad16(tmem_row + uint32_t(32 * half), v[0]);
    TcLoad16(tmem_row + uint32_t(32 * half + 16), v[1]);
    TcWaitLoads();
#pragma unroll
    for (int g = 0; g < 4; ++g)
    {
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            const int c = 8 * g + 2 * q, col = 32 * half + c;
            w[q] = PackBf16(fmaxf(__uint_as_float(v[c / 16][c % 16]) + bias[col], 0.0f),
                            fmaxf(__uint_as_float(v[c / 16][c % 16 + 1]) + bias[col + 1], 0.0f));
        }
        *reinterpret_cast<uint4*>(a_row + (4 * half + g) * kFtLboA) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// The raw inputs of one query and where its output goes (id < 0: no query).
struct QueryIn
{
    float raw[kGuideRaw];
    int64_t id;
};

// One 128-query tile through the network with the weights staged in smem;
// prefetch() runs once the features are written. Returns false if an MMA
// commit did not arrive in time (the tile's outputs are then not written);
// *phase counts the barrier's completed phases.
template <class Prefetch>
__device__ __forceinline__ bool ForwardTcTile(const QueryIn& q, const GuideBounds& bounds, float* out, uint8_t* smem,
                                              uint32_t tmem, uint32_t* phase, Prefetch&& prefetch)
{
    const int r = threadIdx.x & (kFtRows - 1), half = threadIdx.x / kFtRows;
    uint8_t* a_row = smem + kFtOffA + size_t(r) * 16;
    const float* bias = reinterpret_cast<const float*>(smem + kFtOffBias);
    const uint32_t a = SmemAddr(smem + kFtOffA), w = SmemAddr(smem), bar = SmemAddr(smem + kFtOffBar);
    const uint32_t tmem_row = tmem + (uint32_t(r & ~31) << 16);

    // Features 40 half .. 40 half + 39: 20 BF16 pairs, stored as 5 16-byte
    // rows of the A tile.
    {
        uint32_t x[kGuideIn / 4];
        if (q.id >= 0)
        {
            GuideFeatures40(q.raw, bounds, half, [&](int j, float v0, float v1) { x[j >> 1] = PackBf16(v0, v1); });
        }
        else
        {
#pragma unroll
            for (int k = 0; k < kGuideIn / 4; ++k)
            {
                x[k] = 0u;
            }
        }
#pragma unroll
        for (int g = 0; g < kGuideIn / 16; ++g)
        {
            *reinterpret_cast<uint4*>(a_row + (5 * half + g) * kFtLboA) =
                make_uint4(x[4 * g], x[4 * g + 1], x[4 * g + 2], x[4 * g + 3]);
        }
    }
    prefetch();

    const struct
    {
        int w_off, n, k, bias_off;
    } kLayers[4] = { { kTcW0, kGuideHidden, kGuideIn, kCB0 },
                     { kTcW1, kGuideHidden, kGuideHidden, kCB1 },
                     { kTcW2, kGuideHidden, kGuideHidden, kCB2 },
                     { kTcW3, kGuideOutPad, kGuideHidden, kCB3 } };
#pragma unroll
    for (int l = 0; l < 4; ++l)
    {
        TcSyncThreads(); // the A tile is written; the last layer's loads are done
        if (threadIdx.x == 0)
        {
            IssueTcLayer(tmem, a, w + 2 * uint32_t(kLayers[l].w_off), kLayers[l].n, kLayers[l].k, bar);
        }
        const bool done = TcWait(bar, *phase & 1u);
        *phase += 1;
        if (!__syncthreads_and(done))
        {
            return false;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (l < 3)
        {
            HiddenHalfToA(tmem_row, bias + kLayers[l].bias_off, half, a_row);
        }
    }

    // Output layer: half 0 takes columns 0..23, half 1 columns 24..39 (of the
    // 48; the rest are the zero padding).
    const float* b3 = bias + kCB3;
    if (half == 0)
    {
        uint32_t v0[16], v1[8];
        TcLoad16(tmem_row, v0);
        TcLoad8(tmem_row + 16u, v1);
        TcWaitLoads();
        if (q.id >= 0)
        {
            float* o = out + kGuideOut * q.id;
#pragma unroll
            for (int c = 0; c < 16; c += 4)
            {
                *reinterpret_cast<float4*>(o + c) =
                    make_float4(__uint_as_float(v0[c]) + b3[c], __uint_as_float(v0[c + 1]) + b3[c + 1],
                                __uint_as_float(v0[c + 2]) + b3[c + 2], __uint_as_float(v0[c + 3]) + b3[c + 3]);
            }
#pragma unroll
            for (int c = 0; c < 8; c += 4)
            {
                *reinterpret_cast<float4*>(o + 16 + c) = make_float4(
                    __uint_as_float(v1[c]) + b3[16 + c], __uint_as_float(v1[c + 1]) + b3[17 + c],
                    __uint_as_float(v1[c + 2]) + b3[18 + c], __uint_as_float(v1[c + 3]) + b3[19 + c]);
            }
        }
    }
    else
    {
        uint32_t v0[16];
        TcLoad16(tmem_row + 24u, v0);
        TcWaitLoads();
        if (q.id >= 0)
        {
            float* o = out + kGuideOut * q.id + 24;
#pragma unroll
            for (int c = 0; c < 16; c += 4)
            {
                *reinterpret_cast<float4*>(o + c) = make_float4(
                    __uint_as_float(v0[c]) + b3[24 + c], __uint_as_float(v0[c + 1]) + b3[25 + c],
                    __uint_as_float(v0[c + 2]) + b3[26 + c], __uint_as_float(v0[c + 3]) + b3[27 + c]);
            }
        }
    }
    return true;
}

// Tensor memory and the mbarrier of a forward CTA: allocated by warp 0, the
// address published to every thread.
__device__ __forceinline__ uint32_t ForwardTcSetUp(uint8_t* smem)
{
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kFtOffBar + 8);
    if (threadIdx.x < 32)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(slot)),
                     "r"(kFtCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(smem + kFtOffBar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    TcSyncThreads();
    return *slot;
}

__device__ __forceinline__ void ForwardTcTearDown(uint32_t tmem)
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < 32)
    {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kFtCols));
    }
}

// The query behind entry item of the forward's input (index, when set, maps
// entries to record ids; -1 entries are padding).
__device__ __forceinline__ QueryIn FetchQuery(const float* raw, const int32_t* index, int64_t item, int64_t n)
{
    QueryIn q;
    q.id = item < n ? (index ? int64_t(index[item]) : item) : -1;
#pragma unroll
    for (int k = 0; k < kGuideRaw; ++k)
    {
        q.raw[k] = 0.0f;
    }
    if (q.id >= 0)
    {
        const float2* p = reinterpret_cast<const float2*>(raw + kGuideRaw * q.id);
#pragma unroll
        for (int k = 0; k < kGuideRaw / 2; ++k)
        {
            const float2 v = p[k];
            q.raw[2 * k] = v.x;
            q.raw[2 * k + 1] = v.y;
        }
    }
    return q;
}

// Persistent forward: CTA b takes tiles b, b + grid, ...
__global__ void __launch_bounds__(kFtThreads, 4) GuideForwardKernel(const float* raw, const int32_t* index,
                                                                    const int32_t* n_dev, int64_t n_host,
                                                                    GuideBounds bounds, const __nv_bfloat16* wg,
                                                                    const float* pg, float* out, int32_t* status)
{
    extern __shared__ __align__(128) uint8_t ft_smem[];
    const int64_t n = n_dev ? int64_t(*n_dev) : n_host;
    const int64_t tiles = (n + kFtRows - 1) / kFtRows;
    if (int64_t(blockIdx.x) >= tiles)
    {
        return; // the whole CTA, before any tensor-memory use
    }
    const int r = threadIdx.x & (kFtRows - 1);
    QueryIn q = FetchQuery(raw, index, int64_t(blockIdx.x) * kFtRows + r, n);
    StageTcWeights(wg, pg, ft_smem);
    const uint32_t tmem = ForwardTcSetUp(ft_smem);
    uint32_t phase = 0;
    bool ok = true;
    for (int64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x)
    {
        QueryIn next;
        ok = ForwardTcTile(q, bounds, out, ft_smem, tmem, &phase,
                           [&] { next = FetchQuery(raw, index, (tile + gridDim.x) * kFtRows + r, n); });
        q = next;
    }
    if (!ok && threadIdx.x == 0)
    {
        atomicExch(status, 1); // a commit of MMAs did not arrive within the bound
    }
    ForwardTcTearDown(tmem);
}

// Grouped forward: each CTA takes a contiguous run of chunks (one tile each)
// and stages a group's weights whenever the run enters a new group (a chunk
// never spans two groups).
__global__ void __launch_bounds__(kFtThreads, 4) GuideGroupedForwardKernel(const float* raw, const int32_t* index,
                                                                           const int32_t* chunk_start,
                                                                           int32_t n_groups, const GuideGroup* groups,
                                                                           float* out)
{
    extern __shared__ __align__(128) uint8_t ft_smem[];
    const int64_t chunks = chunk_start[n_groups];
    const int64_t c0 = chunks * blockIdx.x / gridDim.x, c1 = chunks * (blockIdx.x + 1) / gridDim.x;
    if (c0 >= c1)
    {
        return;
    }
    const int r = threadIdx.x & (kFtRows - 1);
    const int64_t n = chunks * kGuideGroupChunk;
    QueryIn q = FetchQuery(raw, index, c0 * kFtRows + r, n);
    const uint32_t tmem = ForwardTcSetUp(ft_smem);
    uint32_t phase = 0;
    bool ok = true;
    int32_t staged = -1;
    for (int64_t c = c0; c < c1 && ok; ++c)
    {
        // The group whose chunk range holds c (CTA-uniform).
        int32_t lo = 0, hi = n_groups - 1;
        while (lo < hi)
        {
            int32_t mid = (lo + hi + 1) >> 1;
            if (chunk_start[mid] <= c)
            {
                lo = mid;
            }
            else
            {
                hi = mid - 1;
            }
        }
        if (lo != staged)
        {
            __syncthreads(); // the previous tile's MMAs and loads are done (its commit was awaited)
            StageTcWeights(groups[lo].wg, groups[lo].pg, ft_smem);
            staged = lo;
        }
        QueryIn next;
        ok = ForwardTcTile(q, groups[lo].bounds, out, ft_smem, tmem, &phase,
                           [&] { next = FetchQuery(raw, index, (c + 1 < c1 ? c + 1 : c1) * kFtRows + r, c1 * kFtRows); });
        q = next;
        if (!ok && threadIdx.x == 0)
        {
            atomicExch(groups[lo].status, 1); // a commit of MMAs did not arrive within the bound
        }
    }
    ForwardTcTearDown(tmem);
}

// ---------------------------------------------------------------- training

// Loads BF16 weights (the first n_bf16 values: the training images) and the
// packed biases into shared memory.
__device__ __forceinline__ void StageWeights(const __nv_bfloat16* wg, const float* pg, __nv_bfloat16* ws, float* bs,
                                             int n_bf16)
{
    const uint4* src = reinterpret_cast<const uint4*>(wg);
    uint4* dst = reinterpret_cast<uint4*>(ws);
    for (int i = threadIdx.x; i < n_bf16 / 8; i += blockDim.x)
    {
        dst[i] = src[i];
    }
    for (int i = threadIdx.x; i < kCBias; i += blockDim.x)
    {
        int src_at = i < kCB1 ? kB0 + i : i < kCB2 ? kB1 + (i - kCB1) : i < kCB3 ? kB2 + (i - kCB2) : kB3 + (i - kCB3);
        bs[i] = pg[src_at];
    }
    __syncthreads();
}

// Gradient of -w log q(dir) w.r.t. the 40 raw outputs of one sample, and the
// loss term (q: the vMF mixture of MakeMixture).
__device__ __forceinline__ float MixtureNllGrad(const float* o, V3 dir, float weight, float* g)
{
    VmfMixture m = MakeMixture(o);
    float lp[kLobes];
    float mx = -INFINITY;
    for (int j = 0; j < kLobes; ++j)
    {
        float k = m.kappa[j];
        lp[j] = m.logw[j] + VmfLogNorm(k) + k * (Dot(m.mu[j], dir) - 1.0f);
        mx = fmaxf(mx, lp[j]);
    }
    float s = 0;
    for (int j = 0; j < kLobes; ++j)
    {
        s += expf(lp[j] - mx);
    }
    float logq = mx + logf(s);
    for (int j = 0; j < kLobes; ++j)
    {
        float gamma = expf(lp[j] - logq); // responsibility
        float pi = expf(m.logw[j]);
        float k = m.kappa[j];
        V3 v{ o[5 * j + 1], o[5 * j + 2], o[5 * j + 3] };
        float len = fmaxf(Length(v), 1e-6f);
        float cosm = Dot(m.mu[j], dir);
        V3 dm = (dir - m.mu[j] * cosm) * (gamma * k / len);
        g[5 * j] = -weight * (gamma - pi);
        g[5 * j + 1] = -weight * dm.x;
        g[5 * j + 2] = -weight * dm.y;
        g[5 * j + 3] = -weight * dm.z;
        float r = o[5 * j + 4];
        float two_k = 2.0f * k;
        float dlogf_dlogk = 1.0f - two_k / expm1f(two_k) + k * (cosm - 1.0f);
        bool clamped = r < kKappaLogMin || r > kKappaLogMax;
        g[5 * j + 4] = clamped ? 0.0f : -weight * gamma * dlogf_dlogk;
    }
    return -weight * logq;
}

struct TrainWarp
{
    __nv_bfloat16 x[16 * kXLd];          // [sample][feature], padded rows
    __nv_bfloat16 xt[kGuideIn * 16];     // [feature][sample]
    __nv_bfloat16 h[3][16 * kGuideHidden];   // post-ReLU activations [sample][unit]
    __nv_bfloat16 ht[3][kGuideHidden * 16];  // [unit][sample]
    float y[16 * kGuideOut];             // outputs
    __nv_bfloat16 dy[16 * kGuideOutPad]; // [sample][out], zero padded
    __nv_bfloat16 dyt[kGuideOutPad * 16];
    __nv_bfloat16 dh[16 * kGuideHidden];
    __nv_bfloat16 dht[kGuideHidden * 16];
};

// Shared memory: weights (all images), packed biases, packed bias-gradient
// accumulators, then one TrainWarp per warp.
constexpr size_t kTrainSmem = size_t(kBfAll) * 2 + 2 * size_t(kCBias) * 4 + sizeof(TrainWarp) * kTrainWarps;
static_assert((size_t(kBfAll) * 2 + 2 * size_t(kCBias) * 4) % 16 == 0, "TrainWarp alignment");

// Training scratch (global, bf16, one column per sample, row stride = the
// batch capacity): the transposed layer inputs and output gradients that the
// weight-gradient GEMMs read. Rows: X^T 80, H0^T 64, H1^T 64, H2^T 64,
// dY^T 48 (40 + zero padding), dZ2^T 64, dZ1^T 64, dZ0^T 64.
constexpr int kRowX = 0, kRowH0 = 80, kRowH1 = 144, kRowH2 = 208, kRowDY = 272, kRowDZ2 = 320, kRowDZ1 = 384,
              kRowDZ0 = 448, kScratchRows = 512;

// Copies a warp's [rows][16] bf16 block (16 samples) into scratch rows
// row0.. at sample column col0 (16-byte stores).
__device__ __forceinline__ void StoreColumns(const __nv_bfloat16* src, int rows, __nv_bfloat16* scratch, int64_t ld,
                                             int row0, int64_t col0, int lane)
{
    for (int i = lane; i < 2 * rows; i += 32)
    {
        int r = i >> 1, half = i & 1;
        uint4 v = *reinterpret_cast<const uint4*>(src + r * 16 + half * 8);
        *reinterpret_cast<uint4*>(scratch + (int64_t(row0) + r) * ld + col0 + half * 8) = v;
    }
}

// C fragments (16 rows x 64 cols) -> bf16 [16][64] and [64][16].
__device__ __forceinline__ void StoreActs(const float (&acc)[8][4], __nv_bfloat16* rm, __nv_bfloat16* cm, int lane)
{
    int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
    {
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            int row = g + 8 * half;
            int col = nt * 8 + 2 * t;
            __nv_bfloat16 v0 = __float2bfloat16_rn(acc[nt][2 * half]);
            __nv_bfloat16 v1 = __float2bfloat16_rn(acc[nt][2 * half + 1]);
            rm[row * kGuideHidden + col] = v0;
            rm[row * kGuideHidden + col + 1] = v1;
            cm[col * 16 + row] = v0;
            cm[(col + 1) * 16 + row] = v1;
        }
    }
}

// dZ = (dOut . W) masked by the ReLU of the layer's output h: A = dOut
// [16][K] (ld lda), B = W^T stored [64][K]; writes dZ to dh / dht and adds the
// column sums to the bias gradient.
template <int KT>
__device__ __forceinline__ void BackLayer(const __nv_bfloat16* dout, int lda, const __nv_bfloat16* wt, int ldw,
                                          const __nv_bfloat16* h, __nv_bfloat16* dh, __nv_bfloat16* dht,
                                          float* bias_grad, int lane)
{
    uint32_t a[KT][4];
#pragma unroll
    for (int kt = 0; kt < KT; ++kt)
    {
        LoadA(dout, lda, 0, kt * 16, lane, a[kt]);
    }
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
    {
        acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0;
#pragma unroll
        for (int kt = 0; kt < KT; ++kt)
        {
            uint32_t b0, b1;
            LoadB(wt, ldw, nt * 8, kt * 16, lane, &b0, &b1);
            Mma16816(acc[nt], a[kt], b0, b1);
        }
    }
    __syncwarp(); // every lane has read dout before dh is overwritten
    int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
    {
        float colsum0 = 0, colsum1 = 0;
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            int row = g + 8 * half;
            int col = nt * 8 + 2 * t;
            float v0 = __bfloat162float(h[row * kGuideHidden + col]) > 0.0f ? acc[nt][2 * half] : 0.0f;
            float v1 = __bfloat162float(h[row * kGuideHidden + col + 1]) > 0.0f ? acc[nt][2 * half + 1] : 0.0f;
            colsum0 += v0;
            colsum1 += v1;
            __nv_bfloat16 b0 = __float2bfloat16_rn(v0), b1 = __float2bfloat16_rn(v1);
            dh[row * kGuideHidden + col] = b0;
            dh[row * kGuideHidden + col + 1] = b1;
            dht[col * 16 + row] = b0;
            dht[(col + 1) * 16 + row] = b1;
        }
        // Sum over the 8 row groups (lanes with equal t).
        for (int off = 4; off < 32; off <<= 1)
        {
            colsum0 += __shfl_xor_sync(0xffffffffu, colsum0, off);
            colsum1 += __shfl_xor_sync(0xffffffffu, colsum1, off);
        }
        if (g == 0)
        {
            atomicAdd(bias_grad + nt * 8 + 2 * t, colsum0);
            atomicAdd(bias_grad + nt * 8 + 2 * t + 1, colsum1);
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(32 * kTrainWarps) GuideTrainKernel(const float* raw, const float* dirs,
                                                                      const float* weights, const int32_t* n_dev,
                                                                      int64_t n_host, GuideBounds bounds,
                                                                      const __nv_bfloat16* wg, const float* pg,
                                                                      __nv_bfloat16* scratch, int64_t ld,
                                                                      float* grad_out, float* loss_out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* ws = reinterpret_cast<__nv_bfloat16*>(smem);
    float* bs = reinterpret_cast<float*>(smem + size_t(kBfAll) * 2);
    float* bgs = bs + kCBias; // bias gradients, packed like bs
    TrainWarp* tw = reinterpret_cast<TrainWarp*>(bgs + kCBias);
    StageWeights(wg, pg, ws, bs, kBfAll);
    for (int i = threadIdx.x; i < kCBias; i += blockDim.x)
    {
        bgs[i] = 0;
    }
    __syncthreads();

    const int64_t n = n_dev ? int64_t(*n_dev) : n_host;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    TrainWarp& W = tw[warp];
    const int g = lane >> 2, t = lane & 3;
    float loss = 0;
    const int64_t tiles = (n + 15) / 16;
    for (int64_t tile = int64_t(blockIdx.x) * kTrainWarps + warp; tile < tiles;
         tile += int64_t(gridDim.x) * kTrainWarps)
    {
        // Features, both layouts.
        {
            int row = lane >> 1, half = lane & 1;
            int64_t item = tile * 16 + row;
            bool valid = item < n;
            auto put = [&](int j, float v0, float v1) {
                const int f = half * 40 + j;
                const __nv_bfloat16 a = __float2bfloat16_rn(v0), b = __float2bfloat16_rn(v1);
                W.x[row * kXLd + f] = a;
                W.x[row * kXLd + f + 1] = b;
                W.xt[f * 16 + row] = a;
                W.xt[(f + 1) * 16 + row] = b;
            };
            if (valid)
            {
                float r[kGuideRaw];
                for (int k = 0; k < kGuideRaw; ++k)
                {
                    r[k] = raw[kGuideRaw * item + k];
                }
                GuideFeatures40(r, bounds, half, put);
            }
            else
            {
#pragma unroll
                for (int j = 0; j < 40; j += 2)
                {
                    put(j, 0.0f, 0.0f);
                }
            }
        }
        __syncwarp();

        // Forward, keeping activations.
        uint32_t a0[5][4];
#pragma unroll
        for (int kt = 0; kt < 5; ++kt)
        {
            LoadA(W.x, kXLd, 0, kt * 16, lane, a0[kt]);
        }
        float acc[8][4];
        uint32_t a[4][4];
        HiddenLayer<5>(a0, ws + kBf0, bs + kCB0, lane, acc);
        StoreActs(acc, W.h[0], W.ht[0], lane);
        AccToA(acc, a);
        HiddenLayer<4>(a, ws + kBf1, bs + kCB1, lane, acc);
        StoreActs(acc, W.h[1], W.ht[1], lane);
        AccToA(acc, a);
        HiddenLayer<4>(a, ws + kBf2, bs + kCB2, lane, acc);
        StoreActs(acc, W.h[2], W.ht[2], lane);
        AccToA(acc, a);
        float out[5][4];
        OutputLayer(a, ws + kBf3, bs + kCB3, lane, out);
#pragma unroll
        for (int nt = 0; nt < 5; ++nt)
        {
#pragma unroll
            for (int half = 0; half < 2; ++half)
            {
                int row = g + 8 * half;
                W.y[row * kGuideOut + nt * 8 + 2 * t] = out[nt][2 * half];
                W.y[row * kGuideOut + nt * 8 + 2 * t + 1] = out[nt][2 * half + 1];
            }
        }
        __syncwarp();

        // Output gradient, one lane per sample.
        if (lane < 16)
        {
            int64_t item = tile * 16 + lane;
            float gy[kGuideOut];
            if (item < n)
            {
                V3 dir{ dirs[3 * item], dirs[3 * item + 1], dirs[3 * item + 2] };
                loss += MixtureNllGrad(W.y + lane * kGuideOut, dir, weights[item], gy);
            }
            else
            {
                for (int k = 0; k < kGuideOut; ++k)
                {
                    gy[k] = 0;
                }
            }
            for (int k = 0; k < kGuideOutPad; ++k)
            {
                float v = k < kGuideOut ? gy[k] : 0.0f;
                __nv_bfloat16 b = __float2bfloat16_rn(v);
                W.dy[lane * kGuideOutPad + k] = b;
                W.dyt[k * 16 + lane] = b;
                if (k < kGuideOut && v != 0.0f)
                {
                    atomicAdd(bgs + kCB3 + k, v);
                }
            }
        }
        __syncwarp();

        // Layer 3: dW3 += dY^T H3, dZ2 = (dY W3) * relu'(H3).
        // The layer inputs and output gradients, transposed, go to the
        // scratch columns of these 16 samples; the weight gradients are the
        // GEMMs dW = dZ^T A over the whole batch (GuideWeightGradTcKernel).
        const int64_t col0 = tile * 16;
        StoreColumns(W.xt, kGuideIn, scratch, ld, kRowX, col0, lane);
        StoreColumns(W.ht[0], kGuideHidden, scratch, ld, kRowH0, col0, lane);
        StoreColumns(W.ht[1], kGuideHidden, scratch, ld, kRowH1, col0, lane);
        StoreColumns(W.ht[2], kGuideHidden, scratch, ld, kRowH2, col0, lane);
        StoreColumns(W.dyt, kGuideOutPad, scratch, ld, kRowDY, col0, lane);
        // dZ2 = (dY W3) * relu'(H2), then dZ1, dZ0 likewise.
        BackLayer<3>(W.dy, kGuideOutPad, ws + kBfT3, kGuideOutPad, W.h[2], W.dh, W.dht, bgs + kCB2, lane);
        __syncwarp();
        StoreColumns(W.dht, kGuideHidden, scratch, ld, kRowDZ2, col0, lane);
        BackLayer<4>(W.dh, kGuideHidden, ws + kBfT2, kGuideHidden, W.h[1], W.dh, W.dht, bgs + kCB1, lane);
        __syncwarp();
        StoreColumns(W.dht, kGuideHidden, scratch, ld, kRowDZ1, col0, lane);
        BackLayer<4>(W.dh, kGuideHidden, ws + kBfT1, kGuideHidden, W.h[0], W.dh, W.dht, bgs + kCB0, lane);
        __syncwarp();
        StoreColumns(W.dht, kGuideHidden, scratch, ld, kRowDZ0, col0, lane);
        __syncwarp();
    }
    for (int off = 16; off > 0; off >>= 1)
    {
        loss += __shfl_xor_sync(0xffffffffu, loss, off);
    }
    if (lane == 0 && loss != 0.0f)
    {
        atomicAdd(loss_out, loss);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kCBias; i += blockDim.x)
    {
        float v = bgs[i];
        if (v != 0.0f)
        {
            int dst = i < kCB1 ? kB0 + i : i < kCB2 ? kB1 + (i - kCB1) : i < kCB3 ? kB2 + (i - kCB2) : kB3 + (i - kCB3);
            atomicAdd(grad_out + dst, v);
        }
    }
}

// Weight gradients dW_L[m][n] = sum over the batch of dZ_L[s][m] A_L[s][n]
// (A_L: the layer's input), from the training scratch, per chunk of
// kGradChunk samples (GuideWeightGradTcKernel below); GuideGradReduceKernel
// adds the chunks' partial sums to the gradient (no atomics, a fixed
// summation order). Samples past the batch are zero in the dZ rows.
constexpr int kGradChunk = 256;

struct GradLayer
{
    int dz_row, a_row, m, n, w_off;
};
__constant__ GradLayer kGradLayers[4] = { { kRowDZ0, kRowX, kGuideHidden, kGuideIn, kW0 },
                                          { kRowDZ1, kRowH0, kGuideHidden, kGuideHidden, kW1 },
                                          { kRowDZ2, kRowH1, kGuideHidden, kGuideHidden, kW2 },
                                          { kRowDY, kRowH2, kGuideOut, kGuideHidden, kW3 } };

// grad[w] += sum over chunks of partial[chunk][w], for the weight entries.
__global__ void GuideGradReduceKernel(const float* partial, const int32_t* n_dev, int64_t n_host, float* grad)
{
    const int64_t n = n_dev ? int64_t(*n_dev) : n_host;
    const int64_t chunks = ((n + 15) / 16 * 16 + kGradChunk - 1) / kGradChunk;
    constexpr int kWeights = kGuideParams - kCBias;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kWeights; i += gridDim.x * blockDim.x)
    {
        // The i-th weight entry: W0 b0 W1 b1 W2 b2 W3 b3, biases skipped.
        int w = i < kB0 - kW0 ? kW0 + i
                : i < kB0 - kW0 + (kB1 - kW1) ? kW1 + (i - (kB0 - kW0))
                : i < kB0 - kW0 + (kB1 - kW1) + (kB2 - kW2) ? kW2 + (i - (kB0 - kW0) - (kB1 - kW1))
                : kW3 + (i - (kB0 - kW0) - (kB1 - kW1) - (kB2 - kW2));
        float s = 0;
        for (int64_t c = 0; c < chunks; ++c)
        {
            s += partial[c * kGuideParams + w];
        }
        grad[w] += s;
    }
}

// Weight gradients on the fifth-generation tensor cores (tcgen05, sm_100a):
// one CTA per (chunk of kGradChunk samples, layer) computes the chunk's
// partial dW_L = dZ_L^T A_L with the accumulator in tensor memory. The
// chunk's dZ rows (M, zero-padded to 128) and layer-input rows (N = 80 or 64)
// are staged from the training scratch into shared memory in the canonical
// K-major layout without swizzling: 8-row x 16-byte core matrices, 8-row
// groups kTcSbo bytes apart and 8-sample column groups kTcLbo* bytes apart.
// One thread issues the 16 MMAs of shape 128 x N x 16 (BF16 in, FP32
// accumulate), a commit arrives on an mbarrier, and each warp reads its 32
// accumulator rows back from tensor memory into the chunk's partial sums
// (GuideGradReduceKernel then adds the chunks in a fixed order).
constexpr int kTcRows = 128;                                  // MMA M: dZ rows, zero-padded
constexpr int kTcMaxN = 80;                                   // widest layer input
constexpr int kTcGroups = kGradChunk / 8;                     // 8-sample core-matrix columns
constexpr uint32_t kTcSbo = 128;                              // bytes between 8-row groups
constexpr uint32_t kTcLboA = (kTcRows / 8) * 128;             // bytes between column groups of A
constexpr uint32_t kTcLboB = (kTcMaxN / 8) * 128;             // of B
constexpr size_t kTcSmemA = size_t(kTcGroups) * kTcLboA;      // 64 KB
constexpr size_t kTcSmemB = size_t(kTcGroups) * kTcLboB;      // 40 KB
constexpr size_t kTcSmem = kTcSmemA + kTcSmemB + 16;          // + mbarrier and tensor-memory address
constexpr uint32_t kTcCols = 128;                             // tensor-memory columns (N <= 80)
constexpr int kTcThreads = 256;                               // 8 warps stage; warps 0-3 read 32 rows each

__global__ void __launch_bounds__(kTcThreads) GuideWeightGradTcKernel(const __nv_bfloat16* scratch, int64_t ld,
                                                                        const int32_t* n_dev, int64_t n_host,
                                                                        float* partial, int32_t* status)
{
    extern __shared__ __align__(128) uint8_t tc_smem[];
    uint8_t* sa = tc_smem;
    uint8_t* sb = tc_smem + kTcSmemA;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tc_smem + kTcSmemA + kTcSmemB);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem + kTcSmemA + kTcSmemB + 8);

    const int64_t n = n_dev ? int64_t(*n_dev) : n_host;
    const int64_t n_pad = (n + 15) / 16 * 16;
    const int64_t chunk = blockIdx.x;
    if (chunk * kGradChunk >= n_pad)
    {
        return; // the whole block, before any tensor-memory use
    }
    const GradLayer L = kGradLayers[blockIdx.y];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t k0 = chunk * kGradChunk;
    const int kvalid = int(min(int64_t(kGradChunk), n_pad - k0)); // a multiple of 16

    // Stage the chunk with asynchronous 16-byte copies (all of a thread's
    // copies in flight at once): A = dZ rows (rows >= m zero-filled), B =
    // layer-input rows (rows >= n zero-filled); samples past the batch are
    // zero-filled too (a source size of 0 reads nothing).
    for (int i = tid; i < kTcRows * kTcGroups; i += kTcThreads)
    {
        const int r = i / kTcGroups, g = i % kTcGroups;
        const bool in = r < L.m && g * 8 < kvalid;
        const __nv_bfloat16* src = in ? scratch + (int64_t(L.dz_row) + r) * ld + k0 + g * 8 : scratch;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                         SmemAddr(sa + g * kTcLboA + (r >> 3) * kTcSbo + (r & 7) * 16)),
                     "l"(src), "r"(in ? 16 : 0)
                     : "memory");
    }
    for (int i = tid; i < kTcMaxN * kTcGroups; i += kTcThreads)
    {
        const int r = i / kTcGroups, g = i % kTcGroups;
        const bool in = r < L.n && g * 8 < kvalid;
        const __nv_bfloat16* src = in ? scratch + (int64_t(L.a_row) + r) * ld + k0 + g * 8 : scratch;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                         SmemAddr(sb + g * kTcLboB + (r >> 3) * kTcSbo + (r & 7) * 16)),
                     "l"(src), "r"(in ? 16 : 0)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(tmem_slot)),
                     "r"(kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(1) : "memory");
    }
    // The staged tiles become visible to the tensor cores (the async
    // proxy); the allocated address becomes visible to every thread.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (tid == 0)
    {
        const uint32_t idesc = TcInstr(kTcRows, L.n);
        const uint32_t a0 = SmemAddr(sa), b0 = SmemAddr(sb);
        for (int ks = 0; ks < kvalid / 16; ++ks)
        {
            const uint64_t da = TcDesc(a0 + 2 * ks * kTcLboA, kTcLboA, kTcSbo);
            const uint64_t db = TcDesc(b0 + 2 * ks * kTcLboB, kTcLboB, kTcSbo);
            const uint32_t accumulate = ks > 0 ? 1u : 0u;
            asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                         "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                         "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(SmemAddr(bar))
                     : "memory");
    }
    // Bounded wait for the MMAs' completion (phase 0 of the barrier).
    uint32_t done = 0;
    for (uint32_t poll = 0; poll < kTcMaxPolls && !done; ++poll)
    {
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(SmemAddr(bar)), "r"(0u)
                     : "memory");
        if (!done)
        {
            __nanosleep(64);
        }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // Warps 0-3 read the accumulator rows (warp w may access tensor-memory
    // lanes 32w..32w+31); every warp of them takes the same branch.
    if (warp < kTcRows / 32 && __all_sync(0xffffffffu, done))
    {
        const int r = warp * 32 + lane;
        float* dst = partial + chunk * kGuideParams + L.w_off + r * L.n;
        for (int c = 0; c < L.n; c += 16)
        {
            uint32_t v[16];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                         "%12, %13, %14, %15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                           "=r"(v[14]), "=r"(v[15])
                         : "r"(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (r < L.m)
            {
                for (int q = 0; q < 16; q += 4)
                {
                    *reinterpret_cast<float4*>(dst + c + q) =
                        make_float4(__uint_as_float(v[q]), __uint_as_float(v[q + 1]), __uint_as_float(v[q + 2]),
                                    __uint_as_float(v[q + 3]));
                }
            }
        }
    }
    else if (!done)
    {
        atomicExch(status, 1); // the MMAs did not complete within the bound
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
    {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols));
    }
}

// Counts an Adam step when the batch is not empty. The step number and the
// batch size live in device memory so a captured graph replays correctly.
__global__ void GuideStepKernel(int32_t* step, const int32_t* n_dev, int64_t n_host)
{
    int64_t n = n_dev ? int64_t(*n_dev) : n_host;
    if (n > 0)
    {
        *step += 1;
    }
}

// Adam on the FP32 master parameters (gradient = grad_sum / n), then the
// BF16 images (forward and transposed layouts) are refreshed; the gradient
// accumulator is cleared for the next step. An empty batch changes nothing.
__global__ void GuideAdamKernel(float* params, float* m, float* v, float* grad, const int32_t* step_dev, float lr,
                                float b1, float b2, float eps, const int32_t* n_dev, int64_t n_host)
{
    int64_t n = n_dev ? int64_t(*n_dev) : n_host;
    if (n <= 0)
    {
        return;
    }
    float inv_n = 1.0f / float(n);
    int step = *step_dev;
    float c1 = 1.0f - powf(b1, float(step));
    float c2 = 1.0f - powf(b2, float(step));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGuideParams; i += gridDim.x * blockDim.x)
    {
        float gi = grad[i] * inv_n;
        grad[i] = 0;
        float mi = b1 * m[i] + (1 - b1) * gi;
        float vi = b2 * v[i] + (1 - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void GuideConvertKernel(const float* params, __nv_bfloat16* w)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kBfBuf; i += gridDim.x * blockDim.x)
    {
        float v = 0;
        if (i >= kBfTc)
        {
            // Canonical K-major layout (see kTcW0): locate layer, then (n, k).
            const int j = i - kBfTc;
            const int base = j < kTcW1 ? kTcW0 : j < kTcW2 ? kTcW1 : j < kTcW3 ? kTcW2 : kTcW3;
            const int src = j < kTcW1 ? kW0 : j < kTcW2 ? kW1 : j < kTcW3 ? kW2 : kW3;
            const int n_in = j < kTcW1 ? kGuideIn : kGuideHidden;
            const int n_out = j < kTcW3 ? kGuideHidden : kGuideOutPad;
            const int e = j - base, kg = e / (n_out * 8), rem = e % (n_out * 8);
            const int n = (rem / 64) * 8 + (rem % 64) / 8, k = kg * 8 + rem % 8;
            v = (src != kW3 || n < kGuideOut) ? params[src + n * n_in + k] : 0.0f;
        }
        else if (i < kBfFwd)
        {
            // Fragment order (see kBf0): locate layer, tile, lane, element.
            int base = i < kBf1 ? kBf0 : i < kBf2 ? kBf1 : i < kBf3 ? kBf2 : kBf3;
            int src = i < kBf1 ? kW0 : i < kBf2 ? kW1 : i < kBf3 ? kW2 : kW3;
            int n_in = i < kBf1 ? kGuideIn : kGuideHidden;
            int n_tiles = i < kBf3 ? kGuideHidden / 8 : kGuideOut / 8;
            int j = i - base, e = j & 3, lane = (j >> 2) & 31, tile = j >> 7;
            int n = (tile % n_tiles) * 8 + (lane >> 2);
            int k = (tile / n_tiles) * 16 + 2 * (lane & 3) + (e & 1) + 8 * (e >> 1);
            v = params[src + n * n_in + k];
        }
        else if (i < kBfT2)
        {
            int j = i - kBfT1, r = j / kGuideHidden, c = j % kGuideHidden; // W1^T[r][c] = W1[c][r]
            v = params[kW1 + c * kGuideHidden + r];
        }
        else if (i < kBfT3)
        {
            int j = i - kBfT2, r = j / kGuideHidden, c = j % kGuideHidden;
            v = params[kW2 + c * kGuideHidden + r];
        }
        else
        {
            int j = i - kBfT3, r = j / kGuideOutPad, c = j % kGuideOutPad; // W3^T[r][c] = W3[c][r]
            v = c < kGuideOut ? params[kW3 + c * kGuideHidden + r] : 0.0f;
        }
        w[i] = __float2bfloat16_rn(v);
    }
}

} // namespace

// ---------------------------------------------------------------- launches

// Grid of the persistent forward kernels: as many CTAs per SM as their shared
// memory allows (at most the 4 of their launch bounds; 4 x 64 tensor-memory
// columns fit in an SM's 512). The occupancy calculator is not used: for
// these kernels it reports one CTA per SM.
static int ForwardGrid()
{
    int dev = 0, smem_sm = 0, reserved = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    const int per = int(size_t(smem_sm) / (kFtSmem + size_t(reserved)));
    return CurrentSmCount() * std::min(4, std::max(1, per));
}

bbg_status GuideForward(bbg_guide* G, const float* raw_dev, const int32_t* index_dev, const int32_t* n_dev,
                        int64_t n_host, float* out_dev, cudaStream_t st)
{
    int grid = 0;
    BBG_TRY(GuidePrepare(G, &grid));
    GuideForwardKernel<<<grid, kFtThreads, kFtSmem, st>>>(raw_dev, index_dev, n_dev, n_host, G->bounds, G->bf16.p,
                                                          G->params.p, out_dev, G->tc_status.p);
    BBG_CUDA(cudaGetLastError());
    return BBG_OK;
}

bbg_status GuideForwardGrouped(const float* raw_dev, const int32_t* index_dev, const int32_t* chunk_start_dev,
                               int32_t n_groups, const GuideGroup* groups_dev, float* out_dev, cudaStream_t st)
{
    // Kernel attributes are per device: set once on each device that runs it.
    constexpr int kMaxDevices = 64;
    static std::mutex mutex;
    static int grid_of[kMaxDevices] = {};
    int dev = 0;
    BBG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    }
    int grid = 0;
    {
        std::lock_guard<std::mutex> lock(mutex);
        if (!grid_of[dev])
        {
            BBG_CUDA(cudaFuncSetAttribute(GuideGroupedForwardKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(kFtSmem)));
            grid_of[dev] = ForwardGrid();
        }
        grid = grid_of[dev];
    }
    if (n_groups <= 0)
    {
        return BBG_OK;
    }
    GuideGroupedForwardKernel<<<grid, kFtThreads, kFtSmem, st>>>(raw_dev, index_dev, chunk_start_dev, n_groups,
                                                                        groups_dev, out_dev);
    BBG_CUDA(cudaGetLastError());
    return BBG_OK;
}

bbg_status GuideReserveTraining(bbg_guide* G, int64_t capacity)
{
    const int64_t ld = std::max<int64_t>(16, (capacity + 15) / 16 * 16);
    BBG_TRY(G->scratch.alloc(size_t(kScratchRows) * size_t(ld)));
    const int64_t chunks = (ld + kGradChunk - 1) / kGradChunk;
    BBG_TRY(G->partial.alloc(size_t(chunks) * kGuideParams));
    return BBG_OK;
}

bbg_status GuideAccumulate(bbg_guide* G, const float* raw_dev, const float* dirs_dev, const float* weights_dev,
                           const int32_t* n_dev, int64_t n_host, int64_t capacity, cudaStream_t st)
{
    const int64_t ld = std::max<int64_t>(16, (capacity + 15) / 16 * 16);
    BBG_TRY(GuideReserveTraining(G, capacity));
    const int sms = CurrentSmCount();
    GuideTrainKernel<<<sms, 32 * kTrainWarps, kTrainSmem, st>>>(raw_dev, dirs_dev, weights_dev, n_dev, n_host,
                                                                G->bounds, G->bf16.p, G->params.p, G->scratch.p, ld,
                                                                G->grad.p, G->loss.p);
    const int64_t chunks = (ld + kGradChunk - 1) / kGradChunk;
    // One CTA per (chunk, layer); chunks past the batch exit at once.
    GuideWeightGradTcKernel<<<dim3(unsigned(chunks), 4), kTcThreads, kTcSmem, st>>>(G->scratch.p, ld, n_dev, n_host,
                                                                                     G->partial.p, G->tc_status.p);
    GuideGradReduceKernel<<<(kGuideParams + 255) / 256, 256, 0, st>>>(G->partial.p, n_dev, n_host, G->grad.p);
    BBG_CUDA(cudaGetLastError());
    return BBG_OK;
}

bbg_status GuideApply(bbg_guide* G, float lr, const int32_t* n_dev, int64_t n_host, cudaStream_t st)
{
    GuideStepKernel<<<1, 1, 0, st>>>(G->step_dev.p, n_dev, n_host);
    GuideAdamKernel<<<64, 256, 0, st>>>(G->params.p, G->adam_m.p, G->adam_v.p, G->grad.p, G->step_dev.p, lr, G->beta1,
                                        G->beta2, 1e-8f, n_dev, n_host);
    GuideConvertKernel<<<64, 256, 0, st>>>(G->params.p, G->bf16.p);
    BBG_CUDA(cudaGetLastError());
    return BBG_OK;
}

bbg_status GuideCheckStatus(bbg_guide* G)
{
    int32_t st = 0;
    BBG_CUDA(cudaMemcpy(&st, G->tc_status.p, sizeof(st), cudaMemcpyDeviceToHost));
    if (st != 0)
    {
        return Fail(BBG_ERR_TIMEOUT, "guide: a tensor-core pass (forward or weight gradients) did not complete in time");
    }
    return BBG_OK;
}

bbg_status GuidePrepare(bbg_guide* G, int* grid)
{
    if (!G->smem_set)
    {
        BBG_CUDA(cudaFuncSetAttribute(GuideForwardKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kFtSmem)));
        BBG_CUDA(cudaFuncSetAttribute(GuideTrainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTrainSmem)));
        BBG_CUDA(cudaFuncSetAttribute(GuideWeightGradTcKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(kTcSmem)));
        G->smem_set = true;
    }
    *grid = ForwardGrid();
    return BBG_OK;
}

// Xavier-style uniform initialisation of the hidden layers; the output layer
// starts near an even mixture of broad lobes toward the 8 cube diagonals.
void InitGuideParams(uint64_t seed, float* p)
{
    std::mt19937_64 rng(seed);
    auto fill = [&](int at, int fan_out, int fan_in, float scale) {
        std::uniform_real_distribution<float> u(-scale, scale);
        for (int i = 0; i < fan_out * fan_in; ++i)
        {
            p[at + i] = u(rng);
        }
    };
    fill(kW0, kGuideHidden, kGuideIn, std::sqrt(6.0f / (kGuideIn + kGuideHidden)));
    fill(kW1, kGuideHidden, kGuideHidden, std::sqrt(6.0f / (2 * kGuideHidden)));
    fill(kW2, kGuideHidden, kGuideHidden, std::sqrt(6.0f / (2 * kGuideHidden)));
    fill(kW3, kGuideOut, kGuideHidden, 1e-2f);
    for (int i = 0; i < kGuideHidden; ++i)
    {
        p[kB0 + i] = 0;
        p[kB1 + i] = 0;
        p[kB2 + i] = 0;
    }
    for (int j = 0; j < kLobes; ++j)
    {
        float sx = (j & 1) ? 1.0f : -1.0f, sy = (j & 2) ? 1.0f : -1.0f, sz = (j & 4) ? 1.0f : -1.0f;
        p[kB3 + 5 * j] = 0;
        p[kB3 + 5 * j + 1] = sx;
        p[kB3 + 5 * j + 2] = sy;
        p[kB3 + 5 * j + 3] = sz;
        p[kB3 + 5 * j + 4] = std::log(1.5f);
    }
}

} // namespace bbg

using namespace bbg;

namespace
{

bbg_status Create(const float* aabb, uint64_t seed, bbg_guide* G)
{
    BBG_TRY(CheckDevice());
    BBG_CUDA(cudaGetDevice(&G->device));
    BBG_CUDA(cudaStreamCreateWithFlags(&G->stream, cudaStreamNonBlocking));
    for (int a = 0; a < 3; ++a)
    {
        float ext = aabb[3 + a] - aabb[a];
        G->bounds.lo[a] = aabb[a];
        G->bounds.inv_extent[a] = ext > 0 ? 1.0f / ext : 0.0f;
    }
    std::vector<float> p(kGuideParams);
    InitGuideParams(seed, p.data());
    BBG_TRY(G->params.upload(p.data(), p.size(), G->stream));
    std::vector<float> zeros(kGuideParams, 0.0f);
    BBG_TRY(G->adam_m.upload(zeros.data(), zeros.size(), G->stream));
    BBG_TRY(G->adam_v.upload(zeros.data(), zeros.size(), G->stream));
    BBG_TRY(G->grad.upload(zeros.data(), zeros.size(), G->stream));
    BBG_TRY(G->loss.alloc(1));
    BBG_TRY(G->bf16.alloc(kBfBuf));
    BBG_TRY(G->step_dev.alloc(1));
    BBG_CUDA(cudaMemsetAsync(G->step_dev.p, 0, sizeof(int32_t), G->stream));
    BBG_TRY(G->tc_status.alloc(1));
    BBG_CUDA(cudaMemsetAsync(G->tc_status.p, 0, sizeof(int32_t), G->stream));
    GuideConvertKernel<<<64, 256, 0, G->stream>>>(G->params.p, G->bf16.p);
    BBG_CUDA(cudaGetLastError());
    BBG_CUDA(cudaStreamSynchronize(G->stream));
    return BBG_OK;
}

// Host buffers -> device staging.
bbg_status Stage(bbg_guide* G, const float* raw, const float* dirs, const float* weights, int64_t n)
{
    BBG_TRY(G->s_raw.upload(raw, size_t(n) * kGuideRaw, G->stream));
    if (dirs)
    {
        BBG_TRY(G->s_dirs.upload(dirs, size_t(n) * 3, G->stream));
    }
    if (weights)
    {
        BBG_TRY(G->s_w.upload(weights, size_t(n), G->stream));
    }
    return BBG_OK;
}

} // namespace

namespace bbg
{

// The vMF mixture of each output row, sampled or evaluated as the guided
// renderer does (MakeMixture, MixtureSample, MixturePdf).
__global__ void MixtureSampleKernel(const float* outputs, const float* u, int64_t n, float* dirs, float* pdf)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        VmfMixture m = MakeMixture(outputs + i * kGuideOut);
        V3 w = MixtureSample(m, u[3 * i], u[3 * i + 1], u[3 * i + 2]);
        dirs[3 * i] = w.x;
        dirs[3 * i + 1] = w.y;
        dirs[3 * i + 2] = w.z;
        pdf[i] = MixturePdf(m, w);
    }
}

__global__ void MixturePdfKernel(const float* outputs, const float* dirs, int64_t n, float* pdf)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        VmfMixture m = MakeMixture(outputs + i * kGuideOut);
        pdf[i] = MixturePdf(m, V3{ dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2] });
    }
}

// Host-buffer driver of the two kernels above: stages outputs and the
// second input (uniforms or directions), runs one of them, copies back.
bbg_status MixtureRun(const float* outputs, const float* in, int64_t n, float* dirs_out, float* pdf_out,
                      cudaStream_t st)
{
    DevBuf<float> d_out, d_in, d_dirs, d_pdf;
    BBG_TRY(d_out.upload(outputs, size_t(n) * kGuideOut, st));
    BBG_TRY(d_in.upload(in, size_t(n) * 3, st));
    BBG_TRY(d_pdf.alloc(size_t(n)));
    int grid = int(std::min<int64_t>((n + 255) / 256, 148 * 16));
    if (dirs_out)
    {
        BBG_TRY(d_dirs.alloc(size_t(n) * 3));
        MixtureSampleKernel<<<grid, 256, 0, st>>>(d_out.p, d_in.p, n, d_dirs.p, d_pdf.p);
        BBG_CUDA(cudaGetLastError());
        BBG_CUDA(cudaMemcpyAsync(dirs_out, d_dirs.p, sizeof(float) * 3 * size_t(n), cudaMemcpyDeviceToHost, st));
    }
    else
    {
        MixturePdfKernel<<<grid, 256, 0, st>>>(d_out.p, d_in.p, n, d_pdf.p);
        BBG_CUDA(cudaGetLastError());
    }
    BBG_CUDA(cudaMemcpyAsync(pdf_out, d_pdf.p, sizeof(float) * size_t(n), cudaMemcpyDeviceToHost, st));
    BBG_CUDA(cudaStreamSynchronize(st));
    return BBG_OK;
}

bbg_status MixtureCall(const float* outputs, const float* in, int64_t n, float* dirs_out, float* pdf_out)
{
    BBG_TRY(CheckDevice());
    cudaStream_t st;
    BBG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    bbg_status status = MixtureRun(outputs, in, n, dirs_out, pdf_out, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return status;
}

} // namespace bbg

namespace
{

} // namespace

extern "C" {

bbg_status bbg_guide_mixture_sample(const float* outputs, const float* u, int64_t n, float* dirs_out, float* pdf_out)
{
    if (n < 0 || (n > 0 && (!outputs || !u || !dirs_out || !pdf_out)))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_guide_mixture_sample: bad argument");
    }
    return n == 0 ? BBG_OK : MixtureCall(outputs, u, n, dirs_out, pdf_out);
}

bbg_status bbg_guide_mixture_pdf(const float* outputs, const float* dirs, int64_t n, float* pdf_out)
{
    if (n < 0 || (n > 0 && (!outputs || !dirs || !pdf_out)))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_guide_mixture_pdf: bad argument");
    }
    return n == 0 ? BBG_OK : MixtureCall(outputs, dirs, n, nullptr, pdf_out);
}

bbg_status bbg_guide_create(const float* scene_aabb, uint64_t seed, bbg_guide** out)
{
    if (!scene_aabb || !out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_guide_create: bad argument");
    }
    *out = nullptr;
    auto* G = new bbg_guide;
    bbg_status s = Create(scene_aabb, seed, G);
    if (s != BBG_OK)
    {
        delete G;
        return s;
    }
    *out = G;
    return BBG_OK;
}

bbg_status bbg_guide_destroy(bbg_guide* G)
{
    if (!G)
    {
        return BBG_OK;
    }
    DeviceScope ds(G->device);
    delete G;
    return BBG_OK;
}

bbg_status bbg_guide_get_params(bbg_guide* G, float* out)
{
    if (!G || !out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_guide_get_params: bad argument");
    }
    DeviceScope ds(G->device);
    BBG_CUDA(cudaStreamSynchronize(G->stream));
    BBG_CUDA(cudaMemcpy(out, G->params.p, sizeof(float) * kGuideParams, cudaMemcpyDeviceToHost));
    return BBG_OK;
}

bbg_status bbg_guide_set_params(bbg_guide* G, const float* in)
{
    if (!G || !in)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_guide_set_params: bad argument");
    }
    DeviceScope ds(G->device);
    BBG_CUDA(cudaMemcpy(G->params.p, in, sizeof(float) * kGuideParams, cudaMemcpyHostToDevice));
    GuideConvertKernel<<<64, 256, 0, G->stream>>>(G->params.p, G->bf16.p);
    BBG_CUDA(cudaStreamSynchronize(G->stream));
    return BBG_OK;
}

bbg_status bbg_guide_forward(bbg_guide* G, const float* raw, int64_t n, float* out)
{
    if (!G || n < 0 || (n > 0 && (!raw || !out)))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_guide_forward: bad argument");
    }
    DeviceScope ds(G->device);
    if (n == 0)
    {
        return BBG_OK;
    }
    BBG_TRY(Stage(G, raw, nullptr, nullptr, n));
    BBG_TRY(G->s_out.alloc(size_t(n) * kGuideOut));
    BBG_TRY(GuideForward(G, G->s_raw.p, nullptr, nullptr, n, G->s_out.p, G->stream));
    BBG_CUDA(cudaMemcpyAsync(out, G->s_out.p, sizeof(float) * size_t(n) * kGuideOut, cudaMemcpyDeviceToHost,
                             G->stream));
    BBG_CUDA(cudaStreamSynchronize(G->stream));
    return BBG_OK;
}

bbg_status bbg_guide_gradient(bbg_guide* G, const float* raw, const float* dirs, const float* weights, int64_t n,
                              float* grad_out, float* loss_out)
{
    if (!G || n <= 0 || !raw || !dirs || !weights || !grad_out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_guide_gradient: bad argument");
    }
    DeviceScope ds(G->device);
    int dummy;
    BBG_TRY(GuidePrepare(G, &dummy));
    BBG_TRY(Stage(G, raw, dirs, weights, n));
    BBG_CUDA(cudaMemsetAsync(G->grad.p, 0, sizeof(float) * kGuideParams, G->stream));
    BBG_CUDA(cudaMemsetAsync(G->loss.p, 0, sizeof(float), G->stream));
    BBG_TRY(GuideAccumulate(G, G->s_raw.p, G->s_dirs.p, G->s_w.p, nullptr, n, n, G->stream));
    BBG_CUDA(cudaMemcpyAsync(grad_out, G->grad.p, sizeof(float) * kGuideParams, cudaMemcpyDeviceToHost, G->stream));
    float loss = 0;
    BBG_CUDA(cudaMemcpyAsync(&loss, G->loss.p, sizeof(float), cudaMemcpyDeviceToHost, G->stream));
    BBG_CUDA(cudaMemsetAsync(G->grad.p, 0, sizeof(float) * kGuideParams, G->stream));
    BBG_CUDA(cudaStreamSynchronize(G->stream));
    BBG_TRY(GuideCheckStatus(G));
    if (loss_out)
    {
        *loss_out = loss;
    }
    return BBG_OK;
}

bbg_status bbg_guide_train_step(bbg_guide* G, const float* raw, const float* dirs, const float* weights, int64_t n,
                                float learning_rate, float* loss_out)
{
    if (!G || n <= 0 || !raw || !dirs || !weights)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_guide_train_step: bad argument");
    }
    DeviceScope ds(G->device);
    int dummy;
    BBG_TRY(GuidePrepare(G, &dummy));
    BBG_TRY(Stage(G, raw, dirs, weights, n));
    BBG_CUDA(cudaMemsetAsync(G->loss.p, 0, sizeof(float), G->stream));
    BBG_TRY(GuideAccumulate(G, G->s_raw.p, G->s_dirs.p, G->s_w.p, nullptr, n, n, G->stream));
    BBG_TRY(GuideApply(G, learning_rate, nullptr, n, G->stream));
    float loss = 0;
    BBG_CUDA(cudaMemcpyAsync(&loss, G->loss.p, sizeof(float), cudaMemcpyDeviceToHost, G->stream));
    BBG_CUDA(cudaStreamSynchronize(G->stream));
    BBG_TRY(GuideCheckStatus(G));
    if (loss_out)
    {
        *loss_out = loss / float(n);
    }
    return BBG_OK;
}

} // extern "C"
