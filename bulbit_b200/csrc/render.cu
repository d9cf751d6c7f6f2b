// Wavefront path tracer: PathIntegrator::Li (src/integrator/path_integrator.cpp:26-196)
// recast as queues on the device.
//
// A render is a sequence of waves; a wave holds whole pixels (all their
// samples), one path per slot, slot = path index - wave base, path index =
// (y*W + x)*spp + sample. Per wave:
//   Raygen     seed each path's sampler and sample its camera ray
//   repeat max_bounces + 1 times (one bounce level per iteration):
//     Closest  closest hit of every path in the ray queue
//     Shade    miss / emission MIS, bounce limit, BSDF, next-event estimation
//              (enqueues a shadow ray with its full contribution), BSDF
//              sample, Russian roulette; survivors go to the next ray queue
//     Shadow   any-hit for each shadow ray; if unoccluded L += contribution
//   Film       per pixel, its samples in order, as Film::AddSample does
// The order of additions to each path's L is the reference's (emission of
// vertex k, then its direct light, then vertex k+1), so L agrees up to the
// transcendental functions. Kernels read their queue lengths from device
// memory, so a wave's launches are captured once as a CUDA graph and replayed.

#include "accel.cuh"
#include "dev_bsdf.cuh"
#include "dev_lights.cuh"
#include "guide.cuh"

#include <algorithm>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

namespace bbg
{

constexpr int kBlock = 128;
// Shading kernels are held to 128 registers (4 blocks of kBlock per SM): the
// BSDF dispatch would otherwise take 168 with spills, at 3 blocks per SM.
#ifndef BBG_SHADE_MIN_BLOCKS
#define BBG_SHADE_MIN_BLOCKS 4
#endif

struct SceneDev
{
    AccelView accel;
    const int4* prim_info; // kind, index, material, area light
    const int32_t* tri_indices;
    const float* positions;
    const float* normals;
    const float* tangents;
    const bbg_sphere* spheres;
    const MaterialDev* materials;
    const LightDev* lights;
    const float* light_func;
    const float* light_cdf;
    const float* light_pmf;  // EvaluatePMF per light
    const float* alias_prob;
    const int32_t* alias_idx;
    const int32_t* infinite;  // infinite light indices, in light order
    int32_t n_lights;
    int32_t n_infinite;
    float light_func_integral;
    int32_t light_alias;
    int32_t max_bounces;
    int32_t rr_min_bounces;
    int32_t regularize;
    int32_t spp;
    int32_t seed;
    int32_t sampler_kind; // BBG_SAMPLER_*
    int32_t x_samples;    // stratified: strata along x
    int32_t jitter;       // stratified: jitter within strata
    CameraDev camera;
};

// Per-wave device state (structure of arrays, one entry per slot).
struct WaveDev
{
    float4* o_pdf;   // ray origin, prev_bsdf_pdf
    float4* d_eta;   // ray direction, eta_scale
    float4* beta;    // throughput
    float4* L;       // radiance
    uint64_t* rng;   // PCG32 state
    int32_t* flags;  // bounce | specular << 16 | any_non_specular << 17
    float4* hit;     // prim bits, t, u, v
    int32_t* queue[2];
    float4* sh_o;    // shadow ray origin, t_max
    float4* sh_d;    // shadow ray direction, slot bits
    float4* sh_c;    // contribution
    int32_t* counts; // [0],[1] ray queues, [2] shadow queue, [3],[4] work counters
    unsigned long long* stats; // closest rays, shadow rays
    const int64_t* wave;       // [0] first path, [1] paths in wave
    int32_t* dim;              // stratified sampler: next dimension per slot
    // Shading order (null sorted: queue order): each level's queue sorted by
    // shading kind into `sorted` through per-position keys and kind counts.
    int32_t* sorted;
    uint8_t* keys;
    int32_t* sort_counts; // [0, kShadeKinds) totals, [kShadeKinds, 2 kShadeKinds) cursors
};

// Shading kinds a level's paths are grouped by: escaped, no material, then
// each material type with and without energy compensation.
constexpr int kShadeKinds = 2 + 2 * 4;

constexpr int32_t kSpecularBit = 1 << 16;
constexpr int32_t kAnyNonSpecularBit = 1 << 17;
// flags bits 20-30: the path's scene within a batch of scenes.
constexpr int32_t kSceneShift = 20;
constexpr int32_t kSceneMask = 0x7ff << kSceneShift;
constexpr int32_t kMaxBatchScenes = 0x800;
// Largest batch rendered with guides (one guide per scene).
constexpr int32_t kMaxGuidedScenes = 64;
// Device memory per path slot of a wave (bbg_integrator::Reserve): eight
// float4 records, the sampler state, five int32 arrays and a sort key.
constexpr double kWaveBytesPerPath = 8 * 16 + 8 + 5 * 4 + 1;
// Extra levels after max_bounces + 1 for paths crossing material-less
// surfaces, unless bbg_render_params.pass_through_levels sets another cap.
constexpr int kMaxPassThroughLevels = 4096;

struct FilmDev
{
    float* rgb_sum;
    int32_t* count;
    float* moments;
    float* path_L; // optional
};

// The scenes a render's kernels see. OneScene: a single scene, passed as
// kernel parameters (every path's scene bits are 0). SceneTable: several
// scenes rendered together; per-scene descriptors and films live in device
// memory, the batch's pixels are the scenes' pixels one scene after another
// (pixel_start: prefix sums), and every scene has the same spp.
struct OneScene
{
    SceneDev s;
    FilmDev f;
    __device__ __forceinline__ const SceneDev& Scene(int32_t) const { return s; }
    __device__ __forceinline__ const FilmDev& Film(int32_t) const { return f; }
    __device__ __forceinline__ int32_t Spp() const { return s.spp; }
    __device__ __forceinline__ int32_t Locate(int64_t pixel, int64_t* local) const
    {
        *local = pixel;
        return 0;
    }
};

struct SceneTable
{
    const SceneDev* scenes;
    const FilmDev* films;
    const int64_t* pixel_start; // n + 1 entries
    int32_t n;
    int32_t spp;
    __device__ __forceinline__ const SceneDev& Scene(int32_t i) const { return scenes[i]; }
    __device__ __forceinline__ const FilmDev& Film(int32_t i) const { return films[i]; }
    __device__ __forceinline__ int32_t Spp() const { return spp; }
    __device__ __forceinline__ int32_t Locate(int64_t pixel, int64_t* local) const
    {
        int32_t lo = 0, hi = n - 1;
        while (lo < hi)
        {
            int32_t mid = (lo + hi + 1) >> 1;
            if (pixel_start[mid] <= pixel)
            {
                lo = mid;
            }
            else
            {
                hi = mid - 1;
            }
        }
        *local = pixel - pixel_start[lo];
        return lo;
    }
};

template <class Scenes>
constexpr bool kIsBatch = std::is_same_v<Scenes, SceneTable>;

// Warp-aggregated append of `pred` lanes to a queue counter.
__device__ __forceinline__ int32_t Append(int32_t* counter, bool pred)
{
    unsigned active = __activemask();
    unsigned m = __ballot_sync(active, pred);
    int lane = threadIdx.x & 31;
    int leader = __ffs(active) - 1;
    int32_t base = 0;
    if (lane == leader && m)
    {
        base = atomicAdd(counter, __popc(m));
    }
    base = __shfl_sync(active, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

// The sampler of the path in `slot` (PathSampler), and its write-back. A
// stratified sampler needs the path's pixel and sample (single-scene renders).
__device__ __forceinline__ PathSampler LoadSampler(const SceneDev& s, const WaveDev& w, int32_t slot)
{
    PathSampler p{};
    p.state = w.rng[slot];
    p.stratified = s.sampler_kind == BBG_SAMPLER_STRATIFIED;
    if (p.stratified)
    {
        int64_t path = w.wave[0] + slot;
        int64_t pixel = path / s.spp;
        p.sample = int32_t(path % s.spp);
        p.px = int32_t(pixel % s.camera.width);
        p.py = int32_t(pixel / s.camera.width);
        p.dim = w.dim[slot];
        p.seed = s.seed;
        p.spp = s.spp;
        p.x_samples = s.x_samples;
        p.jitter = s.jitter;
    }
    return p;
}

__device__ __forceinline__ void StoreSampler(const WaveDev& w, int32_t slot, const PathSampler& p)
{
    w.rng[slot] = p.state;
    if (p.stratified)
    {
        w.dim[slot] = p.dim;
    }
}

// Distribution1D::SampleContinuous over a CDF of n + 1 entries
// (include/bulbit/sampling.h:375-393): FindInterval, then the linear offset.
__device__ __forceinline__ float CdfSampleContinuous(const float* cdf, int32_t n, float u, int32_t* off)
{
    int32_t size = n + 1;
    int32_t first = 0, len = size;
    while (len > 0)
    {
        int32_t half = len >> 1, middle = first + half;
        if (cdf[middle] <= u)
        {
            first = middle + 1;
            len -= half + 1;
        }
        else
        {
            len = half;
        }
    }
    int32_t offset = first - 1;
    offset = offset < 0 ? 0 : (offset > size - 2 ? size - 2 : offset);
    *off = offset;
    float du = (u - cdf[offset]) / (cdf[offset + 1] - cdf[offset]);
    return (float(offset) + du) / float(n);
}

// Filter::Sample for the camera's filter (src/reconstruction/box_filter.cpp:17-21,
// tent_filter.cpp:21-29, gaussian_filter.cpp:40-43: Distribution2D::SampleContinuous,
// the marginal over rows first).
__device__ __forceinline__ P2 FilterSample(const CameraDev& c, P2 u)
{
    const float e = c.filter_extent;
    if (c.filter_type == BBG_FILTER_GAUSSIAN)
    {
        int32_t v, dummy;
        float d1 = CdfSampleContinuous(c.filter_cdf, kFilterTable, u.y, &v);
        float d0 = CdfSampleContinuous(c.filter_cdf + (kFilterTable + 1) * (v + 1), kFilterTable, u.x, &dummy);
        return P2{ d0 * e - e / 2, d1 * e - e / 2 };
    }
    if (c.filter_type == BBG_FILTER_TENT)
    {
        float h = e / 2;
        float x = u.x < 0.5f ? h * (sqrtf(2 * u.x) - 1) : h * (1 - sqrtf(1 - 2 * (u.x - 0.5f)));
        float y = u.y < 0.5f ? h * (sqrtf(2 * u.y) - 1) : h * (1 - sqrtf(1 - 2 * (u.y - 0.5f)));
        return P2{ x, y };
    }
    // BoxFilter: (2u - 1) * extent / 2.
    return P2{ (u.x * 2 - 1) * e / 2, (u.y * 2 - 1) * e / 2 };
}

// ---------------------------------------------------------------- raygen

// Render loop body (src/integrator/integrator.cpp:185-190) and
// PerspectiveCamera::SampleRay (src/camera/perspective_camera.cpp:40-52).
template <class Scenes>
__global__ void __launch_bounds__(kBlock) RaygenKernel(Scenes sc, WaveDev w)
{
    const int64_t base = w.wave[0];
    const int64_t n = w.wave[1];
    const int32_t spp = sc.Spp();
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t path = base + i;
        int32_t sample = int32_t(path % spp);
        int64_t pixel;
        int32_t scene = sc.Locate(path / spp, &pixel);
        const SceneDev& s = sc.Scene(scene);
        const CameraDev& c = s.camera;
        int32_t px = int32_t(pixel % c.width);
        int32_t py = int32_t(pixel / c.width);
        PathSampler rng{};
        rng.state = SamplerStart(px, py, s.seed, sample);
        rng.stratified = s.sampler_kind == BBG_SAMPLER_STRATIFIED;
        rng.px = px;
        rng.py = py;
        rng.sample = sample;
        rng.seed = s.seed;
        rng.spp = s.spp;
        rng.x_samples = s.x_samples;
        rng.jitter = s.jitter;
        P2 u1 = Next2D(rng); // lens sample: the right-hand argument, drawn first
        P2 u0 = Next2D(rng); // filter sample

        // pixel offset = filter->Sample(u0) + 0.5.
        P2 f = FilterSample(c, u0);
        P2 off{ f.x + 0.5f, f.y + 0.5f };
        V3 pixel_center = load3(c.lower_left) + load3(c.horizontal) * (px + off.x) / float(c.width) +
                          load3(c.vertical) * (py + off.y) / float(c.height);
        P2 disk = SampleUniformUnitDiskConcentric(u1);
        P2 aperture{ disk.x * c.lens_radius, disk.y * c.lens_radius };
        V3 offset = load3(c.u) * aperture.x + load3(c.v) * aperture.y;
        V3 origin = load3(c.origin) + offset;
        V3 d = Normalize(pixel_center - origin);

        w.o_pdf[i] = make_float4(origin.x, origin.y, origin.z, 0.0f);
        w.d_eta[i] = make_float4(d.x, d.y, d.z, 1.0f);
        w.beta[i] = make_float4(1, 1, 1, 0);
        w.L[i] = make_float4(0, 0, 0, 0);
        w.rng[i] = rng.state;
        if (rng.stratified)
        {
            w.dim[i] = rng.dim;
        }
        w.flags[i] = scene << kSceneShift;
        w.queue[0][i] = int32_t(i);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        w.counts[0] = int32_t(n);
        w.counts[1] = 0;
        w.counts[2] = 0;
    }
}

// ---------------------------------------------------------------- intersect
//
// In a batch, each work item is traced in its own scene's tree (View).

// Work items of the closest-hit pass: queue entry j -> its path's ray.
struct ClosestSrc
{
    const int32_t* q;
    const float4* o_pdf;
    const float4* d_eta;
    float4* hit;

    __device__ __forceinline__ void Load(int32_t j, RayQ* rq, float* t_min, float* t_max) const
    {
        int32_t slot = q[j];
        float4 o = o_pdf[slot];
        float4 d = d_eta[slot];
        *rq = MakeRayQ(V3{ o.x, o.y, o.z }, V3{ d.x, d.y, d.z });
        *t_min = kRayEpsilon;
        *t_max = INFINITY;
    }
    __device__ __forceinline__ void Store(int32_t j, const TraceResult& r) const
    {
        hit[q[j]] = make_float4(__int_as_float(r.prim), r.t, r.u, r.v);
    }
};

// Work items of the shadow pass: an unoccluded shadow ray adds its
// contribution to its path's radiance.
struct ShadowSrc
{
    const float4* sh_o;
    const float4* sh_d;
    const float4* sh_c;
    float4* L;

    __device__ __forceinline__ void Load(int32_t j, RayQ* rq, float* t_min, float* t_max) const
    {
        float4 o = sh_o[j];
        float4 d = sh_d[j];
        *rq = MakeRayQ(V3{ o.x, o.y, o.z }, V3{ d.x, d.y, d.z });
        *t_min = kRayEpsilon;
        *t_max = o.w;
    }
    __device__ __forceinline__ void Store(int32_t j, const TraceResult& r) const
    {
        if (r.prim < 0)
        {
            int32_t slot = __float_as_int(sh_d[j].w);
            float4 c = sh_c[j];
            float4 l = L[slot];
            L[slot] = make_float4(l.x + c.x, l.y + c.y, l.z + c.z, 0.0f);
        }
    }
};

struct ClosestBatchSrc : ClosestSrc
{
    const int32_t* flags;
    const SceneDev* scenes;
    __device__ __forceinline__ AccelView View(int32_t j) const { return scenes[flags[q[j]] >> kSceneShift].accel; }
};

struct ShadowBatchSrc : ShadowSrc
{
    const int32_t* flags;
    const SceneDev* scenes;
    __device__ __forceinline__ AccelView View(int32_t j) const
    {
        return scenes[flags[__float_as_int(sh_d[j].w)] >> kSceneShift].accel;
    }
};

// Launch shapes of the traversal passes the autotuner chooses from: threads
// per block and stack entries per thread kept in shared memory (0: the
// whole traversal stack in local memory). A trace shape passed to the launch
// functions is a shape index, plus kNumShapes when the tree's 8-wide layout is
// traversed (2 kNumShapes when that tree holds triangles only: kernels without
// the sphere test, fewer registers per thread).
struct TraversalShape
{
    int block;
    int short_stack;
};
constexpr int kNumShapes = 4;
constexpr TraversalShape kShapes[kNumShapes] = { { 128, 16 }, { 128, 0 }, { 128, 8 }, { 256, 16 } };

template <class Scenes, int BLOCK = kBlock, int SHORT = kShortStack, bool WIDE = false, bool SPHERES = true>
__global__ void __launch_bounds__(BLOCK) ClosestKernel(Scenes sc, WaveDev w, int parity)
{
    const int32_t n = w.counts[parity];
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        atomicAdd(w.stats, (unsigned long long)n);
    }
    const SceneDev& s = sc.Scene(0);
    if constexpr (kIsBatch<Scenes>)
    {
        // Every scene of a batch uses the ordered traversal, all over the same
        // layout (checked on the host).
        ClosestBatchSrc src{ { w.queue[parity], w.o_pdf, w.d_eta, w.hit }, w.flags, sc.scenes };
        if constexpr (WIDE)
        {
            TracePersistentWide<false, ClosestBatchSrc, BLOCK, SHORT, SPHERES>(s.accel, n, w.counts + 3, src);
        }
        else
        {
            TracePersistent<false, ClosestBatchSrc, BLOCK, SHORT>(s.accel, n, w.counts + 3, src);
        }
        return;
    }
    ClosestSrc src{ w.queue[parity], w.o_pdf, w.d_eta, w.hit };
    if constexpr (WIDE)
    {
        TracePersistentWide<false, ClosestSrc, BLOCK, SHORT, SPHERES>(s.accel, n, w.counts + 3, src);
        return;
    }
    if (s.accel.ordered)
    {
        TracePersistent<false, ClosestSrc, BLOCK, SHORT>(s.accel, n, w.counts + 3, src);
        return;
    }
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        RayQ rq;
        float t_min, t_max;
        src.Load(j, &rq, &t_min, &t_max);
        src.Store(j, TraceReference<false, false>(s.accel, rq, t_min, t_max));
    }
}

template <class Scenes, int BLOCK = kBlock, int SHORT = kShortStack, bool WIDE = false, bool SPHERES = true>
__global__ void __launch_bounds__(BLOCK) ShadowKernel(Scenes sc, WaveDev w)
{
    const int32_t n = w.counts[2];
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        atomicAdd(w.stats + 1, (unsigned long long)n);
    }
    const SceneDev& s = sc.Scene(0);
    if constexpr (kIsBatch<Scenes>)
    {
        ShadowBatchSrc src{ { w.sh_o, w.sh_d, w.sh_c, w.L }, w.flags, sc.scenes };
        if constexpr (WIDE)
        {
            TracePersistentWide<true, ShadowBatchSrc, BLOCK, SHORT, SPHERES>(s.accel, n, w.counts + 4, src);
        }
        else
        {
            TracePersistent<true, ShadowBatchSrc, BLOCK, SHORT>(s.accel, n, w.counts + 4, src);
        }
        return;
    }
    ShadowSrc src{ w.sh_o, w.sh_d, w.sh_c, w.L };
    if constexpr (WIDE)
    {
        TracePersistentWide<true, ShadowSrc, BLOCK, SHORT, SPHERES>(s.accel, n, w.counts + 4, src);
        return;
    }
    if (s.accel.ordered)
    {
        TracePersistent<true, ShadowSrc, BLOCK, SHORT>(s.accel, n, w.counts + 4, src);
        return;
    }
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        RayQ rq;
        float t_min, t_max;
        src.Load(j, &rq, &t_min, &t_max);
        src.Store(j, TraceReference<true, false>(s.accel, rq, t_min, t_max));
    }
}

// ---------------------------------------------------------------- shading

struct Isect
{
    V3 point;
    V3 normal;  // geometric, facing the incoming ray
    V3 sn, st;  // shading normal / tangent
    bool front_face;
    float t;
};

// SetFaceNormal (include/bulbit/shape.h:32-43).
__device__ __forceinline__ void SetFaceNormal(Isect* is, V3 ray_d, V3 outward, V3 sn, V3 st)
{
    bool front_face = Dot(ray_d, outward) < 0;
    float sign = front_face ? 1.0f : -1.0f;
    is->front_face = front_face;
    is->normal = sign * outward;
    is->sn = sign * sn;
    is->st = sign * st;
}

__device__ __forceinline__ void TriVerts(const SceneDev& s, int32_t tri, int32_t v[3], V3 p[3])
{
    v[0] = s.tri_indices[3 * tri];
    v[1] = s.tri_indices[3 * tri + 1];
    v[2] = s.tri_indices[3 * tri + 2];
    for (int k = 0; k < 3; ++k)
    {
        p[k] = load3(s.positions + 3 * size_t(v[k]));
    }
}

// Triangle::Intersect hit record (src/geometry/triangle.cpp:96-109) and
// Sphere::Intersect hit record (src/geometry/sphere.cpp:63-84).
__device__ __forceinline__ Isect MakeIsect(const SceneDev& s, int4 info, float4 hit, V3 ro, V3 rd)
{
    Isect is;
    is.t = hit.y;
    if (info.x == BBG_PRIM_TRIANGLE)
    {
        int32_t v[3];
        V3 p[3];
        TriVerts(s, info.y, v, p);
        float u = hit.z, vv = hit.w;
        float ww = 1 - u - vv;
        is.point = ro + rd * is.t;
        V3 e1 = p[1] - p[0];
        V3 e2 = p[2] - p[0];
        V3 normal = Normalize(Cross(e1, e2));
        V3 n0 = load3(s.normals + 3 * size_t(v[0])), n1 = load3(s.normals + 3 * size_t(v[1])),
           n2 = load3(s.normals + 3 * size_t(v[2]));
        V3 t0 = load3(s.tangents + 3 * size_t(v[0])), t1 = load3(s.tangents + 3 * size_t(v[1])),
           t2 = load3(s.tangents + 3 * size_t(v[2]));
        V3 sn = Normalize(ww * n0 + u * n1 + vv * n2);
        V3 st = Normalize(ww * t0 + u * t1 + vv * t2);
        SetFaceNormal(&is, rd, normal, sn, st);
    }
    else
    {
        const bbg_sphere& sp = s.spheres[info.y];
        V3 c = load3(sp.p), sc = load3(sp.s);
        float4 q = make_float4(sp.q[0], sp.q[1], sp.q[2], sp.q[3]);
        V3 lo = QuatRotateInv(q, ro - c) / sc;
        V3 ld = QuatRotateInv(q, rd / sc);
        V3 point = lo + ld * is.t;
        V3 normal = Normalize(point / sp.radius);
        is.point = QuatRotate(q, sc * point) + c;
        V3 n = QuatRotate(q, normal);
        V3 t;
        if (n.y < 1 - 1e-4f)
        {
            t = Normalize(Cross(V3{ 0, 1, 0 }, n));
        }
        else
        {
            t = Normalize(Cross(n, V3{ 1, 0, 0 }));
        }
        SetFaceNormal(&is, rd, n, n, t);
    }
    return is;
}

// Shape::PDF(isect, ray) for MIS on emitted light
// (src/geometry/triangle.cpp:247-253, src/geometry/sphere.cpp:181-189).
__device__ __forceinline__ float ShapePdf(const SceneDev& s, int4 info, const Isect& is, V3 ro, V3 rd)
{
    if (info.x == BBG_PRIM_TRIANGLE)
    {
        int32_t v[3];
        V3 p[3];
        TriVerts(s, info.y, v, p);
        float distance_squared = is.t * is.t * Length2(rd);
        float cosine = fabsf(Dot(rd, is.normal) / Length(rd));
        float area = 0.5f * Length(Cross(p[1] - p[0], p[2] - p[0]));
        return distance_squared / (cosine * area);
    }
    const bbg_sphere& sp = s.spheres[info.y];
    float distance_squared = Length2(load3(sp.p) - ro);
    float cos_theta_max = sqrtf(1 - sp.radius * sp.radius / distance_squared);
    float solid_angle = kTwoPi * (1 - cos_theta_max);
    return 1 / solid_angle;
}

// PowerLightSampler::Sample: Distribution1D::SampleDiscrete by FindInterval
// (include/bulbit/sampling.h:395-410, include/bulbit/math.h:117-134), or the
// alias table when enabled.
__device__ __forceinline__ int32_t SampleLight(const SceneDev& s, float u, float* pmf)
{
    int32_t n = s.n_lights;
    if (s.light_alias)
    {
        float x = u * n;
        int32_t i = min(int32_t(x), n - 1);
        float frac = x - i;
        int32_t k = frac < s.alias_prob[i] ? i : s.alias_idx[i];
        *pmf = s.light_pmf[k];
        return k;
    }
    int32_t size = n + 1;
    int32_t first = 0, len = size;
    while (len > 0)
    {
        int32_t half = len >> 1, middle = first + half;
        if (s.light_cdf[middle] <= u)
        {
            first = middle + 1;
            len -= half + 1;
        }
        else
        {
            len = half;
        }
    }
    int32_t offset = first - 1;
    offset = offset < 0 ? 0 : (offset > size - 2 ? size - 2 : offset);
    *pmf = s.light_func[offset] / (s.light_func_integral * n);
    return offset;
}

template <class Scenes>
__global__ void __launch_bounds__(kBlock, BBG_SHADE_MIN_BLOCKS) ShadeKernel(Scenes sc, WaveDev w, int parity)
{
    const int32_t* q = w.sorted ? w.sorted : w.queue[parity];
    int32_t* q_next = w.queue[parity ^ 1];
    const int32_t n = w.counts[parity];

    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        int32_t slot = q[j];
        float4 o4 = w.o_pdf[slot], d4 = w.d_eta[slot], b4 = w.beta[slot], L4 = w.L[slot];
        float4 hit = w.hit[slot];
        V3 ro{ o4.x, o4.y, o4.z }, rd{ d4.x, d4.y, d4.z };
        float prev_bsdf_pdf = o4.w, eta_scale = d4.w;
        Spec beta{ b4.x, b4.y, b4.z }, L{ L4.x, L4.y, L4.z };
        int32_t fl = w.flags[slot];
        const SceneDev& s = sc.Scene(fl >> kSceneShift);
        PathSampler rng = LoadSampler(s, w, slot);
        int32_t bounce = fl & 0xffff;
        bool specular_bounce = (fl & kSpecularBit) != 0;
        bool any_non_specular = (fl & kAnyNonSpecularBit) != 0;

        bool cont = false;       // path continues to the next bounce
        bool shadow = false;     // a shadow ray was generated
        V3 sh_o{}, sh_d{};
        float sh_t = 0;
        Spec sh_c{};

        int32_t prim = __float_as_int(hit.x);
        if (prim < 0)
        {
            // Escaped: infinite lights (path_integrator.cpp:41-63).
            for (int32_t k = 0; k < s.n_infinite; ++k)
            {
                const LightDev& l = s.lights[s.infinite[k]];
                Spec Le = l.scale * Spec{ l.L[0], l.L[1], l.L[2] };
                if (bounce == 0 || specular_bounce)
                {
                    L = L + beta * Le;
                }
                else
                {
                    float light_pdf = kInvFourPi * s.light_pmf[s.infinite[k]];
                    float mis_weight = PowerHeuristic(prev_bsdf_pdf, light_pdf);
                    L = L + beta * mis_weight * Le;
                }
            }
        }
        else
        {
            int4 info = s.prim_info[prim];
            Isect is = MakeIsect(s, info, hit, ro, rd);
            V3 wo = Normalize(-rd);

            // Emission from an area light (path_integrator.cpp:67-84).
            if (info.w >= 0)
            {
                const LightDev& l = s.lights[info.w];
                Spec Le = (is.front_face || l.two_sided) ? Spec{ l.L[0], l.L[1], l.L[2] } : spec(0);
                if (!IsBlack(Le))
                {
                    if (bounce == 0 || specular_bounce)
                    {
                        L = L + beta * Le;
                    }
                    else
                    {
                        float light_pdf = ShapePdf(s, info, is, ro, rd) * s.light_pmf[info.w];
                        float mis_weight = PowerHeuristic(prev_bsdf_pdf, light_pdf);
                        L = L + beta * mis_weight * Le;
                    }
                }
            }

            if (bounce++ >= s.max_bounces)
            {
                // terminated
            }
            else if (info.z < 0)
            {
                // No material: a medium boundary; continue straight through
                // without counting a bounce (path_integrator.cpp:95-100).
                ro = is.point;
                rd = -wo;
                --bounce;
                cont = true;
            }
            else
            {
                BSDF bsdf = MakeBSDF(s.materials[info.z], is.sn, is.st, is.front_face);
                if (s.regularize && any_non_specular)
                {
                    bsdf.mf.Regularize();
                    if (bsdf.type == BBG_MAT_CONDUCTOR)
                    {
                        bsdf.flags = bsdf.mf.EffectivelySmooth() ? (kFlagSpecular | kFlagReflection)
                                                                 : (kFlagGlossy | kFlagReflection);
                    }
                    else if (bsdf.type == BBG_MAT_DIELECTRIC)
                    {
                        int32_t f = (bsdf.eta == 1) ? kFlagTransmission : (kFlagReflection | kFlagTransmission);
                        bsdf.flags = f | (bsdf.mf.EffectivelySmooth() ? kFlagSpecular : kFlagGlossy);
                    }
                }

                // Next-event estimation (PathIntegrator::SampleDirectLight).
                if (IsNonSpecular(bsdf.flags))
                {
                    float u0 = Next1D(rng);
                    P2 u12 = Next2D(rng);
                    if (s.n_lights > 0)
                    {
                        float pmf;
                        int32_t li = SampleLight(s, u0, &pmf);
                        const LightDev& l = s.lights[li];
                        V3 tri[3];
                        const bbg_sphere* sph = nullptr;
                        bool on_tri = false;
                        if (l.type == BBG_LIGHT_DIFFUSE_AREA)
                        {
                            int4 linfo = s.prim_info[l.prim];
                            if (linfo.x == BBG_PRIM_TRIANGLE)
                            {
                                int32_t v[3];
                                TriVerts(s, linfo.y, v, tri);
                                on_tri = true;
                            }
                            else
                            {
                                sph = &s.spheres[linfo.y];
                            }
                        }
                        LightSampleLi ls;
                        if (SampleLi(l, is.point, u12, on_tri ? tri : nullptr, sph, &ls))
                        {
                            float bsdf_pdf = bsdf.PDF(wo, ls.wi);
                            if (!(IsBlack(ls.Li) || bsdf_pdf == 0))
                            {
                                float light_pdf = pmf * ls.pdf;
                                Spec f_cos = bsdf.F(wo, ls.wi) * AbsDot(is.sn, ls.wi);
                                if (IsDeltaLight(l.type))
                                {
                                    sh_c = beta * ls.Li * f_cos / light_pdf;
                                }
                                else
                                {
                                    float mis_weight = PowerHeuristic(light_pdf, bsdf_pdf);
                                    sh_c = beta * mis_weight * ls.Li * f_cos / light_pdf;
                                }
                                shadow = true;
                                sh_o = is.point;
                                sh_d = ls.wi;
                                sh_t = ls.visibility;
                            }
                        }
                    }
                }

                // BSDF sample: Next2D (right argument) before Next1D.
                P2 u12 = Next2D(rng);
                float u0 = Next1D(rng);
                BSDFSample bs;
                if (bsdf.Sample(&bs, wo, u0, u12))
                {
                    bool spec_sample = (bs.flags & kFlagSpecular) != 0;
                    specular_bounce = spec_sample;
                    any_non_specular = any_non_specular || !spec_sample;
                    if (bs.flags & kFlagTransmission)
                    {
                        eta_scale *= Sqr(bs.eta);
                    }
                    prev_bsdf_pdf = bs.pdf;
                    beta = beta * (bs.f * AbsDot(is.sn, bs.wi) / bs.pdf);
                    ro = is.point;
                    rd = bs.wi;
                    cont = true;

                    // Russian roulette (path_integrator.cpp:133-146).
                    if (bounce > s.rr_min_bounces)
                    {
                        float p = MaxComponent(beta) * eta_scale;
                        if (p < 1)
                        {
                            if (Next1D(rng) > p)
                            {
                                cont = false;
                            }
                            else
                            {
                                beta = beta / p;
                            }
                        }
                    }
                }
            }
        }

        w.L[slot] = make_float4(L.r, L.g, L.b, 0.0f);
        if (cont)
        {
            w.o_pdf[slot] = make_float4(ro.x, ro.y, ro.z, prev_bsdf_pdf);
            w.d_eta[slot] = make_float4(rd.x, rd.y, rd.z, eta_scale);
            w.beta[slot] = make_float4(beta.r, beta.g, beta.b, 0.0f);
            StoreSampler(w, slot, rng);
            w.flags[slot] = (fl & kSceneMask) | bounce | (specular_bounce ? kSpecularBit : 0) |
                            (any_non_specular ? kAnyNonSpecularBit : 0);
        }
        int32_t qi = Append(&w.counts[parity ^ 1], cont);
        if (cont)
        {
            q_next[qi] = slot;
        }
        int32_t si = Append(&w.counts[2], shadow);
        if (shadow)
        {
            w.sh_o[si] = make_float4(sh_o.x, sh_o.y, sh_o.z, sh_t);
            w.sh_d[si] = make_float4(sh_d.x, sh_d.y, sh_d.z, __int_as_float(slot));
            w.sh_c[si] = make_float4(sh_c.r, sh_c.g, sh_c.b, 0.0f);
        }
    }
}

// ---------------------------------------------------------------- guided shading
//
// With a guide, each level shades in two passes around one batched MLP
// inference: GuidedShadeA does everything up to the BSDF and, at
// non-specular vertices, queues the guide query; GuidedShadeB (after the
// inference) does next-event estimation and the continuation with one-sample
// MIS between the guide and the BSDF (guide selection probability s, 1/2 by
// default): the continuation's density is the mixture s q + (1 - s) p_bsdf.
// Light sampling and the continuation are combined with the plain tracer's
// weights, the power heuristic on the light and BSDF pdfs: any weights that
// sum to one at every direction keep the estimator unbiased, whatever the
// network outputs, and these leave next-event estimation exactly as in the
// plain tracer (the mixture density in them would raise the weight of light
// samples on glossy surfaces, where they are noisy, up to fourfold) and
// bound a continuation sample's weight by 1/(1 - s) times the plain one.
// Specular vertices, and those whose shading frame is not orthonormal
// (kGuideFrameSkew), continue as in the plain tracer. Training records take
// (query, direction, pdf, throughput) at sampled vertices and the radiance
// the rest of the path brings back along that direction.

struct GuideDev
{
    float* raw;        // per slot: query (kGuideRaw floats)
    float* out;        // per slot: network outputs (kGuideOut floats)
    float4* vtx;       // per slot: (point, material), (sn, front), (st, -), (wo, -)
    int32_t* queue;    // slots with a guide query this level
    int32_t* rec_id;   // per slot: open training record or -1
    float* rec;        // per record: raw (10), unit dir (3), pdf, throughput into the vertex over the
                       // RR survival probability (3), L at the next shading pass (3)
    int32_t* rec_slot;
    float* t_raw;      // training batch: raw queries, directions, weights
    float* t_dir;
    float* t_w;
    float* wsum;       // per scene: sum of the training weights
    int32_t* rec_count; // per scene: records appended this wave
    int32_t* rec_n;     // per scene: records kept (at most rec_cap)
    // Batches: the guide queries bucketed by scene for the grouped forward.
    int32_t* bucket;      // per scene: queries this level
    int32_t* cursor;      // per scene: next free bucketed position
    int32_t* chunk_start; // per scene + 1: first chunk of the scene's queries
    int32_t* sorted;      // bucketed queue (-1 pads each scene to whole chunks)
    int32_t rec_cap;   // records per scene (scene k's records start at k rec_cap)
    int32_t n_scenes;
    int32_t stride;    // paths with index % stride == 0 record training samples
    int32_t train;
    float select;      // probability of sampling the guide rather than the BSDF
};

constexpr int kRecFloats = 20;

// Largest |n . t| of a shading frame at which a vertex is guided. The BSDF
// frame is built from the interpolated normal and tangent without
// orthogonalising them (Frame::FromXZ, include/bulbit/frame.h:139-142); when
// they are not orthogonal, the directions the BSDF samples (mapped to world
// space by the skewed frame) and the values f() and PDF() give for a world
// direction (mapped back by dot products) describe different measures, so a
// guide direction, which only f() and PDF() can weigh, would shift the pixel
// estimates. Such vertices use the plain tracer's BSDF sampling. The bound
// keeps the angular error far below the narrowest lobe the materials have.
constexpr float kGuideFrameSkew = 1e-3f;

__device__ __forceinline__ float GuideRoughness(const MaterialDev& m)
{
    return m.type == BBG_MAT_DIFFUSE ? 1.0f : sqrtf(m.alpha_x * m.alpha_y);
}

// Escaped ray: infinite lights with MIS against the previous continuation pdf.
__device__ __forceinline__ void AddEscaped(const SceneDev& s, Spec beta, int32_t bounce, bool specular_bounce,
                                           float prev_pdf, Spec* L)
{
    for (int32_t k = 0; k < s.n_infinite; ++k)
    {
        const LightDev& l = s.lights[s.infinite[k]];
        Spec Le = l.scale * Spec{ l.L[0], l.L[1], l.L[2] };
        if (bounce == 0 || specular_bounce)
        {
            *L = *L + beta * Le;
        }
        else
        {
            float light_pdf = kInvFourPi * s.light_pmf[s.infinite[k]];
            *L = *L + beta * PowerHeuristic(prev_pdf, light_pdf) * Le;
        }
    }
}

// Next-event estimation at a non-specular vertex (PathIntegrator's
// SampleDirectLight, as in ShadeKernel: u0 then u12 drawn, power heuristic
// on the light and BSDF pdfs). Returns whether a shadow ray was made.
__device__ __forceinline__ bool DirectLight(const SceneDev& s, const BSDF& bsdf, V3 point, V3 sn, V3 wo, Spec beta,
                                            PathSampler& rng, V3* sh_d, float* sh_t, Spec* sh_c)
{
    float u0 = Next1D(rng);
    P2 u12 = Next2D(rng);
    if (s.n_lights <= 0)
    {
        return false;
    }
    float pmf;
    int32_t li = SampleLight(s, u0, &pmf);
    const LightDev& l = s.lights[li];
    V3 tri[3];
    const bbg_sphere* sph = nullptr;
    bool on_tri = false;
    if (l.type == BBG_LIGHT_DIFFUSE_AREA)
    {
        int4 linfo = s.prim_info[l.prim];
        if (linfo.x == BBG_PRIM_TRIANGLE)
        {
            int32_t vv[3];
            TriVerts(s, linfo.y, vv, tri);
            on_tri = true;
        }
        else
        {
            sph = &s.spheres[linfo.y];
        }
    }
    LightSampleLi ls;
    if (!SampleLi(l, point, u12, on_tri ? tri : nullptr, sph, &ls))
    {
        return false;
    }
    float bsdf_pdf = bsdf.PDF(wo, ls.wi);
    if (IsBlack(ls.Li) || bsdf_pdf == 0)
    {
        return false;
    }
    float light_pdf = pmf * ls.pdf;
    Spec f_cos = bsdf.F(wo, ls.wi) * AbsDot(sn, ls.wi);
    if (IsDeltaLight(l.type))
    {
        *sh_c = beta * ls.Li * f_cos / light_pdf;
    }
    else
    {
        *sh_c = beta * PowerHeuristic(light_pdf, bsdf_pdf) * ls.Li * f_cos / light_pdf;
    }
    *sh_d = ls.wi;
    *sh_t = ls.visibility;
    return true;
}

template <class Scenes>
__global__ void __launch_bounds__(kBlock, BBG_SHADE_MIN_BLOCKS) GuidedShadeA(Scenes sc, WaveDev w, GuideDev g, int parity)
{
    const int32_t* q = w.sorted ? w.sorted : w.queue[parity];
    int32_t* q_next = w.queue[parity ^ 1];
    const int32_t n = w.counts[parity];
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        int32_t slot = q[j];
        float4 o4 = w.o_pdf[slot], d4 = w.d_eta[slot], b4 = w.beta[slot], L4 = w.L[slot];
        float4 hit = w.hit[slot];
        V3 ro{ o4.x, o4.y, o4.z }, rd{ d4.x, d4.y, d4.z };
        float prev_pdf = o4.w, eta_scale = d4.w;
        Spec beta{ b4.x, b4.y, b4.z }, L{ L4.x, L4.y, L4.z };
        int32_t fl = w.flags[slot];
        const int32_t scene_bits = fl & kSceneMask;
        const SceneDev& s = sc.Scene(fl >> kSceneShift);
        PathSampler rng = LoadSampler(s, w, slot);
        int32_t bounce = fl & 0xffff;
        bool specular_bounce = (fl & kSpecularBit) != 0;
        bool any_non_specular = (fl & kAnyNonSpecularBit) != 0;

        if (g.train)
        {
            int32_t r = g.rec_id[slot];
            if (r >= 0)
            {
                float* rr = g.rec + size_t(r) * kRecFloats;
                rr[17] = L.r;
                rr[18] = L.g;
                rr[19] = L.b;
                g.rec_id[slot] = -1;
            }
        }

        bool cont = false, guided = false, shadow = false;
        V3 sh_o{}, sh_d{};
        float sh_t = 0;
        Spec sh_c{};
        int32_t prim = __float_as_int(hit.x);
        if (prim < 0)
        {
            AddEscaped(s, beta, bounce, specular_bounce, prev_pdf, &L);
        }
        else
        {
            int4 info = s.prim_info[prim];
            Isect is = MakeIsect(s, info, hit, ro, rd);
            V3 wo = Normalize(-rd);
            if (info.w >= 0)
            {
                const LightDev& l = s.lights[info.w];
                Spec Le = (is.front_face || l.two_sided) ? Spec{ l.L[0], l.L[1], l.L[2] } : spec(0);
                if (!IsBlack(Le))
                {
                    if (bounce == 0 || specular_bounce)
                    {
                        L = L + beta * Le;
                    }
                    else
                    {
                        float light_pdf = ShapePdf(s, info, is, ro, rd) * s.light_pmf[info.w];
                        L = L + beta * PowerHeuristic(prev_pdf, light_pdf) * Le;
                    }
                }
            }
            if (bounce++ >= s.max_bounces)
            {
            }
            else if (info.z < 0)
            {
                ro = is.point;
                rd = -wo;
                --bounce;
                cont = true;
            }
            else
            {
                const MaterialDev& mat = s.materials[info.z];
                BSDF bsdf = MakeBSDF(mat, is.sn, is.st, is.front_face);
                if (s.regularize && any_non_specular)
                {
                    RegularizeBSDF(&bsdf);
                }
                if (IsNonSpecular(bsdf.flags) && fabsf(Dot(is.sn, is.st)) <= kGuideFrameSkew)
                {
                    guided = true;
                    float* r = g.raw + size_t(slot) * kGuideRaw;
                    r[0] = is.point.x;
                    r[1] = is.point.y;
                    r[2] = is.point.z;
                    r[3] = is.sn.x;
                    r[4] = is.sn.y;
                    r[5] = is.sn.z;
                    r[6] = wo.x;
                    r[7] = wo.y;
                    r[8] = wo.z;
                    r[9] = GuideRoughness(mat);
                    float4* v = g.vtx + 4 * size_t(slot);
                    v[0] = make_float4(is.point.x, is.point.y, is.point.z, __int_as_float(info.z));
                    v[1] = make_float4(is.sn.x, is.sn.y, is.sn.z, is.front_face ? 1.0f : 0.0f);
                    v[2] = make_float4(is.st.x, is.st.y, is.st.z, 0.0f);
                    v[3] = make_float4(wo.x, wo.y, wo.z, 0.0f);
                }
                else
                {
                    // Specular, or a skewed shading frame: the plain
                    // tracer's next-event estimation and BSDF sampling.
                    if (IsNonSpecular(bsdf.flags))
                    {
                        shadow = DirectLight(s, bsdf, is.point, is.sn, wo, beta, rng, &sh_d, &sh_t, &sh_c);
                        sh_o = is.point;
                    }
                    P2 u12 = Next2D(rng);
                    float u0 = Next1D(rng);
                    BSDFSample bs;
                    if (bsdf.Sample(&bs, wo, u0, u12))
                    {
                        bool spec_sample = (bs.flags & kFlagSpecular) != 0;
                        specular_bounce = spec_sample;
                        any_non_specular = any_non_specular || !spec_sample;
                        if (bs.flags & kFlagTransmission)
                        {
                            eta_scale *= Sqr(bs.eta);
                        }
                        prev_pdf = bs.pdf;
                        beta = beta * (bs.f * AbsDot(is.sn, bs.wi) / bs.pdf);
                        ro = is.point;
                        rd = bs.wi;
                        cont = true;
                        if (bounce > s.rr_min_bounces)
                        {
                            float p = MaxComponent(beta) * eta_scale;
                            if (p < 1)
                            {
                                if (Next1D(rng) > p)
                                {
                                    cont = false;
                                }
                                else
                                {
                                    beta = beta / p;
                                }
                            }
                        }
                    }
                }
            }
        }
        w.L[slot] = make_float4(L.r, L.g, L.b, 0.0f);
        if (cont || guided)
        {
            w.o_pdf[slot] = make_float4(ro.x, ro.y, ro.z, prev_pdf);
            w.d_eta[slot] = make_float4(rd.x, rd.y, rd.z, eta_scale);
            w.beta[slot] = make_float4(beta.r, beta.g, beta.b, 0.0f);
            StoreSampler(w, slot, rng);
            w.flags[slot] =
                scene_bits | bounce | (specular_bounce ? kSpecularBit : 0) | (any_non_specular ? kAnyNonSpecularBit : 0);
        }
        int32_t qi = Append(&w.counts[parity ^ 1], cont);
        if (cont)
        {
            q_next[qi] = slot;
        }
        int32_t gi = Append(&w.counts[5], guided);
        if (guided)
        {
            g.queue[gi] = slot;
        }
        int32_t si = Append(&w.counts[2], shadow);
        if (shadow)
        {
            w.sh_o[si] = make_float4(sh_o.x, sh_o.y, sh_o.z, sh_t);
            w.sh_d[si] = make_float4(sh_d.x, sh_d.y, sh_d.z, __int_as_float(slot));
            w.sh_c[si] = make_float4(sh_c.r, sh_c.g, sh_c.b, 0.0f);
        }
    }
}

template <class Scenes>
__global__ void __launch_bounds__(kBlock, BBG_SHADE_MIN_BLOCKS) GuidedShadeB(Scenes sc, WaveDev w, GuideDev g, int parity)
{
    int32_t* q_next = w.queue[parity ^ 1];
    const int32_t n = w.counts[5];
    const int64_t wave_base = w.wave[0];
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        int32_t slot = g.queue[j];
        float4 d4 = w.d_eta[slot], b4 = w.beta[slot];
        float eta_scale = d4.w;
        Spec beta{ b4.x, b4.y, b4.z };
        int32_t fl = w.flags[slot];
        const int32_t scene = kIsBatch<Scenes> ? (fl >> kSceneShift) : 0;
        const SceneDev& s = sc.Scene(scene);
        PathSampler rng = LoadSampler(s, w, slot);
        int32_t bounce = fl & 0xffff;
        bool any_non_specular = (fl & kAnyNonSpecularBit) != 0;
        const float4* v = g.vtx + 4 * size_t(slot);
        float4 v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3];
        V3 point{ v0.x, v0.y, v0.z }, sn{ v1.x, v1.y, v1.z }, st{ v2.x, v2.y, v2.z }, wo{ v3.x, v3.y, v3.z };
        const MaterialDev& mat = s.materials[__float_as_int(v0.w)];
        BSDF bsdf = MakeBSDF(mat, sn, st, v1.w != 0.0f);
        if (s.regularize && any_non_specular)
        {
            RegularizeBSDF(&bsdf);
        }
        VmfMixture mix = MakeMixture(g.out + size_t(slot) * kGuideOut);

        // Next-event estimation with the plain tracer's weights.
        V3 sh_d{};
        float sh_t = 0;
        Spec sh_c{};
        bool shadow = DirectLight(s, bsdf, point, sn, wo, beta, rng, &sh_d, &sh_t, &sh_c);

        // Continuation: the guide with probability g.select, else the BSDF.
        // A BSDF sample is weighted with its own f and pdf, as the plain
        // tracer does: where the shading frame is not orthonormal (normals
        // and tangents are interpolated independently, see MakeIsect) those
        // differ from f() and PDF() at the world direction, and only the
        // sample's own values keep the plain estimator's expectation. A
        // specular sample is a discrete mass the guide cannot produce; its
        // probability is (1 - select) times the BSDF's.
        bool cont = false;
        float u_sel = Next1D(rng);
        P2 u12 = Next2D(rng);
        float u0 = Next1D(rng);
        V3 wi{}, wdir{};
        Spec f{};
        float pdf = 0, pdf_b = 0, cosv = 0, eta_sample = 1, rr_p = 1;
        bool spec_sample = false, transmit = false;
        const Spec beta_in = beta;
        if (u_sel < g.select)
        {
            wi = MixtureSample(mix, u0, u12.x, u12.y);
            wdir = wi;
            f = bsdf.F(wo, wi);
            pdf_b = bsdf.PDF(wo, wi);
            pdf = g.select * MixturePdf(mix, wi) + (1.0f - g.select) * pdf_b;
            cosv = AbsDot(sn, wi);
            if (mat.type == BBG_MAT_DIELECTRIC)
            {
                float cz_o = Dot(wo, sn), cz_i = Dot(wi, sn);
                transmit = cz_o * cz_i < 0;
                eta_sample = cz_o > 0 ? bsdf.eta : 1 / bsdf.eta;
            }
        }
        else
        {
            BSDFSample bs;
            if (bsdf.Sample(&bs, wo, u0, u12))
            {
                wi = bs.wi;
                wdir = Normalize(wi);
                f = bs.f;
                pdf_b = bs.pdf;
                spec_sample = (bs.flags & kFlagSpecular) != 0;
                pdf = spec_sample ? (1.0f - g.select) * bs.pdf
                                  : g.select * MixturePdf(mix, wdir) + (1.0f - g.select) * bs.pdf;
                cosv = AbsDot(sn, wi);
                transmit = (bs.flags & kFlagTransmission) != 0;
                eta_sample = bs.eta;
            }
        }
        if (pdf > 0 && !IsBlack(f) && cosv > 0)
        {
            if (transmit)
            {
                eta_scale *= Sqr(eta_sample);
            }
            beta = beta * (f * cosv / pdf);
            cont = true;
            if (bounce > s.rr_min_bounces)
            {
                float p = MaxComponent(beta) * eta_scale;
                if (p < 1)
                {
                    if (Next1D(rng) > p)
                    {
                        cont = false;
                    }
                    else
                    {
                        beta = beta / p;
                        rr_p = p;
                    }
                }
            }
        }
        if (g.train && pdf > 0 && !spec_sample && (wave_base + slot) % g.stride == 0)
        {
            int32_t r = atomicAdd(&g.rec_count[scene], 1);
            if (r < g.rec_cap)
            {
                r += scene * g.rec_cap;
                float* rr = g.rec + size_t(r) * kRecFloats;
                const float* raw = g.raw + size_t(slot) * kGuideRaw;
                for (int k = 0; k < kGuideRaw; ++k)
                {
                    rr[k] = raw[k];
                }
                rr[10] = wdir.x;
                rr[11] = wdir.y;
                rr[12] = wdir.z;
                rr[13] = pdf;
                rr[14] = cont ? beta_in.r / rr_p : 0.0f;
                rr[15] = cont ? beta_in.g / rr_p : 0.0f;
                rr[16] = cont ? beta_in.b / rr_p : 0.0f;
                rr[17] = NAN; // filled at the path's next shading pass
                g.rec_slot[r] = slot;
                g.rec_id[slot] = cont ? r : -1;
            }
        }
        if (cont)
        {
            // The emission MIS at the next hit weighs the BSDF pdf against
            // the light's (see above); the throughput carries the mixture's.
            w.o_pdf[slot] = make_float4(point.x, point.y, point.z, pdf_b);
            w.d_eta[slot] = make_float4(wi.x, wi.y, wi.z, eta_scale);
            w.beta[slot] = make_float4(beta.r, beta.g, beta.b, 0.0f);
            w.flags[slot] = (fl & kSceneMask) | bounce | (spec_sample ? kSpecularBit : 0) |
                            ((any_non_specular || !spec_sample) ? kAnyNonSpecularBit : 0);
        }
        StoreSampler(w, slot, rng);
        int32_t qi = Append(&w.counts[parity ^ 1], cont);
        if (cont)
        {
            q_next[qi] = slot;
        }
        int32_t si = Append(&w.counts[2], shadow);
        if (shadow)
        {
            w.sh_o[si] = make_float4(point.x, point.y, point.z, sh_t);
            w.sh_d[si] = make_float4(sh_d.x, sh_d.y, sh_d.z, __int_as_float(slot));
            w.sh_c[si] = make_float4(sh_c.r, sh_c.g, sh_c.b, 0.0f);
        }
    }
}

// Training targets of the wave's records: the integrand's product f cos L_i
// over the sampling pdf (the target of Mueller et al. 2019, "Neural
// Importance Sampling"). The radiance the path gathered after the vertex is
// dL = L(end) - L(at the next shading pass) = beta_in f cos L_i / (pdf p_rr),
// so the weight f cos L_i / pdf = luminance(dL p_rr / beta_in). The next
// hit's emission enters with its MIS weight, so on diffuse surfaces, where
// NEE takes nearly all of it, the guide mostly learns indirect light, and on
// glossy ones it learns the reflected light too. Weights are then
// normalised to mean 1 per scene (GuideNormalizeKernel). Grid row y covers
// scene y's records.
__global__ void GuideFinalizeKernel(WaveDev w, GuideDev g)
{
    const int32_t scene = blockIdx.y;
    const int32_t n = min(g.rec_count[scene], g.rec_cap);
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        g.rec_n[scene] = n;
    }
    float local = 0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const int32_t r = scene * g.rec_cap + i;
        const float* rr = g.rec + size_t(r) * kRecFloats;
        float4 Lf = w.L[g.rec_slot[r]];
        bool started = !isnan(rr[17]);
        Spec cont = started ? Spec{ Lf.x - rr[17], Lf.y - rr[18], Lf.z - rr[19] } : spec(0);
        Spec prod{ rr[14] > 0 ? cont.r / rr[14] : 0.0f, rr[15] > 0 ? cont.g / rr[15] : 0.0f,
                   rr[16] > 0 ? cont.b / rr[16] : 0.0f };
        float wgt = fmaxf(Luminance(prod), 0.0f);
        if (!isfinite(wgt))
        {
            wgt = 0;
        }
        for (int k = 0; k < kGuideRaw; ++k)
        {
            g.t_raw[size_t(r) * kGuideRaw + k] = rr[k];
        }
        g.t_dir[3 * size_t(r)] = rr[10];
        g.t_dir[3 * size_t(r) + 1] = rr[11];
        g.t_dir[3 * size_t(r) + 2] = rr[12];
        g.t_w[r] = wgt;
        local += wgt;
    }
    for (int off = 16; off > 0; off >>= 1)
    {
        local += __shfl_xor_sync(0xffffffffu, local, off);
    }
    if ((threadIdx.x & 31) == 0 && local != 0.0f)
    {
        atomicAdd(&g.wsum[scene], local);
    }
}

__global__ void GuideNormalizeKernel(GuideDev g)
{
    const int32_t scene = blockIdx.y;
    const int32_t n = g.rec_n[scene];
    float sum = g.wsum[scene];
    float scale = sum > 0 ? float(n) / sum : 0.0f;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        g.t_w[size_t(scene) * g.rec_cap + i] *= scale;
    }
}

// Clears the next level's ray queue, the shadow queue, the work counters of
// the persistent closest-hit and shadow passes and the guide-query queue.
__global__ void ResetKernel(WaveDev w, int parity)
{
    w.counts[parity ^ 1] = 0;
    w.counts[2] = 0;
    w.counts[3] = 0;
    w.counts[4] = 0;
    w.counts[5] = 0;
    if (w.sorted)
    {
        for (int k = 0; k < 2 * kShadeKinds; ++k)
        {
            w.sort_counts[k] = 0;
        }
    }
}

// ---------------------------------------------------------------- shading order

template <class Scenes>
__device__ __forceinline__ int32_t ShadeKind(const Scenes& sc, const WaveDev& w, int32_t slot)
{
    int32_t prim = __float_as_int(w.hit[slot].x);
    if (prim < 0)
    {
        return 0;
    }
    const SceneDev& s = sc.Scene(w.flags[slot] >> kSceneShift);
    int32_t m = s.prim_info[prim].z;
    if (m < 0)
    {
        return 1;
    }
    const MaterialDev& md = s.materials[m];
    return 2 + 2 * min(max(md.type, 0), 3) + (md.ms ? 1 : 0);
}

// Counting sort of a level's queue by shading kind, pass 1: the kind of every
// queued path (read from its hit) and the kinds' totals (block-aggregated).
template <class Scenes>
__global__ void __launch_bounds__(kBlock) ShadeKindsKernel(Scenes sc, WaveDev w, int parity)
{
    __shared__ int32_t bc[kShadeKinds];
    const int32_t* q = w.queue[parity];
    const int32_t n = w.counts[parity];
    for (int32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock)
    {
        if (threadIdx.x < kShadeKinds)
        {
            bc[threadIdx.x] = 0;
        }
        __syncthreads();
        const int32_t j = base + int32_t(threadIdx.x);
        if (j < n)
        {
            int32_t k = ShadeKind(sc, w, q[j]);
            w.keys[j] = uint8_t(k);
            atomicAdd(&bc[k], 1);
        }
        __syncthreads();
        if (threadIdx.x < kShadeKinds && bc[threadIdx.x] > 0)
        {
            atomicAdd(&w.sort_counts[threadIdx.x], bc[threadIdx.x]);
        }
        __syncthreads();
    }
}

// Pass 2: every block reserves, per kind, a range after the kinds before it
// (the totals' prefix) and writes its paths' slots there; the order inside a
// kind is arbitrary (paths do not depend on one another).
__global__ void __launch_bounds__(kBlock) ShadeScatterKernel(WaveDev w, int parity)
{
    __shared__ int32_t bc[kShadeKinds], boff[kShadeKinds], start[kShadeKinds];
    const int32_t* q = w.queue[parity];
    const int32_t n = w.counts[parity];
    if (threadIdx.x == 0)
    {
        int32_t acc = 0;
        for (int k = 0; k < kShadeKinds; ++k)
        {
            start[k] = acc;
            acc += w.sort_counts[k];
        }
    }
    for (int32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock)
    {
        if (threadIdx.x < kShadeKinds)
        {
            bc[threadIdx.x] = 0;
        }
        __syncthreads();
        const int32_t j = base + int32_t(threadIdx.x);
        int32_t k = 0, local = 0;
        if (j < n)
        {
            k = w.keys[j];
            local = atomicAdd(&bc[k], 1);
        }
        __syncthreads();
        if (threadIdx.x < kShadeKinds)
        {
            boff[threadIdx.x] =
                bc[threadIdx.x] > 0 ? start[threadIdx.x] + atomicAdd(&w.sort_counts[kShadeKinds + threadIdx.x],
                                                                     bc[threadIdx.x])
                                    : 0;
        }
        __syncthreads();
        if (j < n)
        {
            w.sorted[boff[k] + local] = q[j];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- film


// Film::AddSample over each pixel's samples in order (src/reconstruction/film.cpp:26-37).
template <class Scenes>
__global__ void __launch_bounds__(kBlock) FilmKernel(Scenes sc, WaveDev w)
{
    const int64_t base = w.wave[0];
    const int32_t spp = sc.Spp();
    const int64_t n_pixels = w.wave[1] / spp;
    const int64_t pixel0 = base / spp;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n_pixels; i += int64_t(gridDim.x) * blockDim.x)
    {
        int64_t p;
        const FilmDev& f = sc.Film(sc.Locate(pixel0 + i, &p));
        Spec sum = spec(0);
        int32_t count = 0;
        float m0 = 0, m1 = 0;
        for (int32_t k = 0; k < spp; ++k)
        {
            int64_t slot = i * spp + k;
            float4 L4 = w.L[slot];
            Spec L{ L4.x, L4.y, L4.z };
            if (f.path_L)
            {
                float* dst = f.path_L + 3 * (p * spp + k);
                dst[0] = L.r;
                dst[1] = L.g;
                dst[2] = L.b;
            }
            if (IsNullish(L))
            {
                continue;
            }
            sum = sum + L * 1.0f;
            count += 1;
            float l = Luminance(L);
            float alpha = 1.0f / count;
            m0 = m0 * (1 - alpha) + l * alpha;
            m1 = m1 * (1 - alpha) + (l * l) * alpha;
        }
        f.rgb_sum[3 * p] = sum.r;
        f.rgb_sum[3 * p + 1] = sum.g;
        f.rgb_sum[3 * p + 2] = sum.b;
        f.count[p] = count;
        f.moments[2 * p] = m0;
        f.moments[2 * p + 1] = m1;
    }
}

// ---------------------------------------------------------------- GGX energy tables

constexpr int kEnergySamples = 1024; // 32 x 32 strata, PrepareReflectanceTextures(32, 1024)

// The stratified samples of PrepareReflectanceTextures (src/bxdf/microfacet.cpp:239-275):
// RNG(3); per sample a permuted 1-D stratum u0 and a permuted 2-D stratum
// u12, in that draw order. One thread.
__global__ void EnergySamplesKernel(float* u0s, P2* u12)
{
    uint64_t st = 0; // RNG(3): Seed(initstate = 3, initseq = 1)
    PcgNext(st);
    st += 3;
    PcgNext(st);
    for (int i = 0; i < kEnergySamples; ++i)
    {
        int32_t s0 = int32_t(PermutationElement(uint32_t(i), kEnergySamples, 1));
        u0s[i] = (float(s0) + Next1D(st)) / float(kEnergySamples);
        int32_t s1 = int32_t(PermutationElement(uint32_t(i), kEnergySamples, 2));
        int32_t x = s1 % 32, y = s1 / 32;
        float a = Next1D(st);
        float b = Next1D(st);
        u12[i] = P2{ (float(x) + a) / 32.0f, (float(y) + b) / 32.0f };
    }
}

// E(cos theta, alpha) = rho(wo) of TrowbridgeReitzDistribution(alpha, alpha)
// (include/bulbit/microfacet.h:109-130), one thread per table entry, samples
// summed in order; then E_avg(alpha) = 2 sum_i E cos theta d.
__global__ void GgxEnergyTablesKernel(const P2* u12)
{
    const float d = 1.0f / kEnergyTableSize;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < kEnergyTableSize * kEnergyTableSize)
    {
        int i = e % kEnergyTableSize, j = e / kEnergyTableSize;
        float a = d / 2 + d * float(j);
        float cos_theta = d / 2 + d * float(i);
        float sin_theta = sqrtf(1 - cos_theta * cos_theta);
        V3 wo{ sin_theta, 0, cos_theta };
        TrowbridgeReitz mf{ a, a };
        float r = 0;
        for (int k = 0; k < kEnergySamples; ++k)
        {
            V3 wm = mf.SampleWm(wo, u12[k]);
            V3 wi = Reflect(wo, wm);
            if (!SameHemisphere(wo, wi))
            {
                continue;
            }
            float pdf = mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
            float f = mf.D(wm) * mf.G(wo, wi) / (4 * AbsCosTheta(wo) * AbsCosTheta(wi));
            r += f * AbsCosTheta(wi) / pdf;
        }
        g_ggx_e[e] = r / float(kEnergySamples);
    }
}

__global__ void GgxEnergyAverageKernel()
{
    const float d = 1.0f / kEnergyTableSize;
    int j = threadIdx.x;
    if (j < kEnergyTableSize)
    {
        float r_sum = 0;
        for (int i = 0; i < kEnergyTableSize; ++i)
        {
            float cos_theta = d / 2 + d * float(i);
            r_sum += g_ggx_e[i + kEnergyTableSize * j] * cos_theta * d;
        }
        g_ggx_e_avg[j] = 2 * r_sum;
    }
}

// Energy tables of the rough dielectric (src/bxdf/microfacet.cpp:168-237):
// entry (k, i, j) of E (E_inv) is rho(wo) of DielectricBxDF(ior_k (1 / ior_k),
// GGX(alpha_j)) under importance transport (TransportDirection::ToCamera), the
// samples summed in order (src/bxdf/bxdf.cpp:8-20), then the Spectrum's
// Average of the three equal channels. One thread per entry of both tables.
__global__ void DielectricEnergyTablesKernel(const float* u0s, const P2* u12)
{
    constexpr int n = kEnergyTableSize;
    constexpr int n3 = n * n * n;
    const float d = 1.0f / n;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 2 * n3)
    {
        return;
    }
    bool inv = e >= n3;
    int c = inv ? e - n3 : e;
    int k = c % n, i = (c / n) % n, j = c / (n * n);
    float ior = MapF0toIOR(d / 2 + d * float(k));
    float a = d / 2 + d * float(j);
    float cos_theta = d / 2 + d * float(i);
    float sin_theta = sqrtf(1 - Sqr(cos_theta));
    V3 wo{ sin_theta, 0, cos_theta };
    BSDF b;
    b.type = BBG_MAT_DIELECTRIC;
    b.eta = inv ? 1 / ior : ior;
    b.mf = TrowbridgeReitz{ a, a };
    b.r = spec(1);
    b.ms = 0;
    float r = 0;
    for (int q = 0; q < kEnergySamples; ++q)
    {
        BSDFSample smp;
        if (b.DielectricSample<false>(&smp, wo, u0s[q], u12[q]))
        {
            r += smp.f.r * AbsCosTheta(smp.wi) / smp.pdf;
        }
    }
    r = r / float(kEnergySamples);
    (inv ? g_dms_e_inv : g_dms_e)[c] = (r + r + r) / 3;
}

// E_avg(f0, alpha) = 2 sum_i E(f0, cos theta_i, alpha) cos theta_i d, both
// interfaces. One thread per (k, j).
__global__ void DielectricEnergyAverageKernel()
{
    constexpr int n = kEnergyTableSize;
    const float d = 1.0f / n;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n)
    {
        return;
    }
    int k = e % n, j = e / n;
    float r_sum = 0, r_inv_sum = 0;
    for (int i = 0; i < n; ++i)
    {
        float cos_theta = d / 2 + d * float(i);
        int c = (j * n + i) * n + k;
        r_sum += g_dms_e[c] * cos_theta * d;
        r_inv_sum += g_dms_e_inv[c] * cos_theta * d;
    }
    g_dms_e_avg[j * n + k] = 2 * r_sum;
    g_dms_e_inv_avg[j * n + k] = 2 * r_inv_sum;
}

// ---------------------------------------------------------------- BSDF probe

// Material::GetBSDF at a surface with shading normal +z and tangent +x (so
// local and world directions coincide), then BSDF::f, PDF and Sample_f per
// query; out: f (3), pdf, and the sample's f (3), wi (3), pdf, flags (-1 if
// Sample_f fails) — 12 floats per query.
__global__ void BsdfProbeKernel(MaterialDev m, int32_t front_face, int32_t n, const float* wo, const float* wi,
                                const float* u, float* out)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        BSDF b = MakeBSDF(m, V3{ 0, 0, 1 }, V3{ 1, 0, 0 }, front_face != 0);
        V3 o = load3(wo + 3 * size_t(i)), w = load3(wi + 3 * size_t(i));
        Spec f = b.F(o, w);
        float pdf = b.PDF(o, w);
        BSDFSample s{};
        bool ok = b.Sample(&s, o, u[3 * size_t(i)], P2{ u[3 * size_t(i) + 1], u[3 * size_t(i) + 2] });
        float* r = out + 12 * size_t(i);
        r[0] = f.r, r[1] = f.g, r[2] = f.b, r[3] = pdf;
        r[4] = ok ? s.f.r : 0, r[5] = ok ? s.f.g : 0, r[6] = ok ? s.f.b : 0;
        r[7] = ok ? s.wi.x : 0, r[8] = ok ? s.wi.y : 0, r[9] = ok ? s.wi.z : 0;
        r[10] = ok ? s.pdf : 0, r[11] = ok ? float(s.flags) : -1.0f;
    }
}

// ---------------------------------------------------------------- sampler probe

__global__ void SamplerDrawsKernel(int32_t px, int32_t py, int32_t seed, int32_t sample, int32_t n, float* out)
{
    uint64_t st = SamplerStart(px, py, seed, sample);
    for (int32_t i = 0; i < n; ++i)
    {
        out[i] = Next1D(st);
    }
}

} // namespace bbg

using namespace bbg;

// ---------------------------------------------------------------- handle

struct bbg_integrator
{
    int device = 0; // the accel's device; every call runs there
    bbg_accel* accel = nullptr;
    int32_t n_lights = 0;
    std::vector<float> pmf;
    int32_t max_bounces = 0, rr_min_bounces = 1, regularize = 0;

    DevBuf<int4> prim_info;
    DevBuf<MaterialDev> materials;
    DevBuf<LightDev> lights;
    DevBuf<float> light_func, light_cdf, light_pmf, alias_prob;
    DevBuf<int32_t> alias_idx, infinite;
    float func_integral = 0;
    int32_t n_infinite = 0;

    // Wave state.
    int64_t capacity = 0;
    DevBuf<float4> o_pdf, d_eta, beta, L, hit, sh_o, sh_d, sh_c;
    DevBuf<uint64_t> rng;
    DevBuf<int32_t> flags, queue0, queue1, counts, dim;
    DevBuf<unsigned long long> stats;
    DevBuf<int64_t> wave;
    int64_t* wave_host = nullptr; // pinned

    // Gaussian filter table of the last camera that used one (sigma, extent).
    DevBuf<float> filter_cdf;
    float filter_key[2] = { -1, -1 };
    // Film (device copies for host-memory renders).
    DevBuf<float> film_rgb, film_moments, film_path_L;
    DevBuf<int32_t> film_count;

    // Guided rendering: per-slot query / output / vertex state, training records.
    int64_t g_capacity = 0;
    int64_t g_rec_cap = 0;
    DevBuf<float> g_raw, g_out, g_rec, g_traw, g_tdir, g_tw, g_wsum;
    DevBuf<float4> g_vtx;
    DevBuf<int32_t> g_queue, g_recid, g_recslot, g_slice;
    // Per scene (a batch has several): record counters, bucketed queries.
    DevBuf<int32_t> g_reccount, g_recn, g_bucket, g_cursor, g_chunk, g_sorted;

    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int64_t graph_capacity = -1;
    int graph_iterations = -1;
    FilmDev graph_film{};
    SceneDev graph_scene{};
    GuideDev graph_guide{};
    bbg_guide* graph_guide_handle = nullptr;
    float graph_guide_lr = 0;
    int graph_shape = -1;
    bool graph_shade_sort = false;
    // Shading order of the current render (params.shade_order).
    bool shade_sort = true;
    DevBuf<int32_t> sorted, sort_counts;
    DevBuf<uint8_t> keys;
    // Launch shape of the traversal passes (index into kShapes) and wave size
    // for renders that do not name one (0: 2^22 paths); set by the autotuner.
    int32_t shape = 0;
    int64_t tuned_wave = 0;

    // Guide buffers for waves of n paths over n_scenes scenes, rec_cap
    // training records per scene and steps Adam steps per wave; grouped: the
    // bucketed queries of the grouped forward (batches).
    bbg_status ReserveGuide(int64_t n, int32_t rec_cap, int32_t steps, int32_t n_scenes = 1, bool grouped = false)
    {
        if (n > g_capacity)
        {
            size_t m = size_t(n);
            for (auto* b : { &g_raw, &g_out })
            {
                b->reset();
            }
            g_vtx.reset();
            g_queue.reset();
            g_recid.reset();
            BBG_TRY(g_raw.alloc(m * kGuideRaw));
            BBG_TRY(g_out.alloc(m * kGuideOut));
            BBG_TRY(g_vtx.alloc(4 * m));
            BBG_TRY(g_queue.alloc(m));
            BBG_TRY(g_recid.alloc(m));
            g_capacity = n;
        }
        const int64_t rec_total = int64_t(rec_cap) * n_scenes;
        if (rec_total > g_rec_cap)
        {
            size_t r = size_t(rec_total);
            for (auto* b : { &g_rec, &g_traw, &g_tdir, &g_tw })
            {
                b->reset();
            }
            g_recslot.reset();
            BBG_TRY(g_rec.alloc(r * kRecFloats));
            BBG_TRY(g_traw.alloc(r * kGuideRaw));
            BBG_TRY(g_tdir.alloc(r * 3));
            BBG_TRY(g_tw.alloc(r));
            BBG_TRY(g_recslot.alloc(r));
            g_rec_cap = rec_total;
        }
        const size_t ns = size_t(n_scenes);
        BBG_TRY(g_wsum.alloc(ns));
        BBG_TRY(g_slice.alloc(size_t(std::max(1, steps)) * ns));
        BBG_TRY(g_reccount.alloc(ns));
        BBG_TRY(g_recn.alloc(ns));
        if (grouped)
        {
            BBG_TRY(g_bucket.alloc(ns));
            BBG_TRY(g_cursor.alloc(ns));
            BBG_TRY(g_chunk.alloc(ns + 1));
            BBG_TRY(g_sorted.alloc(size_t(n) + ns * kGuideGroupChunk));
            BBG_CUDA(cudaMemsetAsync(g_bucket.p, 0, ns * sizeof(int32_t), stream));
        }
        return BBG_OK;
    }

    GuideDev Guide(int32_t train, int32_t stride) const
    {
        GuideDev g{};
        g.raw = g_raw.p;
        g.out = g_out.p;
        g.vtx = g_vtx.p;
        g.queue = g_queue.p;
        g.rec_id = g_recid.p;
        g.rec = g_rec.p;
        g.rec_slot = g_recslot.p;
        g.t_raw = g_traw.p;
        g.t_dir = g_tdir.p;
        g.t_w = g_tw.p;
        g.wsum = g_wsum.p;
        g.rec_count = g_reccount.p;
        g.rec_n = g_recn.p;
        g.bucket = g_bucket.p;
        g.cursor = g_cursor.p;
        g.chunk_start = g_chunk.p;
        g.sorted = g_sorted.p;
        g.rec_cap = int32_t(g_rec_cap);
        g.n_scenes = 1;
        g.stride = stride;
        g.train = train;
        return g;
    }

    ~bbg_integrator()
    {
        if (graph) cudaGraphExecDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
        if (wave_host) cudaFreeHost(wave_host);
    }

    WaveDev Wave()
    {
        WaveDev w;
        w.o_pdf = o_pdf.p;
        w.d_eta = d_eta.p;
        w.beta = beta.p;
        w.L = L.p;
        w.rng = rng.p;
        w.flags = flags.p;
        w.hit = hit.p;
        w.queue[0] = queue0.p;
        w.queue[1] = queue1.p;
        w.sh_o = sh_o.p;
        w.sh_d = sh_d.p;
        w.sh_c = sh_c.p;
        w.counts = counts.p;
        w.stats = stats.p;
        w.wave = wave.p;
        w.dim = dim.p;
        w.sorted = shade_sort ? sorted.p : nullptr;
        w.keys = keys.p;
        w.sort_counts = sort_counts.p;
        return w;
    }

    // Path state per wave slot (the arrays below): kWaveBytesPerPath.
    bbg_status Reserve(int64_t n)
    {
        if (n <= capacity) return BBG_OK;
        size_t m = size_t(n);
        for (auto* b : { &o_pdf, &d_eta, &beta, &L, &hit, &sh_o, &sh_d, &sh_c })
        {
            b->reset();
            BBG_TRY(b->alloc(m));
        }
        rng.reset();
        BBG_TRY(rng.alloc(m));
        for (auto* b : { &flags, &queue0, &queue1, &dim, &sorted })
        {
            b->reset();
            BBG_TRY(b->alloc(m));
        }
        keys.reset();
        BBG_TRY(keys.alloc(m));
        BBG_TRY(sort_counts.alloc(2 * kShadeKinds));
        capacity = n;
        return BBG_OK;
    }
};

namespace
{

// Persistent grid sizes of the stage kernels for one kind of scene set.
template <class Scenes>
struct GridsT
{
    int raygen, closest[3 * kNumShapes], shade, shadow[3 * kNumShapes], film, shade_a, shade_b, kinds, scatter;
    GridsT()
    {
        raygen = PersistentGrid(reinterpret_cast<const void*>(RaygenKernel<Scenes>), kBlock);
        Shape<0>();
        Shape<1>();
        Shape<2>();
        Shape<3>();
        shade = PersistentGrid(reinterpret_cast<const void*>(ShadeKernel<Scenes>), kBlock);
        film = PersistentGrid(reinterpret_cast<const void*>(FilmKernel<Scenes>), kBlock);
        shade_a = PersistentGrid(reinterpret_cast<const void*>(GuidedShadeA<Scenes>), kBlock);
        shade_b = PersistentGrid(reinterpret_cast<const void*>(GuidedShadeB<Scenes>), kBlock);
        kinds = PersistentGrid(reinterpret_cast<const void*>(ShadeKindsKernel<Scenes>), kBlock);
        scatter = PersistentGrid(reinterpret_cast<const void*>(ShadeScatterKernel), kBlock);
    }
    template <int K>
    void Shape()
    {
        constexpr TraversalShape t = kShapes[K];
        closest[K] = PersistentGrid(
            reinterpret_cast<const void*>(ClosestKernel<Scenes, t.block, t.short_stack, false>), t.block);
        shadow[K] = PersistentGrid(
            reinterpret_cast<const void*>(ShadowKernel<Scenes, t.block, t.short_stack, false>), t.block);
        closest[kNumShapes + K] = PersistentGrid(
            reinterpret_cast<const void*>(ClosestKernel<Scenes, t.block, t.short_stack, true>), t.block);
        shadow[kNumShapes + K] = PersistentGrid(
            reinterpret_cast<const void*>(ShadowKernel<Scenes, t.block, t.short_stack, true>), t.block);
        closest[2 * kNumShapes + K] = PersistentGrid(
            reinterpret_cast<const void*>(ClosestKernel<Scenes, t.block, t.short_stack, true, false>), t.block);
        shadow[2 * kNumShapes + K] = PersistentGrid(
            reinterpret_cast<const void*>(ShadowKernel<Scenes, t.block, t.short_stack, true, false>), t.block);
    }
};
using Grids = GridsT<OneScene>;

template <int K, bool WIDE, class Scenes, bool SPHERES = true>
void LaunchTraceShape(const GridsT<Scenes>& gr, const Scenes& sc, const WaveDev& w, int parity, bool shadow,
                      cudaStream_t st)
{
    constexpr TraversalShape t = kShapes[K];
    constexpr int g = (WIDE ? (SPHERES ? kNumShapes : 2 * kNumShapes) : 0) + K;
    if (shadow)
    {
        ShadowKernel<Scenes, t.block, t.short_stack, WIDE, SPHERES><<<gr.shadow[g], t.block, 0, st>>>(sc, w);
    }
    else
    {
        ClosestKernel<Scenes, t.block, t.short_stack, WIDE, SPHERES>
            <<<gr.closest[g], t.block, 0, st>>>(sc, w, parity);
    }
}

// The closest-hit (shadow = false) or shadow pass with trace shape
// `shape`: a kShapes index, + kNumShapes over the 8-wide layout, + 2 kNumShapes
// over the 8-wide layout of a tree of triangles only (TraceShapeOf).
template <class Scenes>
void LaunchTrace(int shape, const GridsT<Scenes>& gr, const Scenes& sc, const WaveDev& w, int parity, bool shadow,
                 cudaStream_t st)
{
    switch (shape)
    {
    case 1: LaunchTraceShape<1, false>(gr, sc, w, parity, shadow, st); break;
    case 2: LaunchTraceShape<2, false>(gr, sc, w, parity, shadow, st); break;
    case 3: LaunchTraceShape<3, false>(gr, sc, w, parity, shadow, st); break;
    case kNumShapes + 0: LaunchTraceShape<0, true>(gr, sc, w, parity, shadow, st); break;
    case kNumShapes + 1: LaunchTraceShape<1, true>(gr, sc, w, parity, shadow, st); break;
    case kNumShapes + 2: LaunchTraceShape<2, true>(gr, sc, w, parity, shadow, st); break;
    case kNumShapes + 3: LaunchTraceShape<3, true>(gr, sc, w, parity, shadow, st); break;
    case 2 * kNumShapes + 0: LaunchTraceShape<0, true, Scenes, false>(gr, sc, w, parity, shadow, st); break;
    case 2 * kNumShapes + 1: LaunchTraceShape<1, true, Scenes, false>(gr, sc, w, parity, shadow, st); break;
    case 2 * kNumShapes + 2: LaunchTraceShape<2, true, Scenes, false>(gr, sc, w, parity, shadow, st); break;
    case 2 * kNumShapes + 3: LaunchTraceShape<3, true, Scenes, false>(gr, sc, w, parity, shadow, st); break;
    default: LaunchTraceShape<0, false>(gr, sc, w, parity, shadow, st); break;
    }
}

// Guided-rendering context of one render (guide == nullptr: plain).
struct GuideCtx
{
    bbg_guide* guide = nullptr;
    GuideDev dev{};
    float lr = 0;
    int32_t batch = 0;  // training samples per Adam step
    int32_t steps = 1;  // Adam steps per wave
    int32_t* slice = nullptr; // per step: its number of samples (device)
};

// Splits each scene's training samples of the wave into gc.steps batches of
// gc.batch: slice[scene * steps + k].
__global__ void GuideSliceKernel(GuideDev g, int32_t* slice, int32_t batch, int32_t steps)
{
    for (int32_t i = threadIdx.x; i < g.n_scenes * steps; i += blockDim.x)
    {
        int32_t scene = i / steps, k = i % steps;
        slice[i] = max(0, min(batch, g.rec_n[scene] - k * batch));
    }
}

__global__ void GuideWaveStartKernel(WaveDev w, GuideDev g)
{
    const int64_t n = w.wave[1];
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        g.rec_id[i] = -1;
    }
    if (blockIdx.x == 0)
    {
        for (int32_t k = threadIdx.x; k < g.n_scenes; k += blockDim.x)
        {
            g.rec_count[k] = 0;
            g.wsum[k] = 0;
        }
    }
}

// Bucketing of a level's guide queries by scene for the grouped forward:
// counts, chunk-aligned offsets (with the padding marked -1), scatter.
__global__ void GuideBucketCountKernel(WaveDev w, GuideDev g)
{
    extern __shared__ int32_t hist[];
    for (int32_t k = threadIdx.x; k < g.n_scenes; k += blockDim.x)
    {
        hist[k] = 0;
    }
    __syncthreads();
    const int32_t n = w.counts[5];
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        atomicAdd(&hist[w.flags[g.queue[j]] >> kSceneShift], 1);
    }
    __syncthreads();
    for (int32_t k = threadIdx.x; k < g.n_scenes; k += blockDim.x)
    {
        if (hist[k])
        {
            atomicAdd(&g.bucket[k], hist[k]);
        }
    }
}

__global__ void GuideBucketOffsetKernel(GuideDev g)
{
    __shared__ int32_t start[kMaxGuidedScenes + 1], count[kMaxGuidedScenes];
    if (threadIdx.x == 0)
    {
        int32_t at = 0;
        for (int32_t k = 0; k < g.n_scenes; ++k)
        {
            count[k] = g.bucket[k];
            start[k] = at;
            g.chunk_start[k] = at / kGuideGroupChunk;
            g.cursor[k] = at;
            g.bucket[k] = 0; // ready for the next level
            at += (count[k] + kGuideGroupChunk - 1) / kGuideGroupChunk * kGuideGroupChunk;
        }
        start[g.n_scenes] = at;
        g.chunk_start[g.n_scenes] = at / kGuideGroupChunk;
    }
    __syncthreads();
    for (int32_t k = 0; k < g.n_scenes; ++k)
    {
        for (int32_t i = start[k] + count[k] + threadIdx.x; i < start[k + 1]; i += blockDim.x)
        {
            g.sorted[i] = -1;
        }
    }
}

// Scatter with one atomic per scene per warp: the lanes of a warp that hold
// the same scene (__match_any_sync) take consecutive positions from a range
// their lowest lane reserves (a wave's queries mostly belong to one or two
// scenes, so per-query atomics would all hit one cursor).
__global__ void GuideBucketScatterKernel(WaveDev w, GuideDev g)
{
    const int32_t n = w.counts[5];
    const int lane = threadIdx.x & 31;
    for (int32_t j0 = blockIdx.x * blockDim.x; j0 < n; j0 += gridDim.x * blockDim.x) // warp-uniform
    {
        const int32_t j = j0 + int32_t(threadIdx.x);
        const bool active = j < n;
        const int32_t slot = active ? g.queue[j] : 0;
        const int32_t scene = active ? (w.flags[slot] >> kSceneShift) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, scene);
        const int leader = __ffs(peers) - 1;
        int32_t base = 0;
        if (active && lane == leader)
        {
            base = atomicAdd(&g.cursor[scene], __popc(peers));
        }
        base = __shfl_sync(0xffffffffu, base, leader);
        if (active)
        {
            g.sorted[base + __popc(peers & ((1u << lane) - 1u))] = slot;
        }
    }
}

bbg_status EnqueueLevel(const Grids& gr, const SceneDev& s, const WaveDev& w, const GuideCtx& gc, int parity,
                        int shape, cudaStream_t st)
{
    const OneScene one{ s, FilmDev{} };
    ResetKernel<<<1, 1, 0, st>>>(w, parity);
    LaunchTrace(shape, gr, one, w, parity, false, st);
    if (gc.guide)
    {
        if (w.sorted)
        {
            ShadeKindsKernel<<<gr.kinds, kBlock, 0, st>>>(one, w, parity);
            ShadeScatterKernel<<<gr.scatter, kBlock, 0, st>>>(w, parity);
        }
        GuidedShadeA<<<gr.shade_a, kBlock, 0, st>>>(one, w, gc.dev, parity);
        BBG_TRY(GuideForward(gc.guide, gc.dev.raw, gc.dev.queue, w.counts + 5, 0, gc.dev.out, st));
        GuidedShadeB<<<gr.shade_b, kBlock, 0, st>>>(one, w, gc.dev, parity);
    }
    else
    {
        if (w.sorted)
        {
            ShadeKindsKernel<<<gr.kinds, kBlock, 0, st>>>(one, w, parity);
            ShadeScatterKernel<<<gr.scatter, kBlock, 0, st>>>(w, parity);
        }
        ShadeKernel<<<gr.shade, kBlock, 0, st>>>(one, w, parity);
    }
    LaunchTrace(shape, gr, one, w, parity, true, st);
    return BBG_OK;
}

bbg_status Enqueue(bbg_integrator* I, const Grids& gr, const SceneDev& s, const FilmDev& film, const GuideCtx& gc,
                   int iterations, int shape, cudaStream_t st)
{
    WaveDev w = I->Wave();
    const OneScene one{ s, film };
    RaygenKernel<<<gr.raygen, kBlock, 0, st>>>(one, w);
    if (gc.guide && gc.dev.train)
    {
        GuideWaveStartKernel<<<gr.raygen, kBlock, 0, st>>>(w, gc.dev);
    }
    for (int k = 0; k < iterations; ++k)
    {
        BBG_TRY(EnqueueLevel(gr, s, w, gc, k & 1, shape, st));
    }
    FilmKernel<<<gr.film, kBlock, 0, st>>>(one, w);
    BBG_CUDA(cudaGetLastError());
    return BBG_OK;
}

// The online training steps on the wave's records (after all its levels):
// gc.steps Adam steps of each scene's guide on that scene's records (guides[k]
// for scene k; one scene outside batches). Only scenes first..last can have
// records (the scenes the wave's paths belong to).
bbg_status EnqueueTraining(bbg_integrator* I, const GuideCtx& gc, bbg_guide* const* guides, cudaStream_t st,
                           int32_t first = 0, int32_t last = 0)
{
    WaveDev w = I->Wave();
    const int32_t ns = gc.dev.n_scenes;
    const dim3 grid(unsigned(std::max(1, 256 / ns)), unsigned(ns));
    GuideFinalizeKernel<<<grid, 256, 0, st>>>(w, gc.dev);
    GuideNormalizeKernel<<<grid, 256, 0, st>>>(gc.dev);
    GuideSliceKernel<<<1, 256, 0, st>>>(gc.dev, gc.slice, gc.batch, gc.steps);
    for (int32_t scene = first; scene <= last && scene < ns; ++scene)
    {
        for (int32_t k = 0; k < gc.steps; ++k)
        {
            size_t off = size_t(scene) * size_t(gc.dev.rec_cap) + size_t(k) * size_t(gc.batch);
            const int32_t* n = gc.slice + size_t(scene) * gc.steps + k;
            BBG_TRY(GuideAccumulate(guides[scene], gc.dev.t_raw + off * kGuideRaw, gc.dev.t_dir + off * 3,
                                    gc.dev.t_w + off, n, 0, gc.batch, st));
            BBG_TRY(GuideApply(guides[scene], gc.lr, n, 0, st));
        }
    }
    BBG_CUDA(cudaGetLastError());
    return BBG_OK;
}

bool SameGuide(const GuideDev& a, const GuideDev& b)
{
    return std::memcmp(&a, &b, sizeof(GuideDev)) == 0;
}

bool SameScene(const SceneDev& a, const SceneDev& b)
{
    return std::memcmp(&a, &b, sizeof(SceneDev)) == 0;
}

bool SameFilm(const FilmDev& a, const FilmDev& b)
{
    return std::memcmp(&a, &b, sizeof(FilmDev)) == 0;
}

// Checks a render's sampler and filter choice and prepares the Gaussian
// filter's table (once per sigma and extent) for MakeSceneDev.
bbg_status PrepareSamplerAndFilter(bbg_integrator* I, const bbg_camera* cam, const bbg_render_params* p)
{
    if (p->shade_order != BBG_SHADE_SORTED && p->shade_order != BBG_SHADE_QUEUE)
    {
        return Fail(BBG_ERR_INVALID_ARG, "shade_order %d", p->shade_order);
    }
    I->shade_sort = p->shade_order == BBG_SHADE_SORTED;
    if (p->sampler != BBG_SAMPLER_INDEPENDENT &&
        (p->sampler != BBG_SAMPLER_STRATIFIED || p->x_samples <= 0 || p->spp % p->x_samples != 0))
    {
        return Fail(BBG_ERR_INVALID_ARG, "sampler %d with x_samples %d does not divide spp %d", p->sampler,
                    p->x_samples, p->spp);
    }
    if (cam->filter_type < BBG_FILTER_BOX || cam->filter_type > BBG_FILTER_GAUSSIAN ||
        (cam->filter_type == BBG_FILTER_GAUSSIAN && !(cam->filter_sigma > 0 && cam->filter_extent > 0)))
    {
        return Fail(BBG_ERR_INVALID_ARG, "filter type %d (sigma %g, extent %g)", cam->filter_type,
                    double(cam->filter_sigma), double(cam->filter_extent));
    }
    if (cam->filter_type == BBG_FILTER_GAUSSIAN &&
        (I->filter_key[0] != cam->filter_sigma || I->filter_key[1] != cam->filter_extent || !I->filter_cdf.p))
    {
        std::vector<float> cdf(kFilterCdfFloats);
        GaussianFilterCdf(cam->filter_sigma, cam->filter_extent, cdf.data());
        BBG_TRY(I->filter_cdf.upload(cdf.data(), cdf.size(), I->stream));
        BBG_CUDA(cudaStreamSynchronize(I->stream));
        I->filter_key[0] = cam->filter_sigma;
        I->filter_key[1] = cam->filter_extent;
    }
    return BBG_OK;
}

// The kernels' view of one scene: its accel, shading data, lights and camera.
SceneDev MakeSceneDev(bbg_integrator* I, const bbg_camera* cam, const bbg_render_params* p)
{
    bbg_accel* a = I->accel;
    SceneDev s{};
    s.accel = a->view();
    s.prim_info = I->prim_info.p;
    s.tri_indices = a->tri_indices.p;
    s.positions = a->positions.p;
    s.normals = a->normals.p;
    s.tangents = a->tangents.p;
    s.spheres = a->spheres.p;
    s.materials = I->materials.p;
    s.lights = I->lights.p;
    s.light_func = I->light_func.p;
    s.light_cdf = I->light_cdf.p;
    s.light_pmf = I->light_pmf.p;
    s.alias_prob = I->alias_prob.p;
    s.alias_idx = I->alias_idx.p;
    s.infinite = I->infinite.p;
    s.n_lights = I->n_lights;
    s.n_infinite = I->n_infinite;
    s.light_func_integral = I->func_integral;
    s.light_alias = p->light_alias && I->n_lights > 0 ? 1 : 0;
    s.max_bounces = I->max_bounces;
    s.rr_min_bounces = I->rr_min_bounces;
    s.regularize = I->regularize;
    s.spp = p->spp;
    s.seed = p->seed;
    s.sampler_kind = p->sampler;
    s.x_samples = p->x_samples;
    s.jitter = p->jitter ? 1 : 0;
    s.camera.filter_type = cam->filter_type;
    s.camera.filter_cdf = cam->filter_type == BBG_FILTER_GAUSSIAN ? I->filter_cdf.p : nullptr;
    s.camera.width = cam->width;
    s.camera.height = cam->height;
    std::memcpy(s.camera.origin, cam->origin, sizeof(float) * 3);
    std::memcpy(s.camera.lower_left, cam->lower_left, sizeof(float) * 3);
    std::memcpy(s.camera.horizontal, cam->horizontal, sizeof(float) * 3);
    std::memcpy(s.camera.vertical, cam->vertical, sizeof(float) * 3);
    std::memcpy(s.camera.u, cam->u, sizeof(float) * 3);
    std::memcpy(s.camera.v, cam->v, sizeof(float) * 3);
    s.camera.lens_radius = cam->lens_radius;
    s.camera.filter_extent = cam->filter_extent;
    return s;
}

bbg_status Render(bbg_integrator* I, const bbg_camera* cam, const bbg_render_params* p, bbg_film* film, bbg_memory mem,
                  bbg_render_stats* stats)
{
    if (!cam || !p || !film || !film->rgb_sum || !film->count || !film->moments || p->spp <= 0 || cam->width <= 0 ||
        cam->height <= 0 || (mem != BBG_MEM_HOST && mem != BBG_MEM_DEVICE))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_render: bad argument");
    }
    if (p->guide && p->guide->device != I->device)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_render: the guide lives on device %d, the integrator on device %d",
                    p->guide->device, I->device);
    }
    const int64_t n_pixels = int64_t(cam->width) * cam->height;
    const int64_t n_paths = n_pixels * p->spp;

    // Wave size: whole pixels, at most the requested (or tuned, or default) paths.
    int64_t want = p->wave_paths > 0 ? p->wave_paths : I->tuned_wave > 0 ? I->tuned_wave : (int64_t(1) << 22);
    int64_t px_per_wave = std::max<int64_t>(1, want / p->spp);
    px_per_wave = std::min(px_per_wave, n_pixels);
    const int64_t wave_paths = px_per_wave * p->spp;
    if (wave_paths > (int64_t(1) << 30))
    {
        return Fail(BBG_ERR_INVALID_ARG, "wave of %lld paths exceeds 2^30", (long long)wave_paths);
    }
    BBG_TRY(I->Reserve(wave_paths));
    BBG_TRY(PrepareSamplerAndFilter(I, cam, p));

    SceneDev s = MakeSceneDev(I, cam, p);

    FilmDev f{};
    if (mem == BBG_MEM_DEVICE)
    {
        f.rgb_sum = film->rgb_sum;
        f.count = film->count;
        f.moments = film->moments;
        f.path_L = film->path_L;
    }
    else
    {
        BBG_TRY(I->film_rgb.alloc(3 * size_t(n_pixels)));
        BBG_TRY(I->film_count.alloc(size_t(n_pixels)));
        BBG_TRY(I->film_moments.alloc(2 * size_t(n_pixels)));
        f.rgb_sum = I->film_rgb.p;
        f.count = I->film_count.p;
        f.moments = I->film_moments.p;
        if (film->path_L)
        {
            BBG_TRY(I->film_path_L.alloc(3 * size_t(n_paths)));
            f.path_L = I->film_path_L.p;
        }
    }

    cudaStream_t st = I->stream;
    BBG_CUDA(cudaMemsetAsync(I->stats.p, 0, 2 * sizeof(unsigned long long), st));
    cudaEvent_t e0, e1;
    BBG_CUDA(cudaEventCreate(&e0));
    BBG_CUDA(cudaEventCreate(&e1));

    GuideCtx gc;
    if (p->guide)
    {
        gc.guide = p->guide;
        gc.lr = p->guide_lr > 0 ? p->guide_lr : 1e-2f;
        int32_t batch = p->guide_batch > 0 ? p->guide_batch : (1 << 16);
        int32_t steps = p->guide_steps > 0 ? p->guide_steps : 1;
        if (p->guide_train && int64_t(batch) * steps > (int64_t(1) << 28))
        {
            return Fail(BBG_ERR_INVALID_ARG, "guide_batch x guide_steps exceeds 2^28 training samples per wave");
        }
        // Record every stride-th path so a wave yields about steps batches
        // (about two guided vertices per path).
        int64_t samples = int64_t(batch) * steps;
        int32_t stride = int32_t(std::max<int64_t>(1, (2 * wave_paths + samples - 1) / samples));
        BBG_TRY(I->ReserveGuide(wave_paths, p->guide_train ? int32_t(samples) : 0, steps));
        gc.batch = batch;
        gc.steps = steps;
        gc.dev = I->Guide(p->guide_train ? 1 : 0, stride);
        gc.dev.rec_cap = p->guide_train ? int32_t(samples) : 0;
        gc.slice = I->g_slice.p;
        gc.dev.select = (p->guide_select > 0 && p->guide_select <= 1) ? p->guide_select : 0.5f;
        int dummy;
        BBG_TRY(GuidePrepare(gc.guide, &dummy));
        if (p->guide_train)
        {
            BBG_TRY(GuideReserveTraining(gc.guide, batch));
        }
    }

    const int iterations = I->max_bounces + 1;
    const Grids gr;
    // The tuned launch shape over the accel's layout (8-wide when selected).
    const int trace_shape =
        I->shape + (!I->accel->wide8_active() ? 0 : I->accel->has_spheres ? kNumShapes : 2 * kNumShapes);
    bool use_graph = p->use_graph != 0;
    if (use_graph && (!I->graph || I->graph_capacity != wave_paths || I->graph_iterations != iterations ||
                      !SameScene(I->graph_scene, s) || !SameFilm(I->graph_film, f) ||
                      I->graph_guide_handle != gc.guide || !SameGuide(I->graph_guide, gc.dev) ||
                      I->graph_guide_lr != gc.lr || I->graph_shape != trace_shape ||
                      I->graph_shade_sort != I->shade_sort))
    {
        if (I->graph)
        {
            cudaGraphExecDestroy(I->graph);
            I->graph = nullptr;
        }
        cudaGraph_t g;
        BBG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        bbg_status es = Enqueue(I, gr, s, f, gc, iterations, trace_shape, st);
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        BBG_TRY(es);
        if (ce != cudaSuccess)
        {
            return Fail(BBG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        }
        BBG_CUDA(cudaGraphInstantiate(&I->graph, g, 0));
        cudaGraphDestroy(g);
        I->graph_capacity = wave_paths;
        I->graph_iterations = iterations;
        I->graph_scene = s;
        I->graph_film = f;
        I->graph_guide = gc.dev;
        I->graph_guide_handle = gc.guide;
        I->graph_guide_lr = gc.lr;
        I->graph_shape = trace_shape;
        I->graph_shade_sort = I->shade_sort;
    }

    // Device time of the render itself: buffer set-up and graph capture
    // (once per configuration) are not included.
    BBG_CUDA(cudaEventRecord(e0, st));
    for (int64_t base = 0; base < n_paths; base += wave_paths)
    {
        int64_t count = std::min(wave_paths, n_paths - base);
        BBG_CUDA(cudaStreamSynchronize(st)); // the pinned wave record is reused
        I->wave_host[0] = base;
        I->wave_host[1] = count;
        BBG_CUDA(cudaMemcpyAsync(I->wave.p, I->wave_host, 2 * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        if (use_graph)
        {
            BBG_CUDA(cudaGraphLaunch(I->graph, st));
        }
        else
        {
            BBG_TRY(Enqueue(I, gr, s, f, gc, iterations, trace_shape, st));
        }
        // Paths still queued after max_bounces + 1 levels only come from
        // material-less surfaces, which do not count a bounce
        // (path_integrator.cpp:95-100): drain them level by level.
        int32_t left = 0;
        int parity = iterations & 1;
        BBG_CUDA(cudaMemcpyAsync(&left, I->counts.p + parity, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaStreamSynchronize(st));
        int extra = 0;
        const int max_extra = p->pass_through_levels > 0 ? p->pass_through_levels : kMaxPassThroughLevels;
        while (left > 0)
        {
            if (++extra > max_extra)
            {
                return Fail(BBG_ERR_TIMEOUT, "paths still alive after %d pass-through levels", max_extra);
            }
            BBG_TRY(EnqueueLevel(gr, s, I->Wave(), gc, parity, trace_shape, st));
            parity ^= 1;
            BBG_CUDA(cudaMemcpyAsync(&left, I->counts.p + parity, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            BBG_CUDA(cudaStreamSynchronize(st));
        }
        if (extra > 0)
        {
            // Re-run the film pass for this wave after the extra levels.
            FilmKernel<<<gr.film, kBlock, 0, st>>>(OneScene{ s, f }, I->Wave());
        }
        if (gc.guide && gc.dev.train)
        {
            BBG_TRY(EnqueueTraining(I, gc, &gc.guide, st));
        }
    }
    BBG_CUDA(cudaEventRecord(e1, st));
    BBG_CUDA(cudaStreamSynchronize(st));
    BBG_CUDA(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (gc.guide)
    {
        BBG_TRY(GuideCheckStatus(gc.guide));
    }

    if (mem == BBG_MEM_HOST)
    {
        BBG_CUDA(cudaMemcpy(film->rgb_sum, f.rgb_sum, 3 * sizeof(float) * size_t(n_pixels), cudaMemcpyDeviceToHost));
        BBG_CUDA(cudaMemcpy(film->count, f.count, sizeof(int32_t) * size_t(n_pixels), cudaMemcpyDeviceToHost));
        BBG_CUDA(cudaMemcpy(film->moments, f.moments, 2 * sizeof(float) * size_t(n_pixels), cudaMemcpyDeviceToHost));
        if (film->path_L)
        {
            BBG_CUDA(cudaMemcpy(film->path_L, f.path_L, 3 * sizeof(float) * size_t(n_paths), cudaMemcpyDeviceToHost));
        }
    }
    if (stats)
    {
        unsigned long long c[2];
        BBG_CUDA(cudaMemcpy(c, I->stats.p, sizeof(c), cudaMemcpyDeviceToHost));
        stats->paths = n_paths;
        stats->closest_rays = int64_t(c[0]);
        stats->shadow_rays = int64_t(c[1]);
        stats->device_ms = ms;
    }
    return BBG_OK;
}

// Queue counters, statistics and the pinned wave record of a wave engine
// (an integrator, or the engine of a batch); the stream must exist.
bbg_status InitWaveEngine(bbg_integrator* I)
{
    BBG_TRY(I->counts.alloc(8));
    BBG_TRY(I->stats.alloc(2));
    BBG_TRY(I->wave.alloc(2));
    BBG_CUDA(cudaMallocHost(reinterpret_cast<void**>(&I->wave_host), 2 * sizeof(int64_t)));
    return BBG_OK;
}

// Fills the GGX and rough-dielectric energy tables on the current device,
// once per process and device (they depend on nothing but the reference's
// fixed sample set).
bbg_status EnsureEnergyTables()
{
    static std::mutex mutex;
    static std::vector<bool> done;
    int dev = 0;
    BBG_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mutex);
    if (size_t(dev) < done.size() && done[dev])
    {
        return BBG_OK;
    }
    DevBuf<P2> u12;
    DevBuf<float> u0;
    BBG_TRY(u12.alloc(kEnergySamples));
    BBG_TRY(u0.alloc(kEnergySamples));
    EnergySamplesKernel<<<1, 1>>>(u0.p, u12.p);
    GgxEnergyTablesKernel<<<(kEnergyTableSize * kEnergyTableSize + 127) / 128, 128>>>(u12.p);
    GgxEnergyAverageKernel<<<1, kEnergyTableSize>>>();
    constexpr int kDmsEntries = 2 * kEnergyTableSize * kEnergyTableSize * kEnergyTableSize;
    DielectricEnergyTablesKernel<<<(kDmsEntries + 127) / 128, 128>>>(u0.p, u12.p);
    DielectricEnergyAverageKernel<<<(kEnergyTableSize * kEnergyTableSize + 127) / 128, 128>>>();
    BBG_CUDA(cudaGetLastError());
    BBG_CUDA(cudaDeviceSynchronize());
    if (done.size() <= size_t(dev))
    {
        done.resize(size_t(dev) + 1, false);
    }
    done[dev] = true;
    return BBG_OK;
}

bbg_status CreateIntegrator(bbg_integrator* I, bbg_accel* a, const int32_t* prim_material, const bbg_material* mats,
                            int32_t n_mats, const bbg_light* lights, int32_t n_lights)
{
    if (!a->has_shading)
    {
        return Fail(BBG_ERR_INVALID_ARG, "the accel was created without normals/tangents");
    }
    std::vector<MaterialDev> md(size_t(std::max(n_mats, 1)));
    for (int32_t i = 0; i < n_mats; ++i)
    {
        BBG_TRY(MakeMaterial(mats[i], &md[i]));
        if (md[i].ms)
        {
            BBG_TRY(EnsureEnergyTables());
        }
    }
    std::vector<int4> info(size_t(a->n_prims));
    for (int32_t i = 0; i < a->n_prims; ++i)
    {
        int32_t m = prim_material ? prim_material[i] : -1;
        if (m >= n_mats || m < -1)
        {
            return Fail(BBG_ERR_INVALID_ARG, "primitive %d names material %d of %d", i, m, n_mats);
        }
        info[i] = make_int4(a->host_prim_shape[i].x, a->host_prim_shape[i].y, m, -1);
    }

    // Geometry view for the host-side light set-up.
    bbg_geometry g{};
    g.n_vertices = int32_t(a->host_positions.size() / 3);
    g.positions = a->host_positions.data();
    g.n_triangles = int32_t(a->host_tri_indices.size() / 3);
    g.tri_indices = a->host_tri_indices.data();
    g.n_spheres = int32_t(a->host_spheres.size());
    g.spheres = a->host_spheres.data();
    g.n_prims = a->n_prims;
    std::vector<int32_t> kind(size_t(a->n_prims)), index(size_t(a->n_prims));
    for (int32_t i = 0; i < a->n_prims; ++i)
    {
        kind[i] = a->host_prim_shape[i].x;
        index[i] = a->host_prim_shape[i].y;
    }
    g.prim_kind = kind.data();
    g.prim_index = index.data();

    std::vector<LightDev> ld(size_t(std::max(n_lights, 1)));
    std::vector<float> power(size_t(std::max(n_lights, 1)));
    std::vector<int32_t> infinite;
    for (int32_t i = 0; i < n_lights; ++i)
    {
        BBG_TRY(MakeLight(lights[i], g, a->bounds, &ld[i], &power[i]));
        if (lights[i].type == BBG_LIGHT_UNIFORM_INFINITE)
        {
            infinite.push_back(i);
        }
        if (lights[i].type == BBG_LIGHT_DIFFUSE_AREA)
        {
            // Integrator::Integrator keeps one light per primitive (a HashMap insert).
            if (info[lights[i].prim].w < 0)
            {
                info[lights[i].prim].w = i;
            }
        }
    }
    I->n_lights = n_lights;
    std::vector<float> func(size_t(std::max(n_lights, 1))), cdf(size_t(n_lights + 1)), pmf(size_t(std::max(n_lights, 1)));
    std::vector<float> prob(size_t(std::max(n_lights, 1)));
    std::vector<int32_t> alias(size_t(std::max(n_lights, 1)));
    if (n_lights > 0)
    {
        BuildDistribution(power.data(), n_lights, func.data(), cdf.data(), &I->func_integral);
        for (int32_t i = 0; i < n_lights; ++i)
        {
            pmf[i] = func[i] / (I->func_integral * n_lights);
        }
        BuildAlias(pmf.data(), n_lights, prob.data(), alias.data());
    }
    I->pmf.assign(pmf.begin(), pmf.begin() + n_lights);
    I->n_infinite = int32_t(infinite.size());
    if (infinite.empty())
    {
        infinite.push_back(0);
    }

    BBG_CUDA(cudaStreamCreateWithFlags(&I->stream, cudaStreamNonBlocking));
    BBG_TRY(I->prim_info.upload(info.data(), info.size(), I->stream));
    BBG_TRY(I->materials.upload(md.data(), md.size(), I->stream));
    BBG_TRY(I->lights.upload(ld.data(), ld.size(), I->stream));
    BBG_TRY(I->light_func.upload(func.data(), func.size(), I->stream));
    BBG_TRY(I->light_cdf.upload(cdf.data(), cdf.size(), I->stream));
    BBG_TRY(I->light_pmf.upload(pmf.data(), pmf.size(), I->stream));
    BBG_TRY(I->alias_prob.upload(prob.data(), prob.size(), I->stream));
    BBG_TRY(I->alias_idx.upload(alias.data(), alias.size(), I->stream));
    BBG_TRY(I->infinite.upload(infinite.data(), infinite.size(), I->stream));
    BBG_TRY(InitWaveEngine(I));
    BBG_CUDA(cudaStreamSynchronize(I->stream));
    return BBG_OK;
}


// ---------------------------------------------------------------- batches of scenes

using BatchGrids = GridsT<SceneTable>;

// One bounce level of a batch. With guides (gc.guide set; groups[k] is
// scene k's guide), the level's guide queries are bucketed by scene and the
// scenes' MLPs run as one grouped forward between the two guided passes.
bbg_status EnqueueBatchLevel(const BatchGrids& gr, const SceneTable& t, const WaveDev& w, const GuideCtx& gc,
                             const GuideGroup* groups, int parity, int shape, cudaStream_t st)
{
    ResetKernel<<<1, 1, 0, st>>>(w, parity);
    LaunchTrace(shape, gr, t, w, parity, false, st);
    if (gc.guide)
    {
        if (w.sorted)
        {
            ShadeKindsKernel<<<gr.kinds, kBlock, 0, st>>>(t, w, parity);
            ShadeScatterKernel<<<gr.scatter, kBlock, 0, st>>>(w, parity);
        }
        GuidedShadeA<<<gr.shade_a, kBlock, 0, st>>>(t, w, gc.dev, parity);
        GuideBucketCountKernel<<<gr.scatter, kBlock, size_t(gc.dev.n_scenes) * sizeof(int32_t), st>>>(w, gc.dev);
        GuideBucketOffsetKernel<<<1, 256, 0, st>>>(gc.dev);
        GuideBucketScatterKernel<<<gr.scatter, kBlock, 0, st>>>(w, gc.dev);
        BBG_TRY(GuideForwardGrouped(gc.dev.raw, gc.dev.sorted, gc.dev.chunk_start, gc.dev.n_scenes, groups,
                                    gc.dev.out, st));
        GuidedShadeB<<<gr.shade_b, kBlock, 0, st>>>(t, w, gc.dev, parity);
    }
    else
    {
        if (w.sorted)
        {
            ShadeKindsKernel<<<gr.kinds, kBlock, 0, st>>>(t, w, parity);
            ShadeScatterKernel<<<gr.scatter, kBlock, 0, st>>>(w, parity);
        }
        ShadeKernel<<<gr.shade, kBlock, 0, st>>>(t, w, parity);
    }
    LaunchTrace(shape, gr, t, w, parity, true, st);
    return BBG_OK;
}

bbg_status EnqueueBatch(const BatchGrids& gr, const SceneTable& t, const WaveDev& w, const GuideCtx& gc,
                        const GuideGroup* groups, int iterations, int shape, cudaStream_t st)
{
    RaygenKernel<<<gr.raygen, kBlock, 0, st>>>(t, w);
    if (gc.guide && gc.dev.train)
    {
        GuideWaveStartKernel<<<gr.raygen, kBlock, 0, st>>>(w, gc.dev);
    }
    for (int k = 0; k < iterations; ++k)
    {
        BBG_TRY(EnqueueBatchLevel(gr, t, w, gc, groups, k & 1, shape, st));
    }
    FilmKernel<<<gr.film, kBlock, 0, st>>>(t, w);
    BBG_CUDA(cudaGetLastError());
    return BBG_OK;
}

} // namespace

struct bbg_batch
{
    int device = 0;        // the device that was current at creation; every call runs there
    bbg_integrator engine; // wave buffers, stream and graph of the batch
    bbg::DevBuf<bbg::SceneDev> scenes;
    bbg::DevBuf<bbg::FilmDev> films;
    bbg::DevBuf<int64_t> pixel_start;
    std::vector<bbg::SceneDev> host_scenes;
    std::vector<bbg::FilmDev> host_films;
    std::vector<int64_t> host_pixel_start;
    // Graph of one wave, valid while these stay the same (the tables are read
    // from device memory at run time, so their contents may change).
    int64_t graph_capacity = -1;
    int graph_iterations = -1;
    bbg::SceneTable graph_table{};
    int graph_shape = -1;
    bool graph_shade_sort = false;
    bbg::GuideDev graph_guide{};
    const bbg::GuideGroup* graph_groups = nullptr;
    int32_t shape = 0;      // as bbg_integrator::shape, for the batch
    int64_t tuned_wave = 0; // as bbg_integrator::tuned_wave
    // Guided batches: each scene's guide, as the grouped forward reads them.
    bbg::DevBuf<bbg::GuideGroup> groups;
    std::vector<bbg::GuideGroup> host_groups;
    std::vector<bbg_guide*> guides;
};

namespace
{

bbg_status RenderBatch(bbg_batch* B, int32_t n, bbg_integrator* const* integrators, const bbg_camera* cams,
                       const bbg_render_params* params, bbg_film* films, bbg_memory mem, bbg_render_stats* stats)
{
    if (n <= 0 || n > kMaxBatchScenes || !integrators || !cams || !params || !films ||
        (mem != BBG_MEM_HOST && mem != BBG_MEM_DEVICE))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_batch_render: bad argument");
    }
    const int32_t spp = params[0].spp;
    int iterations = 0;
    B->host_scenes.resize(size_t(n));
    B->host_films.resize(size_t(n));
    B->host_pixel_start.assign(size_t(n) + 1, 0);
    for (int32_t i = 0; i < n; ++i)
    {
        bbg_integrator* I = integrators[i];
        const bbg_camera* cam = &cams[i];
        const bbg_film* film = &films[i];
        if (!I || params[i].spp != spp || spp <= 0 || (params[i].guide != nullptr) != (params[0].guide != nullptr) ||
            cam->width <= 0 || cam->height <= 0 || !film->rgb_sum || !film->count || !film->moments)
        {
            return Fail(BBG_ERR_INVALID_ARG,
                        "bbg_batch_render: scene %d: bad argument (spp must match; a guide for every scene or none)",
                        int(i));
        }
        if (I->device != B->device || (params[i].guide && params[i].guide->device != B->device))
        {
            return Fail(BBG_ERR_INVALID_ARG, "bbg_batch_render: scene %d lives on another device than the batch (%d)",
                        int(i), B->device);
        }
        for (int32_t j = 0; j < i && params[i].guide; ++j)
        {
            if (params[j].guide == params[i].guide)
            {
                return Fail(BBG_ERR_INVALID_ARG, "bbg_batch_render: scenes %d and %d share a guide", int(j), int(i));
            }
        }
        if (!I->accel->ordered)
        {
            return Fail(BBG_ERR_UNSUPPORTED, "bbg_batch_render: scene %d uses the reference-order traversal", int(i));
        }
        const int64_t n_pixels = int64_t(cam->width) * cam->height;
        if (params[i].sampler != BBG_SAMPLER_INDEPENDENT)
        {
            return Fail(BBG_ERR_UNSUPPORTED, "bbg_batch_render: scene %d: batches use the independent sampler",
                        int(i));
        }
        BBG_TRY(PrepareSamplerAndFilter(I, cam, &params[i]));
        B->host_scenes[i] = MakeSceneDev(I, cam, &params[i]);
        FilmDev f{};
        if (mem == BBG_MEM_DEVICE)
        {
            f = FilmDev{ film->rgb_sum, film->count, film->moments, film->path_L };
        }
        else
        {
            BBG_TRY(I->film_rgb.alloc(3 * size_t(n_pixels)));
            BBG_TRY(I->film_count.alloc(size_t(n_pixels)));
            BBG_TRY(I->film_moments.alloc(2 * size_t(n_pixels)));
            f = FilmDev{ I->film_rgb.p, I->film_count.p, I->film_moments.p, nullptr };
            if (film->path_L)
            {
                BBG_TRY(I->film_path_L.alloc(3 * size_t(n_pixels) * size_t(spp)));
                f.path_L = I->film_path_L.p;
            }
        }
        B->host_films[i] = f;
        B->host_pixel_start[i + 1] = B->host_pixel_start[i] + n_pixels;
        iterations = std::max(iterations, I->max_bounces + 1);
    }
    const int64_t total_pixels = B->host_pixel_start[size_t(n)];
    const int64_t n_paths = total_pixels * spp;

    bbg_integrator* E = &B->engine;
    cudaStream_t st = E->stream;
    if (params[0].shade_order != BBG_SHADE_SORTED && params[0].shade_order != BBG_SHADE_QUEUE)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_batch_render: shade_order %d", params[0].shade_order);
    }
    E->shade_sort = params[0].shade_order == BBG_SHADE_SORTED;
    BBG_TRY(B->scenes.upload(B->host_scenes.data(), B->host_scenes.size(), st));
    BBG_TRY(B->films.upload(B->host_films.data(), B->host_films.size(), st));
    BBG_TRY(B->pixel_start.upload(B->host_pixel_start.data(), B->host_pixel_start.size(), st));
    const SceneTable table{ B->scenes.p, B->films.p, B->pixel_start.p, n, spp };

    int64_t want = params[0].wave_paths > 0 ? params[0].wave_paths
                   : B->tuned_wave > 0      ? B->tuned_wave
                                            : (int64_t(1) << 22);
    const int64_t px_per_wave = std::min(std::max<int64_t>(1, want / spp), total_pixels);
    const int64_t wave_paths = px_per_wave * spp;
    if (wave_paths > (int64_t(1) << 30))
    {
        return Fail(BBG_ERR_INVALID_ARG, "wave of %lld paths exceeds 2^30", (long long)wave_paths);
    }
    BBG_TRY(E->Reserve(wave_paths));
    const BatchGrids gr;

    // Guides: one per scene, trained on that scene's records; the training
    // settings are the first scene's.
    GuideCtx gc;
    const bbg_render_params* p0 = &params[0];
    if (p0->guide)
    {
        if (n > kMaxGuidedScenes)
        {
            return Fail(BBG_ERR_UNSUPPORTED, "bbg_batch_render: at most %d scenes with guides", int(kMaxGuidedScenes));
        }
        gc.guide = p0->guide;
        gc.lr = p0->guide_lr > 0 ? p0->guide_lr : 1e-2f;
        const int32_t batch = p0->guide_batch > 0 ? p0->guide_batch : (1 << 16);
        const int32_t steps = p0->guide_steps > 0 ? p0->guide_steps : 1;
        const int64_t samples = int64_t(batch) * steps;
        if (p0->guide_train && samples * n > (int64_t(1) << 28))
        {
            return Fail(BBG_ERR_INVALID_ARG, "guide_batch x guide_steps x scenes exceeds 2^28 training samples");
        }
        const int32_t stride = int32_t(std::max<int64_t>(1, (2 * wave_paths + samples - 1) / samples));
        BBG_TRY(E->ReserveGuide(wave_paths, p0->guide_train ? int32_t(samples) : 0, steps, n, true));
        gc.batch = batch;
        gc.steps = steps;
        gc.dev = E->Guide(p0->guide_train ? 1 : 0, stride);
        gc.dev.rec_cap = p0->guide_train ? int32_t(samples) : 0;
        gc.dev.n_scenes = n;
        gc.slice = E->g_slice.p;
        gc.dev.select = (p0->guide_select > 0 && p0->guide_select <= 1) ? p0->guide_select : 0.5f;
        B->guides.assign(size_t(n), nullptr);
        B->host_groups.resize(size_t(n));
        for (int32_t i = 0; i < n; ++i)
        {
            bbg_guide* G = params[i].guide;
            int dummy;
            BBG_TRY(GuidePrepare(G, &dummy));
            if (p0->guide_train)
            {
                BBG_TRY(GuideReserveTraining(G, batch));
            }
            B->guides[i] = G;
            B->host_groups[i] = GuideGroup{ G->bf16.p, G->params.p, G->tc_status.p, G->bounds };
        }
        BBG_TRY(B->groups.upload(B->host_groups.data(), B->host_groups.size(), st));
    }
    const GuideGroup* groups = p0->guide ? B->groups.p : nullptr;
    // The 8-wide layout only when every scene's accel traverses it.
    bool all_wide = true, any_spheres = false;
    for (int32_t i = 0; i < n; ++i)
    {
        all_wide = all_wide && integrators[i]->accel->wide8_active();
        any_spheres = any_spheres || integrators[i]->accel->has_spheres;
    }
    const int trace_shape = B->shape + (!all_wide ? 0 : any_spheres ? kNumShapes : 2 * kNumShapes);
    const bool use_graph = params[0].use_graph != 0;
    if (use_graph && (!E->graph || B->graph_capacity != wave_paths || B->graph_iterations != iterations ||
                      std::memcmp(&B->graph_table, &table, sizeof(table)) != 0 || B->graph_shape != trace_shape ||
                      B->graph_shade_sort != E->shade_sort || !SameGuide(B->graph_guide, gc.dev) ||
                      B->graph_groups != groups))
    {
        if (E->graph)
        {
            cudaGraphExecDestroy(E->graph);
            E->graph = nullptr;
        }
        cudaGraph_t g;
        BBG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        bbg_status es = EnqueueBatch(gr, table, E->Wave(), gc, groups, iterations, trace_shape, st);
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        BBG_TRY(es);
        if (ce != cudaSuccess)
        {
            return Fail(BBG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        }
        BBG_CUDA(cudaGraphInstantiate(&E->graph, g, 0));
        cudaGraphDestroy(g);
        B->graph_capacity = wave_paths;
        B->graph_iterations = iterations;
        B->graph_table = table;
        B->graph_shape = trace_shape;
        B->graph_shade_sort = E->shade_sort;
        B->graph_guide = gc.dev;
        B->graph_groups = groups;
    }

    BBG_CUDA(cudaMemsetAsync(E->stats.p, 0, 2 * sizeof(unsigned long long), st));
    cudaEvent_t e0, e1;
    BBG_CUDA(cudaEventCreate(&e0));
    BBG_CUDA(cudaEventCreate(&e1));
    BBG_CUDA(cudaEventRecord(e0, st));
    for (int64_t base = 0; base < n_paths; base += wave_paths)
    {
        int64_t count = std::min(wave_paths, n_paths - base);
        BBG_CUDA(cudaStreamSynchronize(st)); // the pinned wave record is reused
        E->wave_host[0] = base;
        E->wave_host[1] = count;
        BBG_CUDA(cudaMemcpyAsync(E->wave.p, E->wave_host, 2 * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        if (use_graph)
        {
            BBG_CUDA(cudaGraphLaunch(E->graph, st));
        }
        else
        {
            BBG_TRY(EnqueueBatch(gr, table, E->Wave(), gc, groups, iterations, trace_shape, st));
        }
        // Paths still queued come from material-less surfaces (no bounce
        // counted): drain them level by level, then redo the film pass.
        int32_t left = 0;
        int parity = iterations & 1;
        BBG_CUDA(cudaMemcpyAsync(&left, E->counts.p + parity, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaStreamSynchronize(st));
        int extra = 0;
        const int max_extra = p0->pass_through_levels > 0 ? p0->pass_through_levels : kMaxPassThroughLevels;
        while (left > 0)
        {
            if (++extra > max_extra)
            {
                return Fail(BBG_ERR_TIMEOUT, "paths still alive after %d pass-through levels", max_extra);
            }
            BBG_TRY(EnqueueBatchLevel(gr, table, E->Wave(), gc, groups, parity, trace_shape, st));
            parity ^= 1;
            BBG_CUDA(cudaMemcpyAsync(&left, E->counts.p + parity, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            BBG_CUDA(cudaStreamSynchronize(st));
        }
        if (extra > 0)
        {
            FilmKernel<<<gr.film, kBlock, 0, st>>>(table, E->Wave());
        }
        if (gc.guide && gc.dev.train)
        {
            // The scenes whose pixels the wave's paths cover.
            const auto& ps = B->host_pixel_start;
            const int64_t px_lo = base / spp, px_hi = (base + count - 1) / spp;
            const int32_t first = int32_t(std::upper_bound(ps.begin(), ps.end(), px_lo) - ps.begin()) - 1;
            const int32_t last = int32_t(std::upper_bound(ps.begin(), ps.end(), px_hi) - ps.begin()) - 1;
            BBG_TRY(EnqueueTraining(E, gc, B->guides.data(), st, first, last));
        }
    }
    BBG_CUDA(cudaEventRecord(e1, st));
    BBG_CUDA(cudaStreamSynchronize(st));
    BBG_CUDA(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (int32_t i = 0; p0->guide && i < n; ++i)
    {
        BBG_TRY(GuideCheckStatus(params[i].guide));
    }
    if (mem == BBG_MEM_HOST)
    {
        for (int32_t i = 0; i < n; ++i)
        {
            const FilmDev& f = B->host_films[i];
            const size_t np = size_t(B->host_pixel_start[i + 1] - B->host_pixel_start[i]);
            BBG_CUDA(cudaMemcpy(films[i].rgb_sum, f.rgb_sum, 3 * sizeof(float) * np, cudaMemcpyDeviceToHost));
            BBG_CUDA(cudaMemcpy(films[i].count, f.count, sizeof(int32_t) * np, cudaMemcpyDeviceToHost));
            BBG_CUDA(cudaMemcpy(films[i].moments, f.moments, 2 * sizeof(float) * np, cudaMemcpyDeviceToHost));
            if (films[i].path_L)
            {
                BBG_CUDA(cudaMemcpy(films[i].path_L, f.path_L, 3 * sizeof(float) * np * size_t(spp),
                                    cudaMemcpyDeviceToHost));
            }
        }
    }
    if (stats)
    {
        unsigned long long c[2];
        BBG_CUDA(cudaMemcpy(c, E->stats.p, sizeof(c), cudaMemcpyDeviceToHost));
        stats->paths = n_paths;
        stats->closest_rays = int64_t(c[0]);
        stats->shadow_rays = int64_t(c[1]);
        stats->device_ms = ms;
    }
    return BBG_OK;
}


// ---------------------------------------------------------------- autotuning

// One probe render of a candidate: launch shape, wave size, spp -> its
// device time and paths.
using ProbeFn = std::function<bbg_status(int shape, int64_t wave, int32_t spp, double* ms, int64_t* paths)>;

std::mutex g_tune_mutex;
std::map<std::vector<int64_t>, bbg_tuning> g_tune_cache;

bbg_tuning TuningOf(int shape, int64_t wave, double per_mpath)
{
    bbg_tuning t{};
    t.block = kShapes[shape].block;
    t.short_stack = kShapes[shape].short_stack;
    t.wave_paths = wave;
    t.probe_ms = per_mpath;
    return t;
}

int ShapeOf(int32_t block, int32_t short_stack)
{
    for (int k = 0; k < kNumShapes; ++k)
    {
        if (kShapes[k].block == block && kShapes[k].short_stack == short_stack)
        {
            return k;
        }
    }
    return -1;
}

// Times each launch shape at the default wave size, then each wave size
// (2^20 .. 2^24 paths) the render can fill with the best shape; every candidate twice, the faster
// run counting, compared per path. A probe of wave w renders enough samples
// per pixel for about two waves (at most the render's spp).
bbg_status Tune(const std::vector<int64_t>& key, int64_t pixels, int32_t spp, const ProbeFn& probe, bbg_tuning* out)
{
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end())
        {
            *out = it->second;
            out->from_cache = 1;
            return BBG_OK;
        }
    }
    const int64_t total = pixels * spp;
    auto measure = [&](int shape, int64_t wave, double* per_mpath) -> bbg_status {
        int32_t ps = int32_t(std::min<int64_t>(spp, std::max<int64_t>(1, (2 * wave + pixels - 1) / pixels)));
        double best = 1e300;
        for (int r = 0; r < 2; ++r)
        {
            double ms = 0;
            int64_t paths = 0;
            BBG_TRY(probe(shape, wave, ps, &ms, &paths));
            best = std::min(best, ms / (double(paths) / 1e6));
        }
        *per_mpath = best;
        return BBG_OK;
    };
    const int64_t w0 = std::min<int64_t>(int64_t(1) << 22, total);
    int best_shape = 0;
    int64_t best_wave = w0;
    double best_t = 1e300;
    for (int k = 0; k < kNumShapes; ++k)
    {
        double t;
        BBG_TRY(measure(k, w0, &t));
        if (t < best_t)
        {
            best_t = t;
            best_shape = k;
        }
    }
    // Larger waves leave fewer bounce levels with few rays, but hold more
    // device memory (kWaveBytesPerPath of path state each): a wave size is
    // tried only if its state fits in a quarter of the free device memory.
    size_t free_bytes = 0, total_bytes = 0;
    BBG_CUDA(cudaMemGetInfo(&free_bytes, &total_bytes));
    for (int e = 20; e <= 26; ++e)
    {
        int64_t wave = int64_t(1) << e;
        if (wave == w0 || wave > total || double(wave) * kWaveBytesPerPath > 0.25 * double(free_bytes))
        {
            continue;
        }
        double t;
        BBG_TRY(measure(best_shape, wave, &t));
        if (t < best_t)
        {
            best_t = t;
            best_wave = wave;
        }
    }
    *out = TuningOf(best_shape, best_wave, best_t);
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = *out;
    return BBG_OK;
}

std::vector<int64_t> SceneKey(const bbg_integrator* I, const bbg_camera* cam, int32_t spp)
{
    const bbg_accel* a = I->accel;
    return { a->n_prims, a->n_nodes, a->max_depth, cam->width, cam->height, spp, I->max_bounces };
}

bbg_status AutotuneIntegrator(bbg_integrator* I, const bbg_camera* cam, const bbg_render_params* p, bbg_tuning* out)
{
    if (!cam || !p || !out || p->spp <= 0 || p->guide || cam->width <= 0 || cam->height <= 0)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_integrator_autotune: bad argument");
    }
    const int64_t pixels = int64_t(cam->width) * cam->height;
    std::vector<float> rgb(3 * static_cast<size_t>(pixels)), mom(2 * static_cast<size_t>(pixels));
    std::vector<int32_t> cnt(static_cast<size_t>(pixels));
    ProbeFn probe = [&](int shape, int64_t wave, int32_t spp, double* ms, int64_t* paths) -> bbg_status {
        const int saved = I->shape;
        I->shape = shape;
        bbg_render_params q = *p;
        q.spp = spp;
        q.wave_paths = wave;
        q.use_graph = 1;
        bbg_film f{ rgb.data(), cnt.data(), mom.data(), nullptr };
        bbg_render_stats st{};
        bbg_status s = Render(I, cam, &q, &f, BBG_MEM_HOST, &st);
        I->shape = saved;
        *ms = st.device_ms;
        *paths = st.paths;
        return s;
    };
    std::vector<int64_t> key = SceneKey(I, cam, p->spp);
    key.insert(key.begin(), 0);
    BBG_TRY(Tune(key, pixels, p->spp, probe, out));
    I->shape = ShapeOf(out->block, out->short_stack);
    I->tuned_wave = out->wave_paths;
    return BBG_OK;
}

bbg_status AutotuneBatch(bbg_batch* B, int32_t n, bbg_integrator* const* integrators, const bbg_camera* cams,
                         const bbg_render_params* params, bbg_tuning* out)
{
    if (n <= 0 || n > kMaxBatchScenes || !integrators || !cams || !params || !out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_batch_autotune: bad argument");
    }
    std::vector<int64_t> key{ 1, n };
    int64_t pixels = 0;
    std::vector<std::vector<float>> rgb(static_cast<size_t>(n)), mom(static_cast<size_t>(n));
    std::vector<std::vector<int32_t>> cnt(static_cast<size_t>(n));
    std::vector<bbg_film> films(static_cast<size_t>(n));
    for (int32_t i = 0; i < n; ++i)
    {
        if (!integrators[i] || cams[i].width <= 0 || cams[i].height <= 0)
        {
            return Fail(BBG_ERR_INVALID_ARG, "bbg_batch_autotune: scene %d: bad argument", int(i));
        }
        std::vector<int64_t> k = SceneKey(integrators[i], &cams[i], params[i].spp);
        key.insert(key.end(), k.begin(), k.end());
        const int64_t px = int64_t(cams[i].width) * cams[i].height;
        pixels += px;
        rgb[i].resize(3 * size_t(px));
        mom[i].resize(2 * size_t(px));
        cnt[i].resize(size_t(px));
        films[i] = bbg_film{ rgb[i].data(), cnt[i].data(), mom[i].data(), nullptr };
    }
    ProbeFn probe = [&](int shape, int64_t wave, int32_t spp, double* ms, int64_t* paths) -> bbg_status {
        const int saved = B->shape;
        B->shape = shape;
        std::vector<bbg_render_params> q(params, params + n);
        for (auto& r : q)
        {
            r.spp = spp;
            r.wave_paths = wave;
            r.use_graph = 1;
        }
        bbg_render_stats st{};
        bbg_status s = RenderBatch(B, n, integrators, cams, q.data(), films.data(), BBG_MEM_HOST, &st);
        B->shape = saved;
        *ms = st.device_ms;
        *paths = st.paths;
        return s;
    };
    BBG_TRY(Tune(key, pixels, params[0].spp, probe, out));
    B->shape = ShapeOf(out->block, out->short_stack);
    B->tuned_wave = out->wave_paths;
    return BBG_OK;
}

} // namespace

extern "C" {

bbg_status bbg_integrator_create(bbg_accel* accel, const int32_t* prim_material, const bbg_material* materials,
                                 int32_t n_materials, const bbg_light* lights, int32_t n_lights, int32_t max_bounces,
                                 int32_t rr_min_bounces, int32_t regularize_bsdf, bbg_integrator** out)
{
    if (!out || !accel || n_materials < 0 || n_lights < 0 || (n_materials > 0 && !materials) ||
        (n_lights > 0 && !lights) || max_bounces < 0)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_integrator_create: bad argument");
    }
    *out = nullptr;
    if (accel->n_prims == 0)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "integrator over an empty scene");
    }
    DeviceScope ds(accel->device);
    auto* I = new bbg_integrator;
    I->device = accel->device;
    I->accel = accel;
    I->max_bounces = max_bounces;
    I->rr_min_bounces = rr_min_bounces;
    I->regularize = regularize_bsdf;
    bbg_status s = CreateIntegrator(I, accel, prim_material, materials, n_materials, lights, n_lights);
    if (s != BBG_OK)
    {
        delete I;
        return s;
    }
    *out = I;
    return BBG_OK;
}

bbg_status bbg_integrator_destroy(bbg_integrator* I)
{
    if (I)
    {
        DeviceScope ds(I->device);
        if (I->stream) cudaStreamSynchronize(I->stream);
        delete I;
    }
    return BBG_OK;
}

bbg_status bbg_integrator_light_pmf(const bbg_integrator* I, float* pmf_out)
{
    if (!I || (!pmf_out && I->n_lights > 0))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_integrator_light_pmf: bad argument");
    }
    std::memcpy(pmf_out, I->pmf.data(), sizeof(float) * I->pmf.size());
    return BBG_OK;
}

bbg_status bbg_render(bbg_integrator* I, const bbg_camera* camera, const bbg_render_params* params, bbg_film* film,
                      bbg_memory mem, bbg_render_stats* stats)
{
    if (!I)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_render: null integrator");
    }
    DeviceScope ds(I->device);
    return Render(I, camera, params, film, mem, stats);
}

bbg_status bbg_ggx_energy_tables(float* e_out, float* e_avg_out)
{
    if (!e_out || !e_avg_out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_ggx_energy_tables: bad argument");
    }
    BBG_TRY(CheckDevice());
    BBG_TRY(EnsureEnergyTables());
    BBG_CUDA(cudaMemcpyFromSymbol(e_out, g_ggx_e, sizeof(g_ggx_e)));
    BBG_CUDA(cudaMemcpyFromSymbol(e_avg_out, g_ggx_e_avg, sizeof(g_ggx_e_avg)));
    return BBG_OK;
}

bbg_status bbg_dielectric_energy_tables(float* e_out, float* e_inv_out, float* e_avg_out, float* e_inv_avg_out)
{
    if (!e_out || !e_inv_out || !e_avg_out || !e_inv_avg_out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_dielectric_energy_tables: bad argument");
    }
    BBG_TRY(CheckDevice());
    BBG_TRY(EnsureEnergyTables());
    BBG_CUDA(cudaMemcpyFromSymbol(e_out, g_dms_e, sizeof(g_dms_e)));
    BBG_CUDA(cudaMemcpyFromSymbol(e_inv_out, g_dms_e_inv, sizeof(g_dms_e_inv)));
    BBG_CUDA(cudaMemcpyFromSymbol(e_avg_out, g_dms_e_avg, sizeof(g_dms_e_avg)));
    BBG_CUDA(cudaMemcpyFromSymbol(e_inv_avg_out, g_dms_e_inv_avg, sizeof(g_dms_e_inv_avg)));
    return BBG_OK;
}

bbg_status bbg_bsdf_probe(const bbg_material* material, int32_t front_face, int32_t n, const float* wo,
                          const float* wi, const float* u, float* out)
{
    if (!material || n < 0 || (n > 0 && (!wo || !wi || !u || !out)))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_bsdf_probe: bad argument");
    }
    BBG_TRY(CheckDevice());
    MaterialDev md{};
    BBG_TRY(MakeMaterial(*material, &md));
    if (md.ms)
    {
        BBG_TRY(EnsureEnergyTables());
    }
    if (n == 0)
    {
        return BBG_OK;
    }
    DevBuf<float> d_wo, d_wi, d_u, d_out;
    BBG_TRY(d_wo.upload(wo, 3 * size_t(n)));
    BBG_TRY(d_wi.upload(wi, 3 * size_t(n)));
    BBG_TRY(d_u.upload(u, 3 * size_t(n)));
    BBG_TRY(d_out.alloc(12 * size_t(n)));
    BsdfProbeKernel<<<std::min((n + 127) / 128, 1024), 128>>>(md, front_face, n, d_wo.p, d_wi.p, d_u.p, d_out.p);
    BBG_CUDA(cudaGetLastError());
    BBG_CUDA(cudaMemcpy(out, d_out.p, 12 * size_t(n) * sizeof(float), cudaMemcpyDeviceToHost));
    return BBG_OK;
}

bbg_status bbg_sampler_draws(int32_t px, int32_t py, int32_t seed, int32_t sample, int32_t n, float* out)
{
    if (!out || n <= 0 || n > (1 << 20))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_sampler_draws: bad argument");
    }
    BBG_TRY(CheckDevice());
    DevBuf<float> d;
    BBG_TRY(d.alloc(size_t(n)));
    SamplerDrawsKernel<<<1, 1>>>(px, py, seed, sample, n, d.p);
    BBG_CUDA(cudaGetLastError());
    BBG_CUDA(cudaMemcpy(out, d.p, sizeof(float) * size_t(n), cudaMemcpyDeviceToHost));
    return BBG_OK;
}

bbg_status bbg_batch_create(bbg_batch** out)
{
    if (!out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_batch_create: bad argument");
    }
    *out = nullptr;
    BBG_TRY(CheckDevice());
    auto* B = new bbg_batch;
    cudaGetDevice(&B->device);
    B->engine.device = B->device;
    cudaError_t e = cudaStreamCreateWithFlags(&B->engine.stream, cudaStreamNonBlocking);
    bbg_status s = e == cudaSuccess ? InitWaveEngine(&B->engine)
                                    : Fail(BBG_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    if (s != BBG_OK)
    {
        delete B;
        return s;
    }
    *out = B;
    return BBG_OK;
}

bbg_status bbg_batch_destroy(bbg_batch* B)
{
    if (B)
    {
        DeviceScope ds(B->device);
        if (B->engine.stream) cudaStreamSynchronize(B->engine.stream);
        delete B;
    }
    return BBG_OK;
}

bbg_status bbg_batch_render(bbg_batch* B, int32_t n, bbg_integrator* const* integrators, const bbg_camera* cameras,
                            const bbg_render_params* params, bbg_film* films, bbg_memory mem, bbg_render_stats* stats)
{
    if (!B)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_batch_render: null batch");
    }
    DeviceScope ds(B->device);
    return RenderBatch(B, n, integrators, cameras, params, films, mem, stats);
}

bbg_status bbg_integrator_autotune(bbg_integrator* I, const bbg_camera* camera, const bbg_render_params* params,
                                   bbg_tuning* out)
{
    if (!I)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_integrator_autotune: null integrator");
    }
    DeviceScope ds(I->device);
    return AutotuneIntegrator(I, camera, params, out);
}

bbg_status bbg_integrator_set_tuning(bbg_integrator* I, const bbg_tuning* t)
{
    if (!I || !t || ShapeOf(t->block, t->short_stack) < 0 || t->wave_paths < 0 || t->wave_paths > (int64_t(1) << 30))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_integrator_set_tuning: not a supported configuration");
    }
    I->shape = ShapeOf(t->block, t->short_stack);
    I->tuned_wave = t->wave_paths;
    return BBG_OK;
}

bbg_status bbg_batch_autotune(bbg_batch* B, int32_t n, bbg_integrator* const* integrators, const bbg_camera* cameras,
                              const bbg_render_params* params, bbg_tuning* out)
{
    if (!B)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_batch_autotune: null batch");
    }
    DeviceScope ds(B->device);
    return AutotuneBatch(B, n, integrators, cameras, params, out);
}

} // extern "C"
