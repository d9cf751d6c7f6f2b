// GPU accel beside the reference BVH: upload of geometry and a flattened SAH
// tree, and the batched closest-hit / any-hit traversal kernels.

#include "accel.cuh"
#include "wide8_build.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace bbg
{

constexpr int kTraceBlock = 128;

bbg_status CheckDevice()
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
    {
        return Fail(BBG_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));
    }
    int dev = 0;
    BBG_CUDA(cudaGetDevice(&dev));
    int major = 0, minor = 0;
    BBG_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    BBG_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
    if (major != 10)
    {
        return Fail(BBG_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a", dev, major, minor);
    }
    return BBG_OK;
}

int CurrentSmCount()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
    {
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    return sms;
}

int PersistentGrid(const void* kernel, int block, size_t smem)
{
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem);
    return CurrentSmCount() * std::max(per_sm, 1);
}

// Reference-order traversal (and the counting run): one thread per ray,
// grid-stride over the batch. Rays are two float4 (o.xyz d.x)(d.yz t_min
// t_max); hits one float4 (prim bits, t, u, v).
template <bool ANY, bool COUNT>
__global__ void __launch_bounds__(kTraceBlock) TraceKernel(AccelView a, const float4* __restrict__ rays, int64_t n,
                                                           float4* __restrict__ hits, uint8_t* __restrict__ occluded,
                                                           unsigned long long* counters)
{
    uint32_t nodes = 0, prims = 0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    {
        float4 r0 = __ldg(rays + 2 * i);
        float4 r1 = __ldg(rays + 2 * i + 1);
        RayQ q = MakeRayQ(V3{ r0.x, r0.y, r0.z }, V3{ r0.w, r1.x, r1.y });
        TraceResult res = TraceReference<ANY, COUNT>(a, q, r1.z, r1.w, &nodes, &prims);
        if (ANY)
        {
            occluded[i] = res.prim >= 0 ? 1 : 0;
        }
        else
        {
            hits[i] = make_float4(__int_as_float(res.prim), res.t, res.u, res.v);
        }
    }
    if (COUNT)
    {
        unsigned long long nv = nodes, np = prims;
        for (int off = 16; off > 0; off >>= 1)
        {
            nv += __shfl_down_sync(0xffffffffu, nv, off);
            np += __shfl_down_sync(0xffffffffu, np, off);
        }
        if ((threadIdx.x & 31) == 0)
        {
            atomicAdd(counters, nv);
            atomicAdd(counters + 1, np);
        }
    }
}

template <bool ANY>
struct BatchSrc
{
    const float4* rays;
    float4* hits;
    uint8_t* occluded;

    __device__ __forceinline__ void Load(int32_t i, RayQ* q, float* t_min, float* t_max) const
    {
        float4 r0 = __ldg(rays + 2 * size_t(i));
        float4 r1 = __ldg(rays + 2 * size_t(i) + 1);
        *q = MakeRayQ(V3{ r0.x, r0.y, r0.z }, V3{ r0.w, r1.x, r1.y });
        *t_min = r1.z;
        *t_max = r1.w;
    }
    __device__ __forceinline__ void Store(int32_t i, const TraceResult& r) const
    {
        if (ANY)
        {
            occluded[i] = r.prim >= 0 ? 1 : 0;
        }
        else
        {
            hits[i] = make_float4(__int_as_float(r.prim), r.t, r.u, r.v);
        }
    }
};

// Ordered traversal: persistent warps pulling rays from a work counter, over
// the child-box layout or (WIDE) the 8-wide layout.
template <bool ANY, bool WIDE, bool SPHERES = true>
__global__ void __launch_bounds__(kTraceBlock) PersistentTraceKernel(AccelView a, const float4* __restrict__ rays,
                                                                     int32_t n, float4* __restrict__ hits,
                                                                     uint8_t* __restrict__ occluded, int32_t* next)
{
    BatchSrc<ANY> src{ rays, hits, occluded };
    if constexpr (WIDE)
    {
        TracePersistentWide<ANY, BatchSrc<ANY>, kTraversalBlock, kShortStack, SPHERES>(a, n, next, src);
    }
    else
    {
        TracePersistent<ANY>(a, n, next, src);
    }
}

template <bool ANY>
static bbg_status LaunchTrace(bbg_accel* a, const float4* rays, int64_t n, float4* hits, uint8_t* occ,
                              cudaStream_t stream)
{
    if (n == 0)
    {
        return BBG_OK;
    }
    if (a->n_prims == 0)
    {
        // No geometry: every query misses (the reference cannot build a tree
        // over zero primitives).
        if (ANY)
        {
            BBG_CUDA(cudaMemsetAsync(occ, 0, size_t(n), stream));
            return BBG_OK;
        }
        return Fail(BBG_ERR_UNSUPPORTED, "closest-hit query on an accel with no primitives");
    }
    if (a->counting || !a->ordered)
    {
        auto k = a->counting ? TraceKernel<ANY, true> : TraceKernel<ANY, false>;
        int grid = PersistentGrid(reinterpret_cast<const void*>(k), kTraceBlock);
        grid = int(std::min<int64_t>(grid, (n + kTraceBlock - 1) / kTraceBlock));
        k<<<grid, kTraceBlock, 0, stream>>>(a->view(), rays, n, hits, occ, a->counters.p);
    }
    else
    {
        auto k = !a->wide8_active() ? PersistentTraceKernel<ANY, false>
                 : a->has_spheres   ? PersistentTraceKernel<ANY, true>
                                    : PersistentTraceKernel<ANY, true, false>;
        int grid = PersistentGrid(reinterpret_cast<const void*>(k), kTraceBlock);
        grid = int(std::min<int64_t>(grid, (n + kTraceBlock - 1) / kTraceBlock));
        const int64_t chunk = int64_t(1) << 30;
        for (int64_t c = 0; c < n; c += chunk)
        {
            int32_t m = int32_t(std::min(chunk, n - c));
            BBG_CUDA(cudaMemsetAsync(a->work.p, 0, sizeof(int32_t), stream));
            k<<<grid, kTraceBlock, 0, stream>>>(a->view(), rays + 2 * c, m, hits ? hits + c : nullptr,
                                                occ ? occ + c : nullptr, a->work.p);
        }
    }
    BBG_CUDA(cudaGetLastError());
    return BBG_OK;
}

bbg_status LaunchIntersect(bbg_accel* a, const float4* rays, int64_t n, float4* hits, cudaStream_t stream)
{
    return LaunchTrace<false>(a, rays, n, hits, nullptr, stream);
}

bbg_status LaunchIntersectAny(bbg_accel* a, const float4* rays, int64_t n, uint8_t* occluded, cudaStream_t stream)
{
    return LaunchTrace<true>(a, rays, n, nullptr, occluded, stream);
}

} // namespace bbg

using namespace bbg;

namespace
{

float BitsToFloat(uint32_t bits)
{
    float f;
    std::memcpy(&f, &bits, sizeof(f));
    return f;
}


// Shading data (the reference Mesh arrays and shapes).
bbg_status UploadShading(bbg_accel* a, const bbg_geometry* g)
{
    BBG_TRY(a->prim_shape.upload(a->host_prim_shape.data(), a->host_prim_shape.size(), a->stream));
    BBG_TRY(a->tri_indices.upload(g->tri_indices, 3 * size_t(g->n_triangles), a->stream));
    BBG_TRY(a->positions.upload(g->positions, 3 * size_t(g->n_vertices), a->stream));
    if (g->n_spheres)
    {
        BBG_TRY(a->spheres.upload(g->spheres, size_t(g->n_spheres), a->stream));
    }
    a->has_shading = g->n_triangles == 0 || (g->normals && g->tangents);
    if (g->normals && g->tangents)
    {
        BBG_TRY(a->normals.upload(g->normals, 3 * size_t(g->n_vertices), a->stream));
        BBG_TRY(a->tangents.upload(g->tangents, 3 * size_t(g->n_vertices), a->stream));
        if (g->uvs)
        {
            BBG_TRY(a->uvs.upload(g->uvs, 2 * size_t(g->n_vertices), a->stream));
        }
    }
    return BBG_OK;
}

// Collapses the binary tree (reference layout) into the 8-wide layout, the
// wide nodes chosen by the surface-area plan (Wide8PlanNode, computed bottom
// up: children follow their parent in the depth-first layout, so a reverse
// sweep sees them first). Nodes are numbered breadth first, a node's
// interior children consecutively. Returns false (no wide layout) if the
// tree is too large for the stack-entry or leaf encodings (2^23 nodes, 2^26
// slots, 31 primitives in a leaf) or too deep for the stack.
bool BuildWide8(const std::vector<bbg_bvh_node>& nodes, std::vector<float4>* out, int32_t* depth_out)
{
    auto child_of = [&](int32_t b) {
        Child8 c;
        std::memcpy(c.lo, nodes[b].bmin, sizeof(c.lo));
        std::memcpy(c.hi, nodes[b].bmax, sizeof(c.hi));
        c.bnode = b;
        return c;
    };
    std::vector<float> cost(8 * nodes.size(), 0.0f); // leaves cost 0
    std::vector<uint8_t> split(8 * nodes.size(), 0);
    for (size_t b = nodes.size(); b-- > 0;)
    {
        if (nodes[b].count == 0)
        {
            Wide8PlanNode(nodes[b], &cost[8 * (b + 1)], &cost[8 * size_t(nodes[b].offset)], &cost[8 * b], &split[8 * b]);
        }
    }
    struct Pending
    {
        int32_t bnode, wnode, depth;
    };
    std::vector<Pending> queue;
    queue.push_back({ 0, 0, 1 });
    out->assign(6, make_float4(0, 0, 0, 0));
    int32_t n_wide = 1, depth = 1;
    for (size_t qi = 0; qi < queue.size(); ++qi)
    {
        Pending pd = queue[qi];
        Child8 cs[8];
        int32_t bs[8];
        const int n = Wide8Gather(nodes.data(), split.data(), pd.bnode, bs);
        for (int c = 0; c < n; ++c)
        {
            cs[c] = child_of(bs[c]);
        }
        float plo[3], phi[3];
        Wide8Union(cs, n, plo, phi);
        int32_t slot_of[8];
        AssignSlots8(cs, n, plo, phi, slot_of);
        int32_t refs[8];
        for (int k = 0; k < 8; ++k) refs[k] = ~0; // empty: a leaf of no primitives
        for (int c = 0; c < n; ++c)
        {
            int32_t b = cs[c].bnode;
            if (nodes[b].count > 0)
            {
                // The leaf's range in the reference, without an indirection.
                if (nodes[b].count >= (1 << kWide8LeafCountBits) ||
                    nodes[b].offset >= (1 << (31 - kWide8LeafCountBits)))
                {
                    return false;
                }
                refs[slot_of[c]] = Wide8LeafRef(nodes[b].offset, int32_t(nodes[b].count));
            }
            else
            {
                if (n_wide >= (1 << 23) - 1)
                {
                    return false;
                }
                refs[slot_of[c]] = n_wide;
                queue.push_back({ b, n_wide, pd.depth + 1 });
                depth = std::max(depth, pd.depth + 1);
                ++n_wide;
            }
        }
        out->resize(6 * size_t(n_wide), make_float4(0, 0, 0, 0));
        QuantizeNode8(cs, n, slot_of, refs, out->data() + 6 * size_t(pd.wnode));
    }
    *depth_out = depth;
    return depth <= kStackCapacity;
}

enum class DeviceTree
{
    None,    // the tree is given or built on the host
    Linear,  // linear BVH built on the device (lbvh.cu)
    Sah,     // the reference's SAH tree built on the device (sah_build.cu)
    SahSplit // the same build over references split on the device (split_build.cu)
};

bbg_status CreateAccel(const bbg_geometry* g, const bbg_bvh* bvh, bbg_accel* a, DeviceTree device_tree = DeviceTree::None,
                       float split_budget = 0)
{
    const bool device_build = device_tree != DeviceTree::None;
    // Host-side checks and the tree come first: a malformed scene or tree is
    // rejected before any device work.
    BBG_TRY(CheckGeometry(g));
    a->n_prims = g->n_prims;

    // Host copies needed later (light set-up on area-light primitives).
    a->host_prim_shape.resize(size_t(g->n_prims));
    for (int32_t i = 0; i < g->n_prims; ++i)
    {
        a->host_prim_shape[i] = make_int2(g->prim_kind[i], g->prim_index[i]);
        a->has_spheres = a->has_spheres || g->prim_kind[i] == BBG_PRIM_SPHERE;
    }
    a->host_tri_indices.assign(g->tri_indices, g->tri_indices + 3 * size_t(g->n_triangles));
    a->host_positions.assign(g->positions, g->positions + 3 * size_t(g->n_vertices));
    a->host_spheres.assign(g->spheres, g->spheres + size_t(g->n_spheres));

    if (g->n_prims == 0)
    {
        BBG_TRY(CheckDevice());
        BBG_CUDA(cudaGetDevice(&a->device));
        BBG_CUDA(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking));
        return BBG_OK;
    }

    // Tree: given (the reference-built one, flattened), built on the host, or
    // (device_build) built on the device after the geometry is uploaded.
    if (device_build)
    {
        a->device_built = device_tree == DeviceTree::Linear;
        a->device_sah = device_tree == DeviceTree::Sah || device_tree == DeviceTree::SahSplit;
        a->ordered = true;
    }
    else if (bvh)
    {
        // A primitive may fill several slots (trees over split references).
        if (!bvh->nodes || !bvh->slot_prims || bvh->n_nodes <= 0 || bvh->n_slots < g->n_prims)
        {
            return Fail(BBG_ERR_INVALID_ARG, "bvh: %d slots for %d primitives", bvh->n_slots, g->n_prims);
        }
        a->host_nodes.assign(bvh->nodes, bvh->nodes + bvh->n_nodes);
        a->host_slots.assign(bvh->slot_prims, bvh->slot_prims + bvh->n_slots);
    }
    else
    {
        std::vector<float> aabbs(6 * size_t(g->n_prims));
        PrimAabbs(*g, aabbs.data());
        a->host_nodes.resize(2 * size_t(g->n_prims) - 1);
        a->host_slots.resize(size_t(g->n_prims));
        int32_t n_nodes = 0;
        BBG_TRY(BuildBvh(aabbs.data(), g->n_prims, a->host_nodes.data(), a->host_slots.data(), &n_nodes));
        a->host_nodes.resize(size_t(n_nodes));
    }
    if (!device_build)
    {
        a->n_nodes = int32_t(a->host_nodes.size());
        a->n_slots = int32_t(a->host_slots.size());
        BBG_TRY(ValidateBvh(a->host_nodes.data(), a->n_nodes, a->n_slots, g->n_prims, a->host_slots.data(),
                            &a->max_depth));
        if (a->max_depth > kStackCapacity)
        {
            return Fail(BBG_ERR_STACK_OVERFLOW, "tree depth %d exceeds the traversal stack (%d)", a->max_depth,
                        kStackCapacity);
        }
        const bbg_bvh_node& root = a->host_nodes[0];
        std::memcpy(a->bounds, root.bmin, 3 * sizeof(float));
        std::memcpy(a->bounds + 3, root.bmax, 3 * sizeof(float));
    }

    // The handle lives on the caller's current device; every later call on it
    // runs there (DeviceScope), whatever device is current then.
    BBG_TRY(CheckDevice());
    BBG_CUDA(cudaGetDevice(&a->device));
    // The allocation-free query's fixed array is reserved now, at set-up
    // (its module loads lazily), not inside that query's first call.
    BBG_TRY(ReserveStaticScratch());
    BBG_CUDA(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking));
    for (int s = 0; s < 2; ++s)
    {
        BBG_CUDA(cudaStreamCreateWithFlags(&a->copy_stream[s], cudaStreamNonBlocking));
    }
    for (int s = 0; s < bbg_accel::kHostStages; ++s)
    {
        BBG_CUDA(cudaEventCreateWithFlags(&a->ev_in[s], cudaEventDisableTiming));
        BBG_CUDA(cudaEventCreateWithFlags(&a->ev_traced[s], cudaEventDisableTiming));
        BBG_CUDA(cudaEventCreateWithFlags(&a->ev_out[s], cudaEventDisableTiming));
    }

    if (device_build)
    {
        BBG_TRY(UploadShading(a, g));
        if (device_tree == DeviceTree::SahSplit)
        {
            DevBuf<float4> ref_box;
            DevBuf<int32_t> ref_prim;
            int32_t n_refs = 0;
            BBG_TRY(SplitReferencesOnDevice(a, split_budget, &ref_box, &ref_prim, &n_refs));
            BBG_TRY(BuildSahOnDevice(a, n_refs, ref_box.p, ref_prim.p));
        }
        else if (device_tree == DeviceTree::Sah)
        {
            BBG_TRY(BuildSahOnDevice(a, g->n_prims, nullptr, nullptr));
        }
        else
        {
            BBG_TRY(BuildLbvh(a, g));
        }
        BBG_TRY(a->counters.alloc(2));
        BBG_TRY(a->work.alloc(1));
        BBG_CUDA(cudaStreamSynchronize(a->stream));
        return BBG_OK;
    }

    // Slot records in leaf order.
    std::vector<float4> slot_rec(3 * size_t(a->n_slots));
    for (int32_t s = 0; s < a->n_slots; ++s)
    {
        int32_t prim = a->host_slots[s];
        float4* r = &slot_rec[3 * size_t(s)];
        if (g->prim_kind[prim] == BBG_PRIM_TRIANGLE)
        {
            const int32_t* v = g->tri_indices + 3 * size_t(g->prim_index[prim]);
            const float* p0 = g->positions + 3 * size_t(v[0]);
            const float* p1 = g->positions + 3 * size_t(v[1]);
            const float* p2 = g->positions + 3 * size_t(v[2]);
            // Edges e1 = p1 - p0, e2 = p2 - p0 as Triangle::Intersect computes them.
            r[0] = make_float4(p0[0], p0[1], p0[2], BitsToFloat(uint32_t(prim)));
            r[1] = make_float4(p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2], 0.0f);
            r[2] = make_float4(p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2], 0.0f);
        }
        else
        {
            const bbg_sphere& sp = g->spheres[g->prim_index[prim]];
            r[0] = make_float4(sp.p[0], sp.p[1], sp.p[2], BitsToFloat(uint32_t(prim) | kSphereBit));
            r[1] = make_float4(sp.q[0], sp.q[1], sp.q[2], sp.q[3]);
            r[2] = make_float4(sp.s[0], sp.s[1], sp.s[2], sp.radius);
        }
    }
    // Child-box layout: one 64-byte record per interior node holding both
    // children's boxes and references (>= 0 interior record, < 0 ~leaf).
    {
        std::vector<int32_t> ref(size_t(a->n_nodes));
        std::vector<int2> leaves;
        int32_t n_wide = 0;
        for (int32_t i = 0; i < a->n_nodes; ++i)
        {
            const bbg_bvh_node& nd = a->host_nodes[i];
            if (nd.count > 0)
            {
                ref[i] = ~int32_t(leaves.size());
                leaves.push_back(make_int2(nd.offset, nd.count));
            }
            else
            {
                ref[i] = n_wide++;
            }
        }
        std::vector<float4> wide(4 * size_t(std::max(n_wide, 1)));
        for (int32_t i = 0; i < a->n_nodes; ++i)
        {
            const bbg_bvh_node& nd = a->host_nodes[i];
            if (nd.count > 0)
            {
                continue;
            }
            const bbg_bvh_node& c0 = a->host_nodes[i + 1];
            const bbg_bvh_node& c1 = a->host_nodes[nd.offset];
            float4* w = &wide[4 * size_t(ref[i])];
            w[0] = make_float4(c0.bmin[0], c0.bmin[1], c0.bmin[2], c0.bmax[0]);
            w[1] = make_float4(c0.bmax[1], c0.bmax[2], c1.bmin[0], c1.bmin[1]);
            w[2] = make_float4(c1.bmin[2], c1.bmax[0], c1.bmax[1], c1.bmax[2]);
            w[3] = make_float4(BitsToFloat(uint32_t(ref[i + 1])), BitsToFloat(uint32_t(ref[nd.offset])), 0.0f, 0.0f);
        }
        a->root = ref[0];
        BBG_TRY(a->wide.upload(wide.data(), wide.size(), a->stream));
        BBG_TRY(a->leaves.upload(leaves.data(), leaves.size(), a->stream));

        std::vector<float4> wide8;
        if (BuildWide8(a->host_nodes, &wide8, &a->depth8))
        {
            a->n_wide8 = int32_t(wide8.size() / 6);
            a->root8 = 0;
            a->use_wide8 = true; // the default traversal where the layout exists
            BBG_TRY(a->wide8.upload(wide8.data(), wide8.size(), a->stream));
        }
    }
    static_assert(sizeof(bbg_bvh_node) == 2 * sizeof(float4), "node layout");
    BBG_TRY(a->nodes.upload(reinterpret_cast<const float4*>(a->host_nodes.data()), 2 * size_t(a->n_nodes), a->stream));
    BBG_TRY(a->slots.upload(slot_rec.data(), slot_rec.size(), a->stream));

    BBG_TRY(UploadShading(a, g));
    BBG_TRY(a->counters.alloc(2));
    BBG_TRY(a->work.alloc(1));
    BBG_CUDA(cudaStreamSynchronize(a->stream));
    return BBG_OK;
}

constexpr int64_t kChunkRays = int64_t(1) << 21;

// Waits for every query queued on the accel's streams; errors of submitted
// queries surface here.
bbg_status Drain(bbg_accel* a)
{
    a->pending = false;
    BBG_CUDA(cudaStreamSynchronize(a->copy_stream[0]));
    BBG_CUDA(cudaStreamSynchronize(a->stream));
    BBG_CUDA(cudaStreamSynchronize(a->copy_stream[1]));
    return BBG_OK;
}

// Host-memory query: chunks of rays staged through two streams so the copies
// of one chunk overlap the traversal of the other. With wait false the call
// returns once everything is queued.
template <bool ANY>
bbg_status TraceHost(bbg_accel* a, const bbg_ray* rays, int64_t n, void* out, bool wait)
{
    // Chunks cycle through the staging ring: the copy in of chunk k + 1 and
    // the copy out of chunk k - 1 overlap the trace of chunk k. Chunk sizes
    // grow from 256K rays to 2M and shrink again towards the end (at most
    // half of what is left), so the first copy in and the last copy out,
    // which nothing overlaps, are short. All traces run in order on one
    // stream (the persistent kernel's work counter is per accel); a slot is
    // refilled only after its trace and its copy out finished, whichever
    // call (an earlier submitted one included) used it last.
    constexpr int R = bbg_accel::kHostStages;
    constexpr int64_t kFirstChunk = int64_t(1) << 18;
    const size_t out_bytes = ANY ? 1 : sizeof(bbg_hit);
    const int64_t chunk = std::min(n, kChunkRays);
    bool grow = false;
    for (int s = 0; s < R; ++s)
    {
        grow |= a->stage_in[s].n < 2 * size_t(chunk) || a->stage_out[s].n < (size_t(chunk) * out_bytes + 15) / 16;
    }
    if (grow && a->pending)
    {
        BBG_TRY(Drain(a)); // a larger slot frees the old one, which queued work may still use
    }
    for (int s = 0; s < R; ++s)
    {
        BBG_TRY(a->stage_in[s].alloc(2 * size_t(chunk)));
        BBG_TRY(a->stage_out[s].alloc((size_t(chunk) * out_bytes + 15) / 16));
    }
    cudaStream_t cin = a->copy_stream[0], cout = a->copy_stream[1], comp = a->stream;
    for (int64_t c = 0, k = 0, m = 0; c < n; c += m, ++k)
    {
        const int s = a->stage_next;
        a->stage_next = (s + 1) % R;
        const int64_t left = n - c;
        const int64_t ramp_up = kFirstChunk << std::min<int64_t>(k, 4);
        const int64_t ramp_down = std::max(left / 2, kFirstChunk);
        m = std::min({ chunk, ramp_up, ramp_down, left });
        // Waiting on an event that was never recorded is no wait.
        BBG_CUDA(cudaStreamWaitEvent(cin, a->ev_traced[s], 0));
        BBG_CUDA(cudaMemcpyAsync(a->stage_in[s].p, rays + c, size_t(m) * sizeof(bbg_ray), cudaMemcpyHostToDevice, cin));
        BBG_CUDA(cudaEventRecord(a->ev_in[s], cin));
        BBG_CUDA(cudaStreamWaitEvent(comp, a->ev_in[s], 0));
        BBG_CUDA(cudaStreamWaitEvent(comp, a->ev_out[s], 0));
        if (ANY)
        {
            BBG_TRY(LaunchIntersectAny(a, a->stage_in[s].p, m, reinterpret_cast<uint8_t*>(a->stage_out[s].p), comp));
        }
        else
        {
            BBG_TRY(LaunchIntersect(a, a->stage_in[s].p, m, a->stage_out[s].p, comp));
        }
        BBG_CUDA(cudaEventRecord(a->ev_traced[s], comp));
        BBG_CUDA(cudaStreamWaitEvent(cout, a->ev_traced[s], 0));
        BBG_CUDA(cudaMemcpyAsync(static_cast<char*>(out) + size_t(c) * out_bytes, a->stage_out[s].p,
                                 size_t(m) * out_bytes, cudaMemcpyDeviceToHost, cout));
        BBG_CUDA(cudaEventRecord(a->ev_out[s], cout));
    }
    return wait ? Drain(a) : BBG_OK;
}

// One batched query. wait false (the submit forms) queues the work on the
// accel's streams and returns; wait true returns with the results in place,
// after any submitted work (the work counter and the staging ring are the
// accel's own, so queries on it never overlap).
template <bool ANY>
bbg_status Query(bbg_accel* a, const bbg_ray* rays, int64_t n, void* out, bbg_memory mem, void* stream,
                 bool wait = true)
{
    if (!a || (n > 0 && (!rays || !out)) || n < 0 || (mem != BBG_MEM_HOST && mem != BBG_MEM_DEVICE))
    {
        return Fail(BBG_ERR_INVALID_ARG, "intersect: bad argument");
    }
    if (!wait && a->counting)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "a counting accel answers only the synchronous queries");
    }
    if (wait && a->pending)
    {
        BBG_TRY(Drain(a));
    }
    if (n == 0)
    {
        a->last_nodes = a->last_prims = 0;
        return BBG_OK;
    }
    if (a->counting)
    {
        BBG_CUDA(cudaMemset(a->counters.p, 0, 2 * sizeof(unsigned long long)));
    }
    if (!wait)
    {
        a->pending = true;
    }
    if (mem == BBG_MEM_HOST)
    {
        BBG_TRY(TraceHost<ANY>(a, rays, n, out, wait));
    }
    else if (!wait)
    {
        const float4* r = reinterpret_cast<const float4*>(rays);
        if (ANY)
        {
            BBG_TRY(LaunchIntersectAny(a, r, n, static_cast<uint8_t*>(out), a->stream));
        }
        else
        {
            BBG_TRY(LaunchIntersect(a, r, n, static_cast<float4*>(out), a->stream));
        }
    }
    else
    {
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : a->stream;
        const float4* r = reinterpret_cast<const float4*>(rays);
        if (ANY)
        {
            BBG_TRY(LaunchIntersectAny(a, r, n, static_cast<uint8_t*>(out), st));
        }
        else
        {
            BBG_TRY(LaunchIntersect(a, r, n, static_cast<float4*>(out), st));
        }
        BBG_CUDA(cudaStreamSynchronize(st));
    }
    if (a->counting)
    {
        unsigned long long c[2];
        BBG_CUDA(cudaMemcpy(c, a->counters.p, sizeof(c), cudaMemcpyDeviceToHost));
        a->last_nodes = int64_t(c[0]);
        a->last_prims = int64_t(c[1]);
    }
    return BBG_OK;
}

} // namespace

extern "C" {

bbg_status bbg_accel_create_device_build(const bbg_geometry* geometry, bbg_accel** out)
{
    if (!out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_create_device_build: out is NULL");
    }
    *out = nullptr;
    auto* a = new bbg_accel;
    bbg_status s = CreateAccel(geometry, nullptr, a, DeviceTree::Linear);
    if (s != BBG_OK)
    {
        bbg_accel_destroy(a);
        return s;
    }
    *out = a;
    return BBG_OK;
}

bbg_status bbg_accel_create_device_sah(const bbg_geometry* geometry, bbg_accel** out)
{
    if (!out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_create_device_sah: out is NULL");
    }
    *out = nullptr;
    auto* a = new bbg_accel;
    bbg_status s = CreateAccel(geometry, nullptr, a, DeviceTree::Sah);
    if (s != BBG_OK)
    {
        bbg_accel_destroy(a);
        return s;
    }
    *out = a;
    return BBG_OK;
}

bbg_status bbg_accel_create_device_split(const bbg_geometry* geometry, float budget, bbg_accel** out)
{
    if (!out || !(budget >= 0.0f) || budget > 64.0f)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_create_device_split: bad argument (budget in [0, 64])");
    }
    *out = nullptr;
    auto* a = new bbg_accel;
    bbg_status s = CreateAccel(geometry, nullptr, a, DeviceTree::SahSplit, budget);
    if (s != BBG_OK)
    {
        bbg_accel_destroy(a);
        return s;
    }
    *out = a;
    return BBG_OK;
}

bbg_status bbg_accel_create_split(const bbg_geometry* geometry, float budget, bbg_accel** out)
{
    if (!out || !(budget >= 0.0f) || budget > 64.0f)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_create_split: bad argument (budget in [0, 64])");
    }
    *out = nullptr;
    BBG_TRY(CheckGeometry(geometry));
    if (geometry->n_prims == 0)
    {
        return bbg_accel_create(geometry, nullptr, out);
    }
    std::vector<float> aabbs;
    std::vector<int32_t> ref_prims;
    BBG_TRY(SplitReferences(*geometry, budget, &aabbs, &ref_prims));
    const int32_t n_refs = int32_t(ref_prims.size());
    std::vector<bbg_bvh_node> nodes(2 * size_t(n_refs) - 1);
    std::vector<int32_t> slots(static_cast<size_t>(n_refs));
    int32_t n_nodes = 0;
    BBG_TRY(BuildBvh(aabbs.data(), n_refs, nodes.data(), slots.data(), &n_nodes));
    for (int32_t& s : slots)
    {
        s = ref_prims[size_t(s)];
    }
    const bbg_bvh tree{ n_nodes, nodes.data(), n_refs, slots.data() };
    return bbg_accel_create(geometry, &tree, out);
}

bbg_status bbg_accel_create(const bbg_geometry* geometry, const bbg_bvh* bvh, bbg_accel** out)
{
    if (!out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_create: out is NULL");
    }
    *out = nullptr;
    auto* a = new bbg_accel;
    bbg_status s = CreateAccel(geometry, bvh, a);
    if (s != BBG_OK)
    {
        bbg_accel_destroy(a);
        return s;
    }
    *out = a;
    return BBG_OK;
}

bbg_status bbg_accel_destroy(bbg_accel* a)
{
    if (!a)
    {
        return BBG_OK;
    }
    DeviceScope ds(a->device);
    if (a->stream)
    {
        cudaStreamSynchronize(a->stream);
        cudaStreamDestroy(a->stream);
    }
    for (int s = 0; s < 2; ++s)
    {
        if (a->copy_stream[s])
        {
            cudaStreamSynchronize(a->copy_stream[s]);
            cudaStreamDestroy(a->copy_stream[s]);
        }
    }
    for (int s = 0; s < bbg_accel::kHostStages; ++s)
    {
        for (cudaEvent_t e : { a->ev_in[s], a->ev_traced[s], a->ev_out[s] })
        {
            if (e)
            {
                cudaEventDestroy(e);
            }
        }
    }
    delete a;
    return BBG_OK;
}

bbg_status bbg_accel_bounds(const bbg_accel* a, float* aabb_out)
{
    if (!a || !aabb_out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_bounds: null argument");
    }
    std::memcpy(aabb_out, a->bounds, sizeof(a->bounds));
    return BBG_OK;
}

bbg_status bbg_accel_export_wide8(const bbg_accel* a, float* nodes_out, int32_t* n_nodes_out)
{
    if (!a || !n_nodes_out)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_export_wide8: bad argument");
    }
    const int32_t n = a->wide8.p ? a->n_wide8 : 0;
    *n_nodes_out = n;
    if (nodes_out && n > 0)
    {
        DeviceScope ds(a->device);
        BBG_CUDA(cudaMemcpy(nodes_out, a->wide8.p, size_t(n) * 6 * sizeof(float4), cudaMemcpyDeviceToHost));
    }
    return BBG_OK;
}

bbg_status bbg_accel_export(const bbg_accel* a, bbg_bvh_node* nodes_out, int32_t* slot_prims_out, int32_t* n_nodes_out,
                            int32_t* n_slots_out)
{
    if (!a)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_export: null accel");
    }
    if (a->device_built)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "bbg_accel_export: the tree was built on the device (no reference layout)");
    }
    if (n_nodes_out) *n_nodes_out = a->n_nodes;
    if (n_slots_out) *n_slots_out = a->n_slots;
    if (a->device_sah)
    {
        // The tree lives on the device only.
        DeviceScope ds(a->device);
        if (nodes_out)
        {
            BBG_CUDA(cudaMemcpy(nodes_out, a->nodes.p, size_t(a->n_nodes) * sizeof(bbg_bvh_node), cudaMemcpyDeviceToHost));
        }
        if (slot_prims_out)
        {
            BBG_CUDA(cudaMemcpy(slot_prims_out, a->slot_prims.p, size_t(a->n_slots) * sizeof(int32_t),
                                cudaMemcpyDeviceToHost));
        }
        return BBG_OK;
    }
    if (nodes_out) std::memcpy(nodes_out, a->host_nodes.data(), a->host_nodes.size() * sizeof(bbg_bvh_node));
    if (slot_prims_out) std::memcpy(slot_prims_out, a->host_slots.data(), a->host_slots.size() * sizeof(int32_t));
    return BBG_OK;
}

bbg_status bbg_intersect(bbg_accel* a, const bbg_ray* rays, int64_t n, bbg_hit* hits, bbg_memory mem, void* stream)
{
    if (!a)
    {
        return Fail(BBG_ERR_INVALID_ARG, "intersect: null accel");
    }
    DeviceScope ds(a->device);
    return Query<false>(a, rays, n, hits, mem, stream);
}

bbg_status bbg_intersect_any(bbg_accel* a, const bbg_ray* rays, int64_t n, uint8_t* occluded, bbg_memory mem,
                             void* stream)
{
    if (!a)
    {
        return Fail(BBG_ERR_INVALID_ARG, "intersect: null accel");
    }
    DeviceScope ds(a->device);
    return Query<true>(a, rays, n, occluded, mem, stream);
}

bbg_status bbg_intersect_submit(bbg_accel* a, const bbg_ray* rays, int64_t n, bbg_hit* hits, bbg_memory mem)
{
    if (!a)
    {
        return Fail(BBG_ERR_INVALID_ARG, "intersect: null accel");
    }
    DeviceScope ds(a->device);
    return Query<false>(a, rays, n, hits, mem, nullptr, false);
}

bbg_status bbg_intersect_any_submit(bbg_accel* a, const bbg_ray* rays, int64_t n, uint8_t* occluded, bbg_memory mem)
{
    if (!a)
    {
        return Fail(BBG_ERR_INVALID_ARG, "intersect: null accel");
    }
    DeviceScope ds(a->device);
    return Query<true>(a, rays, n, occluded, mem, nullptr, false);
}

bbg_status bbg_accel_synchronize(bbg_accel* a)
{
    if (!a)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_synchronize: null accel");
    }
    DeviceScope ds(a->device);
    return Drain(a);
}

bbg_status bbg_accel_set_traversal(bbg_accel* a, int32_t mode)
{
    if (!a || (mode != BBG_TRAVERSAL_ORDERED && mode != BBG_TRAVERSAL_REFERENCE && mode != BBG_TRAVERSAL_WIDE))
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_set_traversal: bad argument");
    }
    if (a->device_built && mode == BBG_TRAVERSAL_REFERENCE)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "a tree built on the device has no reference node layout");
    }
    if (mode == BBG_TRAVERSAL_WIDE && !a->wide8.p && a->n_prims > 0)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "no 8-wide layout for this tree (more than 2^23 nodes or deeper than %d)",
                    kStackCapacity);
    }
    a->ordered = mode != BBG_TRAVERSAL_REFERENCE;
    a->use_wide8 = mode == BBG_TRAVERSAL_WIDE;
    return BBG_OK;
}

bbg_status bbg_accel_set_counting(bbg_accel* a, int32_t enable)
{
    if (!a)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_set_counting: null accel");
    }
    if (a->device_built && enable)
    {
        return Fail(BBG_ERR_UNSUPPORTED, "counting needs the reference-order traversal (not for device-built trees)");
    }
    a->counting = enable != 0;
    return BBG_OK;
}

bbg_status bbg_accel_last_counts(const bbg_accel* a, int64_t* nodes_visited, int64_t* prims_tested)
{
    if (!a)
    {
        return Fail(BBG_ERR_INVALID_ARG, "bbg_accel_last_counts: null accel");
    }
    if (nodes_visited) *nodes_visited = a->last_nodes;
    if (prims_tested) *prims_tested = a->last_prims;
    return BBG_OK;
}

} // extern "C"
