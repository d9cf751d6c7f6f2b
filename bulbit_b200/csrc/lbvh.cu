// Linear BVH built on the device (Karras, "Maximizing Parallelism in the
// Construction of BVHs, Octrees, and k-d Trees", HPG 2012): primitive boxes
// (the same padded boxes the reference's primitives report), 30-bit Morton
// codes of their centres in the centre bounds, one radix sort, the binary
// radix tree over the sorted codes (ties broken by position), and a bottom-up
// pass that writes each interior node's child boxes in the child-box layout
// the ordered traversal reads. One primitive per leaf. The tree differs from
// the reference's SAH tree; closest hits differ only where two primitives are
// hit at exactly the same t (the primitive tests are the same).

#include "accel.cuh"
#include "build_util.cuh"
#include "wide8_build.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cfloat>
#include <cstring>

namespace bbg
{
namespace
{

constexpr int kLbvhBlock = 256;

__global__ void BoxesKernel(const int2* prim_shape, const int32_t* tri, const float* pos, const bbg_sphere* spheres,
                            int32_t n, float4* boxes, uint32_t* cbounds)
{
    uint32_t lo[3] = { 0xffffffffu, 0xffffffffu, 0xffffffffu }, hi[3] = { 0, 0, 0 };
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        float3 mn, mx;
        PrimBox(prim_shape, tri, pos, spheres, i, &mn, &mx);
        boxes[2 * i] = make_float4(mn.x, mn.y, mn.z, 0);
        boxes[2 * i + 1] = make_float4(mx.x, mx.y, mx.z, 0);
        float c[3] = { (mn.x + mx.x) * 0.5f, (mn.y + mx.y) * 0.5f, (mn.z + mx.z) * 0.5f };
        for (int k = 0; k < 3; ++k)
        {
            lo[k] = min(lo[k], FloatKey(c[k]));
            hi[k] = max(hi[k], FloatKey(c[k]));
        }
    }
    for (int k = 0; k < 3; ++k)
    {
        for (int off = 16; off > 0; off >>= 1)
        {
            lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
            hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
        }
        if ((threadIdx.x & 31) == 0)
        {
            atomicMin(&cbounds[k], lo[k]);
            atomicMax(&cbounds[3 + k], hi[k]);
        }
    }
}

__device__ __forceinline__ uint32_t Spread10(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void MortonKernel(const float4* boxes, const uint32_t* cbounds, int32_t n, uint32_t* codes,
                             int32_t* ids)
{
    float lo[3], ext[3];
    for (int k = 0; k < 3; ++k)
    {
        lo[k] = KeyFloat(cbounds[k]);
        float e = KeyFloat(cbounds[3 + k]) - lo[k];
        ext[k] = e > 0 ? e : 1.0f;
    }
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        float4 a = boxes[2 * i], b = boxes[2 * i + 1];
        float c[3] = { (a.x + b.x) * 0.5f, (a.y + b.y) * 0.5f, (a.z + b.z) * 0.5f };
        uint32_t q[3];
        for (int k = 0; k < 3; ++k)
        {
            float t = (c[k] - lo[k]) / ext[k];
            q[k] = uint32_t(fminf(fmaxf(t * 1024.0f, 0.0f), 1023.0f));
        }
        codes[i] = (Spread10(q[0]) << 2) | (Spread10(q[1]) << 1) | Spread10(q[2]);
        ids[i] = i;
    }
}

// Length of the common prefix of keys i and j (sorted codes, ties broken by
// index); -1 outside [0, n).
__device__ __forceinline__ int Delta(const uint32_t* codes, int32_t n, int32_t i, int32_t j)
{
    if (j < 0 || j >= n)
    {
        return -1;
    }
    uint32_t a = codes[i], b = codes[j];
    if (a == b)
    {
        return 32 + __clz(uint32_t(i) ^ uint32_t(j));
    }
    return __clz(a ^ b);
}

// Interior node i of the radix tree: its key range and split, children
// (>= 0 interior, < 0 ~leaf) and the parents of both.
__global__ void HierarchyKernel(const uint32_t* codes, int32_t n, int2* children, int32_t* parent_node,
                                int32_t* parent_leaf)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x)
    {
        int d = (Delta(codes, n, i, i + 1) - Delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
        int dmin = Delta(codes, n, i, i - d);
        int32_t lmax = 2;
        while (Delta(codes, n, i, i + lmax * d) > dmin)
        {
            lmax <<= 1;
        }
        int32_t l = 0;
        for (int32_t t = lmax >> 1; t >= 1; t >>= 1)
        {
            if (Delta(codes, n, i, i + (l + t) * d) > dmin)
            {
                l += t;
            }
        }
        int32_t j = i + l * d;
        int dnode = Delta(codes, n, i, j);
        int32_t s = 0;
        int32_t t = l;
        do
        {
            t = (t + 1) >> 1;
            if (Delta(codes, n, i, i + (s + t) * d) > dnode)
            {
                s += t;
            }
        } while (t > 1);
        int32_t split = i + s * d + min(d, 0);
        int32_t first = min(i, j), last = max(i, j);
        int32_t left = split == first ? ~split : split;
        int32_t right = split + 1 == last ? ~(split + 1) : split + 1;
        children[i] = make_int2(left, right);
        if (left < 0)
        {
            parent_leaf[~left] = i;
        }
        else
        {
            parent_node[left] = i;
        }
        if (right < 0)
        {
            parent_leaf[~right] = i;
        }
        else
        {
            parent_node[right] = i;
        }
    }
}

// Bottom-up: the second child to arrive at a node writes the node's record
// (both children's boxes and references), its own box and its height (leaves
// 0), then goes up; the root's height bounds the traversal stack.
__global__ void RefitKernel(const float4* boxes, const int32_t* sorted_ids, const int2* children,
                            const int32_t* parent_node, const int32_t* parent_leaf, int32_t n, int32_t* arrivals,
                            float4* node_box, int32_t* height, float4* wide)
{
    for (int32_t leaf = blockIdx.x * blockDim.x + threadIdx.x; leaf < n; leaf += gridDim.x * blockDim.x)
    {
        int32_t node = parent_leaf[leaf];
        while (node >= 0)
        {
            __threadfence();
            if (atomicAdd(&arrivals[node], 1) == 0)
            {
                break; // the sibling subtree finishes this node
            }
            __threadfence();
            int2 c = children[node];
            float4 b[4];
            int32_t refs[2] = { c.x, c.y };
            int32_t h = 0;
            for (int k = 0; k < 2; ++k)
            {
                if (refs[k] < 0)
                {
                    int32_t prim = sorted_ids[~refs[k]];
                    b[2 * k] = boxes[2 * prim];
                    b[2 * k + 1] = boxes[2 * prim + 1];
                }
                else
                {
                    b[2 * k] = __ldcg(&node_box[2 * refs[k]]);
                    b[2 * k + 1] = __ldcg(&node_box[2 * refs[k] + 1]);
                    h = max(h, __ldcg(&height[refs[k]]));
                }
            }
            __stcg(&height[node], h + 1);
            float4* w = wide + 4 * size_t(node);
            w[0] = make_float4(b[0].x, b[0].y, b[0].z, b[1].x);
            w[1] = make_float4(b[1].y, b[1].z, b[2].x, b[2].y);
            w[2] = make_float4(b[2].z, b[3].x, b[3].y, b[3].z);
            w[3] = make_float4(__int_as_float(c.x), __int_as_float(c.y), 0.0f, 0.0f);
            __stcg(&node_box[2 * node],
                   make_float4(fminf(b[0].x, b[2].x), fminf(b[0].y, b[2].y), fminf(b[0].z, b[2].z), 0));
            __stcg(&node_box[2 * node + 1],
                   make_float4(fmaxf(b[1].x, b[3].x), fmaxf(b[1].y, b[3].y), fmaxf(b[1].z, b[3].z), 0));
            node = parent_node[node];
        }
    }
}

// Leaf j holds sorted primitive j: its slot record and (first slot, count).
__global__ void SlotsKernel(const int32_t* sorted_ids, const int2* prim_shape, const int32_t* tri, const float* pos,
                            const bbg_sphere* spheres, int32_t n, float4* slots, int2* leaves)
{
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        int32_t prim = sorted_ids[j];
        int2 ps = prim_shape[prim];
        float4* r = slots + 3 * size_t(j);
        if (ps.x == BBG_PRIM_TRIANGLE)
        {
            const int32_t* v = tri + 3 * size_t(ps.y);
            const float* p0 = pos + 3 * size_t(v[0]);
            const float* p1 = pos + 3 * size_t(v[1]);
            const float* p2 = pos + 3 * size_t(v[2]);
            // Edges e1 = p1 - p0, e2 = p2 - p0 as Triangle::Intersect computes them.
            r[0] = make_float4(p0[0], p0[1], p0[2], __uint_as_float(uint32_t(prim)));
            r[1] = make_float4(__fsub_rn(p1[0], p0[0]), __fsub_rn(p1[1], p0[1]), __fsub_rn(p1[2], p0[2]), 0.0f);
            r[2] = make_float4(__fsub_rn(p2[0], p0[0]), __fsub_rn(p2[1], p0[1]), __fsub_rn(p2[2], p0[2]), 0.0f);
        }
        else
        {
            const bbg_sphere& sp = spheres[ps.y];
            r[0] = make_float4(sp.p[0], sp.p[1], sp.p[2], __uint_as_float(uint32_t(prim) | kSphereBit));
            r[1] = make_float4(sp.q[0], sp.q[1], sp.q[2], sp.q[3]);
            r[2] = make_float4(sp.s[0], sp.s[1], sp.s[2], sp.radius);
        }
        leaves[j] = make_int2(j, 1);
    }
}

// One level of the collapse into the 8-wide layout, top down: wide node w
// (w2b[w] names the radix-tree node it stands for) takes that node's two
// children and opens the interior child of largest surface area until it
// holds eight children or only leaves, allocates consecutive wide nodes for
// its interior children (the next level) and writes its record. Leaf j is
// sorted primitive j in slot j.
__global__ void Wide8LevelKernel(const int2* children, const float4* node_box, const float4* boxes,
                                 const int32_t* sorted_ids, int32_t* w2b, int32_t begin, int32_t end,
                                 int32_t capacity, int32_t* counter, int32_t* overflow, float4* wide8)
{
    auto child_of = [&](int32_t r) {
        Child8 c;
        float4 lo, hi;
        if (r < 0)
        {
            int32_t prim = sorted_ids[~r];
            lo = boxes[2 * prim];
            hi = boxes[2 * prim + 1];
        }
        else
        {
            lo = node_box[2 * r];
            hi = node_box[2 * r + 1];
        }
        c.lo[0] = lo.x, c.lo[1] = lo.y, c.lo[2] = lo.z;
        c.hi[0] = hi.x, c.hi[1] = hi.y, c.hi[2] = hi.z;
        c.bnode = r;
        return c;
    };
    for (int32_t w = begin + blockIdx.x * blockDim.x + threadIdx.x; w < end; w += gridDim.x * blockDim.x)
    {
        int32_t b = w2b[w];
        Child8 cs[8];
        int n = 0;
        int2 c2 = children[b];
        cs[n++] = child_of(c2.x);
        cs[n++] = child_of(c2.y);
        while (n < 8)
        {
            int best = -1;
            double best_area = -1;
            for (int j = 0; j < n; ++j)
            {
                if (cs[j].bnode >= 0 && Wide8Area(cs[j]) > best_area)
                {
                    best_area = Wide8Area(cs[j]);
                    best = j;
                }
            }
            if (best < 0)
            {
                break;
            }
            int2 o = children[cs[best].bnode];
            cs[best] = child_of(o.x);
            cs[n++] = child_of(o.y);
        }
        float plo[3], phi[3];
        Wide8Union(cs, n, plo, phi);
        int32_t slot_of[8];
        AssignSlots8(cs, n, plo, phi, slot_of);
        int32_t inner = 0;
        for (int c = 0; c < n; ++c)
        {
            inner += cs[c].bnode >= 0 ? 1 : 0;
        }
        int32_t base = inner > 0 ? atomicAdd(counter, inner) : 0;
        if (base + inner > capacity)
        {
            atomicExch(overflow, 1);
            continue;
        }
        int32_t refs[8];
        for (int k = 0; k < 8; ++k)
        {
            refs[k] = ~0; // empty: a leaf of no primitives
        }
        for (int c = 0, i = 0; c < n; ++c)
        {
            if (cs[c].bnode >= 0)
            {
                refs[slot_of[c]] = base + i;
                w2b[base + i] = cs[c].bnode;
                ++i;
            }
            else
            {
                refs[slot_of[c]] = Wide8LeafRef(~cs[c].bnode, 1);
            }
        }
        QuantizeNode8(cs, n, slot_of, refs, wide8 + 6 * size_t(w));
    }
}

} // namespace

// Collapses the radix tree into the 8-wide layout on the device, one kernel
// per level (the host reads the level sizes back). Leaves it unbuilt (the
// binary layout remains the default) if the tree exceeds the layout's
// encodings; every wide node stands for a distinct interior radix-tree node,
// so n - 1 nodes always suffice.
static bbg_status BuildWide8OnDevice(bbg_accel* a, int32_t n, const DevBuf<int2>& children,
                                     const DevBuf<float4>& node_box, const DevBuf<float4>& boxes,
                                     const DevBuf<int32_t>& sorted_ids, int grid)
{
    const int32_t capacity = n - 1;
    if (n < 2 || capacity >= (1 << 23) - 1 || n >= (1 << (31 - kWide8LeafCountBits)))
    {
        return BBG_OK;
    }
    cudaStream_t st = a->stream;
    DevBuf<int32_t> w2b, counter;
    BBG_TRY(w2b.alloc(size_t(capacity)));
    BBG_TRY(counter.alloc(2)); // [0] nodes allocated, [1] overflow flag
    BBG_TRY(a->wide8.alloc(6 * size_t(capacity)));
    const int32_t init[2] = { 1, 0 };
    const int32_t root = 0;
    BBG_CUDA(cudaMemcpyAsync(counter.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
    BBG_CUDA(cudaMemcpyAsync(w2b.p, &root, sizeof(root), cudaMemcpyHostToDevice, st));
    int32_t begin = 0, end = 1, depth = 0, state[2] = { 1, 0 };
    while (begin < end)
    {
        ++depth;
        if (depth > kStackCapacity)
        {
            a->wide8.reset();
            return BBG_OK;
        }
        int g = std::max(1, std::min((end - begin + kLbvhBlock - 1) / kLbvhBlock, grid));
        Wide8LevelKernel<<<g, kLbvhBlock, 0, st>>>(children.p, node_box.p, boxes.p, sorted_ids.p, w2b.p, begin, end,
                                                   capacity, counter.p, counter.p + 1, a->wide8.p);
        BBG_CUDA(cudaMemcpyAsync(state, counter.p, sizeof(state), cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaStreamSynchronize(st));
        BBG_CUDA(cudaGetLastError());
        if (state[1] != 0)
        {
            a->wide8.reset();
            return BBG_OK;
        }
        begin = end;
        end = state[0];
    }
    a->n_wide8 = end;
    a->root8 = 0;
    a->depth8 = depth;
    a->use_wide8 = true;
    return BBG_OK;
}

bbg_status BuildLbvh(bbg_accel* a, const bbg_geometry* g)
{
    const int32_t n = g->n_prims;
    cudaStream_t st = a->stream;
    const int sms = CurrentSmCount();
    const int grid = std::max(1, std::min((n + kLbvhBlock - 1) / kLbvhBlock, 8 * sms));

    DevBuf<float4> boxes;
    DevBuf<uint32_t> cbounds, codes, codes_sorted;
    DevBuf<int32_t> ids, ids_sorted, parent_node, parent_leaf, arrivals, height;
    DevBuf<int2> children;
    DevBuf<float4> node_box;
    BBG_TRY(boxes.alloc(2 * size_t(n)));
    BBG_TRY(cbounds.alloc(6));
    BBG_TRY(codes.alloc(size_t(n)));
    BBG_TRY(codes_sorted.alloc(size_t(n)));
    BBG_TRY(ids.alloc(size_t(n)));
    BBG_TRY(ids_sorted.alloc(size_t(n)));
    const uint32_t init[6] = { 0xffffffffu, 0xffffffffu, 0xffffffffu, 0, 0, 0 };
    BBG_CUDA(cudaMemcpyAsync(cbounds.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
    BoxesKernel<<<grid, kLbvhBlock, 0, st>>>(a->prim_shape.p, a->tri_indices.p, a->positions.p, a->spheres.p, n,
                                              boxes.p, cbounds.p);
    MortonKernel<<<grid, kLbvhBlock, 0, st>>>(boxes.p, cbounds.p, n, codes.p, ids.p);

    size_t temp_bytes = 0;
    BBG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, codes.p, codes_sorted.p, ids.p, ids_sorted.p, n, 0,
                                             30, st));
    DevBuf<unsigned char> temp;
    BBG_TRY(temp.alloc(std::max<size_t>(temp_bytes, 1)));
    BBG_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, codes.p, codes_sorted.p, ids.p, ids_sorted.p, n, 0,
                                             30, st));

    const int32_t n_inner = std::max(n - 1, 1);
    BBG_TRY(a->slots.alloc(3 * size_t(n)));
    BBG_TRY(a->leaves.alloc(size_t(n)));
    BBG_TRY(a->wide.alloc(4 * size_t(n_inner)));
    SlotsKernel<<<grid, kLbvhBlock, 0, st>>>(ids_sorted.p, a->prim_shape.p, a->tri_indices.p, a->positions.p,
                                              a->spheres.p, n, a->slots.p, a->leaves.p);
    int32_t max_depth = 1;
    float bounds[6];
    if (n == 1)
    {
        a->root = ~0;
        float4 b[2];
        BBG_CUDA(cudaMemcpyAsync(b, boxes.p, sizeof(b), cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaStreamSynchronize(st));
        bounds[0] = b[0].x, bounds[1] = b[0].y, bounds[2] = b[0].z;
        bounds[3] = b[1].x, bounds[4] = b[1].y, bounds[5] = b[1].z;
    }
    else
    {
        BBG_TRY(children.alloc(size_t(n_inner)));
        BBG_TRY(parent_node.alloc(size_t(n_inner)));
        BBG_TRY(parent_leaf.alloc(size_t(n)));
        BBG_TRY(arrivals.alloc(size_t(n_inner)));
        BBG_TRY(height.alloc(size_t(n_inner)));
        BBG_TRY(node_box.alloc(2 * size_t(n_inner)));
        BBG_CUDA(cudaMemsetAsync(arrivals.p, 0, sizeof(int32_t) * size_t(n_inner), st));
        const int32_t minus1 = -1;
        BBG_CUDA(cudaMemcpyAsync(parent_node.p, &minus1, sizeof(int32_t), cudaMemcpyHostToDevice, st)); // root
        HierarchyKernel<<<grid, kLbvhBlock, 0, st>>>(codes_sorted.p, n, children.p, parent_node.p, parent_leaf.p);
        RefitKernel<<<grid, kLbvhBlock, 0, st>>>(boxes.p, ids_sorted.p, children.p, parent_node.p, parent_leaf.p, n,
                                                  arrivals.p, node_box.p, height.p, a->wide.p);
        float4 rb[2];
        BBG_CUDA(cudaMemcpyAsync(rb, node_box.p, sizeof(rb), cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaMemcpyAsync(&max_depth, height.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st)); // root
        BBG_CUDA(cudaStreamSynchronize(st));
        BBG_CUDA(cudaGetLastError());
        a->root = 0;
        bounds[0] = rb[0].x, bounds[1] = rb[0].y, bounds[2] = rb[0].z;
        bounds[3] = rb[1].x, bounds[4] = rb[1].y, bounds[5] = rb[1].z;
        if (max_depth + 1 <= kStackCapacity)
        {
            BBG_TRY(BuildWide8OnDevice(a, n, children, node_box, boxes, ids_sorted, grid));
        }
    }
    BBG_CUDA(cudaGetLastError());
    if (max_depth + 1 > kStackCapacity)
    {
        return Fail(BBG_ERR_STACK_OVERFLOW, "device-built tree depth %d exceeds the traversal stack (%d)", max_depth,
                    kStackCapacity);
    }
    a->max_depth = max_depth;
    a->n_nodes = 2 * n - 1;
    a->n_slots = n;
    std::memcpy(a->bounds, bounds, sizeof(bounds));
    return BBG_OK;
}

} // namespace bbg
