// Host-side set-up of bulbit-b200: the SAH tree build, primitive bounds,
// camera basis, materials, lights and the light-selection distribution.
//
// Each function restates a reference computation whose float results the
// device kernels depend on bit for bit (tree shape, camera rays, light pmf), so
// every expression keeps the reference's operation order; the file is built
// without FMA contraction (x86-64 baseline ISA, no -ffast-math).

#include "bbg_internal.h"
#include "split_util.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <span>
#include <thread>
#include <vector>

namespace bbg
{

// ---------------------------------------------------------------- errors

static thread_local char g_error[512] = "";

void SetError(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

bbg_status Fail(bbg_status s, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    return s;
}

const char* LastError()
{
    return g_error;
}

// ---------------------------------------------------------------- vector math
// Float vector operations in the reference's evaluation order
// (include/bulbit/vectors.h:345-467, include/bulbit/math.h:56).

namespace
{

constexpr float kPi = float(3.14159265358979323846);
constexpr float kTwoPi = float(2 * kPi);
constexpr float kFourPi = float(4 * kPi);
constexpr float kEps = std::numeric_limits<float>::epsilon();
constexpr float kMaxFloat = std::numeric_limits<float>::max();

struct V3
{
    float x, y, z;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

inline V3 operator+(V3 a, V3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline V3 operator-(V3 a, V3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline V3 operator-(V3 a) { return { -a.x, -a.y, -a.z }; }
inline V3 operator*(V3 v, float s) { return { v.x * s, v.y * s, v.z * s }; }
inline V3 operator*(float s, V3 v) { return { v.x * s, v.y * s, v.z * s }; }
inline V3 operator/(V3 v, float s) { return { v.x / s, v.y / s, v.z / s }; }
inline float Dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 Cross(V3 a, V3 b) { return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x }; }
inline float Length2(V3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
inline float Length(V3 v) { return std::sqrt(Length2(v)); }
inline V3 Normalize(V3 v)
{
    float inv_length = 1.0f / Length(v);
    return v * inv_length;
}
// Vector3::Normalize (include/bulbit/vectors.h:121): in place, returns length.
inline float NormalizeInPlace(V3& v)
{
    float length = Length(v);
    if (length < kEps)
    {
        return 0;
    }
    float inv_length = 1.0f / length;
    v.x *= inv_length;
    v.y *= inv_length;
    v.z *= inv_length;
    return length;
}
// std::min / std::max semantics (second argument wins only when strictly less / greater).
inline float SMin(float a, float b) { return (b < a) ? b : a; }
inline float SMax(float a, float b) { return (a < b) ? b : a; }
inline V3 Min(V3 a, V3 b) { return { SMin(a.x, b.x), SMin(a.y, b.y), SMin(a.z, b.z) }; }
inline V3 Max(V3 a, V3 b) { return { SMax(a.x, b.x), SMax(a.y, b.y), SMax(a.z, b.z) }; }

V3 Load3(const float* p) { return { p[0], p[1], p[2] }; }
void Store3(float* d, V3 v)
{
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
}

struct Box
{
    V3 min{ kMaxFloat, kMaxFloat, kMaxFloat };
    V3 max{ -kMaxFloat, -kMaxFloat, -kMaxFloat };
    V3 Center() const { return (min + max) * 0.5f; }
    V3 Extents() const { return max - min; }
    float SurfaceArea() const
    {
        V3 w = max - min;
        return 2 * ((w.x * w.y) + (w.y * w.z) + (w.z * w.x));
    }
    static Box Union(const Box& a, const Box& b) { return { Min(a.min, b.min), Max(a.max, b.max) }; }
    static Box Union(const Box& a, V3 p) { return { Min(a.min, p), Max(a.max, p) }; }
};

} // namespace

// ---------------------------------------------------------------- primitive bounds

// Triangle::GetAABB (src/geometry/triangle.cpp:40-51): vertex bounds padded by
// 10 epsilon; Sphere::GetAABB (src/geometry/sphere.cpp:30-33): p +- radius.
void PrimAabbs(const bbg_geometry& g, float* aabbs)
{
    const V3 pad{ kEps * 10, kEps * 10, kEps * 10 };
    for (int32_t i = 0; i < g.n_prims; ++i)
    {
        V3 mn, mx;
        if (g.prim_kind[i] == BBG_PRIM_TRIANGLE)
        {
            const int32_t* v = g.tri_indices + 3 * size_t(g.prim_index[i]);
            V3 p0 = Load3(g.positions + 3 * size_t(v[0]));
            V3 p1 = Load3(g.positions + 3 * size_t(v[1]));
            V3 p2 = Load3(g.positions + 3 * size_t(v[2]));
            mn = Min(Min(p0, p1), p2) - pad;
            mx = Max(Max(p0, p1), p2) + pad;
        }
        else
        {
            const bbg_sphere& s = g.spheres[g.prim_index[i]];
            V3 p = Load3(s.p);
            V3 r{ s.radius, s.radius, s.radius };
            mn = p - r;
            mx = p + r;
        }
        Store3(aabbs + 6 * size_t(i), mn);
        Store3(aabbs + 6 * size_t(i) + 3, mx);
    }
}

bbg_status CheckGeometry(const bbg_geometry* g)
{
    if (!g || g->n_prims < 0 || g->n_vertices < 0 || g->n_triangles < 0 || g->n_spheres < 0)
    {
        return Fail(BBG_ERR_INVALID_ARG, "geometry: null or negative count");
    }
    if (g->n_prims > 0 && (!g->prim_kind || !g->prim_index))
    {
        return Fail(BBG_ERR_INVALID_ARG, "geometry: prim_kind / prim_index missing");
    }
    if (g->n_triangles > 0 && (!g->tri_indices || !g->positions))
    {
        return Fail(BBG_ERR_INVALID_ARG, "geometry: triangles without indices or positions");
    }
    for (int32_t t = 0; t < 3 * g->n_triangles; ++t)
    {
        if (g->tri_indices[t] < 0 || g->tri_indices[t] >= g->n_vertices)
        {
            return Fail(BBG_ERR_INVALID_ARG, "geometry: triangle vertex %d out of range", g->tri_indices[t]);
        }
    }
    for (int32_t i = 0; i < g->n_prims; ++i)
    {
        int32_t k = g->prim_kind[i], idx = g->prim_index[i];
        bool ok = (k == BBG_PRIM_TRIANGLE && idx >= 0 && idx < g->n_triangles) ||
                  (k == BBG_PRIM_SPHERE && idx >= 0 && idx < g->n_spheres && g->spheres);
        if (!ok)
        {
            return Fail(BBG_ERR_INVALID_ARG, "geometry: primitive %d has kind %d index %d", i, k, idx);
        }
    }
    return BBG_OK;
}

// ---------------------------------------------------------------- reference splitting
// Early split clipping (Ernst & Greiner, "Early Split Clipping for Bounding
// Volume Hierarchies", IEEE RT 2007): a triangle whose box it fills poorly
// (long thin or diagonal triangles, the displaced spheres' slivers) makes the
// tree's boxes overlap. Before the build, the reference whose box wastes the
// most surface area (box area less twice the area of the triangle part it
// holds) is split at the midpoint of its box's longest axis, each half
// keeping the box of the triangle clipped to it, until the budget of extra
// references is spent. Boxes are computed in double precision, rounded
// outward to float and padded by 10 epsilon as Triangle::GetAABB pads
// (src/geometry/triangle.cpp:40-51), so every part of a triangle lies inside
// one of its references' boxes; a ray's closest hit is therefore found, and
// a triangle split across leaves may be tested more than once (same result).

namespace
{

struct SplitRef
{
    double lo[3], hi[3];
    int32_t prim;
};

} // namespace

bbg_status SplitReferences(const bbg_geometry& g, float budget, std::vector<float>* ref_aabbs,
                           std::vector<int32_t>* ref_prims)
{
    const int32_t n = g.n_prims;
    std::vector<float> prim_aabbs(6 * size_t(n));
    PrimAabbs(g, prim_aabbs.data());
    // At most 2^30 references, so a tree over them (2 m - 1 nodes) fits int32.
    const int64_t max_refs = std::min<int64_t>(int64_t(n) + int64_t(double(budget) * n), int64_t(1) << 30);
    if (n > (int32_t(1) << 30))
    {
        return Fail(BBG_ERR_INVALID_ARG, "split references: %d primitives exceed 2^30", n);
    }
    std::vector<SplitRef> refs;
    refs.reserve(size_t(max_refs));
    // Max-heap on wasted box area over the splittable (triangle) references.
    std::vector<std::pair<double, int32_t>> heap;
    for (int32_t i = 0; i < n; ++i)
    {
        SplitRef r;
        r.prim = i;
        if (g.prim_kind[i] == BBG_PRIM_TRIANGLE)
        {
            const int32_t* v = g.tri_indices + 3 * size_t(g.prim_index[i]);
            double tri[3][3];
            for (int c = 0; c < 3; ++c)
            {
                for (int k = 0; k < 3; ++k)
                {
                    tri[k][c] = g.positions[3 * size_t(v[k]) + c];
                }
                r.lo[c] = std::min(std::min(tri[0][c], tri[1][c]), tri[2][c]);
                r.hi[c] = std::max(std::max(tri[0][c], tri[1][c]), tri[2][c]);
            }
            heap.emplace_back(split::BoxArea(r.lo, r.hi) - 2 * split::PolygonArea(tri, 3), int32_t(refs.size()));
        }
        refs.push_back(r);
    }
    std::make_heap(heap.begin(), heap.end());
    while (!heap.empty() && int64_t(refs.size()) < max_refs)
    {
        std::pop_heap(heap.begin(), heap.end());
        int32_t ri = heap.back().second;
        heap.pop_back();
        SplitRef r = refs[size_t(ri)];
        const int axis = split::LongestAxis(r.lo, r.hi);
        const double m = 0.5 * (r.lo[axis] + r.hi[axis]);
        if (!(m > r.lo[axis] && m < r.hi[axis]))
        {
            continue; // too small to split
        }
        const int32_t* v = g.tri_indices + 3 * size_t(g.prim_index[r.prim]);
        double tri[3][3];
        for (int k = 0; k < 3; ++k)
        {
            for (int c = 0; c < 3; ++c)
            {
                tri[k][c] = g.positions[3 * size_t(v[k]) + c];
            }
        }
        double llo[3], lhi[3], rlo[3], rhi[3];
        std::memcpy(llo, r.lo, sizeof(llo));
        std::memcpy(lhi, r.hi, sizeof(lhi));
        std::memcpy(rlo, r.lo, sizeof(rlo));
        std::memcpy(rhi, r.hi, sizeof(rhi));
        lhi[axis] = m;
        rlo[axis] = m;
        SplitRef left{}, right{};
        left.prim = right.prim = r.prim;
        double al = 0, ar = 0;
        bool hl = split::ClippedBox(tri, llo, lhi, left.lo, left.hi, &al);
        bool hr = split::ClippedBox(tri, rlo, rhi, right.lo, right.hi, &ar);
        if (!hl || !hr)
        {
            continue; // the box was not tight on this axis: keep the reference whole
        }
        refs[size_t(ri)] = left;
        heap.emplace_back(split::BoxArea(left.lo, left.hi) - 2 * al, ri);
        std::push_heap(heap.begin(), heap.end());
        heap.emplace_back(split::BoxArea(right.lo, right.hi) - 2 * ar, int32_t(refs.size()));
        std::push_heap(heap.begin(), heap.end());
        refs.push_back(right);
    }
    // Boxes: unsplit references keep the primitive's own box bit for bit.
    const float pad = kEps * 10;
    ref_aabbs->resize(6 * refs.size());
    ref_prims->resize(refs.size());
    for (size_t i = 0; i < refs.size(); ++i)
    {
        const SplitRef& r = refs[i];
        (*ref_prims)[i] = r.prim;
        float* box = ref_aabbs->data() + 6 * i;
        if (g.prim_kind[r.prim] != BBG_PRIM_TRIANGLE)
        {
            std::memcpy(box, prim_aabbs.data() + 6 * size_t(r.prim), 6 * sizeof(float));
            continue;
        }
        for (int c = 0; c < 3; ++c)
        {
            box[c] = split::RoundDown(r.lo[c]) - pad;
            box[3 + c] = split::RoundUp(r.hi[c]) + pad;
        }
    }
    return BBG_OK;
}

// ---------------------------------------------------------------- SAH build
// BVH::BuildRecursive (src/accel/bvh.cpp:56-271) and FlattenBVH (:273-297).
// The same std::partition / std::nth_element calls run on the same element
// order, so the tree and the primitive order inside every leaf come out
// identical; leaves take their slots in depth-first order (the reference's
// single-threaded order; above 64Ki primitives it builds the two halves of a
// node concurrently, which permutes whole leaves inside the slot array but not
// the tree). Here too the halves of nodes above 64Ki primitives are built on
// separate threads (a few levels deep): a node's partition touches only its
// own span, and its right half's leaves start at a slot known in advance (the
// node's first slot + the left half's size), so the tree and the depth-first
// slot order are the same as single-threaded.

namespace
{

struct BuildPrim
{
    size_t index;
    Box aabb;
};

struct BuildNode
{
    Box aabb;
    int32_t axis = 0, offset = 0, count = 0;
    int32_t child1 = -1, child2 = -1;
};

constexpr size_t kParallelBuildSpan = size_t(1) << 16;
// Spans at least this long compute their bounds and SAH buckets on several
// threads (min / max and counts: the same values in any order).
constexpr size_t kParallelReduceSpan = size_t(1) << 18;

// Runs fn(begin, end, chunk) over `threads` contiguous chunks of [0, n).
template <class F>
void ForChunks(size_t n, int threads, F&& fn)
{
    const size_t chunk = (n + size_t(threads) - 1) / size_t(threads);
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t)
    {
        const size_t b = size_t(t) * chunk, e = std::min(n, b + chunk);
        if (b < e)
        {
            pool.emplace_back([&fn, b, e, t] { fn(b, e, t); });
        }
    }
    fn(0, std::min(n, chunk), 0);
    for (std::thread& th : pool)
    {
        th.join();
    }
}

struct Builder
{
    std::vector<BuildNode> nodes;
    int32_t* ordered = nullptr; // slot -> primitive, shared by the threads (disjoint ranges)
    int parallel_levels = 0;    // levels of the recursion that may still fork a thread
    bool too_many_in_leaf = false;

    int32_t MakeLeaf(std::span<BuildPrim> span, const Box& bounds, int32_t offset)
    {
        int32_t count = int32_t(span.size());
        for (int32_t i = 0; i < count; ++i)
        {
            ordered[offset + i] = int32_t(span[i].index);
        }
        if (count > 0xffff)
        {
            too_many_in_leaf = true;
        }
        BuildNode n;
        n.aabb = bounds;
        n.offset = offset;
        n.count = count;
        nodes.push_back(n);
        return int32_t(nodes.size() - 1);
    }

    // Builds the subtree over span; its leaves fill slots from slot_base on.
    int32_t Build(std::span<BuildPrim> span, int32_t slot_base, int depth = 0)
    {
        int32_t primitive_count = int32_t(span.size());
        // Threads for this node's reductions: the machine's, shared among the
        // nodes of this depth that build concurrently.
        const int reduce_threads =
            span.size() >= kParallelReduceSpan ? std::max(1, int(std::thread::hardware_concurrency()) >> depth) : 1;

        Box span_bounds;
        if (reduce_threads > 1)
        {
            std::vector<Box> part(static_cast<size_t>(reduce_threads));
            ForChunks(span.size(), reduce_threads, [&](size_t b, size_t e, int t) {
                Box acc;
                for (size_t i = b; i < e; ++i)
                {
                    acc = Box::Union(acc, span[i].aabb);
                }
                part[size_t(t)] = acc;
            });
            for (const Box& bx : part)
            {
                span_bounds = Box::Union(span_bounds, bx);
            }
        }
        else
        {
            for (const BuildPrim& p : span)
            {
                span_bounds = Box::Union(span_bounds, p.aabb);
            }
        }

        if (span_bounds.SurfaceArea() == 0 || primitive_count == 1)
        {
            return MakeLeaf(span, span_bounds, slot_base);
        }

        Box centroid_bounds;
        if (reduce_threads > 1)
        {
            std::vector<Box> part(static_cast<size_t>(reduce_threads));
            ForChunks(span.size(), reduce_threads, [&](size_t b, size_t e, int t) {
                Box acc;
                for (size_t i = b; i < e; ++i)
                {
                    acc = Box::Union(acc, span[i].aabb.Center());
                }
                part[size_t(t)] = acc;
            });
            for (const Box& bx : part)
            {
                centroid_bounds = Box::Union(centroid_bounds, bx);
            }
        }
        else
        {
            for (const BuildPrim& p : span)
            {
                centroid_bounds = Box::Union(centroid_bounds, p.aabb.Center());
            }
        }

        int32_t axis = 0;
        V3 extents = centroid_bounds.Extents();
        if (extents.y > extents.x)
        {
            axis = 1;
        }
        if (extents.z > extents[axis])
        {
            axis = 2;
        }
        const float extent = extents[axis];

        if (extent == 0)
        {
            return MakeLeaf(span, span_bounds, slot_base);
        }

        int32_t mid;
        if (primitive_count <= 2)
        {
            mid = primitive_count / 2;
            std::nth_element(span.begin(), span.begin() + mid, span.end(),
                             [axis](const BuildPrim& a, const BuildPrim& b) {
                                 return a.aabb.Center()[axis] < b.aabb.Center()[axis];
                             });
        }
        else
        {
            constexpr int32_t bucket_size = 12;
            constexpr int32_t split_planes = bucket_size - 1;
            struct Bucket
            {
                int count = 0;
                Box bounds;
            } buckets[bucket_size];

            auto fill = [&](size_t b0, size_t e0, Bucket* out) {
                for (size_t i = b0; i < e0; ++i)
                {
                    const BuildPrim& p = span[i];
                    int32_t b = int32_t(bucket_size * (p.aabb.Center() - centroid_bounds.min)[axis] / extent);
                    if (b == bucket_size)
                    {
                        b = b - 1;
                    }
                    out[b].count++;
                    out[b].bounds = Box::Union(out[b].bounds, p.aabb);
                }
            };
            if (reduce_threads > 1)
            {
                std::vector<Bucket> part(size_t(reduce_threads) * bucket_size);
                ForChunks(span.size(), reduce_threads,
                          [&](size_t b0, size_t e0, int t) { fill(b0, e0, part.data() + size_t(t) * bucket_size); });
                for (int t = 0; t < reduce_threads; ++t)
                {
                    for (int32_t b = 0; b < bucket_size; ++b)
                    {
                        const Bucket& pb = part[size_t(t) * bucket_size + size_t(b)];
                        buckets[b].count += pb.count;
                        buckets[b].bounds = Box::Union(buckets[b].bounds, pb.bounds);
                    }
                }
            }
            else
            {
                fill(0, span.size(), buckets);
            }

            Box left_bound, right_bound;
            int32_t left_count[split_planes], right_count[split_planes];
            float left_area[split_planes], right_area[split_planes];
            int32_t left_sum = 0, right_sum = 0;
            for (int32_t i = 0; i < split_planes; ++i)
            {
                left_sum += buckets[i].count;
                left_count[i] = left_sum;
                left_bound = Box::Union(left_bound, buckets[i].bounds);
                left_area[i] = left_bound.SurfaceArea();

                right_sum += buckets[split_planes - i].count;
                right_count[split_planes - 1 - i] = right_sum;
                right_bound = Box::Union(right_bound, buckets[split_planes - i].bounds);
                right_area[split_planes - 1 - i] = right_bound.SurfaceArea();
            }

            int32_t min_cost_split_bucket = -1;
            float min_cost = std::numeric_limits<float>::infinity();
            for (int32_t i = 0; i < split_planes; ++i)
            {
                float cost = left_count[i] * left_area[i] + right_count[i] * right_area[i];
                if (cost < min_cost)
                {
                    min_cost = cost;
                    min_cost_split_bucket = i;
                }
            }

            constexpr float traverse_cost = 0.5f;
            min_cost = traverse_cost + min_cost / span_bounds.SurfaceArea();
            const float direct_leaf_cost = float(primitive_count);

            if (min_cost < direct_leaf_cost)
            {
                auto mid_iter = std::partition(span.begin(), span.end(), [=](const BuildPrim& p) {
                    int32_t b = int32_t(bucket_size * (p.aabb.Center() - centroid_bounds.min)[axis] / extent);
                    if (b == bucket_size)
                    {
                        b = bucket_size - 1;
                    }
                    return b <= min_cost_split_bucket;
                });
                mid = int32_t(mid_iter - span.begin());
            }
            else
            {
                return MakeLeaf(span, span_bounds, slot_base);
            }
        }

        int32_t self = int32_t(nodes.size());
        nodes.push_back(BuildNode{});
        int32_t c1, c2;
        if (depth < parallel_levels && span.size() > kParallelBuildSpan)
        {
            Builder right;
            right.ordered = ordered;
            right.parallel_levels = parallel_levels;
            int32_t right_root = -1;
            std::thread t([&] { right_root = right.Build(span.subspan(size_t(mid)), slot_base + mid, depth + 1); });
            c1 = Build(span.subspan(0, size_t(mid)), slot_base, depth + 1);
            t.join();
            // Splice the right subtree's nodes after this builder's.
            const int32_t off = int32_t(nodes.size());
            for (BuildNode bn : right.nodes)
            {
                if (bn.count == 0)
                {
                    bn.child1 += off;
                    bn.child2 += off;
                }
                nodes.push_back(bn);
            }
            c2 = right_root + off;
            too_many_in_leaf = too_many_in_leaf || right.too_many_in_leaf;
        }
        else
        {
            c1 = Build(span.subspan(0, size_t(mid)), slot_base, depth + 1);
            c2 = Build(span.subspan(size_t(mid)), slot_base + mid, depth + 1);
        }
        BuildNode& n = nodes[self];
        n.axis = axis;
        n.child1 = c1;
        n.child2 = c2;
        n.aabb = Box::Union(nodes[c1].aabb, nodes[c2].aabb);
        n.count = 0;
        return self;
    }

    int32_t Flatten(int32_t node, bbg_bvh_node* out, int32_t* offset)
    {
        const BuildNode& n = nodes[node];
        bbg_bvh_node& o = out[*offset];
        std::memset(&o, 0, sizeof(o));
        Store3(o.bmin, n.aabb.min);
        Store3(o.bmax, n.aabb.max);
        int32_t node_offset = (*offset)++;
        if (n.count > 0)
        {
            o.offset = n.offset;
            o.count = uint16_t(n.count);
        }
        else
        {
            o.axis = uint8_t(n.axis);
            o.count = 0;
            Flatten(n.child1, out, offset);
            int32_t c2 = Flatten(n.child2, out, offset);
            out[node_offset].offset = c2;
        }
        return node_offset;
    }
};

} // namespace

bbg_status BuildBvh(const float* aabbs, int32_t n, bbg_bvh_node* nodes_out, int32_t* slots_out, int32_t* n_nodes_out)
{
    std::vector<BuildPrim> prims(static_cast<size_t>(n));
    for (int32_t i = 0; i < n; ++i)
    {
        prims[i].index = size_t(i);
        prims[i].aabb.min = Load3(aabbs + 6 * size_t(i));
        prims[i].aabb.max = Load3(aabbs + 6 * size_t(i) + 3);
    }
    std::vector<int32_t> ordered(static_cast<size_t>(n));
    Builder b;
    b.ordered = ordered.data();
    unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    while ((1u << b.parallel_levels) < hw && b.parallel_levels < 6)
    {
        ++b.parallel_levels;
    }
    b.nodes.reserve(size_t(2) * size_t(std::max(n, 1)));
    int32_t root = b.Build(std::span<BuildPrim>(prims), 0);
    if (b.too_many_in_leaf)
    {
        return Fail(BBG_ERR_BAD_BVH, "a leaf holds more than 65535 primitives (uint16 primitive_count)");
    }
    int32_t offset = 0;
    b.Flatten(root, nodes_out, &offset);
    std::memcpy(slots_out, ordered.data(), sizeof(int32_t) * size_t(n));
    *n_nodes_out = offset;
    return BBG_OK;
}

bbg_status ValidateBvh(const bbg_bvh_node* nodes, int32_t n_nodes, int32_t n_slots, int32_t n_prims,
                       const int32_t* slot_prims, int32_t* max_depth)
{
    if (n_nodes <= 0)
    {
        return Fail(BBG_ERR_BAD_BVH, "empty node array");
    }
    for (int32_t i = 0; i < n_slots; ++i)
    {
        if (slot_prims[i] < 0 || slot_prims[i] >= n_prims)
        {
            return Fail(BBG_ERR_BAD_BVH, "slot %d names primitive %d of %d", i, slot_prims[i], n_prims);
        }
    }
    // Depth-first layout: an interior node's children both lie strictly after
    // it, so every path from the root is finite and the walk below ends.
    std::vector<int32_t> depth(static_cast<size_t>(n_nodes), -1);
    depth[0] = 1;
    int32_t deepest = 1;
    std::vector<int32_t> stack{ 0 };
    while (!stack.empty())
    {
        int32_t i = stack.back();
        stack.pop_back();
        const bbg_bvh_node& n = nodes[i];
        if (n.count > 0)
        {
            if (n.offset < 0 || int64_t(n.offset) + n.count > n_slots)
            {
                return Fail(BBG_ERR_BAD_BVH, "leaf %d covers slots [%d, %d) of %d", i, n.offset,
                            n.offset + n.count, n_slots);
            }
            continue;
        }
        int32_t c1 = i + 1, c2 = n.offset;
        if (c1 >= n_nodes || c2 <= c1 || c2 >= n_nodes || n.axis > 2)
        {
            return Fail(BBG_ERR_BAD_BVH, "interior node %d has children %d, %d (of %d nodes) / axis %d", i, c1, c2,
                        n_nodes, int(n.axis));
        }
        for (int32_t c : { c1, c2 })
        {
            if (depth[c] != -1)
            {
                return Fail(BBG_ERR_BAD_BVH, "node %d is reachable twice", c);
            }
            depth[c] = depth[i] + 1;
            deepest = std::max(deepest, depth[c]);
            stack.push_back(c);
        }
    }
    *max_depth = deepest;
    return BBG_OK;
}

// ---------------------------------------------------------------- camera

namespace
{

struct Quat
{
    float x, y, z, w;
    Quat operator*(float s) const { return { x * s, y * s, z * s, w * s }; }
};

// Quat(const Mat3&) (include/bulbit/quaternion.h:32-57), columns ex, ey, ez.
Quat QuatFromBasis(V3 ex, V3 ey, V3 ez)
{
    if (ez.z < 0)
    {
        if (ex.x > ey.y)
        {
            float t = 1 + ex.x - ey.y - ez.z;
            return Quat{ t, ex.y + ey.x, ez.x + ex.z, ey.z - ez.y } * (0.5f / std::sqrt(t));
        }
        float t = 1 - ex.x + ey.y - ez.z;
        return Quat{ ex.y + ey.x, t, ey.z + ez.y, ez.x - ex.z } * (0.5f / std::sqrt(t));
    }
    if (ex.x < -ey.y)
    {
        float t = 1 - ex.x - ey.y + ez.z;
        return Quat{ ez.x + ex.z, ey.z + ez.y, t, ex.y - ey.x } * (0.5f / std::sqrt(t));
    }
    float t = 1 + ex.x + ey.y + ez.z;
    return Quat{ ey.z - ez.y, ez.x - ex.z, ex.y - ey.x, t } * (0.5f / std::sqrt(t));
}

} // namespace

// Transform::LookAt (include/bulbit/transform.h:108) + Quat(front, up)
// (include/bulbit/quaternion.h:60-70) + PerspectiveCamera::PerspectiveCamera
// (src/camera/perspective_camera.cpp:8-38).
void CameraFromSpec(const bbg_camera_spec& s, bbg_camera* out)
{
    V3 position = Load3(s.position);
    V3 w = Load3(s.target) - position;
    NormalizeInPlace(w);
    V3 up = Load3(s.up);
    V3 ez = w;
    V3 ex = Cross(up, ez);
    NormalizeInPlace(ex);
    V3 ey = Cross(ez, ex);
    Quat q = QuatFromBasis(ex, ey, ez);

    float theta = s.vfov_deg * kPi / 180;
    float h = std::tan(theta / 2);
    float aspect_ratio = (float)s.width / (float)s.height;
    float viewport_height = 2 * h;
    float viewport_width = aspect_ratio * viewport_height;

    // Quat::GetBasisX/Y/Z (include/bulbit/quaternion.h:174-203).
    float x2 = q.x * 2, y2 = q.y * 2, z2 = q.z * 2, w2 = q.w * 2;
    V3 bx{ (q.w * w2) - 1 + q.x * x2, (q.z * w2) + q.y * x2, (-q.y * w2) + q.z * x2 };
    V3 by{ (-q.z * w2) + q.x * y2, (q.w * w2) - 1 + q.y * y2, (q.x * w2) + q.z * y2 };
    V3 bz{ (q.y * w2) + q.x * z2, (-q.x * w2) + q.y * z2, (q.w * w2) - 1 + q.z * z2 };

    V3 u = -bx;
    V3 v = by;
    V3 ww = bz;
    float focus = s.focus_distance;
    V3 horizontal = focus * viewport_width * u;
    V3 vertical = focus * viewport_height * v;
    V3 lower_left = position - horizontal / 2 - vertical / 2 + focus * ww;

    out->width = s.width;
    out->height = s.height;
    Store3(out->origin, position);
    Store3(out->lower_left, lower_left);
    Store3(out->horizontal, horizontal);
    Store3(out->vertical, vertical);
    Store3(out->u, u);
    Store3(out->v, v);
    out->lens_radius = s.aperture_radius;
    out->filter_extent = s.filter_extent;
    out->filter_type = s.filter_type;
    out->filter_sigma = s.filter_sigma;
}

// ---------------------------------------------------------------- materials

bbg_status MakeMaterial(const bbg_material& m, MaterialDev* out)
{
    std::memset(out, 0, sizeof(*out));
    out->type = m.type;
    switch (m.type)
    {
    case BBG_MAT_DIFFUSE:
    {
        // DiffuseMaterial with no roughness texture -> LambertianBxDF
        // (src/material/diffuse_material.cpp:21-35).
        std::memcpy(out->r, m.reflectance, sizeof(out->r));
        bool black = m.reflectance[0] == 0.0f && m.reflectance[1] == 0.0f && m.reflectance[2] == 0.0f;
        out->flags = black ? 0 : (kFlagDiffuse | kFlagReflection);
        return BBG_OK;
    }
    case BBG_MAT_CONDUCTOR:
    {
        // ConductorMaterial::GetBSDF (src/material/conductor_material.cpp:52-99),
        // ConductorBxDF (include/bulbit/bxdfs.h:249-300).
        out->alpha_x = m.roughness[0] * m.roughness[0];
        out->alpha_y = m.roughness[1] * m.roughness[1];
        std::memcpy(out->r, m.reflectance, sizeof(out->r));
        if (m.conductor_from_r)
        {
            for (int c = 0; c < 3; ++c)
            {
                float R = m.k[c];
                float r = R < 0 ? 0.0f : (R > 1 - 1e-4f ? 1 - 1e-4f : R);
                float one_minus = 1.0f - r;
                float mx = (0.0f < one_minus) ? one_minus : 0.0f;
                out->eta[c] = 1;
                out->k[c] = std::sqrt(r) * 2 / std::sqrt(mx);
            }
        }
        else
        {
            std::memcpy(out->eta, m.eta, sizeof(out->eta));
            std::memcpy(out->k, m.k, sizeof(out->k));
        }
        bool smooth = std::max(out->alpha_x, out->alpha_y) < 1e-3f;
        out->flags = smooth ? (kFlagSpecular | kFlagReflection) : (kFlagGlossy | kFlagReflection);
        // energy_compensation = true -> ConductorMultiScatteringBxDF (same
        // flags, include/bulbit/bxdfs.h:303-357).
        out->ms = m.energy_compensation ? 1 : 0;
        return BBG_OK;
    }
    case BBG_MAT_DIELECTRIC:
    {
        // DielectricMaterial::GetBSDF (src/material/dielectric_material.cpp:28-52);
        // DielectricBxDF and DielectricMultiScatteringBxDF store Sqrt(r)
        // (include/bulbit/bxdfs.h:85-90, 148-153). The relative eta and the
        // flags depend on the hit side and are set per hit; the flags are the
        // same with and without energy compensation.
        out->ms = m.energy_compensation ? 1 : 0;
        out->eta[0] = m.eta[0];
        for (int c = 0; c < 3; ++c)
        {
            out->r[c] = std::sqrt(m.reflectance[c]);
        }
        out->alpha_x = m.roughness[0] * m.roughness[0];
        out->alpha_y = m.roughness[1] * m.roughness[1];
        return BBG_OK;
    }
    case BBG_MAT_METALLIC_ROUGHNESS:
    {
        // MetallicRoughnessMaterial::GetBSDF (src/material/metallic_roughness_material.cpp:28-41).
        std::memcpy(out->r, m.reflectance, sizeof(out->r));
        out->metallic = m.metallic;
        out->alpha_x = std::fmax(m.roughness[0] * m.roughness[0], 1e-3f);
        out->alpha_y = std::fmax(m.roughness[1] * m.roughness[1], 1e-3f);
        out->flags = kFlagDiffuse | kFlagGlossy | kFlagReflection;
        return BBG_OK;
    }
    default:
        return Fail(BBG_ERR_INVALID_ARG, "unknown material type %d", m.type);
    }
}

// ---------------------------------------------------------------- lights

namespace
{

float Luminance(const float* c)
{
    return c[0] * 0.2126f + c[1] * 0.7152f + c[2] * 0.0722f;
}

// CoordinateSystem (include/bulbit/frame.h:105-112).
void CoordinateSystem(V3 v1, V3* v2, V3* v3)
{
    float sign = std::copysign(1.0f, v1.z);
    float a = -1 / (sign + v1.z);
    float b = v1.x * v1.y * a;
    *v2 = V3{ 1 + sign * (v1.x * v1.x) * a, sign * b, -sign * v1.x };
    *v3 = V3{ b, sign + (v1.y * v1.y) * a, -v1.y };
}

} // namespace

bbg_status MakeLight(const bbg_light& l, const bbg_geometry& g, const float world[6], LightDev* out,
                     float* power)
{
    std::memset(out, 0, sizeof(*out));
    out->type = l.type;
    out->prim = l.prim;
    out->two_sided = l.two_sided;
    std::memcpy(out->p, l.position, sizeof(out->p));
    std::memcpy(out->L, l.intensity, sizeof(out->L));
    out->scale = l.scale;
    float phi[3];
    switch (l.type)
    {
    case BBG_LIGHT_POINT:
        // PointLight::Phi (src/light/point_light.cpp:118): four_pi * intensity.
        for (int c = 0; c < 3; ++c)
        {
            phi[c] = l.intensity[c] * kFourPi;
        }
        break;
    case BBG_LIGHT_SPOT:
    {
        // SpotLight ctor (src/light/spot_light.cpp:7-24) and Phi (:111).
        V3 n = -Normalize(Load3(l.direction));
        V3 x, y;
        CoordinateSystem(n, &x, &y);
        Store3(out->frame_x, x);
        Store3(out->frame_y, y);
        Store3(out->frame_z, n);
        out->cos_theta_min = std::cos(l.angle_falloff_start * kPi / 180);
        out->cos_theta_max = std::cos(l.angle_max * kPi / 180);
        if (!(out->cos_theta_min > out->cos_theta_max))
        {
            return Fail(BBG_ERR_INVALID_ARG, "spot light needs angle_falloff_start < angle_max");
        }
        float k = (1 - out->cos_theta_min) + (out->cos_theta_min - out->cos_theta_max) / 2;
        for (int c = 0; c < 3; ++c)
        {
            phi[c] = l.intensity[c] * kTwoPi * k;
        }
        break;
    }
    case BBG_LIGHT_UNIFORM_INFINITE:
    {
        // Preprocess -> AABB::ComputeBoundingSphere (include/bulbit/bounding_box.h:524-528);
        // Phi (src/light/uniform_infinite_light.cpp:90).
        Box b{ Load3(world), Load3(world + 3) };
        V3 center = b.Center();
        bool inside = !(b.min.x > center.x || b.max.x < center.x) && !(b.min.y > center.y || b.max.y < center.y) &&
                      !(b.min.z > center.z || b.max.z < center.z);
        float radius = inside ? Length(b.max - center) : 0;
        Store3(out->world_center, center);
        out->world_radius = radius;
        for (int c = 0; c < 3; ++c)
        {
            phi[c] = l.intensity[c] * l.scale * kFourPi * kPi * (radius * radius);
        }
        break;
    }
    case BBG_LIGHT_DIFFUSE_AREA:
    {
        // DiffuseAreaLight::Phi (src/light/diffuse_area_light.cpp:144):
        // emission * Area() * pi * (two_sided ? 2 : 1).
        if (l.prim < 0 || l.prim >= g.n_prims)
        {
            return Fail(BBG_ERR_INVALID_ARG, "area light names primitive %d of %d", l.prim, g.n_prims);
        }
        float area;
        if (g.prim_kind[l.prim] == BBG_PRIM_TRIANGLE)
        {
            const int32_t* v = g.tri_indices + 3 * size_t(g.prim_index[l.prim]);
            V3 p0 = Load3(g.positions + 3 * size_t(v[0]));
            V3 p1 = Load3(g.positions + 3 * size_t(v[1]));
            V3 p2 = Load3(g.positions + 3 * size_t(v[2]));
            area = 0.5f * Length(Cross(p1 - p0, p2 - p0));
        }
        else
        {
            float r = g.spheres[g.prim_index[l.prim]].radius;
            area = kFourPi * (r * r);
        }
        for (int c = 0; c < 3; ++c)
        {
            phi[c] = l.intensity[c] * area * kPi * float(l.two_sided ? 2 : 1);
        }
        break;
    }
    default:
        return Fail(BBG_ERR_INVALID_ARG, "unknown light type %d", l.type);
    }
    *power = Luminance(phi);
    return BBG_OK;
}

// Distribution1D::Distribution1D (include/bulbit/sampling.h:345-371).
void BuildDistribution(const float* f, int32_t n, float* func, float* cdf, float* func_integral)
{
    cdf[0] = 0;
    for (int32_t i = 0; i < n; ++i)
    {
        func[i] = f[i];
    }
    for (int32_t i = 1; i < n + 1; ++i)
    {
        cdf[i] = cdf[i - 1] + func[i - 1] / n;
    }
    *func_integral = cdf[n];
    if (*func_integral == 0)
    {
        for (int32_t i = 1; i < n + 1; ++i)
        {
            cdf[i] = float(i) / float(n);
        }
    }
    else
    {
        for (int32_t i = 1; i < n + 1; ++i)
        {
            cdf[i] /= *func_integral;
        }
    }
}

// GaussianFilter's tabulated distribution (src/reconstruction/gaussian_filter.cpp:8-28):
// 32 x 32 values Gaussian(p.x) Gaussian(p.y) at the cell centres of
// [-extent/2, extent/2]^2, then Distribution2D (include/bulbit/sampling.h:426-446).
// Only the CDFs are kept (SampleContinuous reads nothing else): cdf_out[0..33)
// the marginal, then row v's conditional at 33 + 33 v.
void GaussianFilterCdf(float sigma, float extent, float* cdf_out)
{
    constexpr int32_t n = kFilterTable;
    const float two_pi = float(2 * 3.14159265358979323846);
    auto gaussian = [&](float x) {
        return 1 / std::sqrt(two_pi * sigma * sigma) * std::exp(-((x - 0) * (x - 0)) / (2 * sigma * sigma));
    };
    float values[n * n];
    float half_extent = extent / 2;
    for (int32_t y = 0; y < n; ++y)
    {
        for (int32_t x = 0; x < n; ++x)
        {
            float px = ((float(x) + 0.5f) / float(n)) * extent - half_extent;
            float py = ((float(y) + 0.5f) / float(n)) * extent - half_extent;
            values[y * n + x] = gaussian(px) * gaussian(py);
        }
    }
    float func[n], integral[n];
    for (int32_t v = 0; v < n; ++v)
    {
        BuildDistribution(&values[v * n], n, func, cdf_out + (n + 1) * (v + 1), &integral[v]);
    }
    float marginal_integral;
    BuildDistribution(integral, n, func, cdf_out, &marginal_integral);
}

// Vose's alias method over the pmf (exact in double, stored in float).
void BuildAlias(const float* pmf, int32_t n, float* prob, int32_t* alias)
{
    std::vector<double> scaled(static_cast<size_t>(n));
    std::vector<int32_t> small, large;
    for (int32_t i = 0; i < n; ++i)
    {
        scaled[i] = double(pmf[i]) * n;
        (scaled[i] < 1.0 ? small : large).push_back(i);
        alias[i] = i;
    }
    while (!small.empty() && !large.empty())
    {
        int32_t s = small.back(), l = large.back();
        small.pop_back();
        prob[s] = float(scaled[s]);
        alias[s] = l;
        scaled[l] = (scaled[l] + scaled[s]) - 1.0;
        if (scaled[l] < 1.0)
        {
            large.pop_back();
            small.push_back(l);
        }
    }
    for (int32_t i : large)
    {
        prob[i] = 1.0f;
    }
    for (int32_t i : small)
    {
        prob[i] = 1.0f;
    }
}

} // namespace bbg

// ---------------------------------------------------------------- C ABI (host only)

extern "C" {

bbg_status bbg_bvh_build(const float* prim_aabbs, int32_t n_prims, bbg_bvh_node* nodes_out, int32_t* slot_prims_out,
                         int32_t* n_nodes_out)
{
    if (!prim_aabbs || n_prims <= 0 || !nodes_out || !slot_prims_out || !n_nodes_out)
    {
        return bbg::Fail(BBG_ERR_INVALID_ARG, "bbg_bvh_build: null buffer or n_prims <= 0");
    }
    return bbg::BuildBvh(prim_aabbs, n_prims, nodes_out, slot_prims_out, n_nodes_out);
}

bbg_status bbg_split_references(const bbg_geometry* g, float budget, int32_t capacity, float* aabbs_out,
                                int32_t* prims_out, int32_t* n_out)
{
    if (!g || !aabbs_out || !prims_out || !n_out || !(budget >= 0.0f) || budget > 64.0f || capacity < 0)
    {
        return bbg::Fail(BBG_ERR_INVALID_ARG, "bbg_split_references: bad argument");
    }
    bbg_status st = bbg::CheckGeometry(g);
    if (st != BBG_OK)
    {
        return st;
    }
    std::vector<float> aabbs;
    std::vector<int32_t> prims;
    st = bbg::SplitReferences(*g, budget, &aabbs, &prims);
    if (st != BBG_OK)
    {
        return st;
    }
    if (int64_t(prims.size()) > capacity)
    {
        return bbg::Fail(BBG_ERR_INVALID_ARG, "bbg_split_references: %zu references exceed the capacity %d",
                         prims.size(), capacity);
    }
    std::memcpy(aabbs_out, aabbs.data(), aabbs.size() * sizeof(float));
    std::memcpy(prims_out, prims.data(), prims.size() * sizeof(int32_t));
    *n_out = int32_t(prims.size());
    return BBG_OK;
}

bbg_status bbg_prim_aabbs(const bbg_geometry* g, float* aabbs_out)
{
    if (!g || !aabbs_out)
    {
        return bbg::Fail(BBG_ERR_INVALID_ARG, "bbg_prim_aabbs: null argument");
    }
    bbg::PrimAabbs(*g, aabbs_out);
    return BBG_OK;
}

bbg_status bbg_camera_perspective(const bbg_camera_spec* spec, bbg_camera* out)
{
    if (!spec || !out || spec->width <= 0 || spec->height <= 0)
    {
        return bbg::Fail(BBG_ERR_INVALID_ARG, "bbg_camera_perspective: bad spec");
    }
    bbg::CameraFromSpec(*spec, out);
    return BBG_OK;
}

const char* bbg_last_error(void)
{
    return bbg::LastError();
}

const char* bbg_version(void)
{
    return "bulbit-b200 0.1 (sm_100a)";
}

} // extern "C"
