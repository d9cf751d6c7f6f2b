// BVH traversal and ray-primitive tests on the device.
//
// Restates, operation for operation, BVH::RayCast (include/bulbit/bvh.h:102-155),
// BoundingBox3::TestRay (include/bulbit/bounding_box.h:443-483), the
// Möller-Trumbore test of Triangle::Intersect (src/geometry/triangle.cpp:55-110)
// and Sphere::Intersect (src/geometry/sphere.cpp:35-85), so closest-hit
// primitive ids and t agree bit for bit with the reference, including its
// last-visited-wins rule for equal t.
//
// Layout in HBM (see bbg_internal.h):
//   nodes: 32 B each = two float4 (min.xyz, max.x) (max.yz, offset, count|axis<<16)
//   slots: 48 B each = three float4 per leaf slot, primitives in leaf order
#pragma once

#include "bbg_internal.h"
#include "dev_math.cuh"
#include "wide8_build.cuh"

#include <cuda_fp16.h>

#ifndef BBG_SLAB_FMA
#define BBG_SLAB_FMA 1
#endif

namespace bbg
{

struct AccelView
{
    const float4* nodes;  // reference layout: 2 per node
    const float4* slots;  // 3 per slot
    const float4* wide;   // child-box layout: 4 per interior node
    const int2* leaves;   // (first slot, count) per leaf
    int32_t root;         // child-box layout root reference
    int32_t ordered;      // 1: nearest-first traversal over the child-box layout
    const float4* wide8 = nullptr; // 8-wide layout: 6 per node (null: not built)
    int32_t root8 = 0;             // 8-wide root node
};

struct RayQ
{
    V3 o, d;          // ray as given
    V3 inv_dir;       // 1 / d per component
    V3 dn;            // d after Vector3::Normalize (triangle test)
    float l;          // length returned by that Normalize
    V3 oinv;          // o * (1/d), for the fused slab test of the ordered traversal
    int neg[3];       // inv_dir < 0
};

__device__ __forceinline__ RayQ MakeRayQ(V3 o, V3 d)
{
    RayQ q;
    q.o = o;
    q.d = d;
    q.inv_dir = V3{ 1 / d.x, 1 / d.y, 1 / d.z };
    q.neg[0] = q.inv_dir.x < 0;
    q.neg[1] = q.inv_dir.y < 0;
    q.neg[2] = q.inv_dir.z < 0;
    q.dn = d;
    q.l = NormalizeInPlace(q.dn);
    q.oinv = V3{ o.x * q.inv_dir.x, o.y * q.inv_dir.y, o.z * q.inv_dir.z };
    return q;
}

// BoundingBox3::TestRay: x and y slabs narrow [t_min, t_max], z only tests.
__device__ __forceinline__ bool TestRay(const float4& a, const float4& b, const RayQ& q, float t_min, float t_max)
{
    // a = (min.x, min.y, min.z, max.x), b = (max.y, max.z, ., .)
    float lo_x = q.neg[0] ? a.w : a.x, hi_x = q.neg[0] ? a.x : a.w;
    float lo_y = q.neg[1] ? b.x : a.y, hi_y = q.neg[1] ? a.y : b.x;
    float lo_z = q.neg[2] ? b.y : a.z, hi_z = q.neg[2] ? a.z : b.y;

    float t_min_x = (lo_x - q.o.x) * q.inv_dir.x;
    float t_max_x = (hi_x - q.o.x) * q.inv_dir.x;
    if (t_min > t_max_x || t_max < t_min_x)
    {
        return false;
    }
    if (t_min_x > t_min) t_min = t_min_x;
    if (t_max_x < t_max) t_max = t_max_x;

    float t_min_y = (lo_y - q.o.y) * q.inv_dir.y;
    float t_max_y = (hi_y - q.o.y) * q.inv_dir.y;
    if (t_min > t_max_y || t_max < t_min_y)
    {
        return false;
    }
    if (t_min_y > t_min) t_min = t_min_y;
    if (t_max_y < t_max) t_max = t_max_y;

    float t_min_z = (lo_z - q.o.z) * q.inv_dir.z;
    float t_max_z = (hi_z - q.o.z) * q.inv_dir.z;
    if (t_min > t_max_z || t_max < t_min_z)
    {
        return false;
    }
    return true;
}

// Möller-Trumbore on the normalised direction (src/geometry/triangle.cpp:55-94).
// The edges e1 = p1 - p0 and e2 = p2 - p0 are stored precomputed (the same
// float values the reference computes per test). Returns true and (t, u, v)
// on a hit in [t_min, t_max].
__device__ __forceinline__ bool IntersectTriangle(V3 p0, V3 e1, V3 e2, const RayQ& q, float t_min, float t_max,
                                                  float* t_out, float* u_out, float* v_out)
{
    V3 pvec = Cross(q.dn, e2);
    float det = Dot(e1, pvec);
    if (fabsf(det) < kEpsilon)
    {
        return false;
    }
    float invDet = 1 / det;
    V3 tvec = q.o - p0;
    const float du = Dot(tvec, pvec);
    float u = du * invDet;
    if (u < 0 || u > 1)
    {
        return false;
    }
    V3 qvec = Cross(tvec, e1);
    float v = Dot(q.dn, qvec) * invDet;
    if (v < 0 || u + v > 1)
    {
        return false;
    }
    float t = Dot(e2, qvec) * invDet / q.l;
    if (t < t_min || t > t_max)
    {
        return false;
    }
    *t_out = t;
    *u_out = u;
    *v_out = v;
    return true;
}

// Quat::RotateInv / Rotate (include/bulbit/quaternion.h:140-170).
__device__ __forceinline__ V3 QuatRotateInv(float4 q, V3 v)
{
    float vx = 2 * v.x, vy = 2 * v.y, vz = 2 * v.z;
    float w2 = q.w * q.w - 0.5f;
    float dot2 = (q.x * vx + q.y * vy + q.z * vz);
    return V3{ (vx * w2 - (q.y * vz - q.z * vy) * q.w + q.x * dot2),
               (vy * w2 - (q.z * vx - q.x * vz) * q.w + q.y * dot2),
               (vz * w2 - (q.x * vy - q.y * vx) * q.w + q.z * dot2) };
}

__device__ __forceinline__ V3 QuatRotate(float4 q, V3 v)
{
    float vx = 2 * v.x, vy = 2 * v.y, vz = 2 * v.z;
    float w2 = q.w * q.w - 0.5f;
    float dot2 = (q.x * vx + q.y * vy + q.z * vz);
    return V3{ (vx * w2 + (q.y * vz - q.z * vy) * q.w + q.x * dot2),
               (vy * w2 + (q.z * vx - q.x * vz) * q.w + q.y * dot2),
               (vz * w2 + (q.x * vy - q.y * vx) * q.w + q.z * dot2) };
}

// Sphere::Intersect (src/geometry/sphere.cpp:35-61) in object space:
// MulT(transform, ray) then the half-b quadratic; near root first.
__device__ __forceinline__ bool IntersectSphere(V3 p, float4 rot, V3 s, float radius, V3 o, V3 d, float t_min,
                                                float t_max, float* t_out)
{
    V3 ro = QuatRotateInv(rot, o - p) / s;
    V3 rd = QuatRotateInv(rot, d / s);
    V3 oc = ro;
    float a = Length2(rd);
    float half_b = Dot(oc, rd);
    float c = Length2(oc) - radius * radius;
    float discriminant = half_b * half_b - a * c;
    if (discriminant < 0)
    {
        return false;
    }
    float sqrt_d = sqrtf(discriminant);
    float root = (-half_b - sqrt_d) / a;
    if (root < t_min || t_max < root)
    {
        root = (-half_b + sqrt_d) / a;
        if (root < t_min || t_max < root)
        {
            return false;
        }
    }
    *t_out = root;
    return true;
}

struct TraceResult
{
    int32_t prim; // primitive index, -1 on a miss
    float t, u, v;
};

// One leaf slot: the primitive's test with the current [t_min, t_max].
// SPHERES = false: the tree holds triangles only (no sphere test compiled in,
// which keeps the traversal kernels' register count down).
template <bool SPHERES = true>
__device__ __forceinline__ bool TestSlot(const AccelView& a, int32_t slot, const RayQ& q, float t_min, float t_max,
                                         TraceResult* res)
{
    const float4* s = a.slots + 3 * size_t(slot);
    float4 s0 = __ldg(s);
    float4 s1 = __ldg(s + 1);
    float4 s2 = __ldg(s + 2);
    uint32_t tag = __float_as_uint(s0.w);
    float t, u = 0, v = 0;
    bool hit;
    if (SPHERES && (tag & kSphereBit))
    {
        hit = IntersectSphere(V3{ s0.x, s0.y, s0.z }, s1, V3{ s2.x, s2.y, s2.z }, s2.w, q.o, q.d, t_min, t_max, &t);
    }
    else
    {
        hit = IntersectTriangle(V3{ s0.x, s0.y, s0.z }, V3{ s1.x, s1.y, s1.z }, V3{ s2.x, s2.y, s2.z }, q, t_min,
                                t_max, &t, &u, &v);
    }
    if (hit)
    {
        res->prim = int32_t(tag & ~kSphereBit);
        res->t = t;
        res->u = u;
        res->v = v;
    }
    return hit;
}

// Stack traversal of BVH::RayCast over the reference's own node order. ANY =
// IntersectAny semantics (stop at the first hit); otherwise Intersect
// semantics (shrink t_max; a hit at exactly the current t_max replaces the
// previous one). COUNT accumulates nodes popped and primitive tests.
template <bool ANY, bool COUNT>
__device__ __forceinline__ TraceResult TraceReference(const AccelView& a, const RayQ& q, float t_min, float t_max,
                                                      uint32_t* nodes_visited = nullptr,
                                                      uint32_t* prims_tested = nullptr)
{
    TraceResult res{ -1, t_max, 0, 0 };
    int32_t stack[kStackCapacity];
    int sp = 0;
    stack[sp++] = 0;

    while (sp > 0)
    {
        int32_t index = stack[--sp];
        float4 na = __ldg(a.nodes + 2 * index);
        float4 nb = __ldg(a.nodes + 2 * index + 1);
        if (COUNT) ++*nodes_visited;
        if (!TestRay(na, nb, q, t_min, t_max))
        {
            continue;
        }
        int32_t offset = __float_as_int(nb.z);
        uint32_t packed = __float_as_uint(nb.w);
        int32_t count = int32_t(packed & 0xffffu);
        if (count > 0)
        {
            for (int32_t i = 0; i < count; ++i)
            {
                if (COUNT) ++*prims_tested;
                // The callback's return value: t_min after an any-hit, the
                // hit's t after a closest hit, the running t_max on a miss;
                // RayCast stops when it is <= t_min, else takes it as t_max.
                if (TestSlot(a, offset + i, q, t_min, t_max, &res))
                {
                    if (ANY)
                    {
                        return res;
                    }
                    t_max = res.t;
                }
                if (t_max <= t_min)
                {
                    return res;
                }
            }
        }
        else
        {
            int32_t child1 = index + 1;
            int32_t child2 = offset;
            int axis = int((packed >> 16) & 0xffu);
            if (q.neg[axis])
            {
                stack[sp++] = child1;
                stack[sp++] = child2;
            }
            else
            {
                stack[sp++] = child2;
                stack[sp++] = child1;
            }
        }
    }
    return res;
}

// Slab test of one child box: [entry, exit] of the ray within the box and
// within [t_min, t_max], with the reference's per-axis arithmetic
// (bound - o) * (1/d) (include/bulbit/bounding_box.h:448-480).
__device__ __forceinline__ bool SlabTest(float lx, float ly, float lz, float hx, float hy, float hz, const RayQ& q,
                                         float t_min, float t_max, float* entry)
{
#if BBG_SLAB_FMA
    // bound * (1/d) - o * (1/d) in one fused multiply-add per plane. It may
    // round differently from the reference's (bound - o) * (1/d); it only
    // decides which boxes are opened, and triangle boxes are padded by
    // 10 epsilon (src/geometry/triangle.cpp:42), far beyond that rounding.
    float x0 = __fmaf_rn(q.neg[0] ? hx : lx, q.inv_dir.x, -q.oinv.x);
    float x1 = __fmaf_rn(q.neg[0] ? lx : hx, q.inv_dir.x, -q.oinv.x);
    float y0 = __fmaf_rn(q.neg[1] ? hy : ly, q.inv_dir.y, -q.oinv.y);
    float y1 = __fmaf_rn(q.neg[1] ? ly : hy, q.inv_dir.y, -q.oinv.y);
    float z0 = __fmaf_rn(q.neg[2] ? hz : lz, q.inv_dir.z, -q.oinv.z);
    float z1 = __fmaf_rn(q.neg[2] ? lz : hz, q.inv_dir.z, -q.oinv.z);
#else
    float x0 = ((q.neg[0] ? hx : lx) - q.o.x) * q.inv_dir.x;
    float x1 = ((q.neg[0] ? lx : hx) - q.o.x) * q.inv_dir.x;
    float y0 = ((q.neg[1] ? hy : ly) - q.o.y) * q.inv_dir.y;
    float y1 = ((q.neg[1] ? ly : hy) - q.o.y) * q.inv_dir.y;
    float z0 = ((q.neg[2] ? hz : lz) - q.o.z) * q.inv_dir.z;
    float z1 = ((q.neg[2] ? lz : hz) - q.o.z) * q.inv_dir.z;
#endif
    float t0 = fmaxf(fmaxf(x0, y0), fmaxf(z0, t_min));
    float t1 = fminf(fminf(x1, y1), fminf(z1, t_max));
    *entry = t0;
    return t0 <= t1;
}


// Persistent warp-cooperative traversal over the child-box layout (the
// while-while scheme of Aila & Laine, "Understanding the efficiency of ray
// traversal on GPUs", HPG 2009, with dynamic ray fetch):
//   * a warp takes batches of work items from a global counter whenever fewer
//     than kRefill of its lanes still hold a ray, so lanes that finish early
//     get new rays instead of idling until the slowest ray of the batch ends;
//   * each round first walks interior nodes until every busy lane has found a
//     leaf (a lane that reaches a leaf postpones it and keeps walking), then
//     tests leaves together, so node and leaf work do not serialise the warp.
// Per ray: nearest child first over the child-box layout (each interior node
// holds both children's boxes, so one 64-byte fetch tests two), the farther
// child pushed with its entry distance and skipped on pop once a closer hit
// is known; the same primitive tests as BVH::RayCast in a different order, so
// the closest hit is the same except between hits at exactly equal t.
// Src supplies Load(item, RayQ*, t_min*, t_max*) and Store(item, result).
constexpr int32_t kNoNode = int32_t(0x80000000);
// 28 of 32 measured best for both layouts (16: -9 %, 24: -2.5 %, 32: -9 % on
// the 1M-triangle soup's closest + any-hit rays; path tracing unchanged).
#ifndef BBG_REFILL
#define BBG_REFILL 28
#endif
#ifndef BBG_SHORT_STACK
#define BBG_SHORT_STACK 16
#endif
// A warp fetches new rays when fewer than kRefill of its lanes are busy.
constexpr int kRefill = BBG_REFILL;
// Kernels calling TracePersistent run blocks of this many threads.
constexpr int kTraversalBlock = 128;
// Stack entries kept in shared memory per thread; deeper ones go to local
// memory. The shared part is laid out [depth][thread], so a warp's lanes hit
// distinct banks whatever depth each lane is at.
constexpr int kShortStack = BBG_SHORT_STACK;

// BLOCK: threads per block of the launch; SHORT: stack entries kept in
// shared memory per thread (0: the whole stack in local memory).
template <bool ANY, class Src, int BLOCK = kTraversalBlock, int SHORT = kShortStack>
__device__ __forceinline__ void TracePersistent(const AccelView& a, int32_t n, int32_t* next, Src& src)
{
    const unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int tid = threadIdx.x;
    int32_t item = -1;
    bool exhausted = false;
    RayQ q;
    float t_min = 0, t_max = 0;
    TraceResult res{ -1, 0, 0, 0 };
    __shared__ int32_t s_ref[(SHORT > 0 ? SHORT : 1) * BLOCK];
    __shared__ float s_entry[(SHORT > 0 ? SHORT : 1) * BLOCK];
    int2 spill[kStackCapacity - SHORT];
    int sp = 0;
    int32_t node = kNoNode, leaf = kNoNode;
    // The tree a ray is traced in: the one given, or, when the work source
    // names one per item (several scenes in one launch), that one.
    AccelView av = a;

    auto push = [&](int32_t ref, float entry) {
        if (sp < SHORT)
        {
            s_ref[sp * BLOCK + tid] = ref;
            s_entry[sp * BLOCK + tid] = entry;
        }
        else
        {
            spill[sp - SHORT] = make_int2(ref, __float_as_int(entry));
        }
        ++sp;
    };
    auto pop = [&]() -> int32_t {
        while (sp > 0)
        {
            --sp;
            int32_t ref;
            float entry;
            if (sp < SHORT)
            {
                ref = s_ref[sp * BLOCK + tid];
                entry = s_entry[sp * BLOCK + tid];
            }
            else
            {
                int2 e = spill[sp - SHORT];
                ref = e.x;
                entry = __int_as_float(e.y);
            }
            if (entry <= t_max)
            {
                return ref;
            }
        }
        return kNoNode;
    };

    while (true)
    {
        __syncwarp();
        bool busy = item >= 0;
        unsigned have = __ballot_sync(kFull, busy);
        if (!exhausted && __popc(have) < kRefill)
        {
            unsigned need = ~have;
            int32_t cnt = __popc(need);
            int32_t base = 0;
            if (lane == 0)
            {
                base = atomicAdd(next, cnt);
            }
            base = __shfl_sync(kFull, base, 0);
            exhausted = base + cnt >= n;
            if (!busy)
            {
                int32_t r = base + __popc(need & ((1u << lane) - 1u));
                if (r < n)
                {
                    item = r;
                    src.Load(r, &q, &t_min, &t_max);
                    if constexpr (requires { src.View(r); })
                    {
                        av = src.View(r);
                    }
                    res = TraceResult{ -1, t_max, 0, 0 };
                    sp = 0;
                    node = av.root;
                    leaf = kNoNode;
                    busy = true;
                }
            }
            have = __ballot_sync(kFull, busy);
        }
        if (have == 0)
        {
            break;
        }
        if (busy)
        {
            if (node < 0 && node != kNoNode && leaf == kNoNode)
            {
                leaf = node;
                node = pop();
            }
            // Node phase.
            while (node >= 0)
            {
                const float4* nd = av.wide + 4 * size_t(node);
                float4 f0 = __ldg(nd);
                float4 f1 = __ldg(nd + 1);
                float4 f2 = __ldg(nd + 2);
                int4 f3 = __ldg(reinterpret_cast<const int4*>(nd + 3));
                float e0, e1;
                bool h0 = SlabTest(f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, q, t_min, t_max, &e0);
                bool h1 = SlabTest(f1.z, f1.w, f2.x, f2.y, f2.z, f2.w, q, t_min, t_max, &e1);
                if (h0 && h1)
                {
                    bool swap = e1 < e0;
                    push(swap ? f3.x : f3.y, swap ? e0 : e1);
                    node = swap ? f3.y : f3.x;
                }
                else if (h0 || h1)
                {
                    node = h0 ? f3.x : f3.y;
                }
                else
                {
                    node = pop();
                }
                if (node < 0 && node != kNoNode && leaf == kNoNode)
                {
                    leaf = node;
                    node = pop();
                }
                if (__all_sync(__activemask(), leaf != kNoNode))
                {
                    break;
                }
            }
            // Leaf phase.
            while (leaf != kNoNode)
            {
                int2 lf = __ldg(av.leaves + (~leaf));
                bool stop = false;
                for (int32_t i = 0; i < lf.y; ++i)
                {
                    if (TestSlot(av, lf.x + i, q, t_min, t_max, &res))
                    {
                        if (ANY)
                        {
                            stop = true;
                            break;
                        }
                        t_max = res.t;
                    }
                    if (t_max <= t_min)
                    {
                        stop = true;
                        break;
                    }
                }
                leaf = kNoNode;
                if (stop)
                {
                    node = kNoNode;
                    sp = 0;
                    break;
                }
                if (node < 0 && node != kNoNode)
                {
                    leaf = node;
                    node = pop();
                }
            }
            if (node == kNoNode && leaf == kNoNode)
            {
                src.Store(item, res);
                item = -1;
            }
        }
    }
}

// ---------------------------------------------------------------- 8-wide layout
//
// The reference's binary SAH tree collapsed into nodes of up to eight
// children (the compressed wide BVH of Ylitie, Karras and Laine, "Efficient
// Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017).
// 96 bytes per node, six float4:
//   [0]   origin p (the node box's lower corner), meta = biased exponents
//         e_x | e_y << 8 | e_z << 16 of the per-axis scales s = 2^e, and
//         << 24 the mask of interior-child slots
//   [1-3] child boxes as bytes, child k in byte k & 3 of word k >> 2:
//         qlo_x, qlo_y, qlo_z, qhi_x, qhi_y, qhi_z (two words each)
//   [4-5] child references: >= 0 node, < 0 a leaf ~(first slot << 5 |
//         count); an empty slot is a leaf of no primitives with an inverted
//         box
// Child k's box is [p + qlo s, p + qhi s], rounded outward when built, so it
// contains the binary node it stands for and no ray that reaches a leaf in
// the binary tree is culled here. Slots are assigned so that, for a ray whose
// direction signs form the octant code o (bit a set for a negative axis),
// visiting slots in the order k ^ o for k = 0..7 is roughly front to back.

// Bytes 2 pair and 2 pair + 1 of w as floats: one byte permute assembles the
// half2 (1024 + b0, 1024 + b1) (bits 0x64bb), converted and less 1024, exactly.
__device__ __forceinline__ float2 BytePairAsFloat(uint32_t w, int pair)
{
    uint32_t h = __byte_perm(w, 0x64646464u, pair ? 0x4342u : 0x4140u);
    __half2 v = *reinterpret_cast<__half2*>(&h);
    float2 f = __half22float2(v);
    return make_float2(f.x - 1024.0f, f.y - 1024.0f);
}

// Three-input minimum / maximum (PTX min.f32 / max.f32 with three sources;
// a NaN source is ignored as by fminf / fmaxf).
__device__ __forceinline__ float Max3(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float Min3(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Moves bit k of each byte of m to bit k ^ oct (oct in 0..7).
__device__ __forceinline__ uint32_t PermuteByOctant(uint32_t m, uint32_t oct)
{
    if (oct & 1u) m = ((m & 0x5555u) << 1) | ((m >> 1) & 0x5555u);
    if (oct & 2u) m = ((m & 0x3333u) << 2) | ((m >> 2) & 0x3333u);
    if (oct & 4u) m = ((m & 0x0f0fu) << 4) | ((m >> 4) & 0x0f0fu);
    return m;
}

// Tests the ray against a node's eight child boxes. Bits of *inner / *leaf
// are visit positions (slot ^ octant) of the hit interior / leaf children;
// the node's references are returned for the caller to pick from.
__device__ __forceinline__ void IntersectNode8(const float4* nd, const RayQ& q, uint32_t oct, float t_min, float t_max,
                                               uint32_t* inner, uint32_t* leaf, int4* refs_lo, int4* refs_hi)
{
    float4 h = __ldg(nd);
    uint4 w1 = __ldg(reinterpret_cast<const uint4*>(nd + 1));
    uint4 w2 = __ldg(reinterpret_cast<const uint4*>(nd + 2));
    uint4 w3 = __ldg(reinterpret_cast<const uint4*>(nd + 3));
    *refs_lo = __ldg(reinterpret_cast<const int4*>(nd + 4));
    *refs_hi = __ldg(reinterpret_cast<const int4*>(nd + 5));
    uint32_t meta = __float_as_uint(h.w);
    // Plane k of axis a sits at p_a + q s_a: t = q (s_a / d_a) + (p_a - o_a) / d_a.
    float bx = __uint_as_float((meta & 0xffu) << 23) * q.inv_dir.x;
    float by = __uint_as_float(((meta >> 8) & 0xffu) << 23) * q.inv_dir.y;
    float bz = __uint_as_float(((meta >> 16) & 0xffu) << 23) * q.inv_dir.z;
    // (p - o) / d in the reference's slab form; the ray's signs from 1/d
    // (kept in predicates rather than per-ray registers).
    float ax = (h.x - q.o.x) * q.inv_dir.x;
    float ay = (h.y - q.o.y) * q.inv_dir.y;
    float az = (h.z - q.o.z) * q.inv_dir.z;
    const bool negx = q.inv_dir.x < 0, negy = q.inv_dir.y < 0, negz = q.inv_dir.z < 0;
    // Entry planes are the low bounds on a positive axis, the high ones on a negative axis.
    uint32_t nx0 = negx ? w2.z : w1.x, nx1 = negx ? w2.w : w1.y;
    uint32_t fx0 = negx ? w1.x : w2.z, fx1 = negx ? w1.y : w2.w;
    uint32_t ny0 = negy ? w3.x : w1.z, ny1 = negy ? w3.y : w1.w;
    uint32_t fy0 = negy ? w1.z : w3.x, fy1 = negy ? w1.w : w3.y;
    uint32_t nz0 = negz ? w3.z : w2.x, nz1 = negz ? w3.w : w2.y;
    uint32_t fz0 = negz ? w2.x : w3.z, fz1 = negz ? w2.y : w3.w;
    uint32_t hits = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) // children 2j and 2j + 1
    {
        const int pair = j & 1;
        const bool hi = j >= 2;
        float2 qnx = BytePairAsFloat(hi ? nx1 : nx0, pair), qfx = BytePairAsFloat(hi ? fx1 : fx0, pair);
        float2 qny = BytePairAsFloat(hi ? ny1 : ny0, pair), qfy = BytePairAsFloat(hi ? fy1 : fy0, pair);
        float2 qnz = BytePairAsFloat(hi ? nz1 : nz0, pair), qfz = BytePairAsFloat(hi ? fz1 : fz0, pair);
        float t0a = Max3(__fmaf_rn(qnx.x, bx, ax), __fmaf_rn(qny.x, by, ay), fmaxf(__fmaf_rn(qnz.x, bz, az), t_min));
        float t1a = Min3(__fmaf_rn(qfx.x, bx, ax), __fmaf_rn(qfy.x, by, ay), fminf(__fmaf_rn(qfz.x, bz, az), t_max));
        float t0b = Max3(__fmaf_rn(qnx.y, bx, ax), __fmaf_rn(qny.y, by, ay), fmaxf(__fmaf_rn(qnz.y, bz, az), t_min));
        float t1b = Min3(__fmaf_rn(qfx.y, bx, ax), __fmaf_rn(qfy.y, by, ay), fminf(__fmaf_rn(qfz.y, bz, az), t_max));
        if (t0a <= t1a)
        {
            hits |= 1u << (2 * j);
        }
        if (t0b <= t1b)
        {
            hits |= 1u << (2 * j + 1);
        }
    }
    // Slot-order masks (interior slots from the header), then visit positions.
    uint32_t imask = meta >> 24;
    uint32_t m = PermuteByOctant((hits & imask) | ((hits & ~imask) << 8), oct);
    *inner = m & 0xffu;
    *leaf = m >> 8;
}

__device__ __forceinline__ int32_t ChildRef8(const float4* wide8, int32_t node, uint32_t slot)
{
    return __ldg(reinterpret_cast<const int32_t*>(wide8 + 6 * size_t(node) + 4) + slot);
}

// Reference of slot k (0..7) from the two int4 of a node, by selects (no
// indexed register array, which would live in local memory).
__device__ __forceinline__ int32_t SelectRef8(const int4& a, const int4& b, uint32_t k)
{
    int4 v = (k & 4u) ? b : a;
    int32_t lo = (k & 1u) ? v.y : v.x;
    int32_t hi = (k & 1u) ? v.w : v.z;
    return (k & 2u) ? hi : lo;
}


// Persistent traversal of the 8-wide layout (same work-source protocol as
// TracePersistent). Each iteration opens one node: its hit leaf children's
// primitives are tested at once, and the nearest hit interior child (by the
// octant order) becomes the next node, the rest of them pushed as a group
// (node << 8 | visit positions left). The next node's reference comes from
// the registers of the node just opened; only a group taken off the stack
// reads its reference from memory. Every push is one tree level deeper than
// the last, so the tree depth bounds the stack.
template <bool ANY, class Src, int BLOCK = kTraversalBlock, int SHORT = kShortStack, bool SPHERES = true>
__device__ __forceinline__ void TracePersistentWide(const AccelView& a, int32_t n, int32_t* next, Src& src)
{
    const unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int tid = threadIdx.x;
    int32_t item = -1;
    bool exhausted = false;
    RayQ q;
    float t_min = 0, t_max = 0;
    TraceResult res{ -1, 0, 0, 0 };
    __shared__ int32_t s_stack[(SHORT > 0 ? SHORT : 1) * BLOCK];
    int32_t spill[kStackCapacity - SHORT];
    int sp = 0;
    uint32_t oct = 0;
    int32_t pending = kNoNode; // next node to open
    AccelView av = a;

    auto push = [&](int32_t e) {
        if (sp < SHORT)
        {
            s_stack[sp * BLOCK + tid] = e;
        }
        else
        {
            spill[sp - SHORT] = e;
        }
        ++sp;
    };
    auto pop = [&]() -> int32_t {
        --sp;
        return sp < SHORT ? s_stack[sp * BLOCK + tid] : spill[sp - SHORT];
    };

    while (true)
    {
        __syncwarp();
        bool busy = item >= 0;
        unsigned have = __ballot_sync(kFull, busy);
        if (!exhausted && __popc(have) < kRefill)
        {
            unsigned need = ~have;
            int32_t cnt = __popc(need);
            int32_t base = 0;
            if (lane == 0)
            {
                base = atomicAdd(next, cnt);
            }
            base = __shfl_sync(kFull, base, 0);
            exhausted = base + cnt >= n;
            if (!busy)
            {
                int32_t r = base + __popc(need & ((1u << lane) - 1u));
                if (r < n)
                {
                    item = r;
                    src.Load(r, &q, &t_min, &t_max);
                    if constexpr (requires { src.View(r); })
                    {
                        av = src.View(r);
                    }
                    res = TraceResult{ -1, t_max, 0, 0 };
                    sp = 0;
                    oct = uint32_t(q.inv_dir.x < 0) | (uint32_t(q.inv_dir.y < 0) << 1) | (uint32_t(q.inv_dir.z < 0) << 2);
                    pending = av.root8;
                    busy = true;
                }
            }
            have = __ballot_sync(kFull, busy);
        }
        if (have == 0)
        {
            break;
        }
        if (busy)
        {
            if (pending == kNoNode)
            {
                // The current group is spent: continue with the group below.
                int32_t e = pop();
                int32_t gnode = e >> 8;
                uint32_t gmask = uint32_t(e) & 0xffu;
                uint32_t pos = uint32_t(__ffs(gmask) - 1);
                gmask &= gmask - 1;
                pending = ChildRef8(av.wide8, gnode, pos ^ oct);
                if (gmask != 0)
                {
                    push((gnode << 8) | int32_t(gmask));
                }
            }
            const int32_t node = pending;
            uint32_t im, lm;
            int4 ra, rb;
            IntersectNode8(av.wide8 + 6 * size_t(node), q, oct, t_min, t_max, &im, &lm, &ra, &rb);
            // The node's hit leaves.
            while (lm != 0)
            {
                uint32_t pos = uint32_t(__ffs(lm) - 1);
                lm &= lm - 1;
                uint32_t lf = ~uint32_t(SelectRef8(ra, rb, pos ^ oct));
                int32_t first = int32_t(lf >> kWide8LeafCountBits);
                int32_t count = int32_t(lf & ((1u << kWide8LeafCountBits) - 1u));
                bool stop = false;
                for (int32_t i = 0; i < count; ++i)
                {
                    if (TestSlot<SPHERES>(av, first + i, q, t_min, t_max, &res))
                    {
                        if (ANY)
                        {
                            stop = true;
                            break;
                        }
                        t_max = res.t;
                    }
                    if (t_max <= t_min)
                    {
                        stop = true;
                        break;
                    }
                }
                if (stop)
                {
                    lm = 0;
                    im = 0;
                    sp = 0;
                }
            }
            // The nearest hit interior child next; the others as a group.
            if (im != 0)
            {
                uint32_t pos = uint32_t(__ffs(im) - 1);
                im &= im - 1;
                pending = SelectRef8(ra, rb, pos ^ oct);
                if (im != 0)
                {
                    push((node << 8) | int32_t(im));
                }
            }
            else
            {
                pending = kNoNode;
                if (sp == 0)
                {
                    src.Store(item, res);
                    item = -1;
                }
            }
        }
    }
}


} // namespace bbg
