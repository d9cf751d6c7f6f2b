// The reference's binned SAH tree built on the device, node for node.
//
// BVH::BuildRecursive (src/accel/bvh.cpp:56-271) splits a node's primitive
// span by 12 centroid buckets along the longest centroid axis, with cost
// 0.5 + (n_l A_l + n_r A_r) / A and a leaf when that is not below the count,
// and reorders the span with std::partition (two primitives: std::nth_element).
// Every quantity the decision reads is a float min / max (exact in any order),
// an integer count, or a short sequential float expression evaluated once per
// node, so a parallel build that evaluates the same expressions reproduces the
// same tree. The permutation std::partition leaves (libstdc++'s bidirectional
// algorithm: the k-th element from the left that belongs right is swapped with
// the k-th element from the right that belongs left) is restated as a pairing
// by prefix sums, and two primitives are ordered as insertion sort orders them.
//
// The build runs top down, one launch per tree level (one block per node of
// more than 32 primitives, one warp per smaller node). Each split passes its
// children their primitive and centroid bounds from the bucket bounds, so a
// node reads its primitives twice: once for the buckets, once to partition.
// No node is ever moved: leaves own contiguous ranges of the primitive order,
// in depth-first order, and a node's depth-first index is
//   depth - 1 + 2 * (leaves left of its first primitive) - (right turns on
//   its root path),
// which a scan over leaf starts gives every node at once. The depth-first
// array then feeds the same layouts the host-built tree gets: reference
// nodes, slot records, the binary child-box layout and the 8-wide collapse
// (numbered breadth first in child order, as on the host).
//
// Exactness caveat: min / max in parallel cannot tell +0 from -0 the way a
// sequential std::min does (the first of two equal zeros wins there); a box
// bound that is exactly -0 can print with the other sign. Primitive boxes
// carry a padding (Triangle::GetAABB) or a radius, so their bounds are
// never zero unless a coordinate equals the padding exactly.

#include "accel.cuh"
#include "build_util.cuh"
#include "wide8_build.cuh"

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <vector>

namespace bbg
{
namespace
{

constexpr int kSahBlock = 512;     // threads per node of the block kernel
constexpr int kSahPerThread = 8;   // consecutive primitives per thread in a partition tile
constexpr int kSahTile = kSahBlock * kSahPerThread;
constexpr int kSahWarpTask = 32;   // nodes of at most this many primitives: one warp each
constexpr int kSahWarpBlock = 256; // threads per block of the warp kernel
constexpr int kBuckets = 12;       // bucket_size (src/accel/bvh.cpp:141)
constexpr int kPlanes = kBuckets - 1;
constexpr int kKeys = 12;          // box min xyz, box max xyz, centre min xyz, centre max xyz

struct SahDev
{
    const float4* box; // 2 per primitive: (min xyz, 0) (max xyz, 0)
    const float4* cen; // per primitive: centre (min + max) * 0.5f
    int32_t* idx;      // the primitive order; every node owns a contiguous range of it
    int32_t* scr_l;    // partition: positions left of the split that move right (per node range)
    int32_t* scr_r;    // positions right of the split that move left
    uint32_t* leaf_at; // 1 where a leaf's range starts
    float4* bounds;    // per node: 4 float4: box min, box max, centre min, centre max
    int4* info;        // per node: (start, count, left child id or -1 for a leaf, axis); right = left + 1
    int2* path;        // per node: (depth, right turns on the path from the root)
    int32_t* counters; // [0] nodes created, [1] next big tasks, [2] next small tasks, [3] leaf over 65535
};

__device__ __forceinline__ float SurfaceArea(float3 lo, float3 hi)
{
    // AABB::GetSurfaceArea: 2 * ((w.x * w.y) + (w.y * w.z) + (w.z * w.x)), w = max - min.
    float wx = hi.x - lo.x, wy = hi.y - lo.y, wz = hi.z - lo.z;
    return 2 * ((wx * wy) + (wy * wz) + (wz * wx));
}

__device__ __forceinline__ float Axis(float4 v, int a)
{
    return a == 0 ? v.x : (a == 1 ? v.y : v.z);
}

// The bucket of a centre coordinate: int32(12 * (c - min) / extent), the top
// edge folded into the last bucket (src/accel/bvh.cpp:157-162).
__device__ __forceinline__ int32_t BucketOf(float c, float cmin, float extent)
{
    int32_t b = int32_t(kBuckets * (c - cmin) / extent);
    return b == kBuckets ? kBuckets - 1 : b;
}

// std::min / std::max over boxes kept as order-preserving keys. The empty
// box is the host's default (FLT_MAX, -FLT_MAX).
// FloatKey(FLT_MAX) and FloatKey(-FLT_MAX): FLT_MAX is 0x7f7fffff, positive
// keys set the sign bit, negative ones are complemented.
__host__ __device__ constexpr uint32_t EmptyMinKey() { return 0x7f7fffffu | 0x80000000u; }
__host__ __device__ constexpr uint32_t EmptyMaxKey() { return ~(0x7f7fffffu | 0x80000000u); }

// The split decision of one node from its bucket counts and bounds, evaluated
// in the reference's order (src/accel/bvh.cpp:166-205). Returns the split
// bucket or -1 for a leaf; *mid the left count; the children's box and
// centre bounds (as keys: box min, box max, centre min, centre max).
__device__ int32_t ChooseSplit(const int32_t* cnt, const uint32_t (*bk)[kKeys], int32_t count, float span_area,
                               int32_t* mid, uint32_t left_keys[kKeys], uint32_t right_keys[kKeys])
{
    float lb_lo[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, lb_hi[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
    float rb_lo[3] = { FLT_MAX, FLT_MAX, FLT_MAX }, rb_hi[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
    int32_t left_count[kPlanes], right_count[kPlanes];
    float left_area[kPlanes], right_area[kPlanes];
    int32_t left_sum = 0, right_sum = 0;
    for (int32_t i = 0; i < kPlanes; ++i)
    {
        left_sum += cnt[i];
        left_count[i] = left_sum;
        for (int a = 0; a < 3; ++a)
        {
            float lo = KeyFloat(bk[i][a]), hi = KeyFloat(bk[i][3 + a]);
            lb_lo[a] = lo < lb_lo[a] ? lo : lb_lo[a];
            lb_hi[a] = lb_hi[a] < hi ? hi : lb_hi[a];
        }
        left_area[i] = SurfaceArea(make_float3(lb_lo[0], lb_lo[1], lb_lo[2]), make_float3(lb_hi[0], lb_hi[1], lb_hi[2]));
        const int j = kPlanes - i;
        right_sum += cnt[j];
        right_count[kPlanes - 1 - i] = right_sum;
        for (int a = 0; a < 3; ++a)
        {
            float lo = KeyFloat(bk[j][a]), hi = KeyFloat(bk[j][3 + a]);
            rb_lo[a] = lo < rb_lo[a] ? lo : rb_lo[a];
            rb_hi[a] = rb_hi[a] < hi ? hi : rb_hi[a];
        }
        right_area[kPlanes - 1 - i] =
            SurfaceArea(make_float3(rb_lo[0], rb_lo[1], rb_lo[2]), make_float3(rb_hi[0], rb_hi[1], rb_hi[2]));
    }
    int32_t best = -1;
    float min_cost = __int_as_float(0x7f800000); // infinity
    for (int32_t i = 0; i < kPlanes; ++i)
    {
        float cost = left_count[i] * left_area[i] + right_count[i] * right_area[i];
        if (cost < min_cost)
        {
            min_cost = cost;
            best = i;
        }
    }
    const float traverse_cost = 0.5f;
    min_cost = traverse_cost + min_cost / span_area;
    if (!(min_cost < float(count)))
    {
        return -1;
    }
    *mid = left_count[best];
    for (int k = 0; k < kKeys; ++k)
    {
        const bool is_max = (k % 6) >= 3;
        uint32_t l = is_max ? EmptyMaxKey() : EmptyMinKey(), r = l;
        for (int b = 0; b < kBuckets; ++b)
        {
            if (cnt[b] == 0)
            {
                continue;
            }
            uint32_t v = bk[b][k];
            if (b <= best)
            {
                l = is_max ? max(l, v) : min(l, v);
            }
            else
            {
                r = is_max ? max(r, v) : min(r, v);
            }
        }
        left_keys[k] = l;
        right_keys[k] = r;
    }
    return best;
}

__device__ __forceinline__ void StoreBounds(float4* dst, const uint32_t keys[kKeys])
{
    dst[0] = make_float4(KeyFloat(keys[0]), KeyFloat(keys[1]), KeyFloat(keys[2]), 0.0f);
    dst[1] = make_float4(KeyFloat(keys[3]), KeyFloat(keys[4]), KeyFloat(keys[5]), 0.0f);
    dst[2] = make_float4(KeyFloat(keys[6]), KeyFloat(keys[7]), KeyFloat(keys[8]), 0.0f);
    dst[3] = make_float4(KeyFloat(keys[9]), KeyFloat(keys[10]), KeyFloat(keys[11]), 0.0f);
}

// Bounds of a single primitive (a child of a two-primitive node).
__device__ __forceinline__ void StorePrimBounds(const SahDev& S, float4* dst, int32_t p)
{
    float4 lo = S.box[2 * size_t(p)], hi = S.box[2 * size_t(p) + 1], c = S.cen[p];
    dst[0] = make_float4(lo.x, lo.y, lo.z, 0.0f);
    dst[1] = make_float4(hi.x, hi.y, hi.z, 0.0f);
    dst[2] = make_float4(c.x, c.y, c.z, 0.0f);
    dst[3] = dst[2];
}

// Creates the two children of `node` over [start, start + mid) and
// [start + mid, start + count) and queues them for the next level.
__device__ __forceinline__ int32_t EmitChildren(const SahDev& S, int32_t node, int32_t start, int32_t count, int32_t mid,
                                                int32_t axis, int32_t* next_big, int32_t* next_small)
{
    const int32_t id = atomicAdd(&S.counters[0], 2);
    const int2 pth = S.path[node];
    S.info[id] = make_int4(start, mid, -1, 0);
    S.info[id + 1] = make_int4(start + mid, count - mid, -1, 0);
    S.path[id] = make_int2(pth.x + 1, pth.y);
    S.path[id + 1] = make_int2(pth.x + 1, pth.y + 1);
    S.info[node] = make_int4(start, count, id, axis);
    for (int c = 0; c < 2; ++c)
    {
        const int32_t n = c == 0 ? mid : count - mid;
        if (n > kSahWarpTask)
        {
            next_big[atomicAdd(&S.counters[1], 1)] = id + c;
        }
        else
        {
            next_small[atomicAdd(&S.counters[2], 1)] = id + c;
        }
    }
    return id;
}

__device__ __forceinline__ void EmitLeaf(const SahDev& S, int32_t node, int32_t start, int32_t count)
{
    S.info[node] = make_int4(start, count, -1, 0);
    S.leaf_at[start] = 1;
    if (count > 0xffff)
    {
        S.counters[3] = 1; // uint16 primitive_count
    }
}

// The node's leaf tests: zero box area or one primitive, then a centroid
// extent of zero (src/accel/bvh.cpp:71-123). Returns false for a leaf.
__device__ __forceinline__ bool SplitAxis(const float4* bd, int32_t count, int32_t* axis, float* extent, float* area)
{
    *area = SurfaceArea(make_float3(bd[0].x, bd[0].y, bd[0].z), make_float3(bd[1].x, bd[1].y, bd[1].z));
    if (*area == 0 || count == 1)
    {
        return false;
    }
    float ex = bd[3].x - bd[2].x, ey = bd[3].y - bd[2].y, ez = bd[3].z - bd[2].z;
    int32_t a = 0;
    if (ey > ex)
    {
        a = 1;
    }
    if (ez > (a == 0 ? ex : ey))
    {
        a = 2;
    }
    *axis = a;
    *extent = a == 0 ? ex : (a == 1 ? ey : ez);
    return *extent != 0;
}

// Bins positions [lo, hi) of a node's range (block-wide; every thread of the
// block calls it): counts and the min / max keys of the boxes and centres in
// each bucket, merged into s_cnt / s_key (initialised by the caller).
__device__ __forceinline__ void BinRange(const SahDev& S, int32_t start, int32_t lo, int32_t hi, int32_t axis,
                                         float cmin, float extent, int32_t* s_cnt, uint32_t (*s_key)[kKeys])
{
    const int tid = threadIdx.x, lane = tid & 31;
    int32_t my_cnt = 0;
    uint32_t my_key[kKeys];
    for (int k = 0; k < kKeys; ++k)
    {
        my_key[k] = (k % 6) >= 3 ? EmptyMaxKey() : EmptyMinKey();
    }
    for (int32_t base = lo; base < hi; base += kSahBlock)
    {
        const int32_t i = base + tid;
        int32_t b = -1;
        uint32_t key[kKeys];
        if (i < hi)
        {
            const int32_t p = S.idx[start + i];
            const float4 c = S.cen[p], blo = S.box[2 * size_t(p)], bhi = S.box[2 * size_t(p) + 1];
            b = BucketOf(Axis(c, axis), cmin, extent);
            key[0] = FloatKey(blo.x), key[1] = FloatKey(blo.y), key[2] = FloatKey(blo.z);
            key[3] = FloatKey(bhi.x), key[4] = FloatKey(bhi.y), key[5] = FloatKey(bhi.z);
            key[6] = FloatKey(c.x), key[7] = FloatKey(c.y), key[8] = FloatKey(c.z);
            key[9] = key[6], key[10] = key[7], key[11] = key[8];
        }
        for (int32_t k = 0; k < kBuckets; ++k)
        {
            const unsigned m = __ballot_sync(0xffffffffu, b == k);
            if (m == 0)
            {
                continue;
            }
            const bool in = b == k;
            if (lane == k)
            {
                my_cnt += __popc(m);
            }
            for (int q = 0; q < kKeys; ++q)
            {
                const bool is_max = (q % 6) >= 3;
                const uint32_t v = in ? key[q] : (is_max ? EmptyMaxKey() : EmptyMinKey());
                const uint32_t r = is_max ? __reduce_max_sync(0xffffffffu, v) : __reduce_min_sync(0xffffffffu, v);
                if (lane == k)
                {
                    my_key[q] = is_max ? max(my_key[q], r) : min(my_key[q], r);
                }
            }
        }
    }
    if (lane < kBuckets && my_cnt > 0)
    {
        atomicAdd(&s_cnt[lane], my_cnt);
        for (int q = 0; q < kKeys; ++q)
        {
            if ((q % 6) >= 3)
            {
                atomicMax(&s_key[lane][q], my_key[q]);
            }
            else
            {
                atomicMin(&s_key[lane][q], my_key[q]);
            }
        }
    }
}

// Whether position i of a node's range holds a primitive on the wrong side of
// the split: before mid and belonging right, or from mid on and belonging left.
__device__ __forceinline__ bool Misplaced(const SahDev& S, int32_t start, int32_t i, int32_t mid, int32_t split,
                                          int32_t axis, float cmin, float extent)
{
    const float4 c = S.cen[S.idx[start + i]];
    const bool left = BucketOf(Axis(c, axis), cmin, extent) <= split;
    return i < mid ? !left : left;
}

// Partition ranks over positions [lo, hi) of a node's range (block-wide):
// every misplaced position before mid goes to scr_l, every one from mid on to
// scr_r, each at its rank among the node's misplaced positions of its side
// (*carry_l / *carry_r: those ranked before lo on entry, before hi on return).
__device__ __forceinline__ void RankRange(const SahDev& S, int32_t start, int32_t lo, int32_t hi, int32_t mid,
                                          int32_t split, int32_t axis, float cmin, float extent, int32_t* carry_l,
                                          int32_t* carry_r, int32_t (*s_scan)[kSahBlock / 32], int32_t* s_total)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int kWarps = kSahBlock / 32;
    for (int32_t tile = lo; tile < hi; tile += kSahTile)
    {
        const int32_t first = tile + tid * kSahPerThread;
        uint32_t move = 0; // bit j: element first + j moves
        int32_t nl = 0, nr = 0;
#pragma unroll
        for (int j = 0; j < kSahPerThread; ++j)
        {
            const int32_t i = first + j;
            if (i < hi && Misplaced(S, start, i, mid, split, axis, cmin, extent))
            {
                move |= 1u << j;
                if (i < mid)
                {
                    ++nl;
                }
                else
                {
                    ++nr;
                }
            }
        }
        // Block-wide exclusive prefix of nl and nr.
        int32_t xl = nl, xr = nr;
        for (int off = 1; off < 32; off <<= 1)
        {
            const int32_t yl = __shfl_up_sync(0xffffffffu, xl, off);
            const int32_t yr = __shfl_up_sync(0xffffffffu, xr, off);
            if (lane >= off)
            {
                xl += yl;
                xr += yr;
            }
        }
        if (lane == 31)
        {
            s_scan[0][warp] = xl;
            s_scan[1][warp] = xr;
        }
        __syncthreads();
        if (tid < 2)
        {
            int32_t run = 0;
            for (int w = 0; w < kWarps; ++w)
            {
                const int32_t v = s_scan[tid][w];
                s_scan[tid][w] = run;
                run += v;
            }
            s_total[tid] = run;
        }
        __syncthreads();
        int32_t rl = *carry_l + s_scan[0][warp] + xl - nl;
        int32_t rr = *carry_r + s_scan[1][warp] + xr - nr;
#pragma unroll
        for (int j = 0; j < kSahPerThread; ++j)
        {
            if (move & (1u << j))
            {
                const int32_t i = first + j;
                if (i < mid)
                {
                    S.scr_l[start + rl++] = i;
                }
                else
                {
                    S.scr_r[start + rr++] = i;
                }
            }
        }
        *carry_l += s_total[0];
        *carry_r += s_total[1];
        __syncthreads(); // s_scan / s_total are rewritten by the next tile
    }
}

// One node per block (nodes of more than 32 primitives).
__global__ void __launch_bounds__(kSahBlock) SahBlockKernel(SahDev S, const int32_t* tasks, int32_t n_tasks,
                                                            int32_t* next_big, int32_t* next_small)
{
    __shared__ int32_t s_cnt[kBuckets];
    __shared__ uint32_t s_key[kBuckets][kKeys];
    __shared__ int32_t s_dec[2];           // split bucket (-1: leaf), left count
    __shared__ uint32_t s_child[2][kKeys]; // children's bounds
    __shared__ int32_t s_scan[2][kSahBlock / 32];
    __shared__ int32_t s_total[2];
    const int tid = threadIdx.x;

    for (int32_t t = blockIdx.x; t < n_tasks; t += gridDim.x)
    {
        const int32_t node = tasks[t];
        const int4 inf = S.info[node];
        const int32_t start = inf.x, count = inf.y;
        float4 bd[4];
        for (int k = 0; k < 4; ++k)
        {
            bd[k] = S.bounds[4 * size_t(node) + k];
        }
        int32_t axis = 0;
        float extent = 0, area = 0;
        if (!SplitAxis(bd, count, &axis, &extent, &area))
        {
            if (tid == 0)
            {
                EmitLeaf(S, node, start, count);
            }
            continue; // uniform across the block
        }
        const float cmin = Axis(bd[2], axis);

        // Buckets: counts and the min / max keys of the boxes and centres in each.
        if (tid < kBuckets)
        {
            s_cnt[tid] = 0;
            for (int k = 0; k < kKeys; ++k)
            {
                s_key[tid][k] = (k % 6) >= 3 ? EmptyMaxKey() : EmptyMinKey();
            }
        }
        __syncthreads();
        BinRange(S, start, 0, count, axis, cmin, extent, s_cnt, s_key);
        __syncthreads();
        if (tid == 0)
        {
            int32_t mid = 0;
            const int32_t split = ChooseSplit(s_cnt, s_key, count, area, &mid, s_child[0], s_child[1]);
            s_dec[0] = split;
            s_dec[1] = mid;
        }
        __syncthreads();
        const int32_t split = s_dec[0], mid = s_dec[1];
        if (split < 0)
        {
            if (tid == 0)
            {
                EmitLeaf(S, node, start, count);
            }
            __syncthreads();
            continue;
        }

        // Partition: positions before mid whose primitive belongs right (in
        // order) pair with positions from mid on whose primitive belongs
        // left (in reverse order); each pair swaps.
        int32_t carry_l = 0, carry_r = 0;
        RankRange(S, start, 0, count, mid, split, axis, cmin, extent, &carry_l, &carry_r, s_scan, s_total);
        // carry_l == carry_r: the pairs. The k-th from the left meets the
        // k-th from the right.
        const int32_t pairs = carry_l;
        for (int32_t k = tid; k < pairs; k += kSahBlock)
        {
            const int32_t a = start + S.scr_l[start + k];
            const int32_t b = start + S.scr_r[start + pairs - 1 - k];
            const int32_t pa = S.idx[a], pb = S.idx[b];
            S.idx[a] = pb;
            S.idx[b] = pa;
        }
        if (tid == 0)
        {
            const int32_t id = EmitChildren(S, node, start, count, mid, axis, next_big, next_small);
            StoreBounds(S.bounds + 4 * size_t(id), s_child[0]);
            StoreBounds(S.bounds + 4 * size_t(id + 1), s_child[1]);
        }
        __syncthreads(); // shared state is reused by the next node
    }
}

// Levels with few large nodes (the top of the tree, where one block per node
// leaves most SMs idle): each node is spread over up to kWideMaxChunks blocks,
// each taking a contiguous chunk of the node's range. The bins merge into the
// node's global buckets by the same commutative atomics the block kernel's
// warps use, the decision is ChooseSplit on them, and the partition ranks are
// each chunk's ranks plus the misplaced counts of the chunks before it, so
// the node comes out exactly as the block kernel makes it.
constexpr int kWideMaxTasks = 256;
constexpr int kWideMaxChunks = 1024;

struct SahWide
{
    int32_t* cnt;  // [task][bucket]
    uint32_t* key; // [task][bucket][kKeys]
    int4* dec;     // [task]: split bucket (-1: leaf), left count, axis
    float2* geo;   // [task]: centre min and extent along the axis
    int32_t* nl;   // [task][chunk]: misplaced positions before mid; exclusive offsets after the scan
    int32_t* nr;   // [task][chunk]: misplaced positions from mid on; likewise
    int32_t* pairs; // [task]: swaps
};

// The range [lo, hi) of the node's count that chunk b of n takes.
__device__ __forceinline__ void ChunkOf(int32_t count, int32_t b, int32_t n, int32_t* lo, int32_t* hi)
{
    const int32_t chunk = (count + n - 1) / n;
    *lo = min(count, b * chunk);
    *hi = min(count, *lo + chunk);
}

__global__ void SahWideInitKernel(SahWide W)
{
    const int32_t t = blockIdx.x;
    for (int i = threadIdx.x; i < kBuckets * kKeys; i += blockDim.x)
    {
        W.key[size_t(t) * kBuckets * kKeys + i] = ((i % kKeys) % 6) >= 3 ? EmptyMaxKey() : EmptyMinKey();
    }
    for (int i = threadIdx.x; i < kBuckets; i += blockDim.x)
    {
        W.cnt[t * kBuckets + i] = 0;
    }
}

__global__ void __launch_bounds__(kSahBlock) SahWideBinKernel(SahDev S, SahWide W, const int32_t* tasks)
{
    __shared__ int32_t s_cnt[kBuckets];
    __shared__ uint32_t s_key[kBuckets][kKeys];
    const int32_t t = blockIdx.y, node = tasks[t];
    const int4 inf = S.info[node];
    const int32_t start = inf.x, count = inf.y;
    float4 bd[4];
    for (int k = 0; k < 4; ++k)
    {
        bd[k] = S.bounds[4 * size_t(node) + k];
    }
    int32_t axis = 0, lo = 0, hi = 0;
    float extent = 0, area = 0;
    ChunkOf(count, blockIdx.x, gridDim.x, &lo, &hi);
    if (!SplitAxis(bd, count, &axis, &extent, &area) || lo >= hi)
    {
        return; // a leaf (the decide kernel emits it) or an empty chunk
    }
    const int tid = threadIdx.x;
    if (tid < kBuckets)
    {
        s_cnt[tid] = 0;
        for (int k = 0; k < kKeys; ++k)
        {
            s_key[tid][k] = (k % 6) >= 3 ? EmptyMaxKey() : EmptyMinKey();
        }
    }
    __syncthreads();
    BinRange(S, start, lo, hi, axis, Axis(bd[2], axis), extent, s_cnt, s_key);
    __syncthreads();
    if (tid < kBuckets && s_cnt[tid] > 0)
    {
        atomicAdd(&W.cnt[t * kBuckets + tid], s_cnt[tid]);
        uint32_t* k = W.key + (size_t(t) * kBuckets + tid) * kKeys;
        for (int q = 0; q < kKeys; ++q)
        {
            if ((q % 6) >= 3)
            {
                atomicMax(&k[q], s_key[tid][q]);
            }
            else
            {
                atomicMin(&k[q], s_key[tid][q]);
            }
        }
    }
}

// One thread per node: the leaf tests and ChooseSplit, then the leaf or the
// two children (their ranges and bounds are known before the partition).
__global__ void SahWideDecideKernel(SahDev S, SahWide W, const int32_t* tasks, int32_t n_tasks, int32_t* next_big,
                                    int32_t* next_small)
{
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks)
    {
        return;
    }
    const int32_t node = tasks[t];
    const int4 inf = S.info[node];
    const int32_t start = inf.x, count = inf.y;
    float4 bd[4];
    for (int k = 0; k < 4; ++k)
    {
        bd[k] = S.bounds[4 * size_t(node) + k];
    }
    int32_t axis = 0, mid = 0;
    float extent = 0, area = 0;
    int32_t split = -1;
    uint32_t lk[kKeys], rk[kKeys];
    if (SplitAxis(bd, count, &axis, &extent, &area))
    {
        split = ChooseSplit(W.cnt + t * kBuckets,
                            reinterpret_cast<const uint32_t(*)[kKeys]>(W.key + size_t(t) * kBuckets * kKeys), count,
                            area, &mid, lk, rk);
    }
    W.dec[t] = make_int4(split, mid, axis, 0);
    W.geo[t] = make_float2(Axis(bd[2], axis), extent);
    if (split < 0)
    {
        EmitLeaf(S, node, start, count);
        return;
    }
    const int32_t id = EmitChildren(S, node, start, count, mid, axis, next_big, next_small);
    StoreBounds(S.bounds + 4 * size_t(id), lk);
    StoreBounds(S.bounds + 4 * size_t(id + 1), rk);
}

__global__ void __launch_bounds__(kSahBlock) SahWideCountKernel(SahDev S, SahWide W, const int32_t* tasks)
{
    __shared__ int32_t s_n[2];
    const int32_t t = blockIdx.y, node = tasks[t];
    const int4 dec = W.dec[t];
    const int32_t slot = t * kWideMaxChunks + blockIdx.x;
    if (dec.x < 0)
    {
        return;
    }
    const int4 inf = S.info[node];
    const int32_t start = inf.x, count = inf.y;
    const float2 geo = W.geo[t];
    int32_t lo = 0, hi = 0;
    ChunkOf(count, blockIdx.x, gridDim.x, &lo, &hi);
    if (threadIdx.x < 2)
    {
        s_n[threadIdx.x] = 0;
    }
    __syncthreads();
    int32_t nl = 0, nr = 0;
    for (int32_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
    {
        if (Misplaced(S, start, i, dec.y, dec.x, dec.z, geo.x, geo.y))
        {
            if (i < dec.y)
            {
                ++nl;
            }
            else
            {
                ++nr;
            }
        }
    }
    nl = __reduce_add_sync(0xffffffffu, nl);
    nr = __reduce_add_sync(0xffffffffu, nr);
    if ((threadIdx.x & 31) == 0)
    {
        atomicAdd(&s_n[0], nl);
        atomicAdd(&s_n[1], nr);
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        W.nl[slot] = s_n[0];
        W.nr[slot] = s_n[1];
    }
}

// One thread per node: the chunks' counts become exclusive offsets.
__global__ void SahWideOffsetsKernel(SahWide W, int32_t n_tasks, int32_t n_chunks)
{
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks || W.dec[t].x < 0)
    {
        return;
    }
    int32_t* nl = W.nl + t * kWideMaxChunks;
    int32_t* nr = W.nr + t * kWideMaxChunks;
    int32_t rl = 0, rr = 0;
    for (int32_t b = 0; b < n_chunks; ++b)
    {
        const int32_t vl = nl[b], vr = nr[b];
        nl[b] = rl;
        nr[b] = rr;
        rl += vl;
        rr += vr;
    }
    W.pairs[t] = rl; // == rr
}

__global__ void __launch_bounds__(kSahBlock) SahWideRankKernel(SahDev S, SahWide W, const int32_t* tasks)
{
    __shared__ int32_t s_scan[2][kSahBlock / 32];
    __shared__ int32_t s_total[2];
    const int32_t t = blockIdx.y, node = tasks[t];
    const int4 dec = W.dec[t];
    if (dec.x < 0)
    {
        return;
    }
    const int4 inf = S.info[node];
    const int32_t start = inf.x, count = inf.y;
    const float2 geo = W.geo[t];
    int32_t lo = 0, hi = 0;
    ChunkOf(count, blockIdx.x, gridDim.x, &lo, &hi);
    int32_t carry_l = W.nl[t * kWideMaxChunks + blockIdx.x], carry_r = W.nr[t * kWideMaxChunks + blockIdx.x];
    RankRange(S, start, lo, hi, dec.y, dec.x, dec.z, geo.x, geo.y, &carry_l, &carry_r, s_scan, s_total);
}

__global__ void __launch_bounds__(kSahBlock) SahWideSwapKernel(SahDev S, SahWide W, const int32_t* tasks)
{
    const int32_t t = blockIdx.y, node = tasks[t];
    if (W.dec[t].x < 0)
    {
        return;
    }
    const int32_t start = S.info[node].x, pairs = W.pairs[t];
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < pairs; k += gridDim.x * blockDim.x)
    {
        const int32_t a = start + S.scr_l[start + k];
        const int32_t b = start + S.scr_r[start + pairs - 1 - k];
        const int32_t pa = S.idx[a], pb = S.idx[b];
        S.idx[a] = pb;
        S.idx[b] = pa;
    }
}

// Position of the n-th (0-based, from the least significant end) set bit of m.
__device__ __forceinline__ int32_t NthSetBit(unsigned m, int32_t n)
{
    for (int32_t c = 0; c < n; ++c)
    {
        m &= m - 1u;
    }
    return __ffs(m) - 1;
}

// One node per warp (nodes of at most 32 primitives): lane i holds the i-th
// primitive of the node's range.
__global__ void __launch_bounds__(kSahWarpBlock) SahWarpKernel(SahDev S, const int32_t* tasks, int32_t n_tasks,
                                                               int32_t* next_big, int32_t* next_small)
{
    constexpr int kWarpsPerBlock = kSahWarpBlock / 32;
    __shared__ int32_t s_cnt[kWarpsPerBlock][kBuckets];
    __shared__ uint32_t s_key[kWarpsPerBlock][kBuckets][kKeys];
    __shared__ uint32_t s_child[kWarpsPerBlock][2][kKeys];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int32_t warps = gridDim.x * kWarpsPerBlock;
    for (int32_t t = blockIdx.x * (kSahWarpBlock / 32) + (threadIdx.x >> 5); t < n_tasks; t += warps)
    {
        const int32_t node = tasks[t];
        const int4 inf = S.info[node];
        const int32_t start = inf.x, count = inf.y;
        float4 bd[4];
        for (int k = 0; k < 4; ++k)
        {
            bd[k] = S.bounds[4 * size_t(node) + k];
        }
        int32_t axis = 0;
        float extent = 0, area = 0;
        if (!SplitAxis(bd, count, &axis, &extent, &area))
        {
            if (lane == 0)
            {
                EmitLeaf(S, node, start, count);
            }
            continue;
        }
        const bool have = lane < count;
        const int32_t p = have ? S.idx[start + lane] : -1;
        float4 c = make_float4(0, 0, 0, 0), lo = c, hi = c;
        if (have)
        {
            c = S.cen[p];
            lo = S.box[2 * size_t(p)];
            hi = S.box[2 * size_t(p) + 1];
        }
        if (count == 2)
        {
            // std::nth_element(begin, begin + 1, end) on two elements is an
            // insertion sort: they swap only if the second is strictly less.
            const float c0 = __shfl_sync(0xffffffffu, Axis(c, axis), 0);
            const float c1 = __shfl_sync(0xffffffffu, Axis(c, axis), 1);
            const bool swap = c1 < c0;
            const int32_t p0 = __shfl_sync(0xffffffffu, p, 0), p1 = __shfl_sync(0xffffffffu, p, 1);
            const int32_t first = swap ? p1 : p0, second = swap ? p0 : p1;
            if (lane == 0)
            {
                if (swap)
                {
                    S.idx[start] = first;
                    S.idx[start + 1] = second;
                }
                const int32_t id = EmitChildren(S, node, start, 2, 1, axis, next_big, next_small);
                StorePrimBounds(S, S.bounds + 4 * size_t(id), first);
                StorePrimBounds(S, S.bounds + 4 * size_t(id + 1), second);
            }
            continue;
        }
        const int32_t b = have ? BucketOf(Axis(c, axis), Axis(bd[2], axis), extent) : -1;
        uint32_t key[kKeys];
        key[0] = FloatKey(lo.x), key[1] = FloatKey(lo.y), key[2] = FloatKey(lo.z);
        key[3] = FloatKey(hi.x), key[4] = FloatKey(hi.y), key[5] = FloatKey(hi.z);
        key[6] = FloatKey(c.x), key[7] = FloatKey(c.y), key[8] = FloatKey(c.z);
        key[9] = key[6], key[10] = key[7], key[11] = key[8];
        for (int32_t k = 0; k < kBuckets; ++k)
        {
            const unsigned m = __ballot_sync(0xffffffffu, b == k);
            if (lane == 0)
            {
                s_cnt[wid][k] = __popc(m);
            }
            for (int q = 0; q < kKeys; ++q)
            {
                const bool is_max = (q % 6) >= 3;
                const uint32_t none = is_max ? EmptyMaxKey() : EmptyMinKey();
                const uint32_t v = b == k ? key[q] : none;
                const uint32_t r =
                    m == 0 ? none : (is_max ? __reduce_max_sync(0xffffffffu, v) : __reduce_min_sync(0xffffffffu, v));
                if (lane == q)
                {
                    s_key[wid][k][q] = r;
                }
            }
        }
        __syncwarp();
        int32_t split = -1, mid = 0;
        if (lane == 0)
        {
            split = ChooseSplit(s_cnt[wid], s_key[wid], count, area, &mid, s_child[wid][0], s_child[wid][1]);
        }
        split = __shfl_sync(0xffffffffu, split, 0);
        mid = __shfl_sync(0xffffffffu, mid, 0);
        if (split < 0)
        {
            if (lane == 0)
            {
                EmitLeaf(S, node, start, count);
            }
            __syncwarp();
            continue;
        }
        // The k-th element from the left among those before mid that belong
        // right swaps with the k-th from the right among those from mid on
        // that belong left.
        const bool left = have && b <= split;
        const unsigned fl = __ballot_sync(0xffffffffu, have && lane < mid && !left);
        const unsigned fr = __ballot_sync(0xffffffffu, have && lane >= mid && left);
        int32_t partner = -1;
        if ((fl >> lane) & 1u)
        {
            const int32_t k = __popc(fl & ((1u << lane) - 1u));
            partner = NthSetBit(fr, __popc(fr) - 1 - k);
        }
        else if ((fr >> lane) & 1u)
        {
            const int32_t k = __popc(fr & ~((2u << lane) - 1u)); // rank from the right
            partner = NthSetBit(fl, k);
        }
        const int32_t q = __shfl_sync(0xffffffffu, p, partner < 0 ? lane : partner);
        if (partner >= 0)
        {
            S.idx[start + lane] = q;
        }
        if (lane == 0)
        {
            const int32_t id = EmitChildren(S, node, start, count, mid, axis, next_big, next_small);
            StoreBounds(S.bounds + 4 * size_t(id), s_child[wid][0]);
            StoreBounds(S.bounds + 4 * size_t(id + 1), s_child[wid][1]);
        }
        __syncwarp(); // this warp's shared state is reused by its next node
    }
}

// Primitive boxes and centres, the root's bounds (keys, atomically), and the
// identity order.
__global__ void SahPrimsKernel(const int2* prim_shape, const int32_t* tri, const float* pos, const bbg_sphere* spheres,
                               int32_t n, float4* box, float4* cen, int32_t* idx, uint32_t* root_keys)
{
    uint32_t k[kKeys];
    for (int q = 0; q < kKeys; ++q)
    {
        k[q] = (q % 6) >= 3 ? EmptyMaxKey() : EmptyMinKey();
    }
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        float3 mn, mx;
        PrimBox(prim_shape, tri, pos, spheres, i, &mn, &mx);
        box[2 * size_t(i)] = make_float4(mn.x, mn.y, mn.z, 0);
        box[2 * size_t(i) + 1] = make_float4(mx.x, mx.y, mx.z, 0);
        // AABB::GetCenter: (min + max) * 0.5f.
        const float4 c = make_float4((mn.x + mx.x) * 0.5f, (mn.y + mx.y) * 0.5f, (mn.z + mx.z) * 0.5f, 0);
        cen[i] = c;
        idx[i] = i;
        const uint32_t v[kKeys] = { FloatKey(mn.x), FloatKey(mn.y), FloatKey(mn.z), FloatKey(mx.x),
                                    FloatKey(mx.y), FloatKey(mx.z), FloatKey(c.x),  FloatKey(c.y),
                                    FloatKey(c.z),  FloatKey(c.x),  FloatKey(c.y),  FloatKey(c.z) };
        for (int q = 0; q < kKeys; ++q)
        {
            k[q] = (q % 6) >= 3 ? max(k[q], v[q]) : min(k[q], v[q]);
        }
    }
    for (int q = 0; q < kKeys; ++q)
    {
        const uint32_t r = (q % 6) >= 3 ? __reduce_max_sync(0xffffffffu, k[q]) : __reduce_min_sync(0xffffffffu, k[q]);
        if ((threadIdx.x & 31) == 0)
        {
            if ((q % 6) >= 3)
            {
                atomicMax(&root_keys[q], r);
            }
            else
            {
                atomicMin(&root_keys[q], r);
            }
        }
    }
}

__global__ void SahRootKernel(SahDev S, const uint32_t* root_keys, int32_t n)
{
    StoreBounds(S.bounds, root_keys);
    S.info[0] = make_int4(0, n, -1, 0);
    S.path[0] = make_int2(1, 0);
}

// Depth-first index of a node from its path and the leaves left of it.
__device__ __forceinline__ int32_t PreOrder(const SahDev& S, const uint32_t* leaves_before, int32_t node)
{
    const int2 pth = S.path[node];
    return pth.x - 1 + 2 * int32_t(leaves_before[S.info[node].x]) - pth.y;
}

// Writes every node at its depth-first index in the reference layout
// (LinearBVHNode), its reference in the child-box layout (interior: its index
// among interior nodes in depth-first order; leaf: ~its index among leaves),
// and each leaf's (first slot, count).
__global__ void SahFlattenKernel(SahDev S, const uint32_t* leaves_before, int32_t n_nodes, int32_t n_leaves,
                                 bbg_bvh_node* out, int32_t* ref, int2* leaves, int32_t* bad)
{
    for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n_nodes; v += gridDim.x * blockDim.x)
    {
        const int4 inf = S.info[v];
        const int32_t pre = PreOrder(S, leaves_before, v);
        const int32_t lb = int32_t(leaves_before[inf.x]);
        const int32_t right = inf.z < 0 ? 0 : PreOrder(S, leaves_before, inf.z + 1);
        // Every index written or stored stays in range (a consistency check
        // of the build; the host reports a failure).
        if (pre < 0 || pre >= n_nodes || lb < 0 || (inf.z < 0 && lb >= n_leaves) ||
            (inf.z >= 0 && (right <= pre + 1 || right >= n_nodes || pre - lb < 0 || pre - lb >= n_nodes - n_leaves)))
        {
            *bad = 1;
            continue;
        }
        const float4 lo = S.bounds[4 * size_t(v)], hi = S.bounds[4 * size_t(v) + 1];
        bbg_bvh_node nd;
        nd.bmin[0] = lo.x, nd.bmin[1] = lo.y, nd.bmin[2] = lo.z;
        nd.bmax[0] = hi.x, nd.bmax[1] = hi.y, nd.bmax[2] = hi.z;
        nd.pad = 0;
        if (inf.z < 0)
        {
            nd.offset = inf.x;
            nd.count = uint16_t(inf.y);
            nd.axis = 0;
            ref[pre] = ~lb;
            leaves[lb] = make_int2(inf.x, inf.y);
        }
        else
        {
            nd.offset = right;
            nd.count = 0;
            nd.axis = uint8_t(inf.w);
            ref[pre] = pre - lb;
        }
        out[pre] = nd;
    }
}

// Slot records in leaf order (slot j holds primitive idx[j]).
// As SahPrimsKernel, over given boxes (references: box[2 r], box[2 r + 1]
// are reference r's min and max corners).
__global__ void SahRefsKernel(const float4* ref_box, int32_t n, float4* box, float4* cen, int32_t* idx,
                              uint32_t* root_keys)
{
    uint32_t k[kKeys];
    for (int q = 0; q < kKeys; ++q)
    {
        k[q] = (q % 6) >= 3 ? EmptyMaxKey() : EmptyMinKey();
    }
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const float4 lo = ref_box[2 * size_t(i)], hi = ref_box[2 * size_t(i) + 1];
        box[2 * size_t(i)] = make_float4(lo.x, lo.y, lo.z, 0);
        box[2 * size_t(i) + 1] = make_float4(hi.x, hi.y, hi.z, 0);
        const float4 c = make_float4((lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f, 0);
        cen[i] = c;
        idx[i] = i;
        const uint32_t v[kKeys] = { FloatKey(lo.x), FloatKey(lo.y), FloatKey(lo.z), FloatKey(hi.x),
                                    FloatKey(hi.y), FloatKey(hi.z), FloatKey(c.x),  FloatKey(c.y),
                                    FloatKey(c.z),  FloatKey(c.x),  FloatKey(c.y),  FloatKey(c.z) };
        for (int q = 0; q < kKeys; ++q)
        {
            k[q] = (q % 6) >= 3 ? max(k[q], v[q]) : min(k[q], v[q]);
        }
    }
    for (int q = 0; q < kKeys; ++q)
    {
        const uint32_t r = (q % 6) >= 3 ? __reduce_max_sync(0xffffffffu, k[q]) : __reduce_min_sync(0xffffffffu, k[q]);
        if ((threadIdx.x & 31) == 0)
        {
            if ((q % 6) >= 3)
            {
                atomicMax(&root_keys[q], r);
            }
            else
            {
                atomicMin(&root_keys[q], r);
            }
        }
    }
}

// Primitive of each slot: the build's item order, through the reference map
// when the build ran over references.
__global__ void SahSlotPrimsKernel(const int32_t* idx, const int32_t* ref_prim, int32_t n, int32_t* slot_prims)
{
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        slot_prims[j] = ref_prim ? ref_prim[idx[j]] : idx[j];
    }
}

__global__ void SahSlotsKernel(const int32_t* slot_prims, const int2* prim_shape, const int32_t* tri, const float* pos,
                               const bbg_sphere* spheres, int32_t n, float4* slots)
{
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        const int32_t prim = slot_prims[j];
        const int2 ps = prim_shape[prim];
        float4* r = slots + 3 * size_t(j);
        if (ps.x == BBG_PRIM_TRIANGLE)
        {
            const int32_t* v = tri + 3 * size_t(ps.y);
            const float* p0 = pos + 3 * size_t(v[0]);
            const float* p1 = pos + 3 * size_t(v[1]);
            const float* p2 = pos + 3 * size_t(v[2]);
            // Edges e1 = p1 - p0, e2 = p2 - p0 as Triangle::Intersect computes them.
            r[0] = make_float4(p0[0], p0[1], p0[2], __uint_as_float(uint32_t(prim)));
            r[1] = make_float4(p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2], 0.0f);
            r[2] = make_float4(p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2], 0.0f);
        }
        else
        {
            const bbg_sphere& sp = spheres[ps.y];
            r[0] = make_float4(sp.p[0], sp.p[1], sp.p[2], __uint_as_float(uint32_t(prim) | kSphereBit));
            r[1] = make_float4(sp.q[0], sp.q[1], sp.q[2], sp.q[3]);
            r[2] = make_float4(sp.s[0], sp.s[1], sp.s[2], sp.radius);
        }
    }
}

// The binary child-box layout: one 64-byte record per interior node with
// both children's boxes and references.
__global__ void SahChildBoxKernel(const bbg_bvh_node* nd, const int32_t* ref, int32_t n_nodes, float4* wide)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += gridDim.x * blockDim.x)
    {
        if (nd[i].count > 0)
        {
            continue;
        }
        const bbg_bvh_node& c0 = nd[i + 1];
        const bbg_bvh_node& c1 = nd[nd[i].offset];
        float4* w = wide + 4 * size_t(ref[i]);
        w[0] = make_float4(c0.bmin[0], c0.bmin[1], c0.bmin[2], c0.bmax[0]);
        w[1] = make_float4(c0.bmax[1], c0.bmax[2], c1.bmin[0], c1.bmin[1]);
        w[2] = make_float4(c1.bmin[2], c1.bmax[0], c1.bmax[1], c1.bmax[2]);
        w[3] = make_float4(__int_as_float(ref[i + 1]), __int_as_float(ref[nd[i].offset]), 0.0f, 0.0f);
    }
}

// The surface-area plan of the 8-wide collapse (Wide8PlanNode), bottom up as
// the host computes it: each leaf walks toward the root, and at every node the
// second child to arrive (an atomic count) computes the node's entries from
// both children's and walks on; the first one stops there. No thread waits.
// The children's entries are written by other threads: the writer fences
// before its count, the reader fences after its count and reads through L2.
__global__ void SahPlanParentKernel(const bbg_bvh_node* nd, int32_t n, int32_t* parent)
{
    for (int32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x)
    {
        if (b == 0)
        {
            parent[0] = -1;
        }
        if (nd[b].count == 0)
        {
            parent[b + 1] = b;
            parent[nd[b].offset] = b;
        }
    }
}

__global__ void SahPlanKernel(const bbg_bvh_node* nd, int32_t n, const int32_t* parent, int32_t* arrivals,
                              float* cost, uint8_t* split)
{
    for (int32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x)
    {
        if (nd[b].count == 0)
        {
            continue; // walks start at the leaves (whose entries stay 0)
        }
        for (int32_t p = parent[b]; p >= 0; p = parent[p])
        {
            __threadfence();
            if (atomicAdd(arrivals + p, 1) == 0)
            {
                break; // the other child's walk finishes p
            }
            __threadfence();
            const bbg_bvh_node x = nd[p];
            float cl[8], cr[8], cp[8];
            uint8_t sp[8];
            for (int i = 0; i < 8; ++i)
            {
                cl[i] = __ldcg(cost + 8 * size_t(p + 1) + i);
                cr[i] = __ldcg(cost + 8 * size_t(x.offset) + i);
            }
            Wide8PlanNode(x, cl, cr, cp, sp);
            for (int i = 0; i < 8; ++i)
            {
                __stcg(cost + 8 * size_t(p) + i, cp[i]);
                split[8 * size_t(p) + i] = sp[i];
            }
        }
    }
}

// The 8-wide collapse of one level, as the host collapses a reference tree
// (accel.cu, BuildWide8): wide node w stands for binary node w2b[w] and holds
// the children the plan gives it. Pass 0 counts each wide node's interior
// children (and flags leaves the layout cannot encode); pass 1, with the
// exclusive prefix of those counts, numbers them breadth first in child order
// and writes the node.
__device__ __forceinline__ int Collapse8(const bbg_bvh_node* nd, const uint8_t* split, int32_t b, Child8 cs[8])
{
    int32_t bs[8];
    const int n = Wide8Gather(nd, split, b, bs);
    for (int c = 0; c < n; ++c)
    {
        for (int a = 0; a < 3; ++a)
        {
            cs[c].lo[a] = nd[bs[c]].bmin[a];
            cs[c].hi[a] = nd[bs[c]].bmax[a];
        }
        cs[c].bnode = bs[c];
    }
    return n;
}

__global__ void SahWide8CountKernel(const bbg_bvh_node* nd, const uint8_t* split, const int32_t* w2b, int32_t begin,
                                    int32_t end, int32_t* inner, int32_t* bad)
{
    for (int32_t w = begin + blockIdx.x * blockDim.x + threadIdx.x; w < end; w += gridDim.x * blockDim.x)
    {
        Child8 cs[8];
        const int n = Collapse8(nd, split, w2b[w], cs);
        int32_t k = 0;
        for (int c = 0; c < n; ++c)
        {
            const bbg_bvh_node& x = nd[cs[c].bnode];
            if (x.count == 0)
            {
                ++k;
            }
            else if (x.count >= (1 << kWide8LeafCountBits) || x.offset >= (1 << (31 - kWide8LeafCountBits)))
            {
                *bad = 1;
            }
        }
        inner[w - begin] = k;
    }
}

__global__ void SahWide8WriteKernel(const bbg_bvh_node* nd, const uint8_t* split, int32_t* w2b, int32_t begin,
                                    int32_t end, const int32_t* offsets, float4* wide8)
{
    for (int32_t w = begin + blockIdx.x * blockDim.x + threadIdx.x; w < end; w += gridDim.x * blockDim.x)
    {
        Child8 cs[8];
        const int n = Collapse8(nd, split, w2b[w], cs);
        float plo[3], phi[3];
        Wide8Union(cs, n, plo, phi);
        int32_t slot_of[8];
        AssignSlots8(cs, n, plo, phi, slot_of);
        int32_t refs[8];
        for (int k = 0; k < 8; ++k)
        {
            refs[k] = ~0; // empty: a leaf of no primitives
        }
        int32_t next = end + offsets[w - begin];
        for (int c = 0; c < n; ++c)
        {
            const bbg_bvh_node& x = nd[cs[c].bnode];
            if (x.count > 0)
            {
                refs[slot_of[c]] = Wide8LeafRef(x.offset, int32_t(x.count));
            }
            else
            {
                refs[slot_of[c]] = next;
                w2b[next] = cs[c].bnode;
                ++next;
            }
        }
        QuantizeNode8(cs, n, slot_of, refs, wide8 + 6 * size_t(w));
    }
}

// The 8-wide collapse of the depth-first node array on the device, level by
// level (the host reads each level's size back). Leaves the layout unbuilt if
// a leaf cannot be encoded or the tree exceeds the layout's limits, as the
// host collapse does.
bbg_status SahWide8(bbg_accel* a, const bbg_bvh_node* nd, int32_t n_nodes, int sms)
{
    // Every wide node stands for a distinct interior binary node (or the
    // root leaf), so that many always suffice; the layout encodes at most
    // 2^23 - 1 nodes (the host collapse's limit).
    const int32_t interior = (n_nodes - 1) / 2;
    const int32_t capacity = std::max(interior, 1);
    constexpr int64_t kMaxWide = (int64_t(1) << 23) - 1;
    cudaStream_t st = a->stream;
    DevBuf<int32_t> w2b, inner, offsets, flag, parent, arrivals;
    DevBuf<float> cost;
    DevBuf<uint8_t> split;
    BBG_TRY(parent.alloc(size_t(n_nodes)));
    BBG_TRY(arrivals.alloc(size_t(n_nodes)));
    BBG_TRY(cost.alloc(8 * size_t(n_nodes)));
    BBG_TRY(split.alloc(8 * size_t(n_nodes)));
    BBG_CUDA(cudaMemsetAsync(arrivals.p, 0, sizeof(int32_t) * size_t(n_nodes), st));
    BBG_CUDA(cudaMemsetAsync(cost.p, 0, sizeof(float) * 8 * size_t(n_nodes), st)); // leaves cost 0
    BBG_CUDA(cudaMemsetAsync(split.p, 0, 8 * size_t(n_nodes), st));
    SahPlanParentKernel<<<GridFor(n_nodes, 256, sms), 256, 0, st>>>(nd, n_nodes, parent.p);
    SahPlanKernel<<<GridFor(n_nodes, 256, sms), 256, 0, st>>>(nd, n_nodes, parent.p, arrivals.p, cost.p, split.p);
    BBG_CUDA(cudaGetLastError());
    BBG_TRY(w2b.alloc(size_t(capacity)));
    BBG_TRY(inner.alloc(size_t(capacity) + 1));
    BBG_TRY(offsets.alloc(size_t(capacity) + 1));
    BBG_TRY(flag.alloc(1));
    BBG_TRY(a->wide8.alloc(6 * size_t(capacity)));
    BBG_CUDA(cudaMemsetAsync(w2b.p, 0, sizeof(int32_t), st)); // wide node 0 = binary root 0
    BBG_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int32_t), st));
    size_t scan_bytes = 0;
    BBG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, inner.p, offsets.p, capacity + 1, st));
    DevBuf<uint8_t> scan_tmp;
    BBG_TRY(scan_tmp.alloc(std::max<size_t>(scan_bytes, 1)));
    int32_t begin = 0, end = 1, depth = 0;
    while (begin < end)
    {
        if (++depth > kStackCapacity)
        {
            a->wide8.reset();
            return BBG_OK;
        }
        const int32_t m = end - begin;
        SahWide8CountKernel<<<GridFor(m, 128, sms), 128, 0, st>>>(nd, split.p, w2b.p, begin, end, inner.p, flag.p);
        // offsets[m], the level's total, needs inner[m] = 0.
        BBG_CUDA(cudaMemsetAsync(inner.p + m, 0, sizeof(int32_t), st));
        BBG_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp.p, scan_bytes, inner.p, offsets.p, m + 1, st));
        int32_t state[2] = { 0, 0 };
        BBG_CUDA(cudaMemcpyAsync(&state[0], offsets.p + m, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaMemcpyAsync(&state[1], flag.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaStreamSynchronize(st));
        if (state[1] != 0 || int64_t(end) + state[0] > std::min<int64_t>(capacity, kMaxWide))
        {
            a->wide8.reset();
            return BBG_OK;
        }
        SahWide8WriteKernel<<<GridFor(m, 128, sms), 128, 0, st>>>(nd, split.p, w2b.p, begin, end, offsets.p,
                                                                  a->wide8.p);
        BBG_CUDA(cudaGetLastError());
        begin = end;
        end += state[0];
    }
    a->n_wide8 = end;
    a->root8 = 0;
    a->depth8 = depth;
    a->use_wide8 = true;
    return BBG_OK;
}

} // namespace

bbg_status BuildSahOnDevice(bbg_accel* a, int32_t n, const float4* ref_box, const int32_t* ref_prim)
{
    cudaStream_t st = a->stream;
    const int sms = CurrentSmCount();
    const int64_t max_nodes = 2 * int64_t(n) - 1;
    if (max_nodes >= (int64_t(1) << 31))
    {
        return Fail(BBG_ERR_INVALID_ARG, "device SAH build: %d primitives exceed the node index range", n);
    }

    // Every temporary array of the build in one allocation (carved in
    // 256-byte-aligned pieces), so a build costs one cudaMalloc, not a dozen.
    struct Piece
    {
        void** ptr;
        size_t bytes;
    };
    float4 *box = nullptr, *cen = nullptr, *bounds = nullptr;
    int32_t *idx = nullptr, *scr_l = nullptr, *scr_r = nullptr, *counters = nullptr, *ref = nullptr;
    int32_t* lists[4] = {};
    uint32_t *leaf_at = nullptr, *leaves_before = nullptr, *root_keys = nullptr;
    int4* info = nullptr;
    int2* path = nullptr;
    SahWide W{};
    const size_t un = size_t(n), un1 = size_t(n) + 1, nodes = size_t(max_nodes);
    const Piece pieces[] = {
        { reinterpret_cast<void**>(&box), 2 * un * sizeof(float4) },
        { reinterpret_cast<void**>(&cen), un * sizeof(float4) },
        { reinterpret_cast<void**>(&idx), un * sizeof(int32_t) },
        { reinterpret_cast<void**>(&scr_l), un * sizeof(int32_t) },
        { reinterpret_cast<void**>(&scr_r), un * sizeof(int32_t) },
        { reinterpret_cast<void**>(&leaf_at), un1 * sizeof(uint32_t) },
        { reinterpret_cast<void**>(&leaves_before), un1 * sizeof(uint32_t) },
        { reinterpret_cast<void**>(&bounds), 4 * nodes * sizeof(float4) },
        { reinterpret_cast<void**>(&info), nodes * sizeof(int4) },
        { reinterpret_cast<void**>(&path), nodes * sizeof(int2) },
        { reinterpret_cast<void**>(&ref), nodes * sizeof(int32_t) },
        { reinterpret_cast<void**>(&counters), 4 * sizeof(int32_t) },
        { reinterpret_cast<void**>(&root_keys), kKeys * sizeof(uint32_t) },
        { reinterpret_cast<void**>(&lists[0]), un * sizeof(int32_t) },
        { reinterpret_cast<void**>(&lists[1]), un * sizeof(int32_t) },
        { reinterpret_cast<void**>(&lists[2]), un * sizeof(int32_t) },
        { reinterpret_cast<void**>(&lists[3]), un * sizeof(int32_t) },
        { reinterpret_cast<void**>(&W.cnt), size_t(kWideMaxTasks) * kBuckets * sizeof(int32_t) },
        { reinterpret_cast<void**>(&W.key), size_t(kWideMaxTasks) * kBuckets * kKeys * sizeof(uint32_t) },
        { reinterpret_cast<void**>(&W.dec), size_t(kWideMaxTasks) * sizeof(int4) },
        { reinterpret_cast<void**>(&W.geo), size_t(kWideMaxTasks) * sizeof(float2) },
        { reinterpret_cast<void**>(&W.nl), size_t(kWideMaxTasks) * kWideMaxChunks * sizeof(int32_t) },
        { reinterpret_cast<void**>(&W.nr), size_t(kWideMaxTasks) * kWideMaxChunks * sizeof(int32_t) },
        { reinterpret_cast<void**>(&W.pairs), size_t(kWideMaxTasks) * sizeof(int32_t) },
    };
    size_t total = 0;
    for (const Piece& pc : pieces)
    {
        total += (pc.bytes + 255) / 256 * 256;
    }
    DevBuf<uint8_t> arena;
    BBG_TRY(arena.alloc(total));
    {
        size_t at = 0;
        for (const Piece& pc : pieces)
        {
            *pc.ptr = arena.p + at;
            at += (pc.bytes + 255) / 256 * 256;
        }
    }
    BBG_CUDA(cudaMemsetAsync(leaf_at, 0, sizeof(uint32_t) * (size_t(n) + 1), st));
    uint32_t init_keys[kKeys];
    for (int q = 0; q < kKeys; ++q)
    {
        init_keys[q] = (q % 6) >= 3 ? EmptyMaxKey() : EmptyMinKey();
    }
    BBG_CUDA(cudaMemcpyAsync(root_keys, init_keys, sizeof(init_keys), cudaMemcpyHostToDevice, st));
    if (ref_box)
    {
        SahRefsKernel<<<GridFor(n, 256, sms), 256, 0, st>>>(ref_box, n, box, cen, idx, root_keys);
    }
    else
    {
        SahPrimsKernel<<<GridFor(n, 256, sms), 256, 0, st>>>(a->prim_shape.p, a->tri_indices.p, a->positions.p,
                                                             a->spheres.p, n, box, cen, idx, root_keys);
    }
    SahDev S{ box, cen, idx, scr_l, scr_r, leaf_at, bounds, info, path, counters };
    SahRootKernel<<<1, 1, 0, st>>>(S, root_keys, n);
    const int32_t init_counters[4] = { 1, 0, 0, 0 };
    BBG_CUDA(cudaMemcpyAsync(counters, init_counters, sizeof(init_counters), cudaMemcpyHostToDevice, st));
    const int32_t root = 0;
    // lists[0] / lists[1]: nodes of more than 32 primitives of this level and
    // the next; lists[2] / lists[3]: the smaller ones.
    int cur = 0;
    int32_t n_big = n > kSahWarpTask ? 1 : 0, n_small = 1 - n_big;
    BBG_CUDA(cudaMemcpyAsync(n_big ? lists[0] : lists[2], &root, sizeof(root), cudaMemcpyHostToDevice, st));
    int depth = 0;
    int32_t state[4] = { 1, 0, 0, 0 };
    while (n_big + n_small > 0)
    {
        if (++depth > kStackCapacity)
        {
            return Fail(BBG_ERR_STACK_OVERFLOW, "tree depth exceeds the traversal stack (%d)", kStackCapacity);
        }
        int32_t* big_cur = lists[cur];
        int32_t* big_next = lists[1 - cur];
        int32_t* small_cur = lists[2 + cur];
        int32_t* small_next = lists[3 - cur];
        BBG_CUDA(cudaMemsetAsync(counters + 1, 0, 2 * sizeof(int32_t), st));
        if (n_big > 0 && n_big <= kWideMaxTasks)
        {
            // Few large nodes: about four blocks per SM over them all.
            const int32_t chunks = std::min(kWideMaxChunks, std::max(1, (4 * sms + n_big - 1) / n_big));
            const dim3 grid{ static_cast<unsigned>(chunks), static_cast<unsigned>(n_big), 1u };
            SahWideInitKernel<<<n_big, 256, 0, st>>>(W);
            SahWideBinKernel<<<grid, kSahBlock, 0, st>>>(S, W, big_cur);
            SahWideDecideKernel<<<(n_big + 63) / 64, 64, 0, st>>>(S, W, big_cur, n_big, big_next, small_next);
            SahWideCountKernel<<<grid, kSahBlock, 0, st>>>(S, W, big_cur);
            SahWideOffsetsKernel<<<(n_big + 63) / 64, 64, 0, st>>>(W, n_big, chunks);
            SahWideRankKernel<<<grid, kSahBlock, 0, st>>>(S, W, big_cur);
            SahWideSwapKernel<<<grid, kSahBlock, 0, st>>>(S, W, big_cur);
        }
        else if (n_big > 0)
        {
            SahBlockKernel<<<std::min(n_big, 8 * sms), kSahBlock, 0, st>>>(S, big_cur, n_big, big_next, small_next);
        }
        if (n_small > 0)
        {
            SahWarpKernel<<<GridFor(int64_t(n_small) * 32, kSahWarpBlock, sms), kSahWarpBlock, 0, st>>>(
                S, small_cur, n_small, big_next, small_next);
        }
        BBG_CUDA(cudaMemcpyAsync(state, counters, sizeof(state), cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaStreamSynchronize(st));
        BBG_CUDA(cudaGetLastError());
        n_big = state[1];
        n_small = state[2];
        cur = 1 - cur;
    }
    if (state[3] != 0)
    {
        return Fail(BBG_ERR_BAD_BVH, "a leaf holds more than 65535 primitives (uint16 primitive_count)");
    }
    const int32_t n_nodes = state[0];
    a->max_depth = depth;

    // Leaves left of each position, then every node at its depth-first index.
    size_t scan_bytes = 0;
    BBG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, leaf_at, leaves_before, n + 1, st));
    DevBuf<uint8_t> scan_tmp;
    BBG_TRY(scan_tmp.alloc(std::max<size_t>(scan_bytes, 1)));
    BBG_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp.p, scan_bytes, leaf_at, leaves_before, n + 1, st));
    uint32_t n_leaves = 0;
    BBG_CUDA(cudaMemcpyAsync(&n_leaves, leaves_before + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    BBG_TRY(a->nodes.alloc(2 * size_t(n_nodes)));
    BBG_CUDA(cudaStreamSynchronize(st));
    BBG_TRY(a->leaves.alloc(std::max<size_t>(n_leaves, 1)));
    bbg_bvh_node* nd = reinterpret_cast<bbg_bvh_node*>(a->nodes.p);
    int32_t* bad = counters + 3; // zero: no leaf was too large
    SahFlattenKernel<<<GridFor(n_nodes, 256, sms), 256, 0, st>>>(S, leaves_before, n_nodes, int32_t(n_leaves), nd,
                                                                  ref, a->leaves.p, bad);
    int32_t flat_bad = 0;
    BBG_CUDA(cudaMemcpyAsync(&flat_bad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    BBG_CUDA(cudaStreamSynchronize(st));
    if (flat_bad != 0 || int64_t(n_leaves) > n || int64_t(n_leaves) * 2 - 1 != n_nodes)
    {
        return Fail(BBG_ERR_BAD_BVH, "device SAH build: inconsistent tree (%d nodes, %u leaves)", n_nodes, n_leaves);
    }
    // The primitive of every slot stays on the device (slot records, export).
    BBG_TRY(a->slot_prims.alloc(size_t(n)));
    SahSlotPrimsKernel<<<GridFor(n, 256, sms), 256, 0, st>>>(idx, ref_prim, n, a->slot_prims.p);
    BBG_TRY(a->slots.alloc(3 * size_t(n)));
    SahSlotsKernel<<<GridFor(n, 256, sms), 256, 0, st>>>(a->slot_prims.p, a->prim_shape.p, a->tri_indices.p,
                                                         a->positions.p, a->spheres.p, n, a->slots.p);
    const int32_t n_interior = n_nodes - int32_t(n_leaves);
    BBG_TRY(a->wide.alloc(4 * size_t(std::max(n_interior, 1))));
    SahChildBoxKernel<<<GridFor(n_nodes, 256, sms), 256, 0, st>>>(nd, ref, n_nodes, a->wide.p);
    BBG_CUDA(cudaGetLastError());
    int32_t root_ref = 0;
    BBG_CUDA(cudaMemcpyAsync(&root_ref, ref, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    bbg_bvh_node root_node;
    BBG_CUDA(cudaMemcpyAsync(&root_node, nd, sizeof(root_node), cudaMemcpyDeviceToHost, st));
    BBG_CUDA(cudaStreamSynchronize(st));
    a->root = root_ref;
    a->n_nodes = n_nodes;
    a->n_slots = n;
    std::memcpy(a->bounds, root_node.bmin, 3 * sizeof(float));
    std::memcpy(a->bounds + 3, root_node.bmax, 3 * sizeof(float));
    BBG_TRY(SahWide8(a, nd, n_nodes, sms));
    BBG_CUDA(cudaStreamSynchronize(st));
    return BBG_OK;
}

} // namespace bbg
