// References for a tree over split primitives, made on the device: early
// split clipping (Ernst & Greiner, "Early Split Clipping for Bounding Volume
// Hierarchies", IEEE RT 2007) as the host splitter does it (host_build.cpp,
// SplitReferences), with its greedy order relaxed to rounds. The host pops the
// reference whose box wastes the most area (box surface area less twice the
// area of the triangle part it holds) one at a time; here every round splits
// all references whose wasted area is in the highest occupied power-of-two
// bin, so each round's splits are within a factor of two of the greedy
// choice. A split cuts the box at the midpoint of its longest axis and keeps,
// for each half, the box of the triangle clipped to it (split_util.h, double
// precision, the host's rules); a reference that cannot be split (midpoint
// not strictly inside, or a half empty) is not tried again. Right halves are
// appended in reference order (a prefix sum over the round's splits), so the
// reference set does not depend on thread timing; when a round would exceed
// the budget, the lowest-numbered references split first. Final boxes: an
// unsplit reference keeps its primitive's own box bit for bit (PrimBox), a
// split one its double box rounded outward to float and padded by 10 epsilon
// as Triangle::GetAABB pads, so every part of a triangle lies in one of its
// references' boxes.

#include "accel.cuh"
#include "build_util.cuh"
#include "split_util.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

namespace bbg
{

namespace
{

struct DevRef
{
    double lo[3], hi[3];
    double waste;  // wasted box area; < 0: never split (again)
    int32_t prim;
    int32_t split; // nonzero once the reference holds part of a split triangle
};

constexpr int kWasteBins = 2200; // ilogb(waste) + 1100, clamped
constexpr int kMaxRounds = 4096;

__device__ __forceinline__ int WasteBin(double w)
{
    return min(max(ilogb(w) + 1100, 0), kWasteBins - 1);
}

__device__ __forceinline__ void LoadTriangle(const int2* prim_shape, const int32_t* tri, const float* pos,
                                             int32_t prim, double t[3][3])
{
    const int32_t* v = tri + 3 * size_t(prim_shape[prim].y);
    for (int k = 0; k < 3; ++k)
    {
        for (int c = 0; c < 3; ++c)
        {
            t[k][c] = pos[3 * size_t(v[k]) + c];
        }
    }
}

// The halves of reference r, as the host splits it; false if it cannot be
// split.
__device__ __forceinline__ bool SplitHalves(const DevRef& r, const double tri[3][3], DevRef* left, DevRef* right)
{
    const int axis = split::LongestAxis(r.lo, r.hi);
    const double m = 0.5 * (r.lo[axis] + r.hi[axis]);
    if (!(m > r.lo[axis] && m < r.hi[axis]))
    {
        return false; // too small to split
    }
    double llo[3], lhi[3], rlo[3], rhi[3];
    for (int c = 0; c < 3; ++c)
    {
        llo[c] = rlo[c] = r.lo[c];
        lhi[c] = rhi[c] = r.hi[c];
    }
    lhi[axis] = m;
    rlo[axis] = m;
    double al = 0, ar = 0;
    if (!split::ClippedBox(tri, llo, lhi, left->lo, left->hi, &al) ||
        !split::ClippedBox(tri, rlo, rhi, right->lo, right->hi, &ar))
    {
        return false; // the box was not tight on this axis: keep the reference whole
    }
    left->waste = split::BoxArea(left->lo, left->hi) - 2 * al;
    right->waste = split::BoxArea(right->lo, right->hi) - 2 * ar;
    left->prim = right->prim = r.prim;
    left->split = right->split = 1;
    return true;
}

__global__ void SplitInitKernel(const int2* prim_shape, const int32_t* tri, const float* pos, int32_t n, DevRef* refs)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        DevRef r{};
        r.prim = i;
        r.waste = -1;
        if (prim_shape[i].x == BBG_PRIM_TRIANGLE)
        {
            double t[3][3];
            LoadTriangle(prim_shape, tri, pos, i, t);
            for (int c = 0; c < 3; ++c)
            {
                const double lo01 = t[1][c] < t[0][c] ? t[1][c] : t[0][c];
                const double hi01 = t[0][c] < t[1][c] ? t[1][c] : t[0][c];
                r.lo[c] = t[2][c] < lo01 ? t[2][c] : lo01;
                r.hi[c] = hi01 < t[2][c] ? t[2][c] : hi01;
            }
            r.waste = split::BoxArea(r.lo, r.hi) - 2 * split::PolygonArea(t, 3);
        }
        refs[i] = r;
    }
}

// Histogram of the splittable references' wasted-area bins.
__global__ void SplitHistogramKernel(const DevRef* refs, int32_t m, uint32_t* hist)
{
    __shared__ uint32_t h[kWasteBins];
    for (int b = threadIdx.x; b < kWasteBins; b += blockDim.x)
    {
        h[b] = 0;
    }
    __syncthreads();
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
    {
        const double w = refs[r].waste;
        if (w > 0)
        {
            atomicAdd(&h[WasteBin(w)], 1u);
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kWasteBins; b += blockDim.x)
    {
        if (h[b])
        {
            atomicAdd(&hist[b], h[b]);
        }
    }
}

// Marks the references of bin `bin` that split (flag 1); the others of that
// bin are not tried again.
__global__ void SplitFlagKernel(DevRef* refs, int32_t m, int bin, const int2* prim_shape, const int32_t* tri,
                                const float* pos, int32_t* flags)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    {
        int32_t f = 0;
        const DevRef r = refs[i];
        if (r.waste > 0 && WasteBin(r.waste) == bin)
        {
            double t[3][3];
            LoadTriangle(prim_shape, tri, pos, r.prim, t);
            DevRef left, right;
            if (SplitHalves(r, t, &left, &right))
            {
                f = 1;
            }
            else
            {
                refs[i].waste = -1;
            }
        }
        flags[i] = f;
    }
}

// Splits the flagged references whose place among the round's splits is
// below cap: the left half replaces the reference, the right half goes to
// m + its place.
__global__ void SplitApplyKernel(DevRef* refs, int32_t m, const int32_t* flags, const int32_t* place, int32_t cap,
                                 const int2* prim_shape, const int32_t* tri, const float* pos)
{
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    {
        if (!flags[i] || place[i] >= cap)
        {
            continue;
        }
        const DevRef r = refs[i];
        double t[3][3];
        LoadTriangle(prim_shape, tri, pos, r.prim, t);
        DevRef left, right;
        SplitHalves(r, t, &left, &right); // true, as in the flag pass
        refs[i] = left;
        refs[m + place[i]] = right;
    }
}

__global__ void SplitBoxesKernel(const DevRef* refs, int32_t m, const int2* prim_shape, const int32_t* tri,
                                 const float* pos, const bbg_sphere* spheres, float4* box, int32_t* ref_prim)
{
    const float pad = FLT_EPSILON * 10;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    {
        const DevRef& r = refs[i];
        float3 mn, mx;
        if (!r.split)
        {
            PrimBox(prim_shape, tri, pos, spheres, r.prim, &mn, &mx);
        }
        else
        {
            mn = make_float3(split::RoundDown(r.lo[0]) - pad, split::RoundDown(r.lo[1]) - pad,
                             split::RoundDown(r.lo[2]) - pad);
            mx = make_float3(split::RoundUp(r.hi[0]) + pad, split::RoundUp(r.hi[1]) + pad,
                             split::RoundUp(r.hi[2]) + pad);
        }
        box[2 * size_t(i)] = make_float4(mn.x, mn.y, mn.z, 0);
        box[2 * size_t(i) + 1] = make_float4(mx.x, mx.y, mx.z, 0);
        ref_prim[i] = r.prim;
    }
}

} // namespace

bbg_status SplitReferencesOnDevice(bbg_accel* a, float budget, DevBuf<float4>* ref_box, DevBuf<int32_t>* ref_prim,
                                   int32_t* n_refs)
{
    const int32_t n = a->n_prims;
    cudaStream_t st = a->stream;
    const int sms = CurrentSmCount();
    // At most 2^30 references, so a tree over them (2 m - 1 nodes) fits int32
    // (the host splitter's limit).
    const int64_t max_refs = std::min<int64_t>(int64_t(n) + int64_t(double(budget) * n), int64_t(1) << 30);
    DevBuf<DevRef> refs;
    DevBuf<int32_t> flags, place;
    DevBuf<uint32_t> hist;
    BBG_TRY(refs.alloc(size_t(max_refs)));
    BBG_TRY(flags.alloc(size_t(max_refs)));
    BBG_TRY(place.alloc(size_t(max_refs) + 1));
    BBG_TRY(hist.alloc(kWasteBins));
    size_t scan_bytes = 0;
    BBG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flags.p, place.p, int(max_refs), st));
    DevBuf<uint8_t> scan_tmp;
    BBG_TRY(scan_tmp.alloc(std::max<size_t>(scan_bytes, 1)));

    SplitInitKernel<<<GridFor(n, 256, sms), 256, 0, st>>>(a->prim_shape.p, a->tri_indices.p, a->positions.p, n,
                                                          refs.p);
    int64_t m = n;
    std::vector<uint32_t> h(kWasteBins);
    for (int round = 0; round < kMaxRounds && m < max_refs; ++round)
    {
        BBG_CUDA(cudaMemsetAsync(hist.p, 0, sizeof(uint32_t) * kWasteBins, st));
        SplitHistogramKernel<<<GridFor(m, 256, sms), 256, 0, st>>>(refs.p, int32_t(m), hist.p);
        BBG_CUDA(cudaMemcpyAsync(h.data(), hist.p, sizeof(uint32_t) * kWasteBins, cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaStreamSynchronize(st));
        int bin = kWasteBins - 1;
        while (bin >= 0 && h[size_t(bin)] == 0)
        {
            --bin;
        }
        if (bin < 0)
        {
            break; // nothing left to split
        }
        SplitFlagKernel<<<GridFor(m, 256, sms), 256, 0, st>>>(refs.p, int32_t(m), bin, a->prim_shape.p,
                                                              a->tri_indices.p, a->positions.p, flags.p);
        // Places over m + 1 entries: the last one is the round's split count.
        BBG_CUDA(cudaMemsetAsync(flags.p + m, 0, sizeof(int32_t), st));
        BBG_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp.p, scan_bytes, flags.p, place.p, int(m + 1), st));
        const int32_t cap = int32_t(max_refs - m);
        SplitApplyKernel<<<GridFor(m, 256, sms), 256, 0, st>>>(refs.p, int32_t(m), flags.p, place.p, cap,
                                                               a->prim_shape.p, a->tri_indices.p, a->positions.p);
        int32_t count = 0;
        BBG_CUDA(cudaMemcpyAsync(&count, place.p + m, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        BBG_CUDA(cudaStreamSynchronize(st));
        m += std::min(count, cap);
    }
    BBG_TRY(ref_box->alloc(2 * size_t(m)));
    BBG_TRY(ref_prim->alloc(size_t(m)));
    SplitBoxesKernel<<<GridFor(m, 256, sms), 256, 0, st>>>(refs.p, int32_t(m), a->prim_shape.p, a->tri_indices.p,
                                                           a->positions.p, a->spheres.p, ref_box->p, ref_prim->p);
    BBG_CUDA(cudaStreamSynchronize(st));
    BBG_CUDA(cudaGetLastError());
    *n_refs = int32_t(m);
    return BBG_OK;
}

} // namespace bbg
