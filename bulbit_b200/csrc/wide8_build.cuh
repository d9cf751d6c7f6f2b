// Construction of the 8-wide node layout (see dev_geometry.cuh for the
// format), shared by the collapse of a host-built tree (accel.cu) and of a
// tree built on the device (lbvh.cu): slot assignment by octant and the
// outward-rounding quantisation of the child boxes. Host and device run the
// same double-precision arithmetic, so both produce the same node for the
// same children.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace bbg
{

// One child of a node being collapsed: its box and its binary-tree reference
// (the caller's encoding: an interior node to collapse further, or a leaf).
struct Child8
{
    float lo[3], hi[3];
    int32_t bnode;
};

__host__ __device__ inline float Wide8Bits(uint32_t bits)
{
    float f;
    memcpy(&f, &bits, sizeof(f));
    return f;
}

__host__ __device__ inline double Wide8Area(const Child8& c)
{
    double d[3];
    for (int a = 0; a < 3; ++a)
    {
        d[a] = double(c.hi[a]) - double(c.lo[a]);
    }
    return d[0] * d[1] + d[1] * d[2] + d[2] * d[0];
}

__host__ __device__ inline void Wide8Union(const Child8* cs, int n, float plo[3], float phi[3])
{
    for (int a = 0; a < 3; ++a)
    {
        plo[a] = cs[0].lo[a];
        phi[a] = cs[0].hi[a];
        for (int c = 1; c < n; ++c)
        {
            plo[a] = cs[c].lo[a] < plo[a] ? cs[c].lo[a] : plo[a];
            phi[a] = cs[c].hi[a] > phi[a] ? cs[c].hi[a] : phi[a];
        }
    }
}

// Assigns up to eight children to slots so that slot k holds a child whose
// centroid lies toward corner k of the parent (bit a of k set: the + side of
// axis a); rays with octant code o then meet the children roughly front to
// back in the order k ^ o. Greedy on the largest remaining
// centroid-offset . corner-direction product.
__host__ __device__ inline void AssignSlots8(const Child8* cs, int n, const float plo[3], const float phi[3],
                                             int32_t slot_of[8])
{
    double pc[3];
    for (int a = 0; a < 3; ++a)
    {
        pc[a] = 0.5 * (double(plo[a]) + double(phi[a]));
    }
    double score[8][8];
    for (int c = 0; c < n; ++c)
    {
        for (int k = 0; k < 8; ++k)
        {
            double d = 0;
            for (int a = 0; a < 3; ++a)
            {
                double off = 0.5 * (double(cs[c].lo[a]) + double(cs[c].hi[a])) - pc[a];
                d += ((k >> a) & 1) ? off : -off;
            }
            score[c][k] = d;
        }
    }
    bool child_done[8] = {}, slot_used[8] = {};
    for (int round = 0; round < n; ++round)
    {
        int bc = -1, bk = -1;
        double best = 0;
        for (int c = 0; c < n; ++c)
        {
            if (child_done[c]) continue;
            for (int k = 0; k < 8; ++k)
            {
                if (slot_used[k]) continue;
                if (bc < 0 || score[c][k] > best)
                {
                    best = score[c][k];
                    bc = c;
                    bk = k;
                }
            }
        }
        child_done[bc] = true;
        slot_used[bk] = true;
        slot_of[bc] = bk;
    }
}

// Writes a node: the children's boxes quantised to bytes on a per-axis grid
// p + q 2^e over their union, rounded outward so that every decoded box
// contains its child's box exactly (checked in double precision, where
// p + q 2^e is exact); the interior-slot mask; the references (refs[k] for
// slot k: >= 0 node, < 0 leaf, ~0 for an empty slot).
__host__ __device__ inline void QuantizeNode8(const Child8* cs, int n, const int32_t slot_of[8],
                                              const int32_t refs[8], float4* out)
{
    float plo[3], phi[3];
    Wide8Union(cs, n, plo, phi);
    uint8_t qlo[3][8], qhi[3][8];
    uint32_t meta = 0;
    for (int k = 0; k < 8; ++k)
    {
        meta |= (refs[k] >= 0 ? 1u : 0u) << (24 + k);
    }
    for (int a = 0; a < 3; ++a)
    {
        double p = plo[a];
        double ext = double(phi[a]) - p;
        int e = -126;
        if (ext > 0)
        {
            e = int(ceil(log2(ext / 255.0)));
            e = e < -126 ? -126 : e;
        }
        while (e < 127 && p + 255.0 * ldexp(1.0, e) < double(phi[a]))
        {
            ++e;
        }
        double sc = ldexp(1.0, e);
        meta |= uint32_t(e + 127) << (8 * a);
        for (int k = 0; k < 8; ++k)
        {
            qlo[a][k] = 255; // empty slot: an inverted box
            qhi[a][k] = 0;
        }
        for (int c = 0; c < n; ++c)
        {
            double lo = cs[c].lo[a], hi = cs[c].hi[a];
            double fl = floor((lo - p) / sc), fh = ceil((hi - p) / sc);
            int ql = int(fl < 0.0 ? 0.0 : (fl > 255.0 ? 255.0 : fl));
            int qh = int(fh < 0.0 ? 0.0 : (fh > 255.0 ? 255.0 : fh));
            while (ql > 0 && p + ql * sc > lo) --ql;
            while (qh < 255 && p + qh * sc < hi) ++qh;
            qlo[a][slot_of[c]] = uint8_t(ql);
            qhi[a][slot_of[c]] = uint8_t(qh);
        }
    }
    auto word = [](const uint8_t* b) {
        return Wide8Bits(uint32_t(b[0]) | uint32_t(b[1]) << 8 | uint32_t(b[2]) << 16 | uint32_t(b[3]) << 24);
    };
    out[0] = make_float4(plo[0], plo[1], plo[2], Wide8Bits(meta));
    out[1] = make_float4(word(qlo[0]), word(qlo[0] + 4), word(qlo[1]), word(qlo[1] + 4));
    out[2] = make_float4(word(qlo[2]), word(qlo[2] + 4), word(qhi[0]), word(qhi[0] + 4));
    out[3] = make_float4(word(qhi[1]), word(qhi[1] + 4), word(qhi[2]), word(qhi[2] + 4));
    out[4] = make_float4(Wide8Bits(uint32_t(refs[0])), Wide8Bits(uint32_t(refs[1])), Wide8Bits(uint32_t(refs[2])),
                         Wide8Bits(uint32_t(refs[3])));
    out[5] = make_float4(Wide8Bits(uint32_t(refs[4])), Wide8Bits(uint32_t(refs[5])), Wide8Bits(uint32_t(refs[6])),
                         Wide8Bits(uint32_t(refs[7])));
}

// A leaf child's reference: ~(first slot << 5 | count), count 1..31.
constexpr int kWide8LeafCountBits = 5;
__host__ __device__ inline int32_t Wide8LeafRef(int32_t first_slot, int32_t count)
{
    return ~((first_slot << kWide8LeafCountBits) | count);
}

} // namespace bbg
