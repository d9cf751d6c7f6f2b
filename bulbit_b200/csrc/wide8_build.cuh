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

#include "bbg.h"

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
        // The least e with p + 255 2^e >= phi: frexp (exact, unlike log2,
        // whose last bit the host's and the device's libraries may round
        // differently) places ext / 255 in [2^(x-1), 2^x), so x - 2 is a
        // lower bound, and the exact test below raises it.
        int e = -126;
        if (ext > 0)
        {
            int x = 0;
            frexp(ext / 255.0, &x);
            e = x - 2 < -126 ? -126 : x - 2;
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

// Which binary nodes become wide nodes: the choice that minimises the summed
// surface area of the wide nodes (the surface-area cost of opening them; a
// leaf is tested whenever its own box is hit, whichever wide node holds it,
// so leaves add the same cost to every choice). This is the optimal collapse
// of Ylitie, Karras and Laine (HPG 2017, section 3.1) without merging leaves:
// cost[i - 1] is the least cost of a binary subtree as at most i children of
// one wide node, each child a binary leaf or a binary node that becomes a
// wide node of its own; i > 1 children are shared between the two subtrees,
// the left one taking split[i - 1] (0: as with i - 1 children). Leaves cost
// 0. Interior node x's entries from its children's (cost_l, cost_r); both
// the host and the device run this, in double precision, so they agree.
// split[7] is what x's own wide node holds: the left subtree's share of 8.
__host__ __device__ inline void Wide8PlanNode(const bbg_bvh_node& x, const float cost_l[8], const float cost_r[8],
                                              float cost[8], uint8_t split[8])
{
    Child8 c;
    for (int a = 0; a < 3; ++a)
    {
        c.lo[a] = x.bmin[a];
        c.hi[a] = x.bmax[a];
    }
    double dist[9];
    uint8_t best_k[9] = {};
    for (int j = 2; j <= 8; ++j)
    {
        dist[j] = 1e300;
        for (int k = 1; k < j; ++k)
        {
            const double v = double(cost_l[k - 1]) + double(cost_r[j - k - 1]);
            if (v < dist[j])
            {
                dist[j] = v;
                best_k[j] = uint8_t(k);
            }
        }
    }
    cost[0] = float(Wide8Area(c) + dist[8]); // one child: x is a wide node
    split[0] = 0;
    for (int i = 2; i <= 8; ++i)
    {
        const bool fewer = double(cost[i - 2]) <= dist[i];
        cost[i - 1] = fewer ? cost[i - 2] : float(dist[i]);
        split[i - 1] = fewer ? 0 : best_k[i];
    }
    split[7] = best_k[8];
}

// The children of the wide node that stands for interior binary node b
// (depth-first layout nd, plan split[8 per node]), left subtree's first, in
// order; returns their count. A single-leaf tree's root is its one child.
__host__ __device__ inline int Wide8Gather(const bbg_bvh_node* nd, const uint8_t* split, int32_t b, int32_t out[8])
{
    if (nd[b].count > 0)
    {
        out[0] = b;
        return 1;
    }
    // Pending (subtree, at most so many children), each yielding at least
    // one: the pending budgets and the children out never exceed eight. (A
    // split point outside 1..j-1, which a computed plan never holds, makes
    // the subtree one child, so no plan content can overrun the arrays.)
    int32_t sb[8];
    int si[8];
    int sp = 0, n = 0;
    int k0 = split[8 * size_t(b) + 7];
    k0 = k0 < 1 ? 1 : k0 > 7 ? 7 : k0;
    sb[sp] = nd[b].offset;
    si[sp++] = 8 - k0;
    sb[sp] = b + 1;
    si[sp++] = k0;
    while (sp > 0)
    {
        --sp;
        const int32_t x = sb[sp];
        int j = si[sp];
        while (nd[x].count == 0 && j > 1 && split[8 * size_t(x) + j - 1] == 0)
        {
            --j;
        }
        const int k = nd[x].count == 0 && j > 1 ? split[8 * size_t(x) + j - 1] : 0;
        if (k < 1 || k >= j)
        {
            out[n++] = x;
            continue;
        }
        sb[sp] = nd[x].offset;
        si[sp++] = j - k;
        sb[sp] = x + 1;
        si[sp++] = k;
    }
    return n;
}

} // namespace bbg
