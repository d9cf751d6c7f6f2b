// Device helpers shared by the tree builds on the device (lbvh.cu,
// sah_build.cu): primitive boxes exactly as the host computes them, and an
// order-preserving float <-> uint mapping for atomic and warp-wide min / max.
#pragma once

#include "bbg_internal.h"

#include <cfloat>
#include <cuda_runtime.h>

namespace bbg
{

// Box of primitive i as PrimAabbs (host_build.cpp) computes it: triangles
// padded by 10 FLT_EPSILON (Triangle::GetAABB), spheres centre +- radius.
__device__ __forceinline__ void PrimBox(const int2* prim_shape, const int32_t* tri, const float* pos,
                                        const bbg_sphere* spheres, int32_t i, float3* mn, float3* mx)
{
    int2 ps = prim_shape[i];
    if (ps.x == BBG_PRIM_TRIANGLE)
    {
        const float pad = FLT_EPSILON * 10;
        const int32_t* v = tri + 3 * size_t(ps.y);
        float3 p[3];
        for (int k = 0; k < 3; ++k)
        {
            const float* q = pos + 3 * size_t(v[k]);
            p[k] = make_float3(q[0], q[1], q[2]);
        }
        *mn = make_float3(fminf(fminf(p[0].x, p[1].x), p[2].x) - pad, fminf(fminf(p[0].y, p[1].y), p[2].y) - pad,
                          fminf(fminf(p[0].z, p[1].z), p[2].z) - pad);
        *mx = make_float3(fmaxf(fmaxf(p[0].x, p[1].x), p[2].x) + pad, fmaxf(fmaxf(p[0].y, p[1].y), p[2].y) + pad,
                          fmaxf(fmaxf(p[0].z, p[1].z), p[2].z) + pad);
    }
    else
    {
        const bbg_sphere& s = spheres[ps.y];
        *mn = make_float3(s.p[0] - s.radius, s.p[1] - s.radius, s.p[2] - s.radius);
        *mx = make_float3(s.p[0] + s.radius, s.p[1] + s.radius, s.p[2] + s.radius);
    }
}

// Blocks for a grid-stride loop over items: enough for every item, at most 8
// per SM.
inline int GridFor(int64_t items, int block, int sms)
{
    const int64_t blocks = (items + block - 1) / block;
    return int(blocks < 1 ? 1 : blocks < int64_t(sms) * 8 ? blocks : int64_t(sms) * 8);
}

// Order-preserving float <-> uint mapping for atomic min / max.
__device__ __forceinline__ uint32_t FloatKey(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float KeyFloat(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

} // namespace bbg
