// Lights on the device: PointLight, SpotLight, UniformInfiniteLight and
// DiffuseAreaLight over triangles and spheres, restated from src/light/*.cpp
// and the shape sampling of src/geometry/{triangle,sphere}.cpp.
#pragma once

#include "bbg_internal.h"
#include "dev_geometry.cuh"
#include "dev_sampling.cuh"

namespace bbg
{

struct LightSampleLi
{
    V3 wi;
    float visibility;
    Spec Li;
    float pdf;
};

struct ShapeSample
{
    V3 point;
    V3 normal;
    float pdf;
};

// Triangle::Sample(u) + Triangle::Sample(ref, u) (src/geometry/triangle.cpp:159-234).
__device__ __forceinline__ ShapeSample SampleTriangle(V3 p0, V3 p1, V3 p2, V3 ref, P2 u0)
{
    V3 e1 = p1 - p0;
    V3 e2 = p2 - p0;
    float u = u0.x, v = u0.y;
    if (u + v > 1)
    {
        u = 1 - u;
        v = 1 - v;
    }
    ShapeSample s;
    s.normal = Cross(e1, e2);
    s.point = p0 + e1 * u + e2 * v;
    float area = NormalizeInPlace(s.normal) * 0.5f;
    s.pdf = 1 / area;

    V3 d = s.point - ref;
    float distance_squared = Dot(d, d);
    float cosine = Dot(d, s.normal) / sqrtf(distance_squared);
    if (cosine < 0)
    {
        cosine = -cosine;
    }
    s.pdf *= distance_squared / cosine;
    return s;
}

// Sphere::Sample(ref, u) (src/geometry/sphere.cpp:137-169).
__device__ __forceinline__ ShapeSample SampleSphere(const bbg_sphere& sp, V3 ref, P2 u)
{
    V3 center = load3(sp.p);
    V3 direction = center - ref;
    float distance = NormalizeInPlace(direction);
    float distance_squared = distance * distance;
    float cos_theta_max = sqrtf(1 - sp.radius * sp.radius / distance_squared);
    float z = 1 + u.y * (cos_theta_max - 1);
    float phi = kTwoPi * u.x;
    float sin_theta = sqrtf(1 - z * z);
    float x = dcos(phi) * sin_theta;
    float y = dsin(phi) * sin_theta;
    V3 d{ x, y, z };
    float s = distance * z - sqrtf(sp.radius * sp.radius - distance_squared * sin_theta * sin_theta);
    Frame frame = FrameFromZ(direction);
    V3 ref2p = frame.FromLocal(d) * s;
    float solid_angle = kTwoPi * (1 - cos_theta_max);
    ShapeSample out;
    out.point = ref + ref2p;
    out.normal = Normalize(out.point - center);
    out.pdf = 1 / solid_angle;
    return out;
}

// SmoothStep (include/bulbit/math.h:64-73).
__device__ __forceinline__ float SmoothStep(float a, float b, float x)
{
    if (a == b)
    {
        return (x < a) ? 0.0f : 1.0f;
    }
    float t = Clamp((x - a) / (b - a), 0, 1);
    return t * t * (3 - 2 * t);
}

__device__ __forceinline__ bool IsDeltaLight(int32_t type)
{
    return type == BBG_LIGHT_POINT || type == BBG_LIGHT_SPOT;
}

// Light::Sample_Li for the supported lights. `tri_pos` gives the area light's
// triangle vertices when it sits on a triangle.
__device__ __forceinline__ bool SampleLi(const LightDev& l, V3 ref, P2 u, const V3* tri, const bbg_sphere* sph,
                                         LightSampleLi* out)
{
    switch (l.type)
    {
    case BBG_LIGHT_POINT:
    {
        // src/light/point_light.cpp:35-50
        V3 wi = load3(l.p) - ref;
        float distance = NormalizeInPlace(wi);
        out->wi = wi;
        out->visibility = distance;
        out->pdf = 1;
        out->Li = Spec{ l.L[0], l.L[1], l.L[2] } / (distance * distance);
        return true;
    }
    case BBG_LIGHT_SPOT:
    {
        // src/light/spot_light.cpp:46-68
        V3 wi = load3(l.p) - ref;
        float distance = NormalizeInPlace(wi);
        float cos_theta = -Dot(wi, load3(l.frame_z));
        Spec li = SmoothStep(l.cos_theta_max, l.cos_theta_min, cos_theta) * Spec{ l.L[0], l.L[1], l.L[2] };
        if (IsBlack(li))
        {
            return false;
        }
        out->wi = wi;
        out->visibility = distance;
        out->pdf = 1;
        out->Li = li / (distance * distance);
        return true;
    }
    case BBG_LIGHT_UNIFORM_INFINITE:
    {
        // src/light/uniform_infinite_light.cpp:33-45
        V3 wi = SampleUniformSphere(u);
        out->wi = wi;
        out->pdf = kInvFourPi;
        out->visibility = 2 * l.world_radius;
        out->Li = l.scale * Spec{ l.L[0], l.L[1], l.L[2] };
        return true;
    }
    default:
    {
        // DiffuseAreaLight::Sample_Li (src/light/diffuse_area_light.cpp:43-66)
        ShapeSample ss = tri ? SampleTriangle(tri[0], tri[1], tri[2], ref, u) : SampleSphere(*sph, ref, u);
        V3 wi = ss.point - ref;
        out->visibility = NormalizeInPlace(wi) - kRayEpsilon;
        out->wi = wi;
        out->pdf = ss.pdf;
        bool front_face = Dot(ss.normal, wi) < 0;
        out->Li = (front_face || l.two_sided) ? Spec{ l.L[0], l.L[1], l.L[2] } : spec(0);
        return true;
    }
    }
}

} // namespace bbg
