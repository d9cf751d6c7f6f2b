// Device sampler and sampling routines.
//
// IndependentSampler (src/sampler/independent_sampler.cpp:13-27): for each
// (pixel, sample) the generator is re-seeded with
//   RNG::Seed(MurmurHash64A(bytes{pixel.x, pixel.y, seed, sample}, 16, 0), 1)
// (include/bulbit/hash.h:17-70,111-120; include/bulbit/random.h:27-34) and
// every draw is min(1 - FLT_EPSILON, u32 * 2^-32) (random.h:87-90). The
// stream is identical bit for bit. The reference is built with GCC, which
// evaluates call arguments right to left, so in
//   camera->SampleRay(&ray, pixel, Next2D(), Next2D())    (integrator.cpp:190)
//   bsdf.Sample_f(&bs, wo, Next1D(), Next2D())            (path_integrator.cpp:115)
// the right-hand argument is drawn first; callers here draw in that order.
#pragma once

#include "dev_math.cuh"

namespace bbg
{

constexpr uint64_t kPcgMult = 0x5851f42d4c957f2dull;
constexpr uint64_t kPcgInc = 3; // (initseq = 1) << 1 | 1

__device__ __forceinline__ uint64_t Murmur64A_16(uint64_t k0, uint64_t k1)
{
    const uint64_t m = 0xc6a4a7935bd1e995ull;
    const int r = 47;
    uint64_t h = 0 ^ (16ull * m);
    k0 *= m;
    k0 ^= k0 >> r;
    k0 *= m;
    h ^= k0;
    h *= m;
    k1 *= m;
    k1 ^= k1 >> r;
    k1 *= m;
    h ^= k1;
    h *= m;
    h ^= h >> r;
    h *= m;
    h ^= h >> r;
    return h;
}

__device__ __forceinline__ uint32_t PcgNext(uint64_t& state)
{
    uint64_t old = state;
    state = old * kPcgMult + kPcgInc;
    uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = uint32_t(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((~rot + 1u) & 31));
}

// IndependentSampler::StartPixelSample: the PCG32 state after Seed(hash, 1).
__device__ __forceinline__ uint64_t SamplerStart(int32_t px, int32_t py, int32_t seed, int32_t sample)
{
    uint64_t k0 = uint64_t(uint32_t(px)) | (uint64_t(uint32_t(py)) << 32);
    uint64_t k1 = uint64_t(uint32_t(seed)) | (uint64_t(uint32_t(sample)) << 32);
    uint64_t h = Murmur64A_16(k0, k1);
    uint64_t state = 0;
    PcgNext(state);
    state += h;
    PcgNext(state);
    return state;
}

__device__ __forceinline__ float Next1D(uint64_t& state)
{
    float u = float(PcgNext(state)) * 0x1p-32f;
    return fminf(1 - kEpsilon, u);
}

struct P2
{
    float x, y;
};

// Next2D: Point2{ NextFloat(), NextFloat() } (braced: left to right).
__device__ __forceinline__ P2 Next2D(uint64_t& state)
{
    float a = Next1D(state);
    float b = Next1D(state);
    return P2{ a, b };
}

// PermutationElement (include/bulbit/hash.h:129-159): Kensler's hashed
// permutation of [0, l) ("Correlated Multi-Jittered Sampling", 2013).
__device__ __forceinline__ uint32_t PermutationElement(uint32_t i, uint32_t l, uint32_t p)
{
    uint32_t w = l - 1;
    w |= w >> 1;
    w |= w >> 2;
    w |= w >> 4;
    w |= w >> 8;
    w |= w >> 16;
    do
    {
        i ^= p;
        i *= 0xe170893du;
        i ^= p >> 16;
        i ^= (i & w) >> 4;
        i ^= p >> 8;
        i *= 0x0929eb3fu;
        i ^= p >> 23;
        i ^= (i & w) >> 1;
        i *= 1u | p >> 27;
        i *= 0x6935fa69u;
        i ^= (i & w) >> 11;
        i *= 0x74dcb303u;
        i ^= (i & w) >> 2;
        i *= 0x9e501cc3u;
        i ^= (i & w) >> 2;
        i *= 0xc860a3dfu;
        i &= w;
        i ^= i >> 5;
    } while (i >= l);
    return (i + p) % l;
}

// The per-path sampler: IndependentSampler (src/sampler/independent_sampler.cpp)
// or StratifiedSampler (src/sampler/stratified_sampler.cpp:16-58). Both seed
// the same PCG32 stream from the pixel and sample; the stratified one places
// each draw of dimension d in a stratum chosen by a permutation hashed from
// (seed, pixel, d), jittered by the stream.
struct PathSampler
{
    uint64_t state;
    int32_t dim;        // stratified: next dimension
    int32_t stratified; // 0: independent
    int32_t px, py, sample, seed, spp, x_samples, jitter;
};

__device__ __forceinline__ uint32_t StratumHash(const PathSampler& s)
{
    // Hash(seed, current_pixel, dimension): 16 bytes, little-endian.
    uint64_t k0 = uint64_t(uint32_t(s.seed)) | (uint64_t(uint32_t(s.px)) << 32);
    uint64_t k1 = uint64_t(uint32_t(s.py)) | (uint64_t(uint32_t(s.dim)) << 32);
    return uint32_t(Murmur64A_16(k0, k1));
}

__device__ __forceinline__ float Next1D(PathSampler& s)
{
    if (!s.stratified)
    {
        return Next1D(s.state);
    }
    int32_t stratum = int32_t(PermutationElement(uint32_t(s.sample), uint32_t(s.spp), StratumHash(s)));
    s.dim += 1;
    float delta = s.jitter ? Next1D(s.state) : 0.5f;
    return (float(stratum) + delta) / float(s.spp);
}

__device__ __forceinline__ P2 Next2D(PathSampler& s)
{
    if (!s.stratified)
    {
        return Next2D(s.state);
    }
    int32_t stratum = int32_t(PermutationElement(uint32_t(s.sample), uint32_t(s.spp), StratumHash(s)));
    s.dim += 2;
    int32_t x = stratum % s.x_samples;
    int32_t y = stratum / s.x_samples;
    float dx = s.jitter ? Next1D(s.state) : 0.5f;
    float dy = s.jitter ? Next1D(s.state) : 0.5f;
    int32_t y_samples = s.spp / s.x_samples;
    return P2{ (float(x) + dx) / float(s.x_samples), (float(y) + dy) / float(y_samples) };
}

// PowerHeuristic(1, f, 1, g) (include/bulbit/sampling.h:42-48).
__device__ __forceinline__ float PowerHeuristic(float pdf_f, float pdf_g)
{
    float f = 1 * pdf_f;
    float g = 1 * pdf_g;
    return (f * f) / (f * f + g * g);
}

// SampleUniformUnitDiskConcentric (include/bulbit/sampling.h:114-136).
__device__ __forceinline__ P2 SampleUniformUnitDiskConcentric(P2 u)
{
    P2 uo{ u.x * 2 - 1, u.y * 2 - 1 };
    if (uo.x == 0 && uo.y == 0)
    {
        return P2{ 0, 0 };
    }
    float theta, r;
    if (fabsf(uo.x) > fabsf(uo.y))
    {
        r = uo.x;
        theta = (kPi / 4) * (uo.y / uo.x);
    }
    else
    {
        r = uo.y;
        theta = (kPi / 2) - (kPi / 4) * (uo.x / uo.y);
    }
    return P2{ dcos(theta) * r, dsin(theta) * r };
}

// SampleCosineHemisphere, Malley's method (include/bulbit/sampling.h:160-169).
__device__ __forceinline__ V3 SampleCosineHemisphere(P2 u)
{
    P2 d = SampleUniformUnitDiskConcentric(u);
    float z = sqrtf(SMax(0.0f, 1 - Sqr(d.x) - Sqr(d.y)));
    return V3{ d.x, d.y, z };
}

// SampleUniformSphere (include/bulbit/sampling.h:59-70).
__device__ __forceinline__ V3 SampleUniformSphere(P2 u)
{
    float z = 1 - 2 * u.x;
    float r = sqrtf(fmaxf(0.0f, 1 - z * z));
    float phi = kTwoPi * u.y;
    return V3{ r * dcos(phi), r * dsin(phi), z };
}

// Dupuy & Benyoub spherical-cap VNDF sampling
// (include/bulbit/sampling.h:206-232), including its std::fma.
__device__ __forceinline__ V3 SampleGGXVNDF(V3 wo, float alpha_x, float alpha_y, P2 u)
{
    V3 wo_std = Normalize(V3{ wo.x * alpha_x, wo.y * alpha_y, wo.z });
    float phi = kTwoPi * u.x;
    float z = fmaf((1 - u.y), (1 + wo_std.z), -wo_std.z);
    float sin_theta = sqrtf(Clamp(1 - z * z, 0, 1));
    float x = sin_theta * dcos(phi);
    float y = sin_theta * dsin(phi);
    V3 h = V3{ x, y, z } + wo_std;
    return Normalize(V3{ h.x * alpha_x, h.y * alpha_y, h.z });
}

} // namespace bbg
