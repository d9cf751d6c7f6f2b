// BxDFs on the device: Lambertian, Conductor, Dielectric (each of the last
// two with its energy-compensated form) and Metallic-Roughness with the Trowbridge-Reitz distribution, restated from
// src/bxdf/{lambertian,conductor,dielectric,metallic_roughness}_bxdf.cpp,
// include/bulbit/microfacet.h and include/bulbit/scattering.h with the same
// operation order.
//
// std::complex<float> arithmetic follows GCC/libstdc++: products are the plain
// formula, division is evaluated in double precision and rounded once, |z| is
// a double hypot, real - complex is (-re + x, -im); signed zeros are kept
// because SqrtComplex copies the imaginary part's sign.
#pragma once

#include "bbg_internal.h"
#include "dev_sampling.cuh"

namespace bbg
{

// ---------------------------------------------------------------- microfacet

// Energy tables of the GGX distribution with F = 1, in the reference's layout
// (TrowbridgeReitzDistribution::PrepareReflectanceTexture,
// src/bxdf/microfacet.cpp:28-70): E(cos theta_o, alpha) 32 x 32 (x: cos theta,
// y: alpha) and E_avg(alpha) 32 x 1. Filled on the device by
// GgxEnergyTablesKernel (render.cu) before any energy-compensated material is
// shaded.
constexpr int kEnergyTableSize = 32;
static __device__ float g_ggx_e[kEnergyTableSize * kEnergyTableSize];
static __device__ float g_ggx_e_avg[kEnergyTableSize];

// ImageTexture<Float>::Evaluate: bilinear, texel coordinates clamped
// (include/bulbit/textures.h:55-87).
__device__ __forceinline__ float TableBilinear(const float* img, int w, int h, float u, float v)
{
    float x = u * float(w) - 0.5f;
    float y = v * float(h) - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    int i0 = int(fx), i1 = i0 + 1;
    int j0 = int(fy), j1 = j0 + 1;
    i0 = min(max(i0, 0), w - 1);
    j0 = min(max(j0, 0), h - 1);
    i1 = min(max(i1, 0), w - 1);
    j1 = min(max(j1, 0), h - 1);
    float fu = x - fx;
    float fv = y - fy;
    float v00 = img[i0 + j0 * w], v10 = img[i1 + j0 * w];
    float v01 = img[i0 + j1 * w], v11 = img[i1 + j1 * w];
    return (1 - fu) * (1 - fv) * v00 + (1 - fu) * fv * v01 + fu * (1 - fv) * v10 + fu * fv * v11;
}

// Energy tables of the rough dielectric in the reference's layout
// (DielectricMultiScatteringBxDF::PrepareReflectanceTexture,
// src/bxdf/microfacet.cpp:168-237): E and E_inv 32 x 32 x 32 (x: f0 =
// MapIORtoF0(eta), y: cos theta, z: alpha; E for eta >= 1, E_inv for the
// inverse interface), E_avg and E_inv_avg 32 x 32 (x: f0, y: alpha). Filled on
// the device by DielectricEnergyTablesKernel (render.cu).
static __device__ float g_dms_e[kEnergyTableSize * kEnergyTableSize * kEnergyTableSize];
static __device__ float g_dms_e_inv[kEnergyTableSize * kEnergyTableSize * kEnergyTableSize];
static __device__ float g_dms_e_avg[kEnergyTableSize * kEnergyTableSize];
static __device__ float g_dms_e_inv_avg[kEnergyTableSize * kEnergyTableSize];

// ImageTexture3D<Float>::Evaluate: trilinear, texel coordinates clamped,
// lerped along x, then y, then z (include/bulbit/textures3d.h:33-88).
__device__ __forceinline__ float TableTrilinear(const float* img, int n, float u, float v, float w)
{
    float x = u * float(n) - 0.5f;
    float y = v * float(n) - 0.5f;
    float z = w * float(n) - 0.5f;
    float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    int i0 = int(fx), i1 = i0 + 1;
    int j0 = int(fy), j1 = j0 + 1;
    int k0 = int(fz), k1 = k0 + 1;
    i0 = min(max(i0, 0), n - 1);
    j0 = min(max(j0, 0), n - 1);
    k0 = min(max(k0, 0), n - 1);
    i1 = min(max(i1, 0), n - 1);
    j1 = min(max(j1, 0), n - 1);
    k1 = min(max(k1, 0), n - 1);
    float fu = x - fx;
    float fv = y - fy;
    float fw = z - fz;
    auto at = [&](int i, int j, int k) { return img[(k * n + j) * n + i]; };
    float v00 = (1 - fu) * at(i0, j0, k0) + fu * at(i1, j0, k0);
    float v01 = (1 - fu) * at(i0, j0, k1) + fu * at(i1, j0, k1);
    float v10 = (1 - fu) * at(i0, j1, k0) + fu * at(i1, j1, k0);
    float v11 = (1 - fu) * at(i0, j1, k1) + fu * at(i1, j1, k1);
    float v0 = (1 - fv) * v00 + fv * v10;
    float v1 = (1 - fv) * v01 + fv * v11;
    return (1 - fw) * v0 + fw * v1;
}

// MapF0toIOR / MapIORtoF0 (include/bulbit/scattering.h:189-208).
__device__ __forceinline__ float MapF0toIOR(float f0)
{
    float sqrt_f0 = sqrtf(Sqr(Sqr(f0)));
    return (1 + sqrt_f0) / (1 - sqrt_f0);
}
__device__ __forceinline__ float MapIORtoF0(float ior) { return sqrtf((ior - 1) / (ior + 1)); }

// FresnelDielectricAverage (include/bulbit/scattering.h:154-172): the
// polynomial / rational fits of the hemispherical average of the dielectric
// Fresnel term from the Imageworks 2017 course notes (p. 23).
__device__ __forceinline__ float FresnelDielectricAverage(float eta_p)
{
    if (eta_p < 1)
    {
        const float eta2 = eta_p * eta_p;
        const float eta3 = eta_p * eta2;
        return 0.997118f + 0.1014f * eta_p - 0.965241f * eta2 - 0.130607f * eta3;
    }
    return (eta_p - 1) / (4.08567f + 1.00071f * eta_p);
}

struct TrowbridgeReitz
{
    float alpha_x, alpha_y;

    __device__ __forceinline__ bool EffectivelySmooth() const { return SMax(alpha_x, alpha_y) < 1e-3f; }

    // E(wo), E_avg (include/bulbit/microfacet.h:133-145).
    __device__ __forceinline__ float MeanAlpha() const { return sqrtf(alpha_x * alpha_y); }
    __device__ __forceinline__ float E(V3 wo) const
    {
        return TableBilinear(g_ggx_e, kEnergyTableSize, kEnergyTableSize, wo.z, MeanAlpha());
    }
    __device__ __forceinline__ float EAvg() const
    {
        return TableBilinear(g_ggx_e_avg, kEnergyTableSize, 1, MeanAlpha(), 0.0f);
    }

    __device__ __forceinline__ float D(V3 wm) const
    {
        float tan2_theta = Tan2Theta(wm);
        if (isinf(tan2_theta))
        {
            return 0;
        }
        float cos4_theta = Sqr(Cos2Theta(wm));
        if (cos4_theta < 1e-16f)
        {
            return 0;
        }
        float e = tan2_theta * (Sqr(CosPhi(wm) / alpha_x) + Sqr(SinPhi(wm) / alpha_y));
        return 1 / (kPi * alpha_x * alpha_y * cos4_theta * Sqr(1 + e));
    }

    __device__ __forceinline__ float Lambda(V3 w) const
    {
        float tan2_theta = Tan2Theta(w);
        if (isinf(tan2_theta))
        {
            return 0;
        }
        float alpha2 = Sqr(CosPhi(w) * alpha_x) + Sqr(SinPhi(w) * alpha_y);
        return (sqrtf(1 + alpha2 * tan2_theta) - 1) / 2;
    }

    __device__ __forceinline__ float G1(V3 w) const { return 1 / (1 + Lambda(w)); }
    __device__ __forceinline__ float G(V3 wo, V3 wi) const { return 1 / (1 + Lambda(wo) + Lambda(wi)); }
    __device__ __forceinline__ float PDF(V3 w, V3 wm) const { return G1(w) / AbsCosTheta(w) * D(wm) * AbsDot(w, wm); }
    __device__ __forceinline__ V3 SampleWm(V3 w, P2 u) const { return SampleGGXVNDF(w, alpha_x, alpha_y, u); }

    __device__ __forceinline__ void Regularize()
    {
        if (alpha_x < 0.3f) alpha_x = Clamp(2 * alpha_x, 0.1f, 0.3f);
        if (alpha_y < 0.3f) alpha_y = Clamp(2 * alpha_y, 0.1f, 0.3f);
    }
};

// ---------------------------------------------------------------- Fresnel

__device__ __forceinline__ float FresnelDielectric(float cos_theta_i, float eta)
{
    cos_theta_i = Clamp(cos_theta_i, -1, 1);
    if (cos_theta_i < 0)
    {
        eta = 1 / eta;
        cos_theta_i = -cos_theta_i;
    }
    float sin2_theta_i = 1 - Sqr(cos_theta_i);
    float sin2_theta_t = sin2_theta_i / Sqr(eta);
    if (sin2_theta_t >= 1)
    {
        return 1;
    }
    float cos_theta_t = sqrtf(SMax(0.0f, 1 - sin2_theta_t));
    float r_parl = (eta * cos_theta_i - cos_theta_t) / (eta * cos_theta_i + cos_theta_t);
    float r_perp = (cos_theta_i - eta * cos_theta_t) / (cos_theta_i + eta * cos_theta_t);
    return (Sqr(r_parl) + Sqr(r_perp)) / 2;
}

struct Cx
{
    float re, im;
};

__device__ __forceinline__ Cx CxMul(Cx a, Cx b) { return Cx{ a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re }; }
// GCC's complex float division: the textbook formula in double precision.
__device__ __forceinline__ Cx CxDiv(Cx a, Cx b)
{
    double aa = a.re, bb = a.im, cc = b.re, dd = b.im;
    double denom = cc * cc + dd * dd;
    return Cx{ float((aa * cc + bb * dd) / denom), float((bb * cc - aa * dd) / denom) };
}
__device__ __forceinline__ float CxAbs(Cx z) { return float(sqrt(double(z.re) * z.re + double(z.im) * z.im)); }
__device__ __forceinline__ float CxNorm(Cx z) { return z.re * z.re + z.im * z.im; }

// SqrtComplex (include/bulbit/scattering.h:53-74).
__device__ __forceinline__ Cx SqrtComplex(Cx z)
{
    float n = CxAbs(z);
    float t1 = sqrtf(0.5f * (n + fabsf(z.re)));
    float t2 = 0.5f * z.im / t1;
    if (n == 0)
    {
        return Cx{ 0, 0 };
    }
    if (z.re >= 0)
    {
        return Cx{ t1, t2 };
    }
    return Cx{ fabsf(t2), copysignf(t1, z.im) };
}

// FresnelComplex(cos, complex eta) (include/bulbit/scattering.h:76-95).
__device__ __forceinline__ float FresnelComplex(float cos_theta_i, Cx eta)
{
    cos_theta_i = Clamp(cos_theta_i, 0, 1);
    float sin2_theta_i = 1 - Sqr(cos_theta_i);
    Cx sin2_theta_t = CxDiv(Cx{ sin2_theta_i, 0.0f }, CxMul(eta, eta));
    Cx cos_theta_t = SqrtComplex(Cx{ 1.0f - sin2_theta_t.re, 0.0f - sin2_theta_t.im });
    Cx ec = Cx{ eta.re * cos_theta_i, eta.im * cos_theta_i };
    Cx r_parl = CxDiv(Cx{ ec.re - cos_theta_t.re, ec.im - cos_theta_t.im },
                      Cx{ ec.re + cos_theta_t.re, ec.im + cos_theta_t.im });
    Cx et = CxMul(eta, cos_theta_t);
    Cx r_perp = CxDiv(Cx{ -et.re + cos_theta_i, -et.im }, Cx{ et.re + cos_theta_i, et.im });
    return (CxNorm(r_parl) + CxNorm(r_perp)) / 2;
}

__device__ __forceinline__ Spec FresnelComplex(float cos_theta_i, const float* eta, const float* k)
{
    return Spec{ FresnelComplex(cos_theta_i, Cx{ eta[0], k[0] }), FresnelComplex(cos_theta_i, Cx{ eta[1], k[1] }),
                 FresnelComplex(cos_theta_i, Cx{ eta[2], k[2] }) };
}

// Refract (include/bulbit/scattering.h:9-40).
__device__ __forceinline__ bool Refract(V3* wt, V3 wi, V3 n, float eta, float* eta_p)
{
    float cos_theta_i = Dot(n, wi);
    if (cos_theta_i < 0)
    {
        eta = 1 / eta;
        cos_theta_i = -cos_theta_i;
        n = -n;
    }
    float sin2_theta_i = SMax(0.0f, 1 - Sqr(cos_theta_i));
    float sin2_theta_t = sin2_theta_i / Sqr(eta);
    if (sin2_theta_t >= 1)
    {
        return false;
    }
    float cos_theta_t = sqrtf(1 - sin2_theta_t);
    float inv_eta = 1 / eta;
    *wt = -wi * inv_eta + (cos_theta_i * inv_eta - cos_theta_t) * n;
    *eta_p = eta;
    return true;
}

// Schlick Fresnel of MetallicRoughnessBxDF (include/bulbit/bxdfs.h:480-493).
__device__ __forceinline__ Spec FSchlick(Spec f0, float cos_theta)
{
    return f0 + (spec(1) - f0) * dpow(1 - cos_theta, 5.0f);
}

// ---------------------------------------------------------------- BSDF

struct BSDFSample
{
    Spec f;
    V3 wi;
    float pdf;
    int32_t flags;
    float eta;
};

__device__ __forceinline__ float DotZ(V3 v) { return Dot(v, V3{ 0, 0, 1 }); }

// A BxDF bound to the shading frame (include/bulbit/bsdf.h).
struct BSDF
{
    Frame frame;
    int32_t type;
    int32_t flags;
    Spec r;          // Lambertian r / conductor reflectance / dielectric Sqrt(r) / MR color
    float eta;       // dielectric relative eta (per hit)
    const float* ceta; // conductor eta, k (3 each)
    const float* ck;
    TrowbridgeReitz mf;
    float metallic;
    int32_t ms;      // conductor / dielectric: energy compensation (multiple-scattering lobe)

    // ---- Lambertian (src/bxdf/lambertian_bxdf.cpp)
    __device__ Spec LambertF(V3 wo, V3 wi) const
    {
        if (!SameHemisphere(wo, wi)) return spec(0);
        return r * kInvPi;
    }
    __device__ float LambertPDF(V3 wo, V3 wi) const
    {
        if (!SameHemisphere(wo, wi)) return 0;
        return AbsCosTheta(wi) * kInvPi;
    }
    __device__ bool LambertSample(BSDFSample* s, V3 wo, P2 u12) const
    {
        V3 wi = SampleCosineHemisphere(u12);
        float pdf = wi.z * kInvPi;
        if (wo.z < 0) wi.z = -wi.z;
        *s = BSDFSample{ r * kInvPi, wi, pdf, kFlagDiffuse | kFlagReflection, 1 };
        return true;
    }

    // ---- Conductor (src/bxdf/conductor_bxdf.cpp)
    __device__ Spec ConductorF(V3 wo, V3 wi) const
    {
        if (!SameHemisphere(wo, wi) || mf.EffectivelySmooth()) return spec(0);
        float cos_theta_o = AbsCosTheta(wo);
        float cos_theta_i = AbsCosTheta(wi);
        if (cos_theta_i == 0 || cos_theta_o == 0) return spec(0);
        V3 wm = wo + wi;
        if (Length2(wm) == 0) return spec(0);
        NormalizeInPlace(wm);
        Spec F = FresnelComplex(AbsDot(wo, wm), ceta, ck);
        return r * F * mf.D(wm) * mf.G(wo, wi) / (4 * cos_theta_i * cos_theta_o);
    }
    __device__ float ConductorPDF(V3 wo, V3 wi) const
    {
        if (!SameHemisphere(wo, wi) || mf.EffectivelySmooth()) return 0;
        V3 wm = wo + wi;
        if (Length2(wm) == 0) return 0;
        NormalizeInPlace(wm);
        if (DotZ(wm) < 0) wm = -wm;
        return mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
    }
    __device__ bool ConductorSample(BSDFSample* s, V3 wo, P2 u12) const
    {
        if (mf.EffectivelySmooth())
        {
            V3 wi{ -wo.x, -wo.y, wo.z };
            Spec f = FresnelComplex(AbsCosTheta(wi), ceta, ck) / AbsCosTheta(wi);
            *s = BSDFSample{ r * f, wi, 1, kFlagSpecular | kFlagReflection, 1 };
            return true;
        }
        if (wo.z == 0) return false;
        V3 wm = mf.SampleWm(wo, u12);
        V3 wi = Reflect(wo, wm);
        if (!SameHemisphere(wo, wi)) return false;
        float cos_theta_o = AbsCosTheta(wo);
        float cos_theta_i = AbsCosTheta(wi);
        if (cos_theta_i == 0 || cos_theta_o == 0) return false;
        float pdf = mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
        Spec F = FresnelComplex(AbsDot(wo, wm), ceta, ck);
        Spec f = F * mf.D(wm) * mf.G(wo, wi) / (4 * cos_theta_i * cos_theta_o);
        *s = BSDFSample{ r * f, wi, pdf, kFlagGlossy | kFlagReflection, 1 };
        return true;
    }

    // ---- Energy-compensated conductor (src/bxdf/conductor_multi_scattering_bxdf.cpp):
    // the single-scattering lobe plus a diffuse-like multiple-scattering lobe
    // scaled by the lost energy (1 - E(wo)) (1 - E(wi)).
    __device__ Spec ConductorMsLobe(V3 wo, V3 wi) const
    {
        float E_avg = mf.EAvg();
        Spec F0 = FresnelComplex(1, ceta, ck);
        Spec F90 = FresnelComplex(0, ceta, ck);
        Spec fresnel_avg = (20 * F0 + F90) / 21.0f; // FresnelConductorAverage (scattering.h:174-185)
        Spec fresnel_ms = fresnel_avg * fresnel_avg * E_avg / (spec(1) - fresnel_avg * (1 - E_avg));
        return fresnel_ms * ((1 - mf.E(wo)) * (1 - mf.E(wi))) / (kPi * (1 - E_avg));
    }
    __device__ Spec ConductorMsF(V3 wo, V3 wi) const
    {
        if (!SameHemisphere(wo, wi) || mf.EffectivelySmooth()) return spec(0);
        float cos_theta_o = AbsCosTheta(wo);
        float cos_theta_i = AbsCosTheta(wi);
        if (cos_theta_i == 0 || cos_theta_o == 0) return spec(0);
        V3 wm = wo + wi;
        if (Length2(wm) == 0) return spec(0);
        NormalizeInPlace(wm);
        Spec F = FresnelComplex(AbsDot(wo, wm), ceta, ck);
        Spec f_ss = F * mf.D(wm) * mf.G(wo, wi) / (4 * cos_theta_i * cos_theta_o);
        return r * (f_ss + ConductorMsLobe(wo, wi));
    }
    __device__ float ConductorMsPDF(V3 wo, V3 wi) const
    {
        if (!SameHemisphere(wo, wi) || mf.EffectivelySmooth()) return 0;
        V3 wm = wo + wi;
        if (Length2(wm) == 0) return 0;
        NormalizeInPlace(wm);
        if (DotZ(wm) < 0) wm = -wm;
        float pdf_ss = mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
        float pdf_ms = wi.z * kInvPi; // CosineHemispherePDF(wi.z)
        float e = mf.E(wo);
        return pdf_ms * (1 - e) + pdf_ss * e; // Lerp(pdf_ms, pdf_ss, E(wo))
    }
    __device__ bool ConductorMsSample(BSDFSample* s, V3 wo, float u0, P2 u12) const
    {
        if (mf.EffectivelySmooth())
        {
            V3 wi{ -wo.x, -wo.y, wo.z };
            Spec f = FresnelComplex(AbsCosTheta(wi), ceta, ck) / AbsCosTheta(wi);
            *s = BSDFSample{ r * f, wi, 1, kFlagSpecular | kFlagReflection, 1 };
            return true;
        }
        if (wo.z == 0) return false;
        V3 wm, wi;
        int32_t flag;
        float e = mf.E(wo);
        if (u0 < e)
        {
            wm = mf.SampleWm(wo, u12);
            wi = Reflect(wo, wm);
            flag = kFlagGlossy | kFlagReflection;
        }
        else
        {
            wi = SampleCosineHemisphere(u12);
            wm = Normalize(wo + wi);
            flag = kFlagDiffuse | kFlagReflection;
        }
        if (!SameHemisphere(wo, wi)) return false;
        float cos_theta_o = AbsCosTheta(wo);
        float cos_theta_i = AbsCosTheta(wi);
        if (cos_theta_i == 0 || cos_theta_o == 0) return false;
        Spec F = FresnelComplex(AbsDot(wo, wm), ceta, ck);
        Spec f_ss = F * mf.D(wm) * mf.G(wo, wi) / (4 * cos_theta_i * cos_theta_o);
        Spec f_ms = ConductorMsLobe(wo, wi);
        float pdf_ss = mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
        float pdf_ms = wi.z * kInvPi;
        float pdf = pdf_ms * (1 - e) + pdf_ss * e;
        *s = BSDFSample{ r * (f_ss + f_ms), wi, pdf, flag, 1 };
        return true;
    }

    // ---- Dielectric (src/bxdf/dielectric_bxdf.cpp), radiance transport
    __device__ Spec DielectricF(V3 wo, V3 wi) const
    {
        if (eta == 1 || mf.EffectivelySmooth()) return spec(0);
        float cos_theta_o = wo.z;
        float cos_theta_i = wi.z;
        float eta_p = 1;
        bool reflect = cos_theta_i * cos_theta_o > 0;
        if (!reflect) eta_p = cos_theta_o > 0 ? eta : (1 / eta);
        V3 wm = wi * eta_p + wo;
        if (cos_theta_i == 0 || cos_theta_o == 0 || Length2(wm) == 0) return spec(0);
        NormalizeInPlace(wm);
        if (DotZ(wm) < 0) wm = -wm;
        if (Dot(wm, wi) * cos_theta_i < 0 || Dot(wm, wo) * cos_theta_o < 0) return spec(0);
        float F = FresnelDielectric(Dot(wo, wm), eta);
        if (reflect)
        {
            return spec(F * mf.D(wm) * mf.G(wo, wi) / fabsf(4 * cos_theta_i * cos_theta_o));
        }
        float denom = Sqr(Dot(wi, wm) + Dot(wo, wm) / eta_p) * cos_theta_i * cos_theta_o;
        float ft = (1 - F) * mf.D(wm) * mf.G(wo, wi) * fabsf(Dot(wi, wm) * Dot(wo, wm) / denom);
        ft /= Sqr(eta_p);
        return r * ft;
    }
    __device__ float DielectricPDF(V3 wo, V3 wi) const
    {
        if (eta == 1 || mf.EffectivelySmooth()) return 0;
        float cos_theta_o = wo.z;
        float cos_theta_i = wi.z;
        float eta_p = 1;
        bool reflect = cos_theta_i * cos_theta_o > 0;
        if (!reflect) eta_p = cos_theta_o > 0 ? eta : (1 / eta);
        V3 wm = wi * eta_p + wo;
        if (cos_theta_i == 0 || cos_theta_o == 0 || Length2(wm) == 0) return 0;
        NormalizeInPlace(wm);
        if (DotZ(wm) < 0) wm = -wm;
        if (Dot(wm, wi) * cos_theta_i < 0 || Dot(wm, wo) * cos_theta_o < 0) return 0;
        float R = FresnelDielectric(Dot(wo, wm), eta);
        float T = 1 - R;
        float pr = R, pt = T;
        if (pr == 0 && pt == 0) return 0;
        if (reflect)
        {
            return mf.PDF(wo, wm) / (4 * AbsDot(wo, wm)) * pr / (pr + pt);
        }
        float dwm_dwi = AbsDot(wi, wm) / Sqr(Dot(wi, wm) + Dot(wo, wm) / eta_p);
        return mf.PDF(wo, wm) * dwm_dwi * pt / (pr + pt);
    }
    // kToLight: radiance transport (the integrator); false: importance
    // transport (TransportDirection::ToCamera, the energy-table integrals),
    // which leaves out the 1 / eta'^2 solid-angle factor.
    template <bool kToLight = true>
    __device__ bool DielectricSample(BSDFSample* s, V3 wo, float u0, P2 u12) const
    {
        if (eta == 1 || mf.EffectivelySmooth())
        {
            float R = FresnelDielectric(wo.z, eta);
            float T = 1 - R;
            float pr = R, pt = T;
            if (pr == 0 && pt == 0) return false;
            if (u0 < pr / (pr + pt))
            {
                V3 wi{ -wo.x, -wo.y, wo.z };
                Spec fr = spec(R / AbsCosTheta(wi));
                *s = BSDFSample{ fr, wi, pr / (pr + pt), kFlagSpecular | kFlagReflection, 1 };
            }
            else
            {
                V3 wi;
                float eta_p;
                if (!Refract(&wi, wo, V3{ 0, 0, 1 }, eta, &eta_p)) return false;
                float ft = T / AbsCosTheta(wi);
                if (kToLight) ft /= Sqr(eta_p);
                *s = BSDFSample{ r * ft, wi, pt / (pr + pt), kFlagSpecular | kFlagTransmission, eta_p };
            }
            return true;
        }
        V3 wm = mf.SampleWm(wo, u12);
        float R = FresnelDielectric(Dot(wo, wm), eta);
        float T = 1 - R;
        float pr = R, pt = T;
        if (pr == 0 && pt == 0) return false;
        if (u0 < pr / (pr + pt))
        {
            V3 wi = Reflect(wo, wm);
            if (!SameHemisphere(wo, wi)) return false;
            float pdf = mf.PDF(wo, wm) / (4 * AbsDot(wo, wm)) * pr / (pr + pt);
            Spec fr = spec(R * mf.D(wm) * mf.G(wo, wi) / (4 * wi.z * wo.z));
            *s = BSDFSample{ fr, wi, pdf, kFlagGlossy | kFlagReflection, 1 };
        }
        else
        {
            float eta_p = 1;
            V3 wi{ 0, 0, 0 };
            bool tir = !Refract(&wi, wo, wm, eta, &eta_p);
            if (tir || SameHemisphere(wo, wi) || wi.z == 0) return false;
            float denom = Sqr(Dot(wi, wm) + Dot(wo, wm) / eta_p);
            float dwm_dwi = AbsDot(wi, wm) / denom;
            float pdf = mf.PDF(wo, wm) * dwm_dwi * pt / (pr + pt);
            float ft = T * mf.D(wm) * mf.G(wo, wi) * fabsf(Dot(wi, wm) * Dot(wo, wm) / (wi.z * wo.z * denom));
            if (kToLight) ft /= Sqr(eta_p);
            *s = BSDFSample{ r * ft, wi, pdf, kFlagGlossy | kFlagTransmission, eta_p };
        }
        return true;
    }

    // ---- Energy-compensated dielectric (src/bxdf/dielectric_multi_scattering_bxdf.cpp,
    // include/bulbit/bxdfs.h:145-240), radiance transport: the rough
    // dielectric plus a diffuse-like multiple-scattering lobe on each side,
    // reflection and transmission split by the energy-conserving ratio.
    __device__ float DmsE(V3 w, float e) const
    {
        if (e >= 1)
        {
            return TableTrilinear(g_dms_e, kEnergyTableSize, MapIORtoF0(e), fabsf(w.z), mf.MeanAlpha());
        }
        return TableTrilinear(g_dms_e_inv, kEnergyTableSize, MapIORtoF0(1 / e), fabsf(w.z), mf.MeanAlpha());
    }
    __device__ float DmsEAvg(float e) const
    {
        if (e >= 1)
        {
            return TableBilinear(g_dms_e_avg, kEnergyTableSize, kEnergyTableSize, MapIORtoF0(e), mf.MeanAlpha());
        }
        return TableBilinear(g_dms_e_inv_avg, kEnergyTableSize, kEnergyTableSize, MapIORtoF0(1 / e),
                             mf.MeanAlpha());
    }
    // ComputeScatteringRatio (include/bulbit/bxdfs.h:222-242): the share of
    // the multiple-scattering energy leaving on wo's side.
    __device__ float DmsRatio(float eta_o) const
    {
        float eta_i = eta >= 1 ? eta : 1 / eta;
        float eta_t = 1 / eta_i;
        float a = (1 - FresnelDielectricAverage(eta_i)) / (1 - DmsEAvg(eta_t));
        float b = Sqr(eta_i) * (1 - FresnelDielectricAverage(eta_t)) / (1 - DmsEAvg(eta_i));
        float x = 1 / (a / b + 1);
        if (eta_o >= 1)
        {
            return 1 - x * (1 - FresnelDielectricAverage(eta_o));
        }
        return 1 - (1 - x) * (1 - FresnelDielectricAverage(eta_o));
    }
    __device__ float DmsReflectLobe(V3 wo, V3 wi, float eta_o, float ratio) const
    {
        return ratio * (1 - DmsE(wi, eta_o)) * (1 - DmsE(wo, eta_o)) / fmaxf(1e-4f, kPi * (1 - DmsEAvg(eta_o)));
    }
    __device__ float DmsTransmitLobe(V3 wo, V3 wi, float eta_o, float eta_i, float ratio) const
    {
        return (1 - ratio) * (1 - DmsE(wi, eta_i)) * (1 - DmsE(wo, eta_o)) /
               fmaxf(1e-4f, kPi * (1 - DmsEAvg(eta_i)));
    }
    // Lerp(pdf_ms, pdf_ss, E_o) (include/bulbit/math.h:87-90).
    __device__ static float DmsLerp(float pdf_ms, float pdf_ss, float e_o) { return pdf_ms * (1 - e_o) + pdf_ss * e_o; }

    __device__ Spec DielectricMsF(V3 wo, V3 wi) const
    {
        if (eta == 1 || mf.EffectivelySmooth()) return spec(0);
        float cos_theta_o = wo.z;
        float cos_theta_i = wi.z;
        float eta_p = 1;
        bool reflect = cos_theta_i * cos_theta_o > 0;
        if (!reflect) eta_p = cos_theta_o > 0 ? eta : (1 / eta);
        float eta_o = cos_theta_o > 0 ? eta : 1 / eta;
        float eta_i = cos_theta_o > 0 ? 1 / eta : eta;
        V3 wm = wi * eta_p + wo;
        if (cos_theta_i == 0 || cos_theta_o == 0 || Length2(wm) == 0) return spec(0);
        NormalizeInPlace(wm);
        if (DotZ(wm) < 0) wm = -wm;
        if (Dot(wm, wi) * cos_theta_i < 0 || Dot(wm, wo) * cos_theta_o < 0) return spec(0);
        float ratio = DmsRatio(eta_o);
        float F = FresnelDielectric(Dot(wo, wm), eta);
        if (reflect)
        {
            float fr_ss = F * mf.D(wm) * mf.G(wo, wi) / (4 * cos_theta_i * cos_theta_o);
            return spec(fr_ss + DmsReflectLobe(wo, wi, eta_o, ratio));
        }
        float denom = Sqr(Dot(wi, wm) + Dot(wo, wm) / eta_p);
        float ft_ss =
            (1 - F) * mf.D(wm) * mf.G(wo, wi) * fabsf(Dot(wi, wm) * Dot(wo, wm) / (cos_theta_i * cos_theta_o * denom));
        float ft_ms = DmsTransmitLobe(wo, wi, eta_o, eta_i, ratio);
        ft_ss /= Sqr(eta_p);
        return r * (ft_ss + ft_ms);
    }
    __device__ float DielectricMsPDF(V3 wo, V3 wi) const
    {
        if (eta == 1 || mf.EffectivelySmooth()) return 0;
        float cos_theta_o = wo.z;
        float cos_theta_i = wi.z;
        float eta_p = 1;
        bool reflect = cos_theta_i * cos_theta_o > 0;
        if (!reflect) eta_p = cos_theta_o > 0 ? eta : (1 / eta);
        float eta_o = cos_theta_o > 0 ? eta : 1 / eta;
        V3 wm = wi * eta_p + wo;
        if (cos_theta_i == 0 || cos_theta_o == 0 || Length2(wm) == 0) return 0;
        NormalizeInPlace(wm);
        if (DotZ(wm) < 0) wm = -wm;
        if (Dot(wm, wi) * cos_theta_i < 0 || Dot(wm, wo) * cos_theta_o < 0) return 0;
        float ratio = DmsRatio(eta_o);
        float E_o = Clamp(DmsE(wo, eta_o), 1e-4f, 1 - 1e-4f);
        float R = FresnelDielectric(Dot(wo, wm), eta);
        float T = 1 - R;
        float pr_ss = R, pt_ss = T;
        float pr_ms = ratio, pt_ms = 1 - ratio;
        if (pr_ss == 0 && pt_ss == 0 && pr_ms == 0 && pt_ms == 0) return 0;
        float p_ss_sum = pr_ss + pt_ss;
        float p_ms_sum = pr_ms + pt_ms;
        pr_ss /= p_ss_sum;
        pt_ss /= p_ss_sum;
        pr_ms /= p_ms_sum;
        pt_ms /= p_ms_sum;
        if (reflect)
        {
            float pdf_ss = pr_ss * mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
            float pdf_ms = pr_ms * (AbsCosTheta(wi) * kInvPi);
            return DmsLerp(pdf_ms, pdf_ss, E_o);
        }
        float dwm_dwi = AbsDot(wi, wm) / Sqr(Dot(wi, wm) + Dot(wo, wm) / eta_p);
        float pdf_ss = pt_ss * mf.PDF(wo, wm) * dwm_dwi;
        float pdf_ms = pt_ms * (AbsCosTheta(wi) * kInvPi);
        return DmsLerp(pdf_ms, pdf_ss, E_o);
    }
    __device__ bool DielectricMsSample(BSDFSample* s, V3 wo, float u0, P2 u12) const
    {
        if (eta == 1 || mf.EffectivelySmooth())
        {
            // The perfect specular branch is DielectricBxDF's.
            return DielectricSample(s, wo, u0, u12);
        }
        float eta_o = wo.z > 0 ? eta : 1 / eta;
        float eta_i = wo.z > 0 ? 1 / eta : eta;
        float ratio = DmsRatio(eta_o);
        float E_o = Clamp(DmsE(wo, eta_o), 1e-4f, 1 - 1e-4f);
        if (u0 < E_o)
        {
            // single scattering: a visible microfacet normal, then reflect or refract
            V3 wm = mf.SampleWm(wo, u12);
            NormalizeInPlace(wm);
            if (DotZ(wm) < 0) wm = -wm;
            float R = FresnelDielectric(Dot(wo, wm), eta);
            float T = 1 - R;
            float pr_ss = R, pt_ss = T;
            float pr_ms = ratio, pt_ms = 1 - ratio;
            if (pr_ss == 0 && pt_ss == 0) return false;
            float p_ss_sum = pr_ss + pt_ss;
            float p_ms_sum = pr_ms + pt_ms;
            pr_ss /= p_ss_sum;
            pt_ss /= p_ss_sum;
            pr_ms /= p_ms_sum;
            pt_ms /= p_ms_sum;
            u0 /= E_o;
            if (u0 < pr_ss)
            {
                V3 wi = Reflect(wo, wm);
                if (!SameHemisphere(wo, wi)) return false;
                float pdf_ss = pr_ss * mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
                float pdf_ms = pr_ms * (AbsCosTheta(wi) * kInvPi);
                float fr_ss = R * mf.D(wm) * mf.G(wo, wi) / (4 * wi.z * wo.z);
                float fr_ms = DmsReflectLobe(wo, wi, eta_o, ratio);
                *s = BSDFSample{ spec(fr_ss + fr_ms), wi, DmsLerp(pdf_ms, pdf_ss, E_o), kFlagGlossy | kFlagReflection, 1 };
                return true;
            }
            V3 wi{ 0, 0, 0 };
            float unused;
            bool tir = !Refract(&wi, wo, wm, eta, &unused);
            if (SameHemisphere(wo, wi) || wi.z == 0 || tir) return false;
            float eta_p = wo.z > 0 ? eta : (1 / eta);
            float denom = Sqr(Dot(wi, wm) + Dot(wo, wm) / eta_p);
            float dwm_dwi = AbsDot(wi, wm) / denom;
            float pdf_ss = pt_ss * mf.PDF(wo, wm) * dwm_dwi;
            float pdf_ms = pt_ms * (AbsCosTheta(wi) * kInvPi);
            float ft_ss =
                T * mf.D(wm) * mf.G(wo, wi) * fabsf(Dot(wi, wm) * Dot(wo, wm) / (wi.z * wo.z * denom));
            float ft_ms = DmsTransmitLobe(wo, wi, eta_o, eta_i, ratio);
            ft_ss /= Sqr(eta_p);
            *s = BSDFSample{ r * (ft_ss + ft_ms), wi, DmsLerp(pdf_ms, pdf_ss, E_o), kFlagGlossy | kFlagTransmission,
                             eta_p };
            return true;
        }
        // multiple scattering: a cosine-distributed direction on one side
        float pr_ms = ratio, pt_ms = 1 - ratio;
        if (pr_ms == 0 && pt_ms == 0) return false;
        float p_ms_sum = pr_ms + pt_ms;
        pr_ms /= p_ms_sum;
        pt_ms /= p_ms_sum;
        u0 = (u0 - E_o) / (1 - E_o);
        V3 wi = SampleCosineHemisphere(u12);
        if (u0 < pr_ms)
        {
            if (wo.z < 0) wi = -wi;
            V3 wm = Normalize(wi + wo);
            float R = FresnelDielectric(Dot(wo, wm), eta);
            float pr_ss = R, pt_ss = 1 - R;
            float p_ss_sum = pr_ss + pt_ss;
            pr_ss /= p_ss_sum;
            pt_ss /= p_ss_sum;
            float pdf_ss = pr_ss * mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
            float pdf_ms = pr_ms * (AbsCosTheta(wi) * kInvPi);
            float fr_ss = R * mf.D(wm) * mf.G(wo, wi) / (4 * wi.z * wo.z);
            float fr_ms = DmsReflectLobe(wo, wi, eta_o, ratio);
            *s = BSDFSample{ spec(fr_ss + fr_ms), wi, DmsLerp(pdf_ms, pdf_ss, E_o), kFlagDiffuse | kFlagReflection, 1 };
            return true;
        }
        if (wo.z > 0) wi = -wi;
        V3 wm = Normalize(wi * eta_o + wo);
        if (DotZ(wm) < 0) wm = -wm;
        float R = FresnelDielectric(Dot(wo, wm), eta);
        float T = 1 - R;
        float pr_ss = R, pt_ss = 1 - R;
        float p_ss_sum = pr_ss + pt_ss;
        pr_ss /= p_ss_sum;
        pt_ss /= p_ss_sum;
        float denom = Sqr(Dot(wi, wm) + Dot(wo, wm) / eta_o);
        float dwm_dwi = AbsDot(wi, wm) / denom;
        float pdf_ss = pt_ss * mf.PDF(wo, wm) * dwm_dwi;
        float pdf_ms = pt_ms * (AbsCosTheta(wi) * kInvPi);
        float ft_ss = T * mf.D(wm) * mf.G(wo, wi) * fabsf(Dot(wi, wm) * Dot(wo, wm) / (wi.z * wo.z * denom));
        float ft_ms = DmsTransmitLobe(wo, wi, eta_o, eta_i, ratio);
        ft_ss /= Sqr(eta_o);
        *s = BSDFSample{ r * (ft_ss + ft_ms), wi, DmsLerp(pdf_ms, pdf_ss, E_o), kFlagDiffuse | kFlagTransmission, eta_o };
        return true;
    }

    // ---- Metallic-roughness (src/bxdf/metallic_roughness_bxdf.cpp)
    __device__ Spec MRF0() const { return (1 - metallic) * spec(0.04f) + metallic * r; }
    __device__ Spec MRF(V3 wo, V3 wi) const
    {
        if (!SameHemisphere(wo, wi)) return spec(0);
        float cos_theta_o = AbsCosTheta(wo);
        float cos_theta_i = AbsCosTheta(wi);
        if (cos_theta_i == 0 || cos_theta_o == 0) return spec(0);
        V3 wm = wo + wi;
        if (Length2(wm) == 0) return spec(0);
        NormalizeInPlace(wm);
        Spec F = FSchlick(MRF0(), Dot(wi, wm));
        Spec f_s = F * mf.D(wm) * mf.G(wo, wi) / (4 * cos_theta_i * cos_theta_o);
        Spec f_d = (1 - metallic) * (spec(1) - F) * (r * kInvPi);
        return f_d + f_s;
    }
    __device__ float MRPDF(V3 wo, V3 wi) const
    {
        if (!SameHemisphere(wo, wi) || mf.EffectivelySmooth()) return 0;
        V3 wm = wo + wi;
        if (Length2(wm) == 0) return 0;
        NormalizeInPlace(wm);
        if (DotZ(wm) < 0) wm = -wm;
        float R = FresnelDielectric(Dot(wo, wm), 1.5f);
        float T = 1 - R;
        float pr = R;
        float pt = T * (1 - metallic);
        if (pr == 0 && pt == 0) return 0;
        float p_sum = pr + pt;
        pr /= p_sum;
        pt /= p_sum;
        float pdf_r = mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
        float pdf_d = AbsCosTheta(wi) * kInvPi;
        return pr * pdf_r + pt * pdf_d;
    }
    __device__ bool MRSample(BSDFSample* s, V3 wo, float u0, P2 u12) const
    {
        if (wo.z == 0) return false;
        V3 wm = mf.SampleWm(wo, u12);
        V3 wi = Reflect(wo, wm);
        float R = FresnelDielectric(Dot(wo, wm), 1.5f);
        float T = 1 - R;
        float pr = R;
        float pt = T * (1 - metallic);
        if (pr == 0 && pt == 0) return false;
        float p_sum = pr + pt;
        pr /= p_sum;
        pt /= p_sum;
        int32_t flag;
        if (u0 < pr)
        {
            if (!SameHemisphere(wo, wi)) return false;
            flag = kFlagGlossy | kFlagReflection;
        }
        else
        {
            wi = SampleCosineHemisphere(u12);
            wm = Normalize(wi + wo);
            flag = kFlagDiffuse | kFlagReflection;
        }
        float cos_theta_o = AbsCosTheta(wo);
        float cos_theta_i = AbsCosTheta(wi);
        if (cos_theta_i == 0 || cos_theta_o == 0) return false;
        Spec F = FSchlick(MRF0(), Dot(wi, wm));
        Spec f_r = F * mf.D(wm) * mf.G(wo, wi) / (4 * cos_theta_i * cos_theta_o);
        Spec f_d = (1 - metallic) * (spec(1) - F) * (r * kInvPi);
        float pdf_r = mf.PDF(wo, wm) / (4 * AbsDot(wo, wm));
        float pdf_d = cos_theta_i * kInvPi;
        *s = BSDFSample{ f_r + f_d, wi, pr * pdf_r + pt * pdf_d, flag, 1 };
        return true;
    }

    // ---- dispatch + world/local (include/bulbit/bsdf.h:73-125)
    __device__ Spec F(V3 wo_w, V3 wi_w) const
    {
        V3 wi = frame.ToLocal(wi_w);
        V3 wo = frame.ToLocal(wo_w);
        if (wo.z == 0) return spec(0);
        switch (type)
        {
        case BBG_MAT_DIFFUSE: return LambertF(wo, wi);
        case BBG_MAT_CONDUCTOR: return ms ? ConductorMsF(wo, wi) : ConductorF(wo, wi);
        case BBG_MAT_DIELECTRIC: return ms ? DielectricMsF(wo, wi) : DielectricF(wo, wi);
        default: return MRF(wo, wi);
        }
    }
    __device__ float PDF(V3 wo_w, V3 wi_w) const
    {
        V3 wo = frame.ToLocal(wo_w);
        V3 wi = frame.ToLocal(wi_w);
        if (wo.z == 0) return 0;
        switch (type)
        {
        case BBG_MAT_DIFFUSE: return LambertPDF(wo, wi);
        case BBG_MAT_CONDUCTOR: return ms ? ConductorMsPDF(wo, wi) : ConductorPDF(wo, wi);
        case BBG_MAT_DIELECTRIC: return ms ? DielectricMsPDF(wo, wi) : DielectricPDF(wo, wi);
        default: return MRPDF(wo, wi);
        }
    }
    __device__ bool Sample(BSDFSample* s, V3 wo_w, float u0, P2 u12) const
    {
        V3 wo = frame.ToLocal(wo_w);
        if (wo.z == 0 || !(flags & (kFlagReflection | kFlagTransmission))) return false;
        bool ok;
        switch (type)
        {
        case BBG_MAT_DIFFUSE: ok = LambertSample(s, wo, u12); break;
        case BBG_MAT_CONDUCTOR: ok = ms ? ConductorMsSample(s, wo, u0, u12) : ConductorSample(s, wo, u12); break;
        case BBG_MAT_DIELECTRIC: ok = ms ? DielectricMsSample(s, wo, u0, u12) : DielectricSample(s, wo, u0, u12); break;
        default: ok = MRSample(s, wo, u0, u12); break;
        }
        if (!ok) return false;
        if (IsBlack(s->f) || s->pdf == 0 || s->wi.z == 0) return false;
        s->wi = frame.FromLocal(s->wi);
        return true;
    }
};

// Material::GetBSDF for the four supported materials; `front_face` selects
// the dielectric's relative eta (src/material/dielectric_material.cpp:30).
__device__ __forceinline__ BSDF MakeBSDF(const MaterialDev& m, V3 shading_n, V3 shading_t, bool front_face)
{
    BSDF b;
    b.frame = FrameFromXZ(shading_t, shading_n);
    b.type = m.type;
    b.r = Spec{ m.r[0], m.r[1], m.r[2] };
    b.mf = TrowbridgeReitz{ m.alpha_x, m.alpha_y };
    b.metallic = m.metallic;
    b.ceta = m.eta;
    b.ck = m.k;
    b.ms = m.ms;
    b.eta = 1;
    b.flags = m.flags;
    if (m.type == BBG_MAT_DIELECTRIC)
    {
        float eta = m.eta[0];
        b.eta = front_face ? eta : 1 / eta;
        int32_t f = (b.eta == 1) ? kFlagTransmission : (kFlagReflection | kFlagTransmission);
        b.flags = f | (b.mf.EffectivelySmooth() ? kFlagSpecular : kFlagGlossy);
    }
    return b;
}

__device__ __forceinline__ bool IsNonSpecular(int32_t flags) { return (flags & (kFlagDiffuse | kFlagGlossy)) != 0; }

// BSDF::Regularize (include/bulbit/bsdf.h:134): widen the microfacet lobe,
// then the flags the BxDF reports for the new roughness.
__device__ __forceinline__ void RegularizeBSDF(BSDF* b)
{
    b->mf.Regularize();
    if (b->type == BBG_MAT_CONDUCTOR)
    {
        b->flags = b->mf.EffectivelySmooth() ? (kFlagSpecular | kFlagReflection) : (kFlagGlossy | kFlagReflection);
    }
    else if (b->type == BBG_MAT_DIELECTRIC)
    {
        int32_t f = (b->eta == 1) ? kFlagTransmission : (kFlagReflection | kFlagTransmission);
        b->flags = f | (b->mf.EffectivelySmooth() ? kFlagSpecular : kFlagGlossy);
    }
}

} // namespace bbg
