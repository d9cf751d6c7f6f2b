// Neural path guiding: a small MLP that maps a shading point to an 8-lobe
// von Mises-Fisher mixture over directions, sampled in one-sample MIS with the
// BSDF. No counterpart in the reference renderer; the plain path tracer is
// its fallback and the yardstick of its error.
//
// Network: 80 inputs -> 64 -> 64 -> 64 (ReLU) -> 40 outputs, BF16 weights and
// activations, FP32 accumulation, FP32 biases and master weights. Inference
// runs on tcgen05.mma (128-query tiles, accumulators in tensor memory); the
// training pass's per-sample forward and backward on mma.sync m16n8k16 tiles
// of 16 samples, its weight gradients on tcgen05.mma.
//   inputs  [0, 72): sin / cos(2^k * pi * p_a) for axis a, k = 0..11, where p
//                    is the position scaled to [0, 1] by the scene bounds
//           [72, 75) shading normal, [75, 78) outgoing direction wo,
//           78 roughness (mean microfacet alpha, 1 for Lambertian), 79 = 1
//   outputs 5 per lobe j: weight logit, unnormalised mean (3), log kappa
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "dev_math.cuh"

namespace bbg
{

constexpr int kGuideIn = 80;
constexpr int kGuideHidden = 64;
constexpr int kGuideOut = 40;
constexpr int kGuideOutPad = 48; // output rows padded to a multiple of 16 for the backward MMAs
constexpr int kLobes = 8;
constexpr int kGuideRaw = 10;    // raw query: p(3), n(3), wo(3), roughness

// Parameter offsets in the FP32 master vector: W0 b0 W1 b1 W2 b2 W3 b3,
// each W stored [out][in].
constexpr int kW0 = 0;
constexpr int kB0 = kW0 + kGuideHidden * kGuideIn;      // 5120
constexpr int kW1 = kB0 + kGuideHidden;                  // 5184
constexpr int kB1 = kW1 + kGuideHidden * kGuideHidden;   // 9280
constexpr int kW2 = kB1 + kGuideHidden;                  // 9344
constexpr int kB2 = kW2 + kGuideHidden * kGuideHidden;   // 13440
constexpr int kW3 = kB2 + kGuideHidden;                  // 13504
constexpr int kB3 = kW3 + kGuideOut * kGuideHidden;      // 16064
constexpr int kGuideParams = kB3 + kGuideOut;            // 16104

// Biases packed together (as staged in shared memory by the kernels).
constexpr int kCB0 = 0;
constexpr int kCB1 = kCB0 + kGuideHidden;
constexpr int kCB2 = kCB1 + kGuideHidden;
constexpr int kCB3 = kCB2 + kGuideHidden;
constexpr int kCBias = kCB3 + kGuideOut; // 232

// BF16 weight images used by the kernels: forward layout [out][in] and the
// transposed [in][out] layout for the backward pass (W3 transposed padded to
// 48 columns with zeros).
// The forward image (W0..W3, offsets kBf0..kBf3) is stored in MMA fragment
// order, so a B fragment is one conflict-free 8-byte shared-memory load: for
// a layer of N outputs (NT = N/8 tiles) and K inputs, element
// ((kt * NT + nt) * 32 + lane) * 4 + e holds W[n][k] with n = nt*8 + lane/4
// and k = kt*16 + 2*(lane%4) + {0, 1, 8, 9}[e]. The transposed images
// (kBfT1..kBfT3, backward pass) are row-major.
constexpr int kBf0 = 0;
constexpr int kBf1 = kBf0 + kGuideHidden * kGuideIn;
constexpr int kBf2 = kBf1 + kGuideHidden * kGuideHidden;
constexpr int kBf3 = kBf2 + kGuideHidden * kGuideHidden;
constexpr int kBfFwd = kBf3 + kGuideOut * kGuideHidden;  // 15872
constexpr int kBfT1 = kBfFwd;                            // W1^T [64][64]
constexpr int kBfT2 = kBfT1 + kGuideHidden * kGuideHidden;
constexpr int kBfT3 = kBfT2 + kGuideHidden * kGuideHidden; // W3^T [64][48]
constexpr int kBfAll = kBfT3 + kGuideHidden * kGuideOutPad;
// The forward image for the fifth-generation tensor cores (the inference
// kernels), after the images above: each layer's W [n][k] as the B operand of
// tcgen05.mma in the canonical K-major layout without swizzle, 8 x 8 core
// matrices (8 rows of 16 bytes), 8-row groups 128 bytes apart and 8-column
// groups (N / 8) * 128 bytes apart: element (n, k) at
// (k / 8) * (N / 8) * 64 + (n / 8) * 64 + (n % 8) * 8 + k % 8. W3 is padded to
// N = 48 rows with zeros (the MMA's N is a multiple of 16).
constexpr int kTcW0 = 0;
constexpr int kTcW1 = kTcW0 + kGuideHidden * kGuideIn;
constexpr int kTcW2 = kTcW1 + kGuideHidden * kGuideHidden;
constexpr int kTcW3 = kTcW2 + kGuideHidden * kGuideHidden;
constexpr int kTcImage = kTcW3 + kGuideOutPad * kGuideHidden; // 16384 values, 32 KB
constexpr int kBfTc = kBfAll;                                  // offset of that image in the buffer
constexpr int kBfBuf = kBfTc + kTcImage;                       // all BF16 images of a guide

constexpr float kKappaLogMin = -2.0f;
constexpr float kKappaLogMax = 7.0f;

struct GuideBounds
{
    float lo[3];
    float inv_extent[3];
};

// sin/cos(2^k pi x) for octaves k = k0 .. k0 + count - 1, handed to
// put(j0 + 2 i, sin, cos): sincospif at every fourth octave, the octaves
// between by the double-angle identities sin 2y = 2 sin y cos y,
// cos 2y = 1 - 2 sin^2 y (each doubling at most doubles the absolute error,
// so three steps keep it within a few float ulps of 1, far below the
// features' BF16 rounding). An octave's value depends only on x and k, not
// on where a run starts.
template <class Put>
__device__ __forceinline__ void GuideOctaves(float x, int k0, int count, int j0, Put&& put)
{
    float s = 0, c = 1;
#pragma unroll
    for (int i = 0; i < count; ++i)
    {
        const int k = k0 + i;
        if (i == 0 || (k & 3) == 0)
        {
            sincospif(x * float(1 << k), &s, &c);
        }
        else
        {
            const float s2 = 2.0f * s * c;
            c = 1.0f - 2.0f * s * s;
            s = s2;
        }
        put(j0 + 2 * i, s, c);
    }
}

// Features 40 half .. 40 half + 39 of a raw query (p, n, wo, roughness),
// handed in pairs to put(j, value j, value j + 1) for j = 0, 2, .., 38.
// The 80 features: f < 72 is sin (f even) or cos (f odd) of 2^k pi p_a, with
// axis a = f / 24, octave k = (f % 24) / 2 and p_a the position normalised to
// the scene bounds; then n (3), wo (3), the roughness and a constant 1. Half
// 0 holds axis 0's octaves and axis 1's octaves 0-7, half 1 axis 1's
// octaves 8-11, axis 2's and the rest.
template <class Put>
__device__ __forceinline__ void GuideFeatures40(const float* raw, const GuideBounds& b, int half, Put&& put)
{
    if (half == 0)
    {
        GuideOctaves((raw[0] - b.lo[0]) * b.inv_extent[0], 0, 12, 0, put);
        GuideOctaves((raw[1] - b.lo[1]) * b.inv_extent[1], 0, 8, 24, put);
    }
    else
    {
        GuideOctaves((raw[1] - b.lo[1]) * b.inv_extent[1], 8, 4, 0, put);
        GuideOctaves((raw[2] - b.lo[2]) * b.inv_extent[2], 0, 12, 8, put);
        put(32, raw[3], raw[4]);
        put(34, raw[5], raw[6]);
        put(36, raw[7], raw[8]);
        put(38, raw[9], 1.0f);
    }
}

__device__ __forceinline__ uint32_t PackBf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// D = A * B + D, m16n8k16, BF16 inputs, FP32 accumulation.
__device__ __forceinline__ void Mma16816(float* d, const uint32_t* a, uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                 "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B fragment of an m16n8k16 MMA from a matrix stored [n][k] (k contiguous),
// row stride ld elements: (k = 2t, 2t+1 | 2t+8, 2t+9; n = g).
__device__ __forceinline__ void LoadB(const __nv_bfloat16* w, int ld, int n0, int k0, int lane, uint32_t* b0,
                                      uint32_t* b1)
{
    int g = lane >> 2, t = lane & 3;
    const __nv_bfloat16* row = w + (n0 + g) * ld + k0 + 2 * t;
    *b0 = *reinterpret_cast<const uint32_t*>(row);
    *b1 = *reinterpret_cast<const uint32_t*>(row + 8);
}

// B fragment (b0, b1) of tile (nt, kt) from a fragment-ordered image.
__device__ __forceinline__ void LoadBFrag(const __nv_bfloat16* w, int n_tiles, int nt, int kt, int lane, uint32_t* b0,
                                          uint32_t* b1)
{
    uint2 v = *reinterpret_cast<const uint2*>(w + ((kt * n_tiles + nt) * 32 + lane) * 4);
    *b0 = v.x;
    *b1 = v.y;
}

// Row stride (elements) of the [16][80] feature tiles in shared memory:
// 44 words, so the 8 rows an A-fragment load touches fall in distinct banks.
constexpr int kXLd = 88;

// A fragment from a matrix stored [m][k] (k contiguous), row stride ld.
__device__ __forceinline__ void LoadA(const __nv_bfloat16* x, int ld, int m0, int k0, int lane, uint32_t* a)
{
    int g = lane >> 2, t = lane & 3;
    const __nv_bfloat16* r0 = x + (m0 + g) * ld + k0 + 2 * t;
    const __nv_bfloat16* r1 = x + (m0 + g + 8) * ld + k0 + 2 * t;
    a[0] = *reinterpret_cast<const uint32_t*>(r0);
    a[1] = *reinterpret_cast<const uint32_t*>(r1);
    a[2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
    a[3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
}

// One hidden layer of K inputs -> 64 outputs for the warp's 16 rows: A
// fragments in, ReLU'd accumulators out (as the next layer's A fragments).
template <int KT>
__device__ __forceinline__ void HiddenLayer(const uint32_t (&a)[KT][4], const __nv_bfloat16* w, const float* bias,
                                            int lane, float (&acc)[8][4])
{
    int t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
    {
        float b0 = bias[nt * 8 + 2 * t], b1 = bias[nt * 8 + 2 * t + 1];
        acc[nt][0] = b0;
        acc[nt][1] = b1;
        acc[nt][2] = b0;
        acc[nt][3] = b1;
    }
#pragma unroll
    for (int kt = 0; kt < KT; ++kt)
    {
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
        {
            uint32_t b0, b1;
            LoadBFrag(w, 8, nt, kt, lane, &b0, &b1);
            Mma16816(acc[nt], a[kt], b0, b1);
        }
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
    {
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            acc[nt][i] = fmaxf(acc[nt][i], 0.0f);
        }
    }
}

// Accumulators of 64 columns -> A fragments of a K = 64 layer.
__device__ __forceinline__ void AccToA(const float (&acc)[8][4], uint32_t (&a)[4][4])
{
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
    {
        a[kt][0] = PackBf16(acc[2 * kt][0], acc[2 * kt][1]);
        a[kt][1] = PackBf16(acc[2 * kt][2], acc[2 * kt][3]);
        a[kt][2] = PackBf16(acc[2 * kt + 1][0], acc[2 * kt + 1][1]);
        a[kt][3] = PackBf16(acc[2 * kt + 1][2], acc[2 * kt + 1][3]);
    }
}

// Output layer 64 -> 40 (no activation).
__device__ __forceinline__ void OutputLayer(const uint32_t (&a)[4][4], const __nv_bfloat16* w, const float* bias,
                                            int lane, float (&out)[5][4])
{
    int t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 5; ++nt)
    {
        float b0 = bias[nt * 8 + 2 * t], b1 = bias[nt * 8 + 2 * t + 1];
        out[nt][0] = b0;
        out[nt][1] = b1;
        out[nt][2] = b0;
        out[nt][3] = b1;
    }
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
    {
#pragma unroll
        for (int nt = 0; nt < 5; ++nt)
        {
            uint32_t b0, b1;
            LoadBFrag(w, 5, nt, kt, lane, &b0, &b1);
            Mma16816(out[nt], a[kt], b0, b1);
        }
    }
}

// ---------------------------------------------------------------- vMF mixture

struct VmfMixture
{
    float logw[kLobes]; // log mixture weight (log-softmax of the logits)
    V3 mu[kLobes];
    float kappa[kLobes];
};

// log of the vMF normalisation kappa / (2 pi (1 - exp(-2 kappa))).
__device__ __forceinline__ float VmfLogNorm(float kappa)
{
    return logf(kappa) - logf(kTwoPi) - log1pf(-expf(-2.0f * kappa));
}

__device__ __forceinline__ VmfMixture MakeMixture(const float* o)
{
    VmfMixture m;
    float mx = -INFINITY;
#pragma unroll
    for (int j = 0; j < kLobes; ++j)
    {
        mx = fmaxf(mx, o[5 * j]);
    }
    float s = 0;
#pragma unroll
    for (int j = 0; j < kLobes; ++j)
    {
        s += expf(o[5 * j] - mx);
    }
    float lse = mx + logf(s);
#pragma unroll
    for (int j = 0; j < kLobes; ++j)
    {
        m.logw[j] = o[5 * j] - lse;
        V3 v{ o[5 * j + 1], o[5 * j + 2], o[5 * j + 3] };
        float len = fmaxf(Length(v), 1e-6f);
        m.mu[j] = v / len;
        m.kappa[j] = expf(Clamp(o[5 * j + 4], kKappaLogMin, kKappaLogMax));
    }
    return m;
}

__device__ __forceinline__ float MixturePdf(const VmfMixture& m, V3 w)
{
    float p = 0;
#pragma unroll
    for (int j = 0; j < kLobes; ++j)
    {
        float k = m.kappa[j];
        p += expf(m.logw[j] + VmfLogNorm(k) + k * (Dot(m.mu[j], w) - 1.0f));
    }
    return p;
}

// Samples the mixture: lobe by u_lobe, then the vMF lobe with (u1, u2)
// (W. Jakob, "Numerically stable sampling of the von Mises Fisher
// distribution on S^2", 2012).
__device__ __forceinline__ V3 MixtureSample(const VmfMixture& m, float u_lobe, float u1, float u2)
{
    int j = kLobes - 1;
    float c = 0;
    for (int i = 0; i < kLobes; ++i)
    {
        c += expf(m.logw[i]);
        if (u_lobe < c)
        {
            j = i;
            break;
        }
    }
    float k = m.kappa[j];
    float w = 1.0f + logf(fmaxf(u1 + (1.0f - u1) * expf(-2.0f * k), 1e-30f)) / k;
    w = Clamp(w, -1.0f, 1.0f);
    float r = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    float phi = kTwoPi * u2;
    Frame f = FrameFromZ(m.mu[j]);
    return Normalize(f.FromLocal(V3{ r * cosf(phi), r * sinf(phi), w }));
}

} // namespace bbg
