// Device vector math in the reference's evaluation order
// (include/bulbit/vectors.h, math.h, frame.h, spectrum.h).
//
// Every kernel translation unit of this library is compiled with
// --fmad=false and IEEE division and square root, so each expression below
// rounds exactly like the reference's x86-64 build. Transcendentals are
// evaluated in double precision and rounded to float once; the reference's
// glibc float functions are accurate to well under an ulp, so the two agree
// in nearly every case and differ by one ulp otherwise.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bbg
{

constexpr float kPi = float(3.14159265358979323846);
constexpr float kTwoPi = float(2 * kPi);
constexpr float kFourPi = float(4 * kPi);
constexpr float kInvPi = float(1 / kPi);
constexpr float kInvFourPi = float(1 / (4 * kPi));
constexpr float kEpsilon = 1.1920928955078125e-07f; // FLT_EPSILON
constexpr float kRayEpsilon = 1e-4f;                 // Ray::epsilon (include/bulbit/ray.h:21)

struct V3
{
    float x, y, z;
};

__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{ x, y, z }; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
__device__ __forceinline__ V3 operator-(V3 a) { return { -a.x, -a.y, -a.z }; }
__device__ __forceinline__ V3 operator*(V3 v, float s) { return { v.x * s, v.y * s, v.z * s }; }
__device__ __forceinline__ V3 operator*(float s, V3 v) { return { v.x * s, v.y * s, v.z * s }; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return { a.x * b.x, a.y * b.y, a.z * b.z }; }
__device__ __forceinline__ V3 operator/(V3 v, float s) { return { v.x / s, v.y / s, v.z / s }; }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return { a.x / b.x, a.y / b.y, a.z / b.z }; }
__device__ __forceinline__ float Dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 Cross(V3 a, V3 b)
{
    return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
}
__device__ __forceinline__ float Length2(V3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
__device__ __forceinline__ float Length(V3 v) { return sqrtf(Length2(v)); }
__device__ __forceinline__ float AbsDot(V3 a, V3 b) { return fabsf(Dot(a, b)); }
__device__ __forceinline__ float Sqr(float v) { return v * v; }

// Normalize(v) (include/bulbit/math.h:56).
__device__ __forceinline__ V3 Normalize(V3 v)
{
    float inv_length = 1.0f / Length(v);
    return v * inv_length;
}

// Vector3::Normalize (include/bulbit/vectors.h:121): in place, returns the
// length; vectors shorter than epsilon are left unchanged and 0 is returned.
__device__ __forceinline__ float NormalizeInPlace(V3& v)
{
    float length = Length(v);
    if (length < kEpsilon)
    {
        return 0;
    }
    float inv_length = 1.0f / length;
    v.x *= inv_length;
    v.y *= inv_length;
    v.z *= inv_length;
    return length;
}

// std::min / std::max argument semantics.
__device__ __forceinline__ float SMin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float SMax(float a, float b) { return (a < b) ? b : a; }

// Clamp(v, l, r) (include/bulbit/math.h:50).
__device__ __forceinline__ float Clamp(float v, float l, float r) { return v < l ? l : (v > r ? r : v); }

__device__ __forceinline__ V3 Reflect(V3 v, V3 n) { return -v + 2 * Dot(v, n) * n; }

// Transcendentals: double precision, one rounding to float.
__device__ __forceinline__ float dcos(float x) { return float(cos(double(x))); }
__device__ __forceinline__ float dsin(float x) { return float(sin(double(x))); }
__device__ __forceinline__ float dpow(float x, float y) { return float(pow(double(x), double(y))); }

// ------------------------------------------------------------ spectrum (RGB)

struct Spec
{
    float r, g, b;
};

__device__ __forceinline__ Spec spec(float s) { return { s, s, s }; }
__device__ __forceinline__ Spec operator+(Spec a, Spec b) { return { a.r + b.r, a.g + b.g, a.b + b.b }; }
__device__ __forceinline__ Spec operator-(Spec a, Spec b) { return { a.r - b.r, a.g - b.g, a.b - b.b }; }
__device__ __forceinline__ Spec operator*(Spec a, Spec b) { return { a.r * b.r, a.g * b.g, a.b * b.b }; }
__device__ __forceinline__ Spec operator*(Spec a, float s) { return { a.r * s, a.g * s, a.b * s }; }
__device__ __forceinline__ Spec operator*(float s, Spec a) { return { a.r * s, a.g * s, a.b * s }; }
__device__ __forceinline__ Spec operator/(Spec a, float s) { return { a.r / s, a.g / s, a.b / s }; }
__device__ __forceinline__ Spec operator/(Spec a, Spec b) { return { a.r / b.r, a.g / b.g, a.b / b.b }; }
__device__ __forceinline__ bool IsBlack(Spec s) { return s.r == 0.0f && s.g == 0.0f && s.b == 0.0f; }
__device__ __forceinline__ bool IsNullish(Spec s)
{
    return isnan(s.r) || isinf(s.r) || isnan(s.g) || isinf(s.g) || isnan(s.b) || isinf(s.b);
}
// std::max({r, g, b}): first largest by operator<.
__device__ __forceinline__ float MaxComponent(Spec s)
{
    float m = s.r;
    if (m < s.g) m = s.g;
    if (m < s.b) m = s.b;
    return m;
}
__device__ __forceinline__ float Luminance(Spec s) { return s.r * 0.2126f + s.g * 0.7152f + s.b * 0.0722f; }

// ------------------------------------------------------------ frames

// Shading-frame helpers (include/bulbit/frame.h).
__device__ __forceinline__ float AbsCosTheta(V3 w) { return fabsf(w.z); }
__device__ __forceinline__ float Cos2Theta(V3 w) { return Sqr(w.z); }
__device__ __forceinline__ float Sin2Theta(V3 w) { return SMax(0.0f, 1 - Cos2Theta(w)); }
__device__ __forceinline__ float SinTheta(V3 w) { return sqrtf(Sin2Theta(w)); }
__device__ __forceinline__ float Tan2Theta(V3 w) { return Sin2Theta(w) / Cos2Theta(w); }
__device__ __forceinline__ float CosPhi(V3 w)
{
    float sin_theta = SinTheta(w);
    return (sin_theta == 0) ? 1 : Clamp(w.x / sin_theta, -1, 1);
}
__device__ __forceinline__ float SinPhi(V3 w)
{
    float sin_theta = SinTheta(w);
    return (sin_theta == 0) ? 0 : Clamp(w.y / sin_theta, -1, 1);
}
__device__ __forceinline__ bool SameHemisphere(V3 a, V3 b) { return a.z * b.z > 0; }

struct Frame
{
    V3 x, y, z;
    // Frame::ToLocal / FromLocal (include/bulbit/frame.h:157-167).
    __device__ __forceinline__ V3 ToLocal(V3 v) const { return { Dot(v, x), Dot(v, y), Dot(v, z) }; }
    __device__ __forceinline__ V3 FromLocal(V3 v) const { return v.x * x + v.y * y + v.z * z; }
};

// CoordinateSystem (include/bulbit/frame.h:105-112).
__device__ __forceinline__ void CoordinateSystem(V3 v1, V3* v2, V3* v3)
{
    float sign = copysignf(1.0f, v1.z);
    float a = -1 / (sign + v1.z);
    float b = v1.x * v1.y * a;
    *v2 = V3{ 1 + sign * (v1.x * v1.x) * a, sign * b, -sign * v1.x };
    *v3 = V3{ b, sign + (v1.y * v1.y) * a, -v1.y };
}

// Frame::FromXZ (include/bulbit/frame.h:125).
__device__ __forceinline__ Frame FrameFromXZ(V3 x, V3 z) { return Frame{ x, Cross(z, x), z }; }

// Frame(const Vec3& n) (include/bulbit/frame.h:145).
__device__ __forceinline__ Frame FrameFromZ(V3 n)
{
    Frame f;
    f.z = n;
    CoordinateSystem(n, &f.x, &f.y);
    return f;
}

__device__ __forceinline__ V3 load3(const float* p) { return { p[0], p[1], p[2] }; }

} // namespace bbg
