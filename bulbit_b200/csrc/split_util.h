// Geometry of reference splitting (early split clipping), shared by the host
// splitter (host_build.cpp) and the device splitter (split_build.cu) so both
// clip, measure and round the same way: a triangle clipped to an axis-aligned
// box in double precision (Sutherland-Hodgman), the clipped part's area, a
// box's surface area, and the outward rounding of a double bound to float.
// Compiled by g++ for the host and by nvcc for both sides.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define BBG_SPLIT_FN __host__ __device__ inline
#else
#define BBG_SPLIT_FN inline
#endif

namespace bbg
{
namespace split
{

// A triangle clipped to one axis-aligned half-space (coordinate `axis` below
// or above m); the polygon's corners go to out, their count is returned. A
// triangle clipped by six planes has at most 9 corners.
BBG_SPLIT_FN int ClipAxis(const double (*in)[3], int n, int axis, double m, bool keep_below, double (*out)[3])
{
    int k = 0;
    for (int i = 0; i < n; ++i)
    {
        const double* a = in[i];
        const double* b = in[(i + 1) % n];
        const bool ia = keep_below ? a[axis] <= m : a[axis] >= m;
        const bool ib = keep_below ? b[axis] <= m : b[axis] >= m;
        if (ia)
        {
            out[k][0] = a[0];
            out[k][1] = a[1];
            out[k][2] = a[2];
            ++k;
        }
        if (ia != ib)
        {
            const double t = (m - a[axis]) / (b[axis] - a[axis]);
            for (int c = 0; c < 3; ++c)
            {
                out[k][c] = a[c] + t * (b[c] - a[c]);
            }
            out[k][axis] = m;
            ++k;
        }
    }
    return k;
}

// Area of a planar convex polygon (fan of triangles from corner 0).
BBG_SPLIT_FN double PolygonArea(const double (*p)[3], int n)
{
    double c[3] = { 0, 0, 0 };
    for (int i = 1; i + 1 < n; ++i)
    {
        double u[3], v[3];
        for (int k = 0; k < 3; ++k)
        {
            u[k] = p[i][k] - p[0][k];
            v[k] = p[i + 1][k] - p[0][k];
        }
        c[0] += u[1] * v[2] - u[2] * v[1];
        c[1] += u[2] * v[0] - u[0] * v[2];
        c[2] += u[0] * v[1] - u[1] * v[0];
    }
    return 0.5 * sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
}

// Box (and area) of the triangle clipped to [lo, hi]; false if nothing is left.
BBG_SPLIT_FN bool ClippedBox(const double tri[3][3], const double lo[3], const double hi[3], double out_lo[3],
                             double out_hi[3], double* area)
{
    double a[12][3], b[12][3];
    int n = 3;
    for (int k = 0; k < 3; ++k)
    {
        for (int c = 0; c < 3; ++c)
        {
            a[k][c] = tri[k][c];
        }
    }
    for (int axis = 0; axis < 3 && n > 0; ++axis)
    {
        n = ClipAxis(a, n, axis, lo[axis], false, b);
        n = ClipAxis(b, n, axis, hi[axis], true, a);
    }
    if (n == 0)
    {
        return false;
    }
    *area = PolygonArea(a, n);
    for (int c = 0; c < 3; ++c)
    {
        out_lo[c] = out_hi[c] = a[0][c];
    }
    for (int i = 1; i < n; ++i)
    {
        for (int c = 0; c < 3; ++c)
        {
            out_lo[c] = a[i][c] < out_lo[c] ? a[i][c] : out_lo[c];
            out_hi[c] = out_hi[c] < a[i][c] ? a[i][c] : out_hi[c];
        }
    }
    // The clipped polygon lies inside the box it was clipped to.
    for (int c = 0; c < 3; ++c)
    {
        out_lo[c] = out_lo[c] < lo[c] ? lo[c] : out_lo[c];
        out_hi[c] = hi[c] < out_hi[c] ? hi[c] : out_hi[c];
    }
    return true;
}

BBG_SPLIT_FN double BoxArea(const double lo[3], const double hi[3])
{
    const double d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
    return 2 * (d0 * d1 + d1 * d2 + d2 * d0);
}

// The largest float not above v / the smallest float not below v.
BBG_SPLIT_FN float RoundDown(double v)
{
    const float f = float(v);
    return double(f) > v ? nextafterf(f, -INFINITY) : f;
}

BBG_SPLIT_FN float RoundUp(double v)
{
    const float f = float(v);
    return double(f) < v ? nextafterf(f, INFINITY) : f;
}

// Index of the longest axis of [lo, hi] (the first on a tie).
BBG_SPLIT_FN int LongestAxis(const double lo[3], const double hi[3])
{
    int axis = 0;
    for (int c = 1; c < 3; ++c)
    {
        if (hi[c] - lo[c] > hi[axis] - lo[axis])
        {
            axis = c;
        }
    }
    return axis;
}

} // namespace split
} // namespace bbg
