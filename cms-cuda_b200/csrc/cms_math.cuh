// Fixed-order FP64 3-vector arithmetic shared by every surface kernel.
//
// The library is compiled with -fmad=false, so `a*b + c` is a rounded multiply
// followed by a rounded add, exactly like NumPy.  Three-term sums come in the
// two orders NumPy uses for the reference CPU calculator (cms-cuda/_core.py):
//
//   dot_seq : (p0 + p1) + p2  -- np.sum(..., -1), np.linalg.norm, scipy cdist
//   dot_alt : (p0 + p2) + p1  -- np.einsum('...i,...i->...')
//
// `normalize` divides each component by the norm (NumPy `a / norm(a)`), never
// multiplies by a reciprocal.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

struct V3 { double x, y, z; };

__host__ __device__ __forceinline__ V3 v3(double x, double y, double z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator/(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }

__device__ __forceinline__ double dot_seq(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ double dot_alt(V3 a, V3 b) { return (a.x * b.x + a.z * b.z) + a.y * b.y; }
__device__ __forceinline__ double sq_seq(V3 a) { return dot_seq(a, a); }
__device__ __forceinline__ double sq_alt(V3 a) { return dot_alt(a, a); }
__device__ __forceinline__ double norm3(V3 a) { return sqrt(dot_seq(a, a)); }
__device__ __forceinline__ V3 normalize3(V3 a) { double n = norm3(a); return v3(a.x / n, a.y / n, a.z / n); }
__device__ __forceinline__ V3 cross3(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ V3 ld3(const double* p) { return v3(p[0], p[1], p[2]); }
__device__ __forceinline__ void st3(double* p, V3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
__device__ __forceinline__ V3 xyz_of(double4 a) { return v3(a.x, a.y, a.z); }

#define CMS_TWO_PI 6.283185307179586
#define CMS_MAX_SUBDIV 100

// Number of subdivision points of an arc of `angle` radians on a circle of
// radius `rad` at `density` points per unit area (the reference's vec_sub_div,
// _core.py:2429-2486): point i exists iff delta*(i+0.5) <= angle, i < 100,
// with delta = 1/(sqrt(density)*rad).  NaN angle or infinite delta give 0.
__device__ __forceinline__ int subdiv_count(double delta, double angle)
{
    int n = 0;
    while (n < CMS_MAX_SUBDIV && delta * ((double)n + 0.5) <= angle) ++n;
    return n;
}

// subdiv_count for long circles (latitudes of a sphere: tens of points).  For
// delta > 0 the rounded products delta*(n + 0.5) do not decrease with n
// (n + 0.5 is exact and rounding is monotone), so the points that exist are a
// prefix: start from an FP32 estimate of the quotient and settle the exact
// boundary with the same FP64 comparisons the loop makes.  Inputs outside the
// FP32 range take the loop.
__device__ __forceinline__ int subdiv_count_long(double delta, double angle)
{
    int n = 0;
    if (delta > 1e-30 && delta < 1e30 && fabs(angle) < 1e30) {
        const float e = __fdividef((float)angle, (float)delta) + 0.5f;
        n = !(e > 0.f) ? 0 : (e >= (float)CMS_MAX_SUBDIV ? CMS_MAX_SUBDIV : (int)e);
        while (n > 0 && !(delta * ((double)(n - 1) + 0.5) <= angle)) --n;
        while (n < CMS_MAX_SUBDIV && delta * ((double)n + 0.5) <= angle) ++n;
        return n;
    }
    while (n < CMS_MAX_SUBDIV && delta * ((double)n + 0.5) <= angle) ++n;
    return n;
}

__device__ __forceinline__ double subdiv_delta(double density, double rad)
{
    return 1.0 / (sqrt(density) * rad);
}

// In-plane frame of a full circle around `axis` (vec_sub_cir, _core.py:2488-2523).
__device__ __forceinline__ void circle_frame(V3 axis_in, V3& x, V3& y)
{
    V3 axis = normalize3(axis_in);
    V3 v1 = v3(axis.y * axis.y + axis.z * axis.z,
               axis.x * axis.x + axis.z * axis.z,
               axis.x * axis.x + axis.y * axis.y);
    v1 = normalize3(v1);
    double dt = dot_seq(v1, axis);
    if (fabs(dt) > 0.99) v1 = v3(1.0, 0.0, 0.0);
    V3 v2 = normalize3(cross3(axis, v1));
    x = normalize3(cross3(axis, v2));
    y = cross3(axis, x);
}

// Arc angle of vec_sub_arc (_core.py:2407-2427): y = axis x x; the angle from
// x to v measured in the (x, y) plane, mapped to [0, 2pi); NaN when v is
// (numerically) perpendicular to the plane.
__device__ __forceinline__ double arc_angle(V3 axis, V3 x, V3 v, V3& y)
{
    y = cross3(axis, x);
    double dt1 = dot_seq(v, x);
    double dt2 = dot_seq(v, y);
    double ang = atan2(dt2, dt1);
    if (ang < 0.0) ang = ang + CMS_TWO_PI;
    if (fabs(dt1) <= 1e-08 && fabs(dt2) <= 1e-08) ang = __longlong_as_double(0x7ff8000000000000LL);
    return ang;
}

// Subdivision point i: (cen + x*(rad*cos a)) + y*(rad*sin a), a = delta*(i+0.5).
__device__ __forceinline__ V3 subdiv_point(V3 cen, double rad, V3 x, V3 y, double delta, int i)
{
    double a = delta * ((double)i + 0.5);
    double s, c;
    sincos(a, &s, &c);
    double rc = rad * c, rs = rad * s;
    return (cen + x * rc) + y * rs;
}

// Arc length per point: rad*angle/count (0 when count is 0).
__device__ __forceinline__ double subdiv_ps(double rad, double angle, int count)
{
    return count > 0 ? (rad * angle) / (double)count : 0.0;
}
