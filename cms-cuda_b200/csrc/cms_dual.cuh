// Forward-mode dual numbers and the dot geometry written once for doubles and
// duals.
//
// Dn<K> carries a value and K tangents.  Every operation computes its value
// with exactly the operation the surface kernels use (same order, no
// contraction: the library is built with -fmad=false), so the value part of a
// dual computation reproduces the kernels' doubles bit for bit; the tangents
// follow the usual derivative rules.  Branches (the |dt| > 0.99 frame switch,
// the cusp case, argmax / argmin picks, subdivision counts) are taken on the
// values, which is what holding the dot topology fixed means.
#pragma once
#include "cms_math.cuh"

namespace cms {

template <int K>
struct Dn {
    double v;
    double d[K];
};

template <int K>
__device__ __forceinline__ Dn<K> dn_c(double v)
{
    Dn<K> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = 0.0;
    return r;
}

template <int K>
__device__ __forceinline__ Dn<K> dn_var(double v, int k0)
{
    Dn<K> r = dn_c<K>(v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = k == k0 ? 1.0 : 0.0;
    return r;
}

template <int K> __device__ __forceinline__ Dn<K> operator+(const Dn<K>& a, const Dn<K>& b)
{
    Dn<K> r; r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator+(const Dn<K>& a, double b)
{
    Dn<K> r = a; r.v = a.v + b; return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator+(double a, const Dn<K>& b)
{
    Dn<K> r = b; r.v = a + b.v; return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator-(const Dn<K>& a, const Dn<K>& b)
{
    Dn<K> r; r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator-(const Dn<K>& a, double b)
{
    Dn<K> r = a; r.v = a.v - b; return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator-(double a, const Dn<K>& b)
{
    Dn<K> r; r.v = a - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -b.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator-(const Dn<K>& a)
{
    Dn<K> r; r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator*(const Dn<K>& a, const Dn<K>& b)
{
    Dn<K> r; r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator*(const Dn<K>& a, double b)
{
    Dn<K> r; r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator*(double a, const Dn<K>& b)
{
    Dn<K> r; r.v = a * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a * b.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator/(const Dn<K>& a, const Dn<K>& b)
{
    Dn<K> r; r.v = a.v / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator/(const Dn<K>& a, double b)
{
    Dn<K> r; r.v = a.v / b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] / b;
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> operator/(double a, const Dn<K>& b)
{
    Dn<K> r; r.v = a / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -(r.v * b.d[k]) / b.v;
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> dsqrt(const Dn<K>& a)
{
    Dn<K> r; r.v = sqrt(a.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] / (2.0 * r.v);
    return r;
}
template <int K> __device__ __forceinline__ void dsincos(const Dn<K>& a, Dn<K>& s, Dn<K>& c)
{
    double sv, cv;
    sincos(a.v, &sv, &cv);
    s.v = sv; c.v = cv;
#pragma unroll
    for (int k = 0; k < K; ++k) { s.d[k] = cv * a.d[k]; c.d[k] = -sv * a.d[k]; }
}
template <int K> __device__ __forceinline__ Dn<K> dsin(const Dn<K>& a)
{
    Dn<K> r; r.v = sin(a.v);
    const double cv = cos(a.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = cv * a.d[k];
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> datan2(const Dn<K>& y, const Dn<K>& x)
{
    Dn<K> r; r.v = atan2(y.v, x.v);
    const double den = x.v * x.v + y.v * y.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (x.v * y.d[k] - y.v * x.d[k]) / den;
    return r;
}
template <int K> __device__ __forceinline__ Dn<K> dacos(const Dn<K>& a)
{
    Dn<K> r; r.v = acos(a.v);
    const double s = sqrt(1.0 - a.v * a.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k] / s;
    return r;
}

// scalar helpers that work on doubles and duals alike
template <class T> struct Lift { __device__ static double c(double v) { return v; } };
template <int K> struct Lift<Dn<K>> { __device__ static Dn<K> c(double v) { return dn_c<K>(v); } };
template <class T> __device__ __forceinline__ T lift(double v) { return Lift<T>::c(v); }

__device__ __forceinline__ double val(double a) { return a; }
template <int K> __device__ __forceinline__ double val(const Dn<K>& a) { return a.v; }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ void dsincos(double a, double& s, double& c) { sincos(a, &s, &c); }
__device__ __forceinline__ double dsin(double a) { return sin(a); }
__device__ __forceinline__ double datan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ double dacos(double a) { return acos(a); }

template <class T> struct TV3 { T x, y, z; };

template <class T> __device__ __forceinline__ TV3<T> tv3(const T& x, const T& y, const T& z)
{
    TV3<T> r; r.x = x; r.y = y; r.z = z; return r;
}
template <class T> __device__ __forceinline__ TV3<T> tconst(V3 a)
{
    TV3<T> r; r.x = lift<T>(a.x); r.y = lift<T>(a.y); r.z = lift<T>(a.z); return r;
}
template <class T> __device__ __forceinline__ TV3<T> operator+(const TV3<T>& a, const TV3<T>& b) { return tv3<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> __device__ __forceinline__ TV3<T> operator-(const TV3<T>& a, const TV3<T>& b) { return tv3<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> __device__ __forceinline__ TV3<T> operator-(const TV3<T>& a) { return tv3<T>(-a.x, -a.y, -a.z); }
template <class T, class S> __device__ __forceinline__ TV3<T> operator*(const TV3<T>& a, const S& s) { return tv3<T>(a.x * s, a.y * s, a.z * s); }
template <class T, class S> __device__ __forceinline__ TV3<T> operator/(const TV3<T>& a, const S& s) { return tv3<T>(a.x / s, a.y / s, a.z / s); }

template <class T> __device__ __forceinline__ T tdot_seq(const TV3<T>& a, const TV3<T>& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class T> __device__ __forceinline__ T tdot_alt(const TV3<T>& a, const TV3<T>& b) { return (a.x * b.x + a.z * b.z) + a.y * b.y; }
template <class T> __device__ __forceinline__ T tnorm(const TV3<T>& a) { return dsqrt(tdot_seq(a, a)); }
template <class T> __device__ __forceinline__ TV3<T> tnormalize(const TV3<T>& a)
{
    const T n = tnorm(a);
    return tv3<T>(a.x / n, a.y / n, a.z / n);
}
template <class T> __device__ __forceinline__ TV3<T> tcross(const TV3<T>& a, const TV3<T>& b)
{
    return tv3<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class T> __device__ __forceinline__ V3 tval(const TV3<T>& a) { return v3(val(a.x), val(a.y), val(a.z)); }

// circle_frame of cms_math.cuh
template <class T> __device__ __forceinline__ void tcircle_frame(const TV3<T>& axis_in, TV3<T>& x, TV3<T>& y)
{
    const TV3<T> axis = tnormalize(axis_in);
    TV3<T> v1 = tv3<T>(axis.y * axis.y + axis.z * axis.z, axis.x * axis.x + axis.z * axis.z,
                       axis.x * axis.x + axis.y * axis.y);
    v1 = tnormalize(v1);
    const T dt = tdot_seq(v1, axis);
    if (fabs(val(dt)) > 0.99) v1 = tv3<T>(lift<T>(1.0), lift<T>(0.0), lift<T>(0.0));
    const TV3<T> v2 = tnormalize(tcross(axis, v1));
    x = tnormalize(tcross(axis, v2));
    y = tcross(axis, x);
}

// arc_angle of cms_math.cuh (the NaN case carries no tangent)
template <class T> __device__ __forceinline__ T tarc_angle(const TV3<T>& axis, const TV3<T>& x, const TV3<T>& v, TV3<T>& y)
{
    y = tcross(axis, x);
    const T dt1 = tdot_seq(v, x);
    const T dt2 = tdot_seq(v, y);
    T ang = datan2(dt2, dt1);
    if (val(ang) < 0.0) ang = ang + CMS_TWO_PI;
    if (fabs(val(dt1)) <= 1e-08 && fabs(val(dt2)) <= 1e-08) ang = lift<T>(__longlong_as_double(0x7ff8000000000000LL));
    return ang;
}

template <class T> __device__ __forceinline__ T tsubdiv_delta(double density, const T& rad)
{
    return 1.0 / (sqrt(density) * rad);
}

template <class T, class R, class D>
__device__ __forceinline__ TV3<T> tsubdiv_point(const TV3<T>& cen, const R& rad, const TV3<T>& x, const TV3<T>& y,
                                                const D& delta, int i)
{
    const D a = delta * ((double)i + 0.5);
    D s, c;
    dsincos(a, s, c);
    const auto rc = rad * c;
    const auto rs = rad * s;
    return (cen + x * rc) + y * rs;
}

template <class T, class R> __device__ __forceinline__ T tsubdiv_ps(const R& rad, const T& angle, int count)
{
    return count > 0 ? (rad * angle) / (double)count : lift<T>(0.0);
}

}  // namespace cms
