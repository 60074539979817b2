// Atom lists pruned to a circle.
//
// A probe that touches two atoms i and j sits on one circle (centre tij,
// unit axis uij, radius rij): the torus points of the pair, the probe centres
// of its toroidal dots and the probes of every triple (i, j, k).  An atom
// whose sphere of radius r + rp stays more than CMS_CIRCLE_MARGIN away from
// that circle collides with, or buries, no point of it, so the collision and
// burial tests can run over the atoms that pass circle_prune and give the
// same answer as over the full list for every point within CMS_CIRCLE_TOL of
// the circle.  Both bounds are far above the FP64 rounding of the points.
#pragma once
#include "cms_internal.cuh"

namespace cms {

#define CMS_CIRCLE_MARGIN 1e-4   // A, added to r + rp when pruning
#define CMS_CIRCLE_TOL 1e-5      // A, largest distance of a point from the circle for the pruned test

// A toroid pair (i, j): its pair geometry and the subdivision of its torus
// circle.  A kernel after the pair loop makes it once per toroid (tor_pair_of,
// kept in Dev::tor_geo); the toroidal count and emit passes load it
// (tor_pair_load), adding the per-atom values again with the same operations.
struct TorPair {
    int i, j;
    V3 xi, xj, uij, tij;
    double ri, rj, eri, erj, rij, density, ts, dtor, darc;
    bool between;
    int ns;
    V3 fx, fy;
};

__device__ __forceinline__ TorPair tor_pair_of(const Dev& d, int i, int j)
{
    TorPair T;
    const double rp = d.st.rp;
    T.i = i; T.j = j;
    double4 a = d.xyzr[T.i], b = d.xyzr[T.j];
    T.xi = v3(a.x, a.y, a.z); T.xj = v3(b.x, b.y, b.z);
    T.ri = a.w; T.rj = b.w;
    // pair geometry, as second_loop computes it (_core.py:1372-1416)
    V3 diff = T.xj - T.xi;
    double dij_sq = sq_alt(diff);
    double dij = sqrt(dij_sq);
    T.eri = T.ri + rp; T.erj = T.rj + rp;
    double asymm = (T.eri * T.eri - T.erj * T.erj) / dij;
    T.between = fabs(asymm) < dij;
    T.uij = diff / dij;
    T.tij = ((T.xi + T.xj) * 0.5) + T.uij * (asymm * 0.5);
    double far_sq = (T.eri + T.erj) * (T.eri + T.erj) - dij_sq;
    double rd = T.ri - T.rj;
    double cont_sq = dij_sq - rd * rd;
    T.rij = ((0.5 * sqrt(far_sq)) * sqrt(cont_sq)) / dij;
    // torus circle subdivision (_core.py:1863-1885)
    T.density = (d.dens[T.i] + d.dens[T.j]) * 0.5;
    double rci = (T.rij * T.ri) / T.eri;
    double rcj = (T.rij * T.rj) / T.erj;
    double rbt = T.rij - rp;
    double rb = rbt < 0.0 ? 0.0 : rbt;                 // np.maximum keeps NaN
    double rs = ((rci + 2.0 * rb) + rcj) * 0.25;
    double e = rs / T.rij;
    double edens = (e * e) * T.density;
    circle_frame(T.uij, T.fx, T.fy);
    T.dtor = subdiv_delta(edens, T.rij);
    T.ns = subdiv_count(T.dtor, CMS_TWO_PI);
    T.ts = subdiv_ps(T.rij, CMS_TWO_PI, T.ns);
    T.darc = subdiv_delta(T.density, rp);
    return T;
}

// a probe's spherical-triangle frame for the concave dots (k_probe_geo): the
// three plane normals, the top vertex and the latitude arc's second axis, the
// frame of the latitude circles, the latitude spacing and count, the arc step
struct ConcGeo {
    double v0[3], v1[3], v2[3], top[3], ylat[3], fx[3], fy[3];
    double dl, cs;
    int nl;
};

// a convex atom's frame (k_convex_geo): the pole, the latitude arc's second
// axis, the frame of the latitude circles, the latitude spacing, step and count
struct CvGeo {
    double north[3], ylat[3], fx[3], fy[3];
    double dl, cs;
    int nl;
};

struct TorGeo {
    double ux, uy, uz, tx, ty, tz, fxx, fxy, fxz, fyx, fyy, fyz;
    double rij, ts, dtor, darc;
    int ns, between;
};

__device__ __forceinline__ void tor_geo_store(const Dev& d, long long q, const TorPair& T)
{
    TorGeo G;
    G.ux = T.uij.x; G.uy = T.uij.y; G.uz = T.uij.z;
    G.tx = T.tij.x; G.ty = T.tij.y; G.tz = T.tij.z;
    G.fxx = T.fx.x; G.fxy = T.fx.y; G.fxz = T.fx.z;
    G.fyx = T.fy.x; G.fyy = T.fy.y; G.fyz = T.fy.z;
    G.rij = T.rij; G.ts = T.ts; G.dtor = T.dtor; G.darc = T.darc;
    G.ns = T.ns; G.between = T.between ? 1 : 0;
    d.tor_geo[q] = G;
}

__device__ __forceinline__ TorPair tor_pair_load(const Dev& d, long long q)
{
    TorPair T;
    const double rp = d.st.rp;
    T.i = d.tor_i[q]; T.j = d.tor_j[q];
    const double4 a = d.xyzr[T.i], b = d.xyzr[T.j];
    T.xi = v3(a.x, a.y, a.z); T.xj = v3(b.x, b.y, b.z);
    T.ri = a.w; T.rj = b.w;
    T.eri = T.ri + rp; T.erj = T.rj + rp;
    T.density = (d.dens[T.i] + d.dens[T.j]) * 0.5;
    const TorGeo G = d.tor_geo[q];
    T.uij = v3(G.ux, G.uy, G.uz); T.tij = v3(G.tx, G.ty, G.tz);
    T.fx = v3(G.fxx, G.fxy, G.fxz); T.fy = v3(G.fyx, G.fyy, G.fyz);
    T.rij = G.rij; T.ts = G.ts; T.dtor = G.dtor; T.darc = G.darc;
    T.ns = G.ns; T.between = G.between != 0;
    return T;
}

// squared distance of x from the circle
__device__ __forceinline__ double circle_dist2(V3 x, V3 c, V3 u, double R)
{
    const V3 v = x - c;
    const double h = dot_seq(v, u);
    const double rho = sqrt(fmax(sq_seq(v) - h * h, 0.0));
    const double dr = rho - R;
    return h * h + dr * dr;
}

// true when the pruned lists are valid for point x (a NaN distance is not)
__device__ __forceinline__ bool near_circle(V3 x, V3 c, V3 u, double R)
{
    return circle_dist2(x, c, u, R) <= CMS_CIRCLE_TOL * CMS_CIRCLE_TOL;
}

// Warp-cooperative: compact into out[] (room for cap ids) the atoms ids[s, e)
// other than `skip` whose sphere of radius r + rp may reach the circle; -1
// when they do not fit (the caller then scans the full list).  A non-finite
// distance keeps the atom.  Every lane returns the same count.  With `cover`,
// also reports whether one of the atoms holds the whole circle strictly
// inside its sphere, CMS_CIRCLE_MARGIN to spare: then every point of the
// circle collides with it (strict < test).
__device__ __forceinline__ int circle_prune(const Dev& d, V3 c, V3 u, double R, const int* ids, long long s,
                                            long long e, int skip, int* out, int cap, bool* cover = nullptr)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const double rp = d.st.rp;
    int n = 0;
    bool cov = false;
    for (long long b = s; b < e; b += 32) {
        const long long k = b + lane;
        bool keep = false;
        int id = -1;
        if (k < e) {
            id = ids[k];
            if (id != skip) {
                const double4 a = d.xyzr[id];
                const V3 v = v3(a.x, a.y, a.z) - c;
                const double h = dot_seq(v, u);
                const double rho = sqrt(fmax(sq_seq(v) - h * h, 0.0));
                const double dr = rho - R;
                const double t = a.w + rp + CMS_CIRCLE_MARGIN;
                keep = !(h * h + dr * dr > t * t);
                if (cover && keep) {
                    const double far = rho + R, ti = a.w + rp - CMS_CIRCLE_MARGIN;
                    cov |= ti > 0.0 && h * h + far * far < ti * ti;
                }
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        const int pos = n + __popc(m & lt);
        if (keep && pos < cap) out[pos] = id;
        n += __popc(m);
    }
    if (cover) *cover = __any_sync(0xffffffffu, cov);
    __syncwarp();
    return n > cap ? -1 : n;
}

}  // namespace cms
