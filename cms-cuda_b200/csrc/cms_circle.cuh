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
