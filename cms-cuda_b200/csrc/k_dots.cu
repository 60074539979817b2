// Surface pipeline, back half: convex, toroidal and concave dot generation
// with the burial test, in two passes (count, then emit) that share one code
// path so the two passes agree by construction.  The count passes keep what
// the emit passes need (convex: the accepted candidates; toroidal: the torus
// points with arc dots; concave: the finished dots) in buffers sized by the
// capacities; a unit that does not fit is recomputed by the emit pass.
//
// Reference behaviour (cms-cuda/_core.py):
//   generate_convex_surface        _core.py:1646-1840
//   generate_toroidal_surface(s)   _core.py:1234-1248, 1847-2067
//   generate_concave_surface       _core.py:2069-2333
//   add_dots                       _core.py:2337-2377
//   vec_sub_arc / vec_sub_div / vec_sub_cir / vec_distance_point_to_line
//                                  _core.py:2380-2527
//
// Dot order per complex and molecule is the reference's: all convex dots
// (atom, latitude, point), then all arc-1 toroidal dots (toroid pair, torus
// point, arc point), then all arc-2 toroidal dots, then all concave dots
// (probe, latitude, point).  Each unit's dots start at
// seg.dot0 + (unit scan - seg.scan0); inside a unit a warp orders its dots
// with ballots.
#include "cms_circle.cuh"
#include "cms_kernels.cuh"

namespace cms {

static constexpr int SM_COUNT = 148;

static inline unsigned grid_for(long long items, int per_block, int max_blocks_per_sm = 16)
{
    long long b = (items + per_block - 1) / per_block;
    long long cap = (long long)SM_COUNT * max_blocks_per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

// buried = any buried partner b of the owner with |pcen - x_b|^2 <= (r_b + rp)^2 (seq order)
__device__ __forceinline__ int8_t buried_test(const Dev& d, int owner, V3 pcen)
{
    const long long s = d.bu_off[owner], e = d.bu_off[owner + 1];
    const double rp = d.st.rp;
    for (long long p = s; p < e; ++p) {
        double4 b = d.xyzr[d.bu_id[p]];
        double t = b.w + rp;
        if (sq_seq(v3(b.x, b.y, b.z) - pcen) <= t * t) return 1;
    }
    return 0;
}

// buried_test for one probe centre and up to three owners, the warp's lanes
// spread over each owner's buried partners (same result: any partner within reach)
__device__ __forceinline__ int8_t buried_warp(const Dev& d, int owner, V3 pcen)
{
    const int lane = threadIdx.x & 31;
    const long long s = d.bu_off[owner], e = d.bu_off[owner + 1];
    const double rp = d.st.rp;
    for (long long b0 = s; b0 < e; b0 += 32) {
        bool hit = false;
        if (b0 + lane < e) {
            const double4 b = d.xyzr[d.bu_id[b0 + lane]];
            const double t = b.w + rp;
            hit = sq_seq(v3(b.x, b.y, b.z) - pcen) <= t * t;
        }
        if (__any_sync(0xffffffffu, hit)) return 1;
    }
    return 0;
}

__device__ __forceinline__ void write_dot_b(const Dev& d, long long q, V3 pt, V3 pcen, double area, int owner,
                                            int type, int unit, int sub, int8_t bur)
{
    if (q >= d.dot_cap) return;
    const double rp = d.st.rp;
    V3 nml = rp <= 0.0 ? pt - atom_xyz(d, owner) : (pcen - pt) / rp;
    st3(d.dxyz + 3 * q, pt);
    st3(d.dnml + 3 * q, nml);
    d.darea[q] = area;
    d.dbur[q] = bur;
    d.dtype[q] = (int8_t)type;
    d.datom[q] = owner;
    d.dunit[q] = unit;
    d.dsub[q] = sub;
}

__device__ __forceinline__ void write_dot(const Dev& d, long long q, V3 pt, V3 pcen, double area, int owner,
                                          int type, int unit, int sub)
{
    if (q >= d.dot_cap) return;
    write_dot_b(d, q, pt, pcen, area, owner, type, unit, sub, buried_test(d, owner, pcen));
}

__device__ __forceinline__ long long unit_base(const Dev& d, int c, int m, int t, long long unit_scan)
{
    const Seg s = d.seg[(c * 2 + m) * 4 + t];
    return s.dot0 + (unit_scan - s.scan0);
}

// Kept candidates of a unit: the count pass collects them in shared memory
// (up to KS_CAP) and moves them to the kept-candidate buffer at the unit's
// end; the emit pass then computes and writes those dots alone.  -1: not
// stashed (too many, or the buffer is full), the emit pass tests every
// candidate again.
static constexpr int KS_CAP = 512;

__device__ __forceinline__ int ks_stash(const Dev& d, const int* list, int kept, StashCursor& cur)
{
    const int lane = threadIdx.x & 31;
    if (kept <= 0 || kept > KS_CAP) return -1;
    const long long off = stash_take(d.ks_top, d.ks_cap, cur, kept);
    if (off < 0) return -1;
    for (int e = lane; e < kept; e += 32) d.ks_buf[off + e] = list[e];
    return (int)off;
}

// ---------------------------------------------------------------------------
// convex dots: one warp per atom of the convex queue
// ---------------------------------------------------------------------------
static constexpr int CV_WARPS = 2;
static constexpr int CV_ROW = 128;    // neighbour rows up to this long are cached in shared memory

// Latitude table of one sphere: each latitude's offset dt along the polar
// axis (its circle's centre is recomputed as the table was made: xi + north dt
// for convex, south dt for concave), radius, subdivision step, dot area and
// first point in the sphere's enumeration.
struct LatTable {
    double dt[CMS_MAX_SUBDIV], rad[CMS_MAX_SUBDIV], delta[CMS_MAX_SUBDIV], area[CMS_MAX_SUBDIV];
    int start[CMS_MAX_SUBDIV + 1];
};

__device__ __forceinline__ int find_lat(const LatTable& L, int nl, int t)
{
    // largest l with start[l] <= t
    int lo = 0, hi = nl - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (L.start[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void lat_prefix(LatTable& L, const int* nc, int nl)
{
    if ((threadIdx.x & 31) == 0) {
        int s = 0;
        for (int l = 0; l < nl; ++l) { L.start[l] = s; s += nc[l]; }
        L.start[nl] = s;
    }
    __syncwarp();
}

template <bool EMIT>
__global__ void __launch_bounds__(CV_WARPS * 32, EMIT ? 10 : 12) k_convex(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ LatTable tab[CV_WARPS];
    __shared__ int ncs[CV_WARPS][CMS_MAX_SUBDIV];
    __shared__ int ksl[EMIT ? 1 : CV_WARPS][KS_CAP];
    __shared__ double4 nrow[CV_WARPS][CV_ROW];   // the atom's neighbours: x, y, z, r + rp
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    LatTable& L = tab[w];
    StashCursor kcur{0, 0};
    const double rp = d.st.rp;
    const long long wid = blockIdx.x * (long long)CV_WARPS + w;
    const long long nw = (long long)gridDim.x * CV_WARPS;
    for (long long gg = wid; gg < d.N; gg += nw) {
        const int g = (int)gg;
        const int K = d.nnb[g];
        if (!(K > 0 && d.access[g] != 0 && d.atten[g] > 1)) {
            if (!EMIT && lane == 0) d.conv_cnt[g] = 0;
            continue;
        }
        if (EMIT && d.conv_cnt[g] == 0) continue;                      // no dots: nothing to write
        const double4 ai = d.xyzr[g];
        const V3 xi = v3(ai.x, ai.y, ai.z);
        const double ri = ai.w, eri = ri + rp, dens = d.dens[g];
        const long long off = d.nb_off[g];
        // frame from the nearest neighbour (_core.py:1665-1726), made by k_convex_geo
        const CvGeo G = d.cv_geo[g];
        const V3 north = v3(G.north[0], G.north[1], G.north[2]), ylat = v3(G.ylat[0], G.ylat[1], G.ylat[2]);
        const V3 fx = v3(G.fx[0], G.fx[1], G.fx[2]), fy = v3(G.fy[0], G.fy[1], G.fy[2]);
        const double dl = G.dl, cs = G.cs;
        const int nl = G.nl;
        for (int l = lane; l < nl; l += 32) {
            V3 lat = subdiv_point(v3(0.0, 0.0, 0.0), ri, north, ylat, dl, l);
            double dt = dot_seq(lat, north);
            double rsq = ri * ri - dt * dt;
            double rad = rsq > 0.0 ? sqrt(rsq) : 0.0;
            int nc = 0;
            double delta = 0.0, ps = 0.0;
            if (rad > 0.0) {
                delta = subdiv_delta(dens, rad);
                nc = subdiv_count_long(delta, CMS_TWO_PI);
                ps = subdiv_ps(rad, CMS_TWO_PI, nc);
            }
            L.dt[l] = dt;
            L.rad[l] = rad; L.delta[l] = delta; L.area[l] = ps * cs;
            ncs[w][l] = nc;
        }
        __syncwarp();
        lat_prefix(L, ncs[w], nl);
        const int total = nl > 0 ? L.start[nl] : 0;
        long long base = 0;
        if (EMIT) base = unit_base(d, d.cplx[g], d.mol[g], 0, d.conv_off[g]);
        int kept = 0;
        const double scale = eri / ri;
        if (EMIT) {
            const int so = d.cv_soff[g];
            if (so >= 0) {
                // the count pass's kept candidates
                const int cnt = d.conv_cnt[g];
                for (int e = lane; e < cnt; e += 32) {
                    const int sub = d.ks_buf[so + e];
                    const int l = sub >> 16, i = sub & 0xffff;
                    const V3 pt = subdiv_point(xi + north * L.dt[l], L.rad[l], fx, fy, L.delta[l], i);
                    write_dot(d, base + e, pt, xi + (pt - xi) * scale, L.area[l], g, 1, g, sub);
                }
                __syncwarp();
                continue;
            }
        }
        // the neighbour row in shared memory (the collision test reads it for every point)
        const bool cached = K <= CV_ROW;
        if (cached) {
            for (int s = lane; s < K; s += 32) {
                const double4 b = d.xyzr[d.nb_id[off + s]];
                nrow[w][s] = make_double4(b.x, b.y, b.z, b.w + rp);
            }
            __syncwarp();
        }
        for (int t0 = 0; t0 < total; t0 += 32) {
            const int t = t0 + lane;
            bool keep = false;
            V3 pt, pcen;
            int l = 0, i = 0;
            if (t < total) {
                l = find_lat(L, nl, t);
                i = t - L.start[l];
                pt = subdiv_point(xi + north * L.dt[l], L.rad[l], fx, fy, L.delta[l], i);
                pcen = xi + (pt - xi) * scale;
                keep = true;
                if (cached) {
                    for (int s = 1; s < K; ++s) {    // slot 0 (the frame atom) is skipped
                        const double4 b = nrow[w][s];
                        if (sq_seq(v3(b.x, b.y, b.z) - pcen) <= b.w * b.w) { keep = false; break; }
                    }
                } else {
                    for (int s = 1; s < K; ++s) {
                        double4 b = d.xyzr[d.nb_id[off + s]];
                        double tt = b.w + rp;
                        if (sq_seq(v3(b.x, b.y, b.z) - pcen) <= tt * tt) { keep = false; break; }
                    }
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (EMIT && keep) write_dot(d, base + kept + __popc(m & lt), pt, pcen, L.area[l], g, 1, g, (l << 16) | i);
            if (!EMIT && keep && kept + __popc(m & lt) < KS_CAP) ksl[EMIT ? 0 : w][kept + __popc(m & lt)] = (l << 16) | i;
            kept += __popc(m);
        }
        if (!EMIT) {
            __syncwarp();
            const int so = ks_stash(d, ksl[EMIT ? 0 : w], kept, kcur);
            if (lane == 0) { d.conv_cnt[g] = kept; d.cv_soff[g] = so; }
        }
        __syncwarp();
    }
}

// Each convex atom's frame, one thread per atom (the convex count and emit
// passes load it; a warp per atom computing it on every lane spent a long FP64
// chain per atom before its points)
__global__ void k_convex_geo(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const double rp = d.st.rp;
    for (long long gg = blockIdx.x * (long long)blockDim.x + threadIdx.x; gg < d.N; gg += (long long)gridDim.x * blockDim.x) {
        const int g = (int)gg;
        const int K = d.nnb[g];
        if (!(K > 0 && d.access[g] != 0 && d.atten[g] > 1)) continue;
        const double4 ai = d.xyzr[g];
        const V3 xi = v3(ai.x, ai.y, ai.z);
        const double ri = ai.w, eri = ri + rp, dens = d.dens[g];
        const long long off = d.nb_off[g];
        // frame from the nearest neighbour (_core.py:1665-1726)
        const int n0 = d.nb_id[off];
        const double4 an = d.xyzr[n0];
        const V3 xn = v3(an.x, an.y, an.z);
        const V3 north = normalize3(xi - xn);
        V3 vt = v3(north.y * north.y + north.z * north.z, north.x * north.x + north.z * north.z,
                   north.x * north.x + north.y * north.y);
        vt = normalize3(vt);
        if (fabs(dot_seq(vt, north)) > 0.99) vt = v3(1.0, 0.0, 0.0);
        const V3 eq = normalize3(cross3(north, vt));
        const V3 vql = cross3(eq, north);
        V3 south = v3(0.0, 0.0, -1.0);
        {
            const double rj = an.w, erj = rj + rp;
            const double dij = norm3(xn - xi);
            const V3 uij = (xn - xi) / dij;
            const double asymm = (eri * eri - erj * erj) / dij;
            const V3 tij = ((xi + xn) * 0.5) + uij * (asymm * 0.5);
            const double far_sq = (eri + erj) * (eri + erj) - dij * dij;
            const double rd = ri - rj;
            const double contain_sq = dij * dij - rd * rd;
            if (far_sq > 0.0 && contain_sq > 0.0) {
                const double rij = ((0.5 * sqrt(far_sq)) * sqrt(contain_sq)) / dij;
                const V3 pij = tij + vql * rij;
                south = (pij - xi) / eri;
            }
        }
        // latitude arc from north to south in the (north, eq x north) plane
        V3 ylat;
        const double ang = arc_angle(eq, north, south, ylat);
        const double dl = subdiv_delta(dens, ri);
        const int nl = subdiv_count_long(dl, ang);
        const double cs = subdiv_ps(ri, ang, nl);
        V3 fx, fy;
        circle_frame(north, fx, fy);
        CvGeo G;
        G.north[0] = north.x; G.north[1] = north.y; G.north[2] = north.z;
        G.ylat[0] = ylat.x; G.ylat[1] = ylat.y; G.ylat[2] = ylat.z;
        G.fx[0] = fx.x; G.fx[1] = fx.y; G.fx[2] = fx.z;
        G.fy[0] = fy.x; G.fy[1] = fy.y; G.fy[2] = fy.z;
        G.dl = dl; G.cs = cs; G.nl = nl;
        d.cv_geo[g] = G;
    }
}

void launch_convex_geo(const Dev& d, cudaStream_t s)
{
    k_convex_geo<<<grid_for(d.N, 128), 128, 0, s>>>(d);
}

void launch_convex(const Dev& d, bool emit, cudaStream_t s)
{
    if (emit) k_convex<true><<<grid_for(d.N, CV_WARPS), CV_WARPS * 32, 0, s>>>(d);
    else k_convex<false><<<grid_for(d.N, CV_WARPS), CV_WARPS * 32, 0, s>>>(d);
}

// ---------------------------------------------------------------------------
// toroidal dots: one warp per toroid pair, lanes over torus points
// ---------------------------------------------------------------------------
// Every torus point of a pair lies on one circle (centre tij, axis uij,
// radius rij), and so does the probe centre of each of its arc dots.  Before
// the points, the warp keeps the atoms whose sphere (radius r + rp) can reach
// that circle: atom i's neighbours for the collision test and, when emitting,
// the buried partners of i and j for the burial test.  The others fail those
// tests at every point of the circle (a 1e-4 A margin covers the rounding of
// the points), so the tests give the reference's results on the short lists
// (cms_circle.cuh).
// The burial test depends on the probe centre alone, so each torus point
// takes it once per arc instead of once per dot.
//
// A torus circle has few points (often under a dozen), so a warp takes
// TO_PAIRS pairs at a time and spreads their points over its lanes; when
// emitting, the dots of the 32 points of a chunk are spread over the lanes
// again, so consecutive lanes write consecutive dots.
//
// Three shapes, picked per batch shape by the autotuner: NPB pairs per warp
// batch, NW warps per CTA and registers for MINB CTAs per SM -- (16, 4, 4),
// (32, 2, any), (16, 4, 6).  Per batch up to
// NPB * 32 pruned atom ids (past it: the full lists are scanned) and as many
// kept torus points (past it: the batch is not kept).


// atoms of ids[s, e) other than `skip` that may reach the torus circle of T
__device__ __forceinline__ int tor_prune(const Dev& d, const TorPair& T, const int* ids, long long s, long long e,
                                         int skip, int* out, int cap, bool* cover = nullptr)
{
    return circle_prune(d, T.tij, T.uij, T.rij, ids, s, e, skip, out, cap, cover);
}

struct TorPoint {
    V3 pij, pi, pj, axis, pqi, pqj;
    bool valid;    // survives the neighbour collision test (gives access)
    bool arcs;     // also passes the angle test (generates dots)
};

// atom i's neighbours except atom j, strict <
__device__ __forceinline__ bool tor_collides(const Dev& d, const TorPair& T, V3 pij, const int* near, int nnear)
{
    const double rp = d.st.rp;
    if (nnear >= 0) {
        for (int k = 0; k < nnear; ++k) {
            const double4 b = d.xyzr[near[k]];
            const double t = b.w + rp;
            if (sq_alt(pij - v3(b.x, b.y, b.z)) < t * t) return true;
        }
        return false;
    }
    const long long off = d.nb_off[T.i];
    const int K = d.nnb[T.i];
    for (int k = 0; k < K; ++k) {
        const int n = d.nb_id[off + k];
        if (n == T.j) continue;
        const double4 b = d.xyzr[n];
        const double t = b.w + rp;
        if (sq_alt(pij - v3(b.x, b.y, b.z)) < t * t) return true;
    }
    return false;
}

// burial of a probe centre on the torus circle: buried_test on the pruned list
__device__ __forceinline__ int8_t tor_buried(const Dev& d, int owner, V3 pcen, const int* near, int nnear)
{
    if (nnear < 0) return buried_test(d, owner, pcen);
    const double rp = d.st.rp;
    for (int k = 0; k < nnear; ++k) {
        const double4 b = d.xyzr[near[k]];
        const double t = b.w + rp;
        if (sq_seq(v3(b.x, b.y, b.z) - pcen) <= t * t) return 1;
    }
    return 0;
}

__device__ __forceinline__ TorPoint tor_point(const Dev& d, const TorPair& T, int s, const int* near, int nnear)
{
    TorPoint P;
    const double rp = d.st.rp;
    P.pij = subdiv_point(T.tij, T.rij, T.fx, T.fy, T.dtor, s);
    P.valid = !tor_collides(d, T, P.pij, near, nnear);
    P.arcs = false;
    if (!P.valid) return P;
    P.pi = (T.xi - P.pij) / T.eri;
    P.pj = (T.xj - P.pij) / T.erj;
    P.axis = normalize3(cross3(P.pi, P.pj));
    const double dtq = rp * rp - T.rij * T.rij;
    if (dtq > 0.0 && T.between) {
        double dtq_s = sqrt(dtq);
        V3 qij = T.tij - T.uij * dtq_s;
        P.pqi = (qij - P.pij) / rp;
        P.pqj = v3(0.0, 0.0, 0.0);
    } else {
        V3 mid = normalize3(P.pi + P.pj);
        P.pqi = mid;
        P.pqj = mid;
    }
    double dt1 = dot_seq(P.pqi, P.pi);
    double dt2 = dot_seq(P.pqj, P.pj);
    P.arcs = fabs(dt1) < 1.0 && fabs(dt2) < 1.0;
    return P;
}

// area of a toroidal dot: ps * ts * (distance of the point from the torus axis) / rij
__device__ __forceinline__ double tor_area(const TorPair& T, double ps, V3 pt)
{
    V3 vec = pt - T.tij;
    double dt = dot_seq(vec, T.uij);
    double d2 = sq_seq(vec) - dt * dt;
    double dist = d2 < 0.0 ? 0.0 : sqrt(d2);
    return ((ps * T.ts) * dist) / T.rij;
}

// one arc of a torus point: x -> v around `axis` on the probe sphere at pij
struct Arc { V3 x, y; double angle, ps; int n; };

__device__ __forceinline__ Arc tor_arc(const TorPair& T, const TorPoint& P, V3 x, V3 v, double rp)
{
    Arc A;
    A.x = x;
    A.angle = arc_angle(P.axis, x, v, A.y);
    A.n = subdiv_count(T.darc, A.angle);
    A.ps = subdiv_ps(rp, A.angle, A.n);
    return A;
}

__device__ __forceinline__ bool fin3(V3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// Dots of an arc whose area is a number.  With every input finite and rij
// non-zero the points and areas are finite, so all A.n dots count.
__device__ __forceinline__ int arc_count(const TorPair& T, const TorPoint& P, const Arc& A, double rp, bool& fast)
{
    if (A.n <= 0) return 0;
    if (isfinite(A.ps) && isfinite(T.ts) && isfinite(T.rij) && T.rij != 0.0 && isfinite(T.darc) && isfinite(rp) &&
        fin3(P.pij) && fin3(A.x) && fin3(A.y) && fin3(T.tij) && fin3(T.uij))
        return A.n;
    fast = false;
    int c = 0;
    for (int t = 0; t < A.n; ++t) {
        V3 pt = subdiv_point(P.pij, rp, A.x, A.y, T.darc, t);
        if (!isnan(tor_area(T, A.ps, pt))) ++c;
    }
    return c;
}

__device__ __forceinline__ void arc_emit(const Dev& d, const TorPair& T, const TorPoint& P, const Arc& A, double rp,
                                         long long q0, int owner, long long unit, int s, int arcbit, int8_t bur)
{
    int c = 0;
    for (int t = 0; t < A.n; ++t) {
        V3 pt = subdiv_point(P.pij, rp, A.x, A.y, T.darc, t);
        double area = tor_area(T, A.ps, pt);
        if (isnan(area)) continue;
        write_dot_b(d, q0 + c, pt, P.pij, area, owner, 2, (int)unit, (s << 16) | arcbit | t, bur);
        ++c;
    }
}

__device__ __forceinline__ int warp_excl_scan(int v, int& total)
{
    const int lane = threadIdx.x & 31;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

// one lane's arc, staged for the spread-out dot loop
struct TorArcS {
    V3 p, x, y;
    double ps;
    long long pos;     // dot index of the arc's first dot
    int k, s, bur;     // pair slot in the batch, torus point, burial of its probe centre
};

// Emit the dots of the warp's arcs (c dots for this lane's arc, e its
// exclusive scan, tot the warp's total), one dot per lane per step.  Every
// arc here took the finite path, so its dots are 0 .. c-1 in order.
__device__ __forceinline__ void tor_emit_spread(const Dev& d, TorArcS* S, int* X, const TorPair* tps, const int* tq,
                                                int c, int e, int tot, V3 pij, const Arc& A, long long pos, int k,
                                                int s, int8_t bur, int arcbit)
{
    const int lane = threadIdx.x & 31;
    const double rp = d.st.rp;
    __syncwarp();
    if (c > 0) {
        TorArcS& a = S[lane];
        a.p = pij; a.x = A.x; a.y = A.y; a.ps = A.ps; a.pos = pos; a.k = k; a.s = s; a.bur = bur;
    }
    X[lane] = e;
    if (lane == 31) X[32] = e + c;
    __syncwarp();
    for (int g = lane; g < tot; g += 32) {
        int lo = 0, hi = 31;                  // the lane whose dots cover g: largest o with X[o] <= g
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (X[mid] <= g) lo = mid; else hi = mid - 1;
        }
        const TorArcS& a = S[lo];
        const TorPair& T = tps[a.k];
        const int t = g - X[lo];
        const V3 pt = subdiv_point(a.p, rp, a.x, a.y, T.darc, t);
        write_dot_b(d, a.pos + t, pt, a.p, tor_area(T, a.ps, pt), arcbit ? T.j : T.i, 2, tq[a.k],
                    (a.s << 16) | arcbit | t, (int8_t)a.bur);
    }
}

template <bool EMIT, int NPB, int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) k_toroidal(Dev d)
{
    constexpr int TO_WARPS = NW, TO_PAIRS = NPB, TO_POOL = NPB * 32, TO_KEEP = NPB * 32;
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ TorPair tp[TO_WARPS][TO_PAIRS];
    __shared__ int tq[TO_WARPS][TO_PAIRS];                  // pair index of each batch slot
    __shared__ int nsv[TO_WARPS][TO_PAIRS];                 // torus points of each pair (0: circle covered)
    __shared__ int pool[TO_WARPS][TO_POOL];
    __shared__ int pst[TO_WARPS][TO_PAIRS + 1];             // exclusive scan of torus points per pair
    __shared__ int l_off[TO_WARPS][3][TO_PAIRS];            // pruned lists: neighbours of i, partners of i, of j
    __shared__ int l_cnt[TO_WARPS][3][TO_PAIRS];
    __shared__ int run[TO_WARPS][2][TO_PAIRS];              // arc dots of each pair before the current chunk
    __shared__ int hasf[TO_WARPS][TO_PAIRS];
    __shared__ unsigned char arcf[TO_WARPS][TO_PAIRS];      // bit 0: arc 1 dots, bit 1: arc 2 dots
    __shared__ long long base[EMIT ? TO_WARPS : 1][2][TO_PAIRS];
    __shared__ TorArcS arcs[EMIT ? TO_WARPS : 1][32];
    __shared__ int arcx[EMIT ? TO_WARPS : 1][33];
    // count: the batch's torus points with arc dots in (pair, point) order and their number per pair;
    // emit: each pair's first kept point in the kept-candidate buffer
    __shared__ int tpl[EMIT ? 1 : TO_WARPS][TO_KEEP];
    __shared__ int spc[TO_WARPS][TO_PAIRS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int wc = EMIT ? 0 : w;
    StashCursor kcur{0, 0};
    const int we = EMIT ? w : 0;
    const double rp = d.st.rp;
    // count: every pair; emit: only the pairs with dots (the work list)
    const long long NT = EMIT ? d.tor_loff[d.tor_cap] : min(d.tor_off[d.N], d.tor_cap);
    const long long nbatch = (NT + TO_PAIRS - 1) / TO_PAIRS;
    for (long long bt = blockIdx.x * (long long)TO_WARPS + w; bt < nbatch; bt += (long long)gridDim.x * TO_WARPS) {
        const long long q0 = bt * TO_PAIRS;
        const int np = (int)min((long long)TO_PAIRS, NT - q0);
        __syncwarp();
        bool kok = true;                           // emit: the pair's torus points with arc dots were kept
        if (lane < np) {
            const long long q = EMIT ? (long long)d.tor_list[q0 + lane] : q0 + lane;
            const TorPair T = tor_pair_load(d, q);
            tp[w][lane] = T;
            tq[w][lane] = (int)q;
            nsv[w][lane] = T.ns;
            spc[w][lane] = 0;
            if (EMIT) {
                spc[w][lane] = d.tor_soff[q];
                kok = spc[w][lane] >= 0;
                if (kok) nsv[w][lane] = d.tor_sn[q];
            }
            run[w][0][lane] = 0; run[w][1][lane] = 0;
            hasf[w][lane] = 0;
            arcf[w][lane] = (unsigned char)((d.atten[T.i] >= 2 ? 1 : 0) | (d.atten[T.j] >= 2 ? 2 : 0));
            if (EMIT) {
                const int c = d.cplx[T.i], m = d.mol[T.i];
                base[we][0][lane] = unit_base(d, c, m, 1, d.tor1_off[q]);
                base[we][1][lane] = unit_base(d, c, m, 2, d.tor2_off[q]);
            }
        }
        // emit with every pair's points kept: those points only, all free (no collision list)
        const bool kept_pts = EMIT && __all_sync(0xffffffffu, kok);
        if (EMIT && !kept_pts && lane < np) nsv[w][lane] = tp[w][lane].ns;
        __syncwarp();
        // pruned lists of the batch's pairs; a circle inside one neighbour's
        // sphere has no free point, so its pair takes no torus points
        int used = 0;
        for (int k = 0; k < np; ++k) {
            const TorPair& T = tp[w][k];
            int c = 0;
            if (!kept_pts) {
                bool cov;
                c = tor_prune(d, T, d.nb_id, d.nb_off[T.i], d.nb_off[T.i] + d.nnb[T.i], T.j, pool[w] + used,
                              TO_POOL - used, &cov);
                if (lane == 0 && cov) nsv[w][k] = 0;
            }
            if (lane == 0) { l_off[w][0][k] = used; l_cnt[w][0][k] = c; }
            if (c > 0) used += c;
            if (EMIT) {
                const int af = arcf[w][k];
                c = (af & 1) ? tor_prune(d, T, d.bu_id, d.bu_off[T.i], d.bu_off[T.i + 1], -1, pool[w] + used,
                                         TO_POOL - used) : 0;
                if (lane == 0) { l_off[w][1][k] = used; l_cnt[w][1][k] = c; }
                if (c > 0) used += c;
                c = (af & 2) ? tor_prune(d, T, d.bu_id, d.bu_off[T.j], d.bu_off[T.j + 1], -1, pool[w] + used,
                                         TO_POOL - used) : 0;
                if (lane == 0) { l_off[w][2][k] = used; l_cnt[w][2][k] = c; }
                if (c > 0) used += c;
            }
        }
        __syncwarp();
        int tot;
        const int ex = warp_excl_scan(lane < np ? nsv[w][lane] : 0, tot);
        if (lane < np) pst[w][lane] = ex;
        if (lane == 0) pst[w][np] = tot;
        __syncwarp();
        // torus points, 32 at a time; lanes of one pair are contiguous
        int tn = 0;                                // count: kept torus points of the batch
        for (int c0 = 0; c0 < tot; c0 += 32) {
            const int g = c0 + lane;
            const bool on = g < tot;
            int k = 0;
            if (on) {
                int lo = 0, hi = np - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (pst[w][mid] <= g) lo = mid; else hi = mid - 1;
                }
                k = lo;
            }
            const TorPair& T = tp[w][k];
            const int s = !on ? 0 : (kept_pts ? d.ks_buf[spc[w][k] + (g - pst[w][k])] : g - pst[w][k]);
            int c1 = 0, c2 = 0;
            bool valid = false, fast = true;
            TorPoint P;
            Arc A1, A2;
            if (on) {
                P = tor_point(d, T, s, pool[w] + l_off[w][0][k], l_cnt[w][0][k]);
                valid = P.valid;
                if (P.arcs) {
                    const int af = arcf[w][k];
                    if (af & 1) { A1 = tor_arc(T, P, P.pi, P.pqi, rp); c1 = arc_count(T, P, A1, rp, fast); }
                    if (af & 2) { A2 = tor_arc(T, P, P.pqj, P.pj, rp); c2 = arc_count(T, P, A2, rp, fast); }
                }
            }
            const int first = on ? max(pst[w][k] - c0, 0) : lane;
            const int knext = __shfl_down_sync(0xffffffffu, k, 1);
            const int onnext = __shfl_down_sync(0xffffffffu, on ? 1 : 0, 1);
            const bool last = on && (lane == 31 || !onnext || knext != k);
            int t1, t2;
            const int e1 = warp_excl_scan(c1, t1), e2 = warp_excl_scan(c2, t2);
            const int f1 = __shfl_sync(0xffffffffu, e1, first), f2 = __shfl_sync(0xffffffffu, e2, first);
            const unsigned vm = __ballot_sync(0xffffffffu, valid);
            const unsigned km = __ballot_sync(0xffffffffu, on && c1 + c2 > 0);
            if (!EMIT) {
                if (on && c1 + c2 > 0 && tn + __popc(km & ((1u << lane) - 1u)) < TO_KEEP)
                    tpl[wc][tn + __popc(km & ((1u << lane) - 1u))] = s;
                tn += __popc(km);
            }
            if (EMIT) {
                const long long pos1 = on ? base[we][0][k] + run[w][0][k] + (e1 - f1) : 0;
                const long long pos2 = on ? base[we][1][k] + run[w][1][k] + (e2 - f2) : 0;
                int8_t bur1 = 0, bur2 = 0;
                if (c1) bur1 = tor_buried(d, T.i, P.pij, pool[w] + l_off[w][1][k], l_cnt[w][1][k]);
                if (c2) bur2 = tor_buried(d, T.j, P.pij, pool[w] + l_off[w][2][k], l_cnt[w][2][k]);
                if (__all_sync(0xffffffffu, fast)) {
                    if (t1) tor_emit_spread(d, arcs[we], arcx[we], tp[w], tq[w], c1, e1, t1, P.pij, A1, pos1, k, s, bur1,
                                            0);
                    if (t2) tor_emit_spread(d, arcs[we], arcx[we], tp[w], tq[w], c2, e2, t2, P.pij, A2, pos2, k, s, bur2,
                                            1 << 15);
                } else {
                    if (c1) arc_emit(d, T, P, A1, rp, pos1, T.i, tq[w][k], s, 0, bur1);
                    if (c2) arc_emit(d, T, P, A2, rp, pos2, T.j, tq[w][k], s, 1 << 15, bur2);
                }
            }
            __syncwarp();
            if (last) {
                run[w][0][k] += (e1 + c1) - f1;
                run[w][1][k] += (e2 + c2) - f2;
                const unsigned seg = ((2u << lane) - 1u) & ~((1u << first) - 1u);
                if (vm & seg) hasf[w][k] = 1;
                if (!EMIT) spc[w][k] += __popc(km & seg);
            }
            __syncwarp();
        }
        if (!EMIT) {
            // keep the batch's torus points with arc dots for the emit pass
            long long koff = -1;
            if (tn > 0 && tn <= TO_KEEP) {
                const long long o = stash_take(d.ks_top, d.ks_cap, kcur, tn);
                if (o >= 0) {
                    for (int e = lane; e < tn; e += 32) d.ks_buf[o + e] = tpl[wc][e];
                    koff = o;
                }
            }
            int kt;
            const int kx = warp_excl_scan(lane < np ? spc[w][lane] : 0, kt);
            if (lane < np) {
                d.tor_sn[q0 + lane] = spc[w][lane];
                d.tor_soff[q0 + lane] = koff >= 0 ? (int)(koff + kx) : -1;
            }
        }
        if (!EMIT && lane < np) {
            d.tor1_cnt[q0 + lane] = run[w][0][lane];
            d.tor2_cnt[q0 + lane] = run[w][1][lane];
            d.tor_has[q0 + lane] = (int8_t)hasf[w][lane];
        }
    }
}

void launch_toroidal(const Dev& d, long long tor_grid, bool emit, int variant, cudaStream_t s)
{
    if (variant == 1) {
        const long long batches = (tor_grid + 31) / 32;
        if (emit) k_toroidal<true, 32, 2, 1><<<grid_for(batches, 2), 2 * 32, 0, s>>>(d);
        else k_toroidal<false, 32, 2, 1><<<grid_for(batches, 2), 2 * 32, 0, s>>>(d);
        return;
    }
    const long long batches = (tor_grid + 15) / 16;
    if (variant == 0) {
        if (emit) k_toroidal<true, 16, 4, 4><<<grid_for(batches, 4), 4 * 32, 0, s>>>(d);
        else k_toroidal<false, 16, 4, 4><<<grid_for(batches, 4), 4 * 32, 0, s>>>(d);
    } else {      // registers capped for 6 CTAs per SM (24 warps)
        if (emit) k_toroidal<true, 16, 4, 6><<<grid_for(batches, 4), 4 * 32, 0, s>>>(d);
        else k_toroidal<false, 16, 4, 6><<<grid_for(batches, 4), 4 * 32, 0, s>>>(d);
    }
}

// ---------------------------------------------------------------------------
// concave dots: one warp per probe
// ---------------------------------------------------------------------------
// subdiv_point with its FP64 sincos as one called copy: the concave kernel calls it from three places, and
// inlining each copy made a kernel large enough to stall on instruction fetch (concave count 25.1 -> 24.3 ms
// with the call; the convex and toroidal kernels are faster with it inlined)
static __device__ __noinline__ void sincos_called(double a, double* s, double* c) { sincos(a, s, c); }

__device__ __forceinline__ V3 subdiv_point_called(V3 cen, double rad, V3 x, V3 y, double delta, int i)
{
    const double a = delta * ((double)i + 0.5);
    double s, c;
    sincos_called(a, &s, &c);
    const double rc = rad * c, rs = rad * s;
    return (cen + x * rc) + y * rs;
}
static constexpr int CC_WARPS = 4;

// MINB: CTAs per SM the register allocation must allow -- 4 (128 registers),
// 5 (102) or 6 (85: more warps to hide the FP64 latency, more spills); the
// autotuner picks per batch shape
template <bool EMIT, int MINB>
__global__ void __launch_bounds__(CC_WARPS * 32, MINB) k_concave(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ LatTable tab[CC_WARPS];
    __shared__ int ncs[CC_WARPS][CMS_MAX_SUBDIV];
    __shared__ int nears[CC_WARPS][CMS_NEAR_CAP];
    __shared__ int cpre[CC_WARPS][33];                 // low-probe cell columns: exclusive scan of lengths
    __shared__ long long cbeg[CC_WARPS][32];           // and each column's first entry
    __shared__ int ksl[EMIT ? 1 : CC_WARPS][KS_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    LatTable& L = tab[w];
    StashCursor kcur{0, 0};
    const double rp = d.st.rp, rp2 = rp * rp;
    const long long NP = min(d.plus_off[d.N] + d.minus_off[d.N], d.probe_cap);
    const long long wid = blockIdx.x * (long long)CC_WARPS + w;
    const long long nw = (long long)gridDim.x * CC_WARPS;
    for (long long p = wid; p < NP; p += nw) {
        if (EMIT && d.conc_cnt[p] == 0) continue;                      // no dots: nothing to write
        const int so = EMIT ? d.cc_soff[p] : -1;                         // >= 0: the count pass made the dots
        if (EMIT && so >= 0) {
            const long long base = unit_base(d, d.cplx[d.pa0[p]], d.mol[d.pa0[p]], 3, d.conc_off[p]);
            const V3 pijk = ld3(d.pxyz + 3 * p);
            const int cnt = d.conc_cnt[p];
            for (int e = lane; e < cnt; e += 32) {
                const long long k = (long long)so + e;
                write_dot_b(d, base + e, ld3(d.cs_xyz + 3 * k), pijk, d.cs_area[k], d.cs_own[k], 3, (int)p,
                            d.cs_sub[k], d.cs_bur[k]);
            }
            continue;
        }
        const int ia[3] = {d.pa0[p], d.pa1[p], d.pa2[p]};
        V3 xa[3];
        double ra[3];
        for (int k = 0; k < 3; ++k) { double4 a = d.xyzr[ia[k]]; xa[k] = v3(a.x, a.y, a.z); ra[k] = a.w; }
        const double density = ((d.dens[ia[0]] + d.dens[ia[1]]) + d.dens[ia[2]]) / 3.0;
        const V3 pijk = ld3(d.pxyz + 3 * p);
        const V3 uijk = ld3(d.palt + 3 * p);
        const bool low = d.ph[p] < rp;
        const int c = d.cplx[ia[0]];
        // nearby low probes of the same complex (d2 <= 4 rp^2), self excluded.  A complex with few low
        // probes has them scanned in list order; one with many (a whole molecule's surface) has them looked
        // up through its cells (clamped to the complex's grid) that meet the box of the 2 rp ball, one
        // (x, y) column per lane, each column's cells contiguous, then one probe per lane.
        int nnear = 0;
        const Cplx C = d.cx[c];
        long long ls = 0, le = 0;
        if (low) {
            const int s0 = C.a0, e1 = C.a0 + C.n;
            const long long pb = min(d.plus_off[s0] + d.minus_off[s0], d.probe_cap);
            const long long pe = min(d.plus_off[e1] + d.minus_off[e1], d.probe_cap);
            ls = d.plow_off[pb]; le = d.plow_off[pe];
        }
        if (low && le - ls <= CMS_LOW_CELL_MIN) {
            for (long long b = ls; b < le; b += 32) {
                long long li = b + lane;
                bool near = false;
                int qi = -1;
                if (li < le) {
                    qi = d.plow_list[li];
                    if (qi != p) near = sq_seq(pijk - ld3(d.pxyz + 3 * (long long)qi)) <= 4 * rp2;
                }
                unsigned m = __ballot_sync(0xffffffffu, near);
                int pos = nnear + __popc(m & lt);
                if (near && pos < CMS_NEAR_CAP) nears[w][pos] = qi;
                nnear += __popc(m);
            }
        } else if (low) {
            const double re = (2.0 * rp) * (1.0 + 1e-9) + 1e-9;
            const int x0 = cell_coord(pijk.x - re, C.org[0], C.h, C.dims[0]);
            const int x1 = cell_coord(pijk.x + re, C.org[0], C.h, C.dims[0]);
            const int y0 = cell_coord(pijk.y - re, C.org[1], C.h, C.dims[1]);
            const int y1 = cell_coord(pijk.y + re, C.org[1], C.h, C.dims[1]);
            const int z0 = cell_coord(pijk.z - re, C.org[2], C.h, C.dims[2]);
            const int z1 = cell_coord(pijk.z + re, C.org[2], C.h, C.dims[2]);
            const int ny = y1 - y0 + 1;
            const int ncol = (x1 - x0 + 1) * ny;
            const long long c0 = d.ncell_scan[c];
            for (int cb = 0; cb < ncol; cb += 32) {
                const int col = cb + lane;
                long long s0 = 0;
                int len = 0;
                if (col < ncol) {
                    const long long base = c0 + ((long long)(x0 + col / ny) * C.dims[1] + (y0 + col % ny)) * C.dims[2];
                    if (base + z1 < d.cells_cap) {
                        s0 = d.plc_start[base + z0];
                        len = (int)(d.plc_start[base + z1 + 1] - s0);
                    }
                }
                int tot;
                const int ex = warp_excl_scan(len, tot);
                __syncwarp();
                cpre[w][lane] = ex;
                cbeg[w][lane] = s0;
                if (lane == 31) cpre[w][32] = tot;
                __syncwarp();
                for (int b = 0; b < tot; b += 32) {
                    const int i = b + lane;
                    bool near = false;
                    int qi = -1;
                    if (i < tot) {
                        int lo = 0, hi = 31;          // column holding i: largest k with cpre[k] <= i
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (cpre[w][mid] <= i) lo = mid; else hi = mid - 1;
                        }
                        qi = d.plc_item[cbeg[w][lo] + (i - cpre[w][lo])];
                        if (qi != p) near = sq_seq(pijk - ld3(d.pxyz + 3 * (long long)qi)) <= 4 * rp2;
                    }
                    unsigned m = __ballot_sync(0xffffffffu, near);
                    int pos = nnear + __popc(m & lt);
                    if (near && pos < CMS_NEAR_CAP) nears[w][pos] = qi;
                    nnear += __popc(m);
                }
                __syncwarp();
            }
        }
        if (low) {
            if (nnear > CMS_NEAR_CAP) {
                if (lane == 0) atomicOr(&d.status[c], ST_NEAR_OVERFLOW);
                nnear = CMS_NEAR_CAP;
            }
            __syncwarp();
        }
        // spherical-triangle frame (_core.py:2140-2164), made by k_probe_geo
        const ConcGeo G = d.cc_geo[p];
        const V3 vec0 = v3(G.v0[0], G.v0[1], G.v0[2]), vec1 = v3(G.v1[0], G.v1[1], G.v1[2]);
        const V3 vec2 = v3(G.v2[0], G.v2[1], G.v2[2]);
        const V3 south = -uijk;
        const V3 vtop = v3(G.top[0], G.top[1], G.top[2]), ylat = v3(G.ylat[0], G.ylat[1], G.ylat[2]);
        const V3 fx = v3(G.fx[0], G.fx[1], G.fx[2]), fy = v3(G.fy[0], G.fy[1], G.fy[2]);
        const double dl = G.dl, cs = G.cs;
        const int nl = G.nl;
        for (int l = lane; l < nl; l += 32) {
            V3 lat = subdiv_point_called(v3(0.0, 0.0, 0.0), rp, vtop, ylat, dl, l);
            double dt = dot_seq(lat, south);
            double rsq = rp2 - dt * dt;
            double rad = sqrt(rsq < 0.0 ? 0.0 : rsq);
            int nc = 0;
            double delta = 0.0, ps = 0.0;
            if (rad > 0.0) {
                delta = subdiv_delta(density, rad);
                nc = subdiv_count_long(delta, CMS_TWO_PI);
                ps = subdiv_ps(rad, CMS_TWO_PI, nc);
            }
            L.dt[l] = dt;
            L.rad[l] = rad; L.delta[l] = delta; L.area[l] = ps * cs;
            ncs[w][l] = nc;
        }
        __syncwarp();
        lat_prefix(L, ncs[w], nl);
        const int total = nl > 0 ? L.start[nl] : 0;
        long long base = 0;
        // burial depends on the probe centre and the owner: one test per atom of the probe
        int8_t bur3[3] = {0, 0, 0};
        if (EMIT) {
            base = unit_base(d, c, d.mol[ia[0]], 3, d.conc_off[p]);
            if (d.conc_cnt[p] > 0) {
                for (int k = 0; k < 3; ++k) bur3[k] = buried_warp(d, ia[k], pijk);
            }
        }
        int kept = 0;
        for (int t0 = 0; t0 < total; t0 += 32) {
            const int t = t0 + lane;
            bool keep = false;
            V3 pts;
            int l = 0, i = 0, mc = 0;
            if (t < total) {
                l = find_lat(L, nl, t);
                i = t - L.start[l];
                V3 pt = subdiv_point_called(south * L.dt[l], L.rad[l], fx, fy, L.delta[l], i);
                keep = !(dot_seq(pt, vec0) >= 0 || dot_seq(pt, vec1) >= 0 || dot_seq(pt, vec2) >= 0);
                if (keep) {
                    pts = pt + pijk;
                    if (low) {
                        for (int k = 0; k < nnear; ++k) {
                            if (sq_alt(pts - ld3(d.pxyz + 3 * (long long)nears[w][k])) < rp2) { keep = false; break; }
                        }
                    }
                }
                if (keep) {
                    double dd[3];
                    for (int k = 0; k < 3; ++k) dd[k] = norm3(pts - xa[k]) - ra[k];
                    mc = 0;                            // np.argmin: first minimum, NaN wins
                    if (!isnan(dd[0])) {
                        for (int k = 1; k < 3; ++k) {
                            if (isnan(dd[k])) { mc = k; break; }
                            if (dd[k] < dd[mc]) mc = k;
                        }
                    }
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (EMIT && keep)
                write_dot_b(d, base + kept + __popc(m & lt), pts, pijk, L.area[l], ia[mc], 3, (int)p, (l << 16) | i,
                            mc == 0 ? bur3[0] : (mc == 1 ? bur3[1] : bur3[2]));
            if (!EMIT && keep && kept + __popc(m & lt) < KS_CAP) ksl[EMIT ? 0 : w][kept + __popc(m & lt)] = (l << 16) | i;
            kept += __popc(m);
        }
        if (!EMIT) {
            // make the probe's dots now (point, owner, burial) for the emit pass to copy
            __syncwarp();
            long long sp = -1;
            if (kept > 0 && kept <= KS_CAP) sp = stash_take(d.cs_top, d.cs_cap, kcur, kept);
            if (sp >= 0) {
                int8_t b3[3];
                for (int k = 0; k < 3; ++k) b3[k] = buried_warp(d, ia[k], pijk);
                for (int e = lane; e < kept; e += 32) {
                    const int sub = ksl[EMIT ? 0 : w][e];
                    const int l = sub >> 16, i = sub & 0xffff;
                    const V3 pts = subdiv_point_called(south * L.dt[l], L.rad[l], fx, fy, L.delta[l], i) + pijk;
                    double dd[3];
                    for (int k = 0; k < 3; ++k) dd[k] = norm3(pts - xa[k]) - ra[k];
                    int mc = 0;                        // np.argmin: first minimum, NaN wins
                    if (!isnan(dd[0])) {
                        for (int k = 1; k < 3; ++k) {
                            if (isnan(dd[k])) { mc = k; break; }
                            if (dd[k] < dd[mc]) mc = k;
                        }
                    }
                    const long long q = sp + e;
                    st3(d.cs_xyz + 3 * q, pts);
                    d.cs_area[q] = L.area[l];
                    d.cs_own[q] = ia[mc];
                    d.cs_sub[q] = sub;
                    d.cs_bur[q] = mc == 0 ? b3[0] : (mc == 1 ? b3[1] : b3[2]);
                }
            }
            if (lane == 0) { d.conc_cnt[p] = kept; d.cc_soff[p] = (int)sp; }
        }
        __syncwarp();
    }
}

// Each probe's spherical-triangle frame, one thread per probe (the concave
// count and emit passes load it; a warp per probe computing it on every lane
// spent a long FP64 chain per probe before its points)
__global__ void k_probe_geo(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const double rp = d.st.rp;
    const long long NP = min(d.plus_off[d.N] + d.minus_off[d.N], d.probe_cap);
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < NP; p += (long long)gridDim.x * blockDim.x) {
        const int ia[3] = {d.pa0[p], d.pa1[p], d.pa2[p]};
        V3 xa[3];
        for (int k = 0; k < 3; ++k) { const double4 a = d.xyzr[ia[k]]; xa[k] = v3(a.x, a.y, a.z); }
        const double density = ((d.dens[ia[0]] + d.dens[ia[1]]) + d.dens[ia[2]]) / 3.0;
        const V3 pijk = ld3(d.pxyz + 3 * p);
        const V3 uijk = ld3(d.palt + 3 * p);
        V3 vp[3];
        for (int k = 0; k < 3; ++k) vp[k] = normalize3(xa[k] - pijk);
        const V3 vec0 = normalize3(cross3(vp[0], vp[1]));
        const V3 vec1 = normalize3(cross3(vp[1], vp[2]));
        const V3 vec2 = normalize3(cross3(vp[2], vp[0]));
        double dts[3];
        for (int k = 0; k < 3; ++k) dts[k] = dot_seq(uijk, vp[k]);
        int mm = 0;                                   // np.argmax: first maximum, NaN wins
        if (!isnan(dts[0])) {
            for (int k = 1; k < 3; ++k) {
                if (isnan(dts[k])) { mm = k; break; }
                if (dts[k] > dts[mm]) mm = k;
            }
        }
        const V3 south = -uijk;
        const V3 vtop = vp[mm];
        const V3 axis = normalize3(cross3(vtop, south));
        V3 ylat;
        const double ang = arc_angle(axis, vtop, south, ylat);
        ConcGeo G;
        G.dl = subdiv_delta(density, rp);
        G.nl = subdiv_count_long(G.dl, ang);
        G.cs = subdiv_ps(rp, ang, G.nl);
        V3 fx, fy;
        circle_frame(south, fx, fy);
        G.v0[0] = vec0.x; G.v0[1] = vec0.y; G.v0[2] = vec0.z;
        G.v1[0] = vec1.x; G.v1[1] = vec1.y; G.v1[2] = vec1.z;
        G.v2[0] = vec2.x; G.v2[1] = vec2.y; G.v2[2] = vec2.z;
        G.top[0] = vtop.x; G.top[1] = vtop.y; G.top[2] = vtop.z;
        G.ylat[0] = ylat.x; G.ylat[1] = ylat.y; G.ylat[2] = ylat.z;
        G.fx[0] = fx.x; G.fx[1] = fx.y; G.fx[2] = fx.z;
        G.fy[0] = fy.x; G.fy[1] = fy.y; G.fy[2] = fy.z;
        d.cc_geo[p] = G;
    }
}

void launch_probe_geo(const Dev& d, long long probe_grid, cudaStream_t s)
{
    k_probe_geo<<<grid_for(probe_grid, 128), 128, 0, s>>>(d);
}

void launch_concave(const Dev& d, long long probe_grid, bool emit, int variant, cudaStream_t s)
{
    if (variant == 0) {
        if (emit) k_concave<true, 4><<<grid_for(probe_grid, CC_WARPS), CC_WARPS * 32, 0, s>>>(d);
        else k_concave<false, 4><<<grid_for(probe_grid, CC_WARPS), CC_WARPS * 32, 0, s>>>(d);
    } else if (variant == 1) {
        if (emit) k_concave<true, 5><<<grid_for(probe_grid, CC_WARPS), CC_WARPS * 32, 0, s>>>(d);
        else k_concave<false, 5><<<grid_for(probe_grid, CC_WARPS), CC_WARPS * 32, 0, s>>>(d);
    } else {
        if (emit) k_concave<true, 6><<<grid_for(probe_grid, CC_WARPS), CC_WARPS * 32, 0, s>>>(d);
        else k_concave<false, 6><<<grid_for(probe_grid, CC_WARPS), CC_WARPS * 32, 0, s>>>(d);
    }
}

// ---------------------------------------------------------------------------
// layout: dot segment offsets per complex, molecule and type
// ---------------------------------------------------------------------------
struct SegCounts { long long cnt[2][4], scan0[2][4]; };

__device__ __forceinline__ SegCounts seg_counts(const Dev& d, int c)
{
    SegCounts S;
    const Cplx C = d.cx[c];
    const int s0 = C.a0, s1 = C.a0 + C.n0, e1 = C.a0 + C.n;
    const int as[2] = {s0, s1}, ae[2] = {s1, e1};
    const long long pb = d.plus_off[s0] + d.minus_off[s0];
    const long long P0 = (d.plus_off[s1] - d.plus_off[s0]) + (d.minus_off[s1] - d.minus_off[s0]);
    const long long P1 = (d.plus_off[e1] - d.plus_off[s1]) + (d.minus_off[e1] - d.minus_off[s1]);
    const long long ps[2] = {pb, pb + P0}, pe[2] = {pb + P0, pb + P0 + P1};
    for (int m = 0; m < 2; ++m) {
        S.scan0[m][0] = d.conv_off[as[m]];
        S.cnt[m][0] = d.conv_off[ae[m]] - S.scan0[m][0];
        // clamped to the capacities: past them the run is flagged and redone
        const long long ts = min(d.tor_off[as[m]], d.tor_cap), te = min(d.tor_off[ae[m]], d.tor_cap);
        S.scan0[m][1] = d.tor1_off[ts];
        S.cnt[m][1] = d.tor1_off[te] - S.scan0[m][1];
        S.scan0[m][2] = d.tor2_off[ts];
        S.cnt[m][2] = d.tor2_off[te] - S.scan0[m][2];
        S.scan0[m][3] = d.conc_off[min(ps[m], d.probe_cap)];
        S.cnt[m][3] = d.conc_off[min(pe[m], d.probe_cap)] - S.scan0[m][3];
    }
    return S;
}

__global__ void k_layout_counts(Dev d, int* cm_count)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.B; c += gridDim.x * blockDim.x) {
        SegCounts S = seg_counts(d, c);
        for (int m = 0; m < 2; ++m)
            cm_count[c * 2 + m] = (int)(S.cnt[m][0] + S.cnt[m][1] + S.cnt[m][2] + S.cnt[m][3]);
    }
}

__global__ void k_layout_seg(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.B; c += gridDim.x * blockDim.x) {
        SegCounts S = seg_counts(d, c);
        for (int m = 0; m < 2; ++m) {
            long long pos = d.dot_off[c * 2 + m];
            for (int t = 0; t < 4; ++t) {
                Seg g;
                g.dot0 = pos;
                g.scan0 = S.scan0[m][t];
                d.seg[(c * 2 + m) * 4 + t] = g;
                pos += S.cnt[m][t];
            }
        }
    }
}

void launch_layout(const Dev& d, long long* cm_count_tmp, long long* scan_tmp, cudaStream_t s)
{
    int* cm = reinterpret_cast<int*>(cm_count_tmp);
    k_layout_counts<<<grid_for(d.B, 128), 128, 0, s>>>(d, cm);
    scan_counts(cm, d.dot_off, 2LL * d.B, scan_tmp, s);
    k_layout_seg<<<grid_for(d.B, 128), 128, 0, s>>>(d);
}

// ---------------------------------------------------------------------------
// toroidal access flags: access[natoms1] |= has, then access[natoms2] |= has,
// where NumPy's fancy-index read-modify-write keeps, for a repeated atom, the
// value computed for its last occurrence (_core.py:1247-1248)
// ---------------------------------------------------------------------------
__global__ void k_tor_last(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NT = min(d.tor_off[d.N], d.tor_cap);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < NT; q += (long long)gridDim.x * blockDim.x)
        atomicMax(&d.tor_last2[d.tor_j[q]], (unsigned long long)(q + 1));
}

__global__ void k_tor_access_apply(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (long long a = blockIdx.x * (long long)blockDim.x + threadIdx.x; a < d.N; a += (long long)gridDim.x * blockDim.x) {
        int8_t v = d.access[a];
        if (d.tor_off[a + 1] > d.tor_off[a]) v |= d.tor_has[d.tor_off[a + 1] - 1];   // rows are grouped by atom1
        unsigned long long l2 = d.tor_last2[a];
        if (l2 > 0) v |= d.tor_has[l2 - 1];
        d.access[a] = v;
    }
}

// work list of the emit pass: the toroid pairs with at least one dot, in pair order
__global__ void k_tor_flag(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.tor_cap; q += (long long)gridDim.x * blockDim.x)
        d.tor_lflag[q] = (d.tor1_cnt[q] | d.tor2_cnt[q]) != 0 ? 1 : 0;
}

__global__ void k_tor_list(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < d.tor_cap; q += (long long)gridDim.x * blockDim.x)
        if (d.tor_lflag[q]) d.tor_list[d.tor_loff[q]] = (int)q;
}

void launch_tor_list(const Dev& d, long long tor_grid, long long* scan_tmp, cudaStream_t s)
{
    k_tor_flag<<<grid_for(tor_grid, 256), 256, 0, s>>>(d);
    scan_counts(d.tor_lflag, d.tor_loff, tor_grid, scan_tmp, s);
    k_tor_list<<<grid_for(tor_grid, 256), 256, 0, s>>>(d);
}

void launch_tor_access(const Dev& d, long long tor_grid, cudaStream_t s)
{
    cudaMemsetAsync(d.tor_last2, 0, sizeof(unsigned long long) * d.N, s);
    k_tor_last<<<grid_for(tor_grid, 256), 256, 0, s>>>(d);
    k_tor_access_apply<<<grid_for(d.N, 256), 256, 0, s>>>(d);
}

}  // namespace cms
