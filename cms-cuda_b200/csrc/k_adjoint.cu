// FP64 adjoint of the contact molecular surface: d(sum_c g_c CMS_c)/d(xyz)
// with the dot topology held fixed.
//
// CMS of one side of a complex (cms-cuda/_core.py:946-1004) is
//   sum over the side's buried dots q of  area_q * exp(-w |p_q - p_r(q)|^2)
// where r(q) is the nearest buried dot of the other side (first index on
// ties).  Holding the topology fixed means keeping which dots exist, their
// burial, their (latitude, point) / (torus point, arc point) indices, every
// branch of the construction and r(q); positions and areas then are smooth
// functions of the atom coordinates:
//   convex dot of atom i      -- coordinates of i and of its first neighbour
//                                (the frame atom), _core.py:1646-1840
//   toroidal dot of pair i, j -- coordinates of i and j, _core.py:1847-2067
//   concave dot of a probe    -- coordinates of its three atoms, through the
//                                probe solve of _core.py:1445-1643 and the
//                                cap construction of _core.py:2069-2333
//
// Passes:
//   1. per query dot: the adjoints of its area and position, and the
//      contribution to its nearest dot's position;
//   2. per reference dot: the sum of the contributions from the queries that
//      picked it, in query order (counting sort by reference dot);
//   3. per unit (atom / toroid pair / probe) holding a dot with a non-zero
//      adjoint: the unit's geometry in forward-mode duals (6 or 9 tangents,
//      cms_dual.cuh), the Jacobian-transpose products summed over its dots in
//      dot order, one 3-vector per atom of the unit;
//   4. per atom: the unit contributions gathered by one warp, lanes over the
//      atom's row and units, summed in a fixed tree.
// Every sum has a fixed order, so the gradient is deterministic.
//
// The same unit code run on plain doubles recomputes the dots; that recompute
// must equal the surface kernels' output bit for bit, which ties the
// differentiated formula to the generated surface.
#include "cms_dual.cuh"
#include <algorithm>

#include "cms_readout.cuh"

namespace cms {

static constexpr int SM_COUNT_ADJ = 148;

static inline unsigned grid_adj(long long items, int per_block)
{
    long long b = (items + per_block - 1) / per_block;
    const long long cap = (long long)SM_COUNT_ADJ * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

__device__ __forceinline__ long long adj_doff(const Dev& d, long long i) { return min(d.dot_off[i], d.dot_cap); }

__device__ __forceinline__ long long adj_unit_base(const Dev& d, int c, int m, int t, long long unit_scan)
{
    const Seg s = d.seg[(c * 2 + m) * 4 + t];
    return s.dot0 + (unit_scan - s.scan0);
}

// ---------------------------------------------------------------------------
// unit geometry, templated on double / Dn<K>
// ---------------------------------------------------------------------------
template <class T> struct DotV { TV3<T> p; T area; };

// convex unit of atom g with frame atom n0 (k_convex in k_dots.cu)
template <class T> struct ConvexU {
    TV3<T> xi, north, ylat, fx, fy;
    T cs;
    double ri, dl, dens;
    int nl;
};

template <class T>
__device__ __forceinline__ ConvexU<T> convex_unit(const Dev& d, int g, const TV3<T>& xi, const TV3<T>& xn, double ri,
                                                  double rj)
{
    ConvexU<T> U;
    const double rp = d.st.rp;
    const double eri = ri + rp;
    U.xi = xi; U.ri = ri; U.dens = d.dens[g];
    U.north = tnormalize(xi - xn);
    const TV3<T>& n = U.north;
    TV3<T> vt = tv3<T>(n.y * n.y + n.z * n.z, n.x * n.x + n.z * n.z, n.x * n.x + n.y * n.y);
    vt = tnormalize(vt);
    if (fabs(val(tdot_seq(vt, n))) > 0.99) vt = tconst<T>(v3(1.0, 0.0, 0.0));
    const TV3<T> eq = tnormalize(tcross(n, vt));
    const TV3<T> vql = tcross(eq, n);
    TV3<T> south = tconst<T>(v3(0.0, 0.0, -1.0));
    {
        const double erj = rj + rp;
        const T dij = tnorm(xn - xi);
        const TV3<T> uij = (xn - xi) / dij;
        const T asymm = (eri * eri - erj * erj) / dij;
        const TV3<T> tij = ((xi + xn) * 0.5) + uij * (asymm * 0.5);
        const T far_sq = (eri + erj) * (eri + erj) - dij * dij;
        const double rd = ri - rj;
        const T contain_sq = dij * dij - rd * rd;
        if (val(far_sq) > 0.0 && val(contain_sq) > 0.0) {
            const T rij = ((0.5 * dsqrt(far_sq)) * dsqrt(contain_sq)) / dij;
            const TV3<T> pij = tij + vql * rij;
            south = (pij - xi) / eri;
        }
    }
    const T ang = tarc_angle(eq, n, south, U.ylat);
    U.dl = subdiv_delta(U.dens, ri);
    U.nl = subdiv_count_long(U.dl, val(ang));
    U.cs = tsubdiv_ps(ri, ang, U.nl);
    tcircle_frame(n, U.fx, U.fy);
    return U;
}

template <class T> struct LatU { TV3<T> cen; T rad, delta, area; };

template <class T>
__device__ __forceinline__ LatU<T> convex_lat(const ConvexU<T>& U, int l)
{
    LatU<T> L;
    const TV3<T> lat = tsubdiv_point(tconst<T>(v3(0.0, 0.0, 0.0)), U.ri, U.north, U.ylat, U.dl, l);
    const T dt = tdot_seq(lat, U.north);
    L.cen = U.xi + U.north * dt;
    const T rsq = U.ri * U.ri - dt * dt;
    L.rad = val(rsq) > 0.0 ? dsqrt(rsq) : lift<T>(0.0);
    L.delta = lift<T>(0.0);
    L.area = lift<T>(0.0);
    if (val(L.rad) > 0.0) {
        L.delta = tsubdiv_delta(U.dens, L.rad);
        const int nc = subdiv_count_long(val(L.delta), CMS_TWO_PI);
        const T ps = nc > 0 ? (L.rad * CMS_TWO_PI) / (double)nc : lift<T>(0.0);
        L.area = ps * U.cs;
    }
    return L;
}

// toroidal unit of pair (i, j) (tor_pair / tor_point / tor_arc / tor_area in k_dots.cu)
template <class T> struct TorU {
    TV3<T> xi, xj, uij, tij, fx, fy;
    T rij, ts, dtor;
    double eri, erj, darc;
    bool between;
};

template <class T>
__device__ __forceinline__ TorU<T> tor_unit(const Dev& d, int i, int j, const TV3<T>& xi, const TV3<T>& xj)
{
    TorU<T> U;
    const double rp = d.st.rp;
    const double ri = d.xyzr[i].w, rj = d.xyzr[j].w;
    U.xi = xi; U.xj = xj;
    const TV3<T> diff = xj - xi;
    const T dij_sq = tdot_alt(diff, diff);
    const T dij = dsqrt(dij_sq);
    U.eri = ri + rp; U.erj = rj + rp;
    const T asymm = (U.eri * U.eri - U.erj * U.erj) / dij;
    U.between = fabs(val(asymm)) < val(dij);
    U.uij = diff / dij;
    U.tij = ((xi + xj) * 0.5) + U.uij * (asymm * 0.5);
    const T far_sq = (U.eri + U.erj) * (U.eri + U.erj) - dij_sq;
    const double rd = ri - rj;
    const T cont_sq = dij_sq - rd * rd;
    U.rij = ((0.5 * dsqrt(far_sq)) * dsqrt(cont_sq)) / dij;
    const double density = (d.dens[i] + d.dens[j]) * 0.5;
    const T rci = (U.rij * ri) / U.eri;
    const T rcj = (U.rij * rj) / U.erj;
    const T rbt = U.rij - rp;
    const T rb = val(rbt) < 0.0 ? lift<T>(0.0) : rbt;
    const T rs = ((rci + 2.0 * rb) + rcj) * 0.25;
    const T e = rs / U.rij;
    const T edens = (e * e) * density;
    tcircle_frame(U.uij, U.fx, U.fy);
    U.dtor = 1.0 / (dsqrt(edens) * U.rij);
    const int ns = subdiv_count(val(U.dtor), CMS_TWO_PI);
    U.ts = tsubdiv_ps(U.rij, lift<T>(CMS_TWO_PI), ns);
    U.darc = subdiv_delta(density, rp);
    return U;
}

// one arc of torus point s: start x, frame y, per-point length ps
template <class T> struct TorArcU { TV3<T> pij, x, y; T ps; };

template <class T>
__device__ __forceinline__ TorArcU<T> tor_point_arc(const Dev& d, const TorU<T>& U, int s, bool arc2)
{
    const double rp = d.st.rp;
    TorArcU<T> A;
    A.pij = tsubdiv_point(U.tij, U.rij, U.fx, U.fy, U.dtor, s);
    const TV3<T> pi = (U.xi - A.pij) / U.eri;
    const TV3<T> pj = (U.xj - A.pij) / U.erj;
    const TV3<T> axis = tnormalize(tcross(pi, pj));
    const T dtq = rp * rp - U.rij * U.rij;
    TV3<T> pqi, pqj;
    if (val(dtq) > 0.0 && U.between) {
        const T dtq_s = dsqrt(dtq);
        const TV3<T> qij = U.tij - U.uij * dtq_s;
        pqi = (qij - A.pij) / rp;
        pqj = tconst<T>(v3(0.0, 0.0, 0.0));
    } else {
        const TV3<T> mid = tnormalize(pi + pj);
        pqi = mid;
        pqj = mid;
    }
    const TV3<T> x = arc2 ? pqj : pi;
    const TV3<T> v = arc2 ? pj : pqi;
    A.x = x;
    const T ang = tarc_angle(axis, x, v, A.y);
    const int n = subdiv_count(U.darc, val(ang));
    A.ps = tsubdiv_ps(rp, ang, n);
    return A;
}

template <class T>
__device__ __forceinline__ DotV<T> tor_dot(const Dev& d, const TorU<T>& U, const TorArcU<T>& A, int t)
{
    DotV<T> D;
    D.p = tsubdiv_point(A.pij, d.st.rp, A.x, A.y, U.darc, t);
    const TV3<T> vec = D.p - U.tij;
    const T dt = tdot_seq(vec, U.uij);
    const T d2 = tdot_seq(vec, vec) - dt * dt;
    const T dist = val(d2) < 0.0 ? lift<T>(0.0) : dsqrt(d2);
    D.area = ((A.ps * U.ts) * dist) / U.rij;
    return D;
}

// probe solve of the triple loop (triples_flush in k_surface.cu): the probe
// of sign sg (+1 / -1) over atoms i, j, k and its direction (alt = sg * uijk)
template <class T>
__device__ __forceinline__ void probe_solve(const Dev& d, const TV3<T>& xi, double ri, const TV3<T>& xj, double rj,
                                            const TV3<T>& xk, double rk, double sg, TV3<T>& pijk, TV3<T>& alt)
{
    const double rp = d.st.rp;
    const double eri = ri + rp, erj = rj + rp, erk = rk + rp;
    const TV3<T> diff = xj - xi;
    const T dij_sq = tdot_alt(diff, diff);
    const T dij = dsqrt(dij_sq);
    const T asymm_j = (eri * eri - erj * erj) / dij;
    const TV3<T> uij = diff / dij;
    const TV3<T> tij = ((xi + xj) * 0.5) + uij * (asymm_j * 0.5);
    const TV3<T> vk = xk - xi;
    const T dik = tnorm(vk);
    const TV3<T> uik = vk / dik;
    const T dt = tdot_alt(uij, uik);
    const T dtc = val(dt) < -1.0 ? lift<T>(-1.0) : (val(dt) > 1.0 ? lift<T>(1.0) : dt);
    const T wijk = dacos(dtc);
    const T swijk = dsin(wijk);
    const TV3<T> uijk = tcross(uij, uik) / swijk;
    const TV3<T> utb = tcross(uijk, uij);
    const T asymm = (eri * eri - erk * erk) / dik;
    const TV3<T> tik = (xi + xk) * 0.5 + uik * (asymm * 0.5);
    const T dtb = tdot_alt(uik, tik - tij);
    const TV3<T> bijk = tij + utb * (dtb / swijk);
    const TV3<T> bma = bijk - xi;
    const T h2 = eri * eri - tdot_alt(bma, bma);
    const T h = dsqrt(h2);
    pijk = bijk + uijk * (h * sg);
    alt = uijk * sg;
}

// concave unit of a probe (k_concave in k_dots.cu)
template <class T> struct ConcU {
    TV3<T> pijk, south, vtop, ylat, fx, fy;
    T cs;
    double density, dl;
    int nl;
};

template <class T>
__device__ __forceinline__ ConcU<T> conc_unit(const Dev& d, const TV3<T>* xa, const int* ia, const TV3<T>& pijk,
                                              const TV3<T>& uijk)
{
    ConcU<T> U;
    const double rp = d.st.rp;
    U.pijk = pijk;
    U.density = ((d.dens[ia[0]] + d.dens[ia[1]]) + d.dens[ia[2]]) / 3.0;
    TV3<T> vp[3];
    for (int k = 0; k < 3; ++k) vp[k] = tnormalize(xa[k] - pijk);
    double dts[3];
    for (int k = 0; k < 3; ++k) dts[k] = val(tdot_seq(uijk, vp[k]));
    int mm = 0;                                   // np.argmax: first maximum, NaN wins
    if (!isnan(dts[0])) {
        for (int k = 1; k < 3; ++k) {
            if (isnan(dts[k])) { mm = k; break; }
            if (dts[k] > dts[mm]) mm = k;
        }
    }
    U.south = -uijk;
    U.vtop = vp[mm];
    const TV3<T> axis = tnormalize(tcross(U.vtop, U.south));
    const T ang = tarc_angle(axis, U.vtop, U.south, U.ylat);
    U.dl = subdiv_delta(U.density, rp);
    U.nl = subdiv_count_long(U.dl, val(ang));
    U.cs = tsubdiv_ps(rp, ang, U.nl);
    tcircle_frame(U.south, U.fx, U.fy);
    return U;
}

template <class T>
__device__ __forceinline__ LatU<T> conc_lat(const Dev& d, const ConcU<T>& U, int l)
{
    const double rp = d.st.rp, rp2 = rp * rp;
    LatU<T> L;
    const TV3<T> lat = tsubdiv_point(tconst<T>(v3(0.0, 0.0, 0.0)), rp, U.vtop, U.ylat, U.dl, l);
    const T dt = tdot_seq(lat, U.south);
    L.cen = U.south * dt;
    const T rsq = rp2 - dt * dt;
    L.rad = dsqrt(val(rsq) < 0.0 ? lift<T>(0.0) : rsq);
    L.delta = lift<T>(0.0);
    L.area = lift<T>(0.0);
    if (val(L.rad) > 0.0) {
        L.delta = tsubdiv_delta(U.density, L.rad);
        const int nc = subdiv_count_long(val(L.delta), CMS_TWO_PI);
        const T ps = nc > 0 ? (L.rad * CMS_TWO_PI) / (double)nc : lift<T>(0.0);
        L.area = ps * U.cs;
    }
    return L;
}

// the sign of probe p and the index of its triple's atom i among (a0, a1, a2):
// probes are laid out per complex as [+mol0 | -mol0 | +mol1 | -mol1]
__device__ __forceinline__ bool probe_is_plus(const Dev& d, long long p, int a0)
{
    const int c = d.cplx[a0];
    const Cplx C = d.cx[c];
    const int s0 = C.a0, s1 = C.a0 + C.n0, e1 = C.a0 + C.n;
    const int m = d.mol[a0];
    const int ms = m == 0 ? s0 : s1, me = m == 0 ? s1 : e1;
    const long long cbase = d.plus_off[s0] + d.minus_off[s0];
    const long long m0 = (d.plus_off[s1] - d.plus_off[s0]) + (d.minus_off[s1] - d.minus_off[s0]);
    const long long mb = cbase + (m == 0 ? 0 : m0);
    return p < mb + (d.plus_off[me] - d.plus_off[ms]);
}

// ---------------------------------------------------------------------------
// per-unit drivers: f.want(dot) selects dots, f.take(dot, DotV) consumes them
// ---------------------------------------------------------------------------
// Seeds of the atom coordinates: Plain (doubles), Lane (one tangent: the
// coordinate 3 * slot + axis equal to the lane's k gets derivative 1)
struct SeedPlain {
    __device__ TV3<double> atom(const Dev& d, int a, int) const
    {
        const double4 x = d.xyzr[a];
        return tv3<double>(x.x, x.y, x.z);
    }
};

// A lane's NT tangents: coordinates [NT k, NT k + NT) of the unit's atoms
// (x, y, z of atom slot 0, then of slot 1, ...)
template <int NT>
struct SeedLane {
    int k;
    __device__ TV3<Dn<NT>> atom(const Dev& d, int a, int slot) const
    {
        const double4 x = d.xyzr[a];
        const int b = 3 * slot - NT * k;         // tangent index of this atom's x coordinate
        return tv3<Dn<NT>>(dn_var<NT>(x.x, b), dn_var<NT>(x.y, b + 1), dn_var<NT>(x.z, b + 2));
    }
};

// the first dot in [q, e) the consumer wants (e when none): the unit loops step from wanted dot to wanted dot,
// so the lanes of a warp, whose units hold about as many such dots (the units are ordered by that count), run
// their k-th wanted dots together
template <class F>
__device__ __forceinline__ long long next_wanted(const Dev& d, const F& f, long long q, long long e)
{
    while (q < e && (q >= d.dot_cap || !f.want(q))) ++q;
    return q;
}

template <class T, class S, class F>
__device__ __forceinline__ void convex_unit_dots(const Dev& d, int g, const S& seed, F& f)
{
    const long long base = adj_unit_base(d, d.cplx[g], d.mol[g], 0, d.conv_off[g]);
    const int cnt = d.conv_cnt[g];
    const int n0 = d.nb_id[d.nb_off[g]];
    const ConvexU<T> U = convex_unit<T>(d, g, seed.atom(d, g, 0), seed.atom(d, n0, 1), d.xyzr[g].w, d.xyzr[n0].w);
    int cur = -1;
    LatU<T> L;
    for (long long q = next_wanted(d, f, base, base + cnt); q < base + cnt; q = next_wanted(d, f, q + 1, base + cnt)) {
        const int sub = d.dsub[q];
        const int l = sub >> 16, i = sub & 0xffff;
        if (l != cur) { L = convex_lat(U, l); cur = l; }
        DotV<T> D;
        D.p = tsubdiv_point(L.cen, L.rad, U.fx, U.fy, L.delta, i);
        D.area = L.area;
        f.take(q, D);
    }
}

template <class T, class S, class F>
__device__ __forceinline__ void tor_unit_dots(const Dev& d, long long qp, const S& seed, F& f)
{
    const int i = d.tor_i[qp], j = d.tor_j[qp];
    const int c = d.cplx[i], m = d.mol[i];
    const TorU<T> U = tor_unit<T>(d, i, j, seed.atom(d, i, 0), seed.atom(d, j, 1));
    for (int arc = 0; arc < 2; ++arc) {
        const long long base = adj_unit_base(d, c, m, 1 + arc, arc ? d.tor2_off[qp] : d.tor1_off[qp]);
        const int cnt = arc ? d.tor2_cnt[qp] : d.tor1_cnt[qp];
        int cur = -1;
        TorArcU<T> A;
        for (long long q = next_wanted(d, f, base, base + cnt); q < base + cnt; q = next_wanted(d, f, q + 1, base + cnt)) {
            const int sub = d.dsub[q];
            const int s = sub >> 16, t = sub & 0x7fff;
            if (s != cur) { A = tor_point_arc(d, U, s, arc == 1); cur = s; }
            f.take(q, tor_dot(d, U, A, t));
        }
    }
}

template <class T, class S, class F>
__device__ __forceinline__ void conc_unit_dots(const Dev& d, long long p, const S& seed, F& f)
{
    const int ia[3] = {d.pa0[p], d.pa1[p], d.pa2[p]};
    TV3<T> xa[3];
    for (int k = 0; k < 3; ++k) xa[k] = seed.atom(d, ia[k], k);
    const bool plus = probe_is_plus(d, p, ia[0]);
    // the triple's (i, j): (a0, a1) for a "+" probe, (a1, a0) for a "-" probe
    const int si = plus ? 0 : 1, sj = plus ? 1 : 0;
    TV3<T> pijk, uijk;
    probe_solve<T>(d, xa[si], d.xyzr[ia[si]].w, xa[sj], d.xyzr[ia[sj]].w, xa[2], d.xyzr[ia[2]].w, plus ? 1.0 : -1.0,
                   pijk, uijk);
    const ConcU<T> U = conc_unit<T>(d, xa, ia, pijk, uijk);
    const int c = d.cplx[ia[0]];
    const long long base = adj_unit_base(d, c, d.mol[ia[0]], 3, d.conc_off[p]);
    const int cnt = d.conc_cnt[p];
    int cur = -1;
    LatU<T> L;
    for (long long q = next_wanted(d, f, base, base + cnt); q < base + cnt; q = next_wanted(d, f, q + 1, base + cnt)) {
        const int sub = d.dsub[q];
        const int l = sub >> 16, i = sub & 0xffff;
        if (l != cur) { L = conc_lat(d, U, l); cur = l; }
        DotV<T> D;
        D.p = tsubdiv_point(L.cen, L.rad, U.fx, U.fy, L.delta, i) + U.pijk;
        D.area = L.area;
        f.take(q, D);
    }
}

// ---------------------------------------------------------------------------
// recompute (plain doubles): positions and areas of every dot
// ---------------------------------------------------------------------------
struct RecomputeF {
    double* xyz; double* area;
    __device__ bool want(long long) const { return true; }
    __device__ void take(long long q, const DotV<double>& D)
    {
        xyz[3 * q] = D.p.x; xyz[3 * q + 1] = D.p.y; xyz[3 * q + 2] = D.p.z;
        area[q] = D.area;
    }
};

__global__ void k_recompute(Dev d, double* xyz, double* area)
{
    RecomputeF f{xyz, area};
    const SeedPlain seed;
    const long long NT = min(d.tor_off[d.N], d.tor_cap);
    const long long NP = min(d.plus_off[d.N] + d.minus_off[d.N], d.probe_cap);
    const long long total = d.N + NT + NP;
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < total; u += (long long)gridDim.x * blockDim.x) {
        if (u < d.N) {
            if (d.conv_cnt[u] > 0) convex_unit_dots<double>(d, (int)u, seed, f);
        } else if (u < d.N + NT) {
            tor_unit_dots<double>(d, u - d.N, seed, f);
        } else {
            conc_unit_dots<double>(d, u - d.N - NT, seed, f);
        }
    }
}

void launch_recompute(const Dev& d, double* xyz, double* area, cudaStream_t s)
{
    k_recompute<<<grid_adj((long long)d.N + d.tor_cap + d.probe_cap, 128), 128, 0, s>>>(d, xyz, area);
}

// ---------------------------------------------------------------------------
// adjoint
// ---------------------------------------------------------------------------
// a dot given an adjoint makes its unit active and counts toward the unit's work
__device__ __forceinline__ void mark_unit(const Dev& d, const AdjBuf& a, int dot)
{
    const int t = d.dtype[dot], u = d.dunit[dot];
    atomicAdd(t == 1 ? &a.act_conv[u] : (t == 2 ? &a.act_tor[u] : &a.act_conc[u]), 1);
}

// pass 1: query dots of `side`; A = (d/dp, d/darea) per dot
__global__ void k_adj_queries(Dev d, Rd r, AdjBuf a, const NNTask* task, int side)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NB = r.bur_scan[adj_doff(d, 2LL * d.B)];
    const double w = d.st.weight;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < NB; k += (long long)gridDim.x * blockDim.x) {
        a.ref_ent[k] = -1;
        const int cm = r.bur_cm[k];
        if ((cm & 1) != side) continue;
        const NNTask T = task[cm];
        const int idx = a.cms_idx[k];
        if (T.rn <= 0 || idx < 0 || idx >= T.rn) continue;
        const int q = r.bur_idx[k];
        const long long re = T.r0 + idx;            // the reference's buried entry
        const int rd = r.bur_idx[re];
        const double g = a.gtot[cm >> 1];
        const double* pq = d.dxyz + 3LL * q;
        const double* pr = d.dxyz + 3LL * rd;
        // cdist(ref, query) order, as the search computed it
        const double dx = pr[0] - pq[0], dy = pr[1] - pq[1], dz = pr[2] - pq[2];
        const double d2 = (dx * dx + dy * dy) + dz * dz;
        const double e = exp((-d2) * w);
        const double area = d.darea[q];
        // d(area e)/dp_q = area e (-w) 2 (p_q - p_r) = area e 2w (p_r - p_q)
        const double s = g * area * e * 2.0 * w;
        a.A[q] = make_double4(s * dx, s * dy, s * dz, g * e);
        mark_unit(d, a, q);
        a.ref_ent[k] = (int)re;
        a.ref_vec[k] = make_double4(-s * dx, -s * dy, -s * dz, 0.0);
    }
}

// pass 2: reference contributions, counting sort by the reference's buried entry
__global__ void k_adj_ref_count(Dev d, Rd r, AdjBuf a)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NB = r.bur_scan[adj_doff(d, 2LL * d.B)];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < NB; k += (long long)gridDim.x * blockDim.x) {
        const int re = a.ref_ent[k];
        if (re >= 0) atomicAdd(&a.rcnt[re], 1);
    }
}

__global__ void k_adj_ref_fill(Dev d, Rd r, AdjBuf a)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NB = r.bur_scan[adj_doff(d, 2LL * d.B)];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < NB; k += (long long)gridDim.x * blockDim.x) {
        const int re = a.ref_ent[k];
        if (re >= 0) a.rslot[a.roff[re] + atomicAdd(&a.rfill[re], 1)] = (int)k;
    }
}

__global__ void k_adj_ref_sum(Dev d, Rd r, AdjBuf a)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NB = r.bur_scan[adj_doff(d, 2LL * d.B)];
    for (long long re = blockIdx.x * (long long)blockDim.x + threadIdx.x; re < NB; re += (long long)gridDim.x * blockDim.x) {
        const int n = a.rcnt[re];
        if (n == 0) continue;
        int* s = a.rslot + a.roff[re];
        for (int i = 1; i < n; ++i) {          // query order
            const int v = s[i];
            int k = i - 1;
            while (k >= 0 && s[k] > v) { s[k + 1] = s[k]; --k; }
            s[k + 1] = v;
        }
        double x = 0.0, y = 0.0, z = 0.0;
        for (int i = 0; i < n; ++i) {
            const double4 v = a.ref_vec[s[i]];
            x += v.x; y += v.y; z += v.z;
        }
        const int rd = r.bur_idx[re];
        const double4 o = a.A[rd];
        a.A[rd] = make_double4(o.x + x, o.y + y, o.z + z, o.w);
        mark_unit(d, a, rd);
    }
}

// active units of each kind, in any order (each unit owns its output slots)
__global__ void k_adj_collect(Dev d, AdjBuf a)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NT = min(d.tor_off[d.N], d.tor_cap);
    const long long NP = min(d.plus_off[d.N] + d.minus_off[d.N], d.probe_cap);
    const long long total = d.N + NT + NP;
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < total; u += (long long)gridDim.x * blockDim.x) {
        if (u < d.N) {
            if (a.act_conv[u]) a.list_conv[atomicAdd(&a.nact[0], 1)] = (int)u;
        } else if (u < d.N + NT) {
            if (a.act_tor[u - d.N]) a.list_tor[atomicAdd(&a.nact[1], 1)] = (int)(u - d.N);
        } else {
            if (a.act_conc[u - d.N - NT]) a.list_conc[atomicAdd(&a.nact[2], 1)] = (int)(u - d.N - NT);
        }
    }
}

// Active units ordered by the number of their dots given an adjoint, largest
// first, so the units that share a warp run loops of similar length (a
// counting sort on the clamped count; the order inside a key does not matter:
// every unit writes its own slots and the gather sums them in a fixed order).
static constexpr int ADJ_KEYS = 256;

__device__ __forceinline__ int adj_unit_key(const AdjBuf& a, int kind, int u)
{
    const int c = kind == 0 ? a.act_conv[u] : (kind == 1 ? a.act_tor[u] : a.act_conc[u]);
    return ADJ_KEYS - 1 - min(max(c, 0), ADJ_KEYS - 1);
}

__device__ __forceinline__ bool adj_entry(const AdjBuf& a, long long e, int& kind, int& u)
{
    const long long n0 = a.nact[0], n1 = a.nact[1], n2 = a.nact[2];
    if (e < n0) { kind = 0; u = a.list_conv[e]; return true; }
    if (e < n0 + n1) { kind = 1; u = a.list_tor[e - n0]; return true; }
    if (e < n0 + n1 + n2) { kind = 2; u = a.list_conc[e - n0 - n1]; return true; }
    return false;
}

__global__ void k_adj_key_count(Dev d, AdjBuf a)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ int h[3 * ADJ_KEYS];
    for (int i = threadIdx.x; i < 3 * ADJ_KEYS; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const long long total = (long long)a.nact[0] + a.nact[1] + a.nact[2];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        int kind, u;
        if (adj_entry(a, e, kind, u)) atomicAdd(&h[kind * ADJ_KEYS + adj_unit_key(a, kind, u)], 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * ADJ_KEYS; i += blockDim.x)
        if (h[i]) atomicAdd(&a.skey[i], h[i]);
}

// one warp per kind: exclusive scan of its key counts
__global__ void k_adj_key_scan(Dev d, AdjBuf a)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const int lane = threadIdx.x & 31, kind = threadIdx.x >> 5;
    if (kind >= 3) return;
    constexpr int PER = ADJ_KEYS / 32;
    int* k = a.skey + kind * ADJ_KEYS + lane * PER;
    int sum = 0;
    for (int i = 0; i < PER; ++i) sum += k[i];
    int x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    int run = x - sum;
    for (int i = 0; i < PER; ++i) { const int c = k[i]; k[i] = run; run += c; }
}

__global__ void k_adj_key_scatter(Dev d, AdjBuf a)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const long long total = (long long)a.nact[0] + a.nact[1] + a.nact[2];
    const long long stride = (long long)gridDim.x * blockDim.x;
    // warp-uniform trip count: every lane takes part in the match below
    for (long long e0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); e0 < total; e0 += stride) {
        int kind = 0, u = 0, slot = -1;
        const bool on = adj_entry(a, e0 + lane, kind, u);
        if (on) slot = kind * ADJ_KEYS + adj_unit_key(a, kind, u);
        const unsigned peers = __match_any_sync(0xffffffffu, slot);
        int base = 0;
        if (on && (peers & lt) == 0) base = atomicAdd(&a.skey[slot], __popc(peers));
        base = __shfl_sync(0xffffffffu, base, __ffs(peers) - 1);
        if (on) {
            int* out = kind == 0 ? a.slist_conv : (kind == 1 ? a.slist_tor : a.slist_conc);
            out[base + __popc(peers & lt)] = u;
        }
    }
}

// pass 3: per active unit, one lane per coordinate of its atoms (K lanes);
// lane k accumulates sum over the unit's dots of A . d(dot)/d(coordinate k)
template <int NT>
struct AdjLaneF {
    const double4* A;
    const int8_t* bur;      // only buried dots carry an adjoint (the others' slots are not cleared)
    double g[NT];
    __device__ bool want(long long q) const
    {
        if (!bur[q]) return false;
        const double4 v = A[q];
        return v.x != 0.0 || v.y != 0.0 || v.z != 0.0 || v.w != 0.0;
    }
    __device__ void take(long long q, const DotV<Dn<NT>>& D)
    {
        const double4 v = A[q];
#pragma unroll
        for (int t = 0; t < NT; ++t)
            g[t] += ((v.x * D.p.x.d[t] + v.y * D.p.y.d[t]) + v.z * D.p.z.d[t]) + v.w * D.area.d[t];
    }
};

// One active unit per group of K / NT lanes, each lane carrying NT of the
// unit's K coordinates as dual-number tangents through the unit's geometry.
// four CTAs per SM: twice the warps of the unbounded register count, which
// outweighs the spills it costs (measured)
template <int KIND, int NT>
__global__ void __launch_bounds__(128, 4) k_adj_units(Dev d, AdjBuf a)
{
    CMS_EXIT_ON_OVERFLOW(d);
    constexpr int K = KIND == 2 ? 9 : 6;       // coordinates of the unit's atoms
    constexpr int L = K / NT;                  // lanes per unit
    constexpr int G = 32 / L;                  // units per warp
    const int lane = threadIdx.x & 31;
    const int grp = lane / L, k = lane % L;
    const int* list = KIND == 0 ? a.slist_conv : (KIND == 1 ? a.slist_tor : a.slist_conc);
    const long long n = a.nact[KIND];
    const long long wid = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = wid * G; base < n; base += nw * G) {
        const long long e = base + grp;
        if (grp >= G || e >= n) continue;
        const int u = list[e];
        AdjLaneF<NT> f;
        f.A = a.A;
        f.bur = d.dbur;
#pragma unroll
        for (int t = 0; t < NT; ++t) f.g[t] = 0.0;
        const SeedLane<NT> seed{k};
        double* out;
        if (KIND == 0) {
            convex_unit_dots<Dn<NT>>(d, u, seed, f);
            out = a.gconv + 6LL * u;
            if (k == 0) { a.act_atom[u] = 1; a.act_atom[d.nb_id[d.nb_off[u]]] = 1; }
        } else if (KIND == 1) {
            tor_unit_dots<Dn<NT>>(d, u, seed, f);
            out = a.gtor + 6LL * u;
            if (k == 0) { a.act_atom[d.tor_i[u]] = 1; a.act_atom[d.tor_j[u]] = 1; }
        } else {
            conc_unit_dots<Dn<NT>>(d, u, seed, f);
            out = a.gconc + 9LL * u;
            if (k == 0) { a.act_atom[d.pa0[u]] = 1; a.act_atom[d.pa1[u]] = 1; a.act_atom[d.pa2[u]] = 1; }
        }
#pragma unroll
        for (int t = 0; t < NT; ++t) out[NT * k + t] = f.g[t];
    }
}

// probe range of atom g's triples: "+" probes [pb, pe), "-" probes [mb, me)
__device__ __forceinline__ void atom_probe_ranges(const Dev& d, int g, long long& pb, long long& pe, long long& mb,
                                                  long long& me)
{
    const int c = d.cplx[g];
    const Cplx C = d.cx[c];
    const int s0 = C.a0, s1 = C.a0 + C.n0, e1 = C.a0 + C.n;
    const int ms = d.mol[g] == 0 ? s0 : s1, mend = d.mol[g] == 0 ? s1 : e1;
    const long long cbase = d.plus_off[s0] + d.minus_off[s0];
    const long long m0 = (d.plus_off[s1] - d.plus_off[s0]) + (d.minus_off[s1] - d.minus_off[s0]);
    const long long blk = cbase + (d.mol[g] == 0 ? 0 : m0);
    pb = blk + (d.plus_off[g] - d.plus_off[ms]);
    pe = pb + (d.plus_off[g + 1] - d.plus_off[g]);
    mb = blk + (d.plus_off[mend] - d.plus_off[ms]) + (d.minus_off[g] - d.minus_off[ms]);
    me = mb + (d.minus_off[g + 1] - d.minus_off[g]);
}

// clears the per-dot adjoint of the buried dots (the only ones that get one)
// and the per-entry and per-unit counters
__global__ void k_adj_zero(Dev d, Rd r, AdjBuf a, long long dcap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long nf = (long long)d.N + d.tor_cap + d.probe_cap;
    const long long n = max(dcap, nf);
    const long long NB = r.bur_scan[adj_doff(d, 2LL * d.B)];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (i < NB) a.A[r.bur_idx[i]] = make_double4(0.0, 0.0, 0.0, 0.0);
        if (i < dcap) {
            a.rcnt[i] = 0;
            a.rfill[i] = 0;
        }
        if (i < d.N) { a.act_conv[i] = 0; a.act_atom[i] = 0; }
        if (i < d.tor_cap) a.act_tor[i] = 0;
        if (i < d.probe_cap) a.act_conc[i] = 0;
        if (i < 3) a.nact[i] = 0;
    }
}

// pass 4, one warp per active atom: the lanes take the atom's neighbour-row
// slots (the convex units it frames, the pairs (i, atom) of lower-index
// neighbours i, their triples' probes) and its own pairs and probes, and the
// warp sums the lanes' partial sums in a fixed tree; inactive atoms get zeros
__device__ __forceinline__ void add_probe_range_lanes(const Dev& d, const AdjBuf& a, int atom, long long b, long long e,
                                                      int start, int step, double& x, double& y, double& z)
{
    for (long long p = b + start; p < e && p < d.probe_cap; p += step) {
        if (!a.act_conc[p]) continue;
        const int ia[3] = {d.pa0[p], d.pa1[p], d.pa2[p]};
        for (int s = 0; s < 3; ++s) {
            if (ia[s] != atom) continue;
            const double* v = a.gconc + 9 * p + 3 * s;
            x += v[0]; y += v[1]; z += v[2];
        }
    }
}

__global__ void k_adj_gather_w(Dev d, AdjBuf a, double* grad)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const int lane = threadIdx.x & 31;
    const long long wid = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long NT = min(d.tor_off[d.N], d.tor_cap);
    for (long long b0 = wid * 32; b0 < d.N; b0 += nw * 32) {
        const long long me = b0 + lane;
        const bool act = me < d.N && a.act_atom[me];
        if (me < d.N && !act) { grad[3 * me] = 0.0; grad[3 * me + 1] = 0.0; grad[3 * me + 2] = 0.0; }
        unsigned m = __ballot_sync(0xffffffffu, act);
        while (m) {
            const int at = (int)(b0 + __ffs(m) - 1);
            m &= m - 1;
            double x = 0.0, y = 0.0, z = 0.0;
            if (lane == 0 && a.act_conv[at]) {
                x = a.gconv[6LL * at]; y = a.gconv[6LL * at + 1]; z = a.gconv[6LL * at + 2];
            }
            const long long off = d.nb_off[at];
            const int K = d.nnb[at];
            for (int s = lane; s < K; s += 32) {
                const int g = d.nb_id[off + s];
                if (a.act_conv[g] && d.nb_id[d.nb_off[g]] == at) {
                    const double* v = a.gconv + 6LL * g + 3;
                    x += v[0]; y += v[1]; z += v[2];
                }
                if (g < at) {
                    for (long long q = d.tor_off[g]; q < d.tor_off[g + 1] && q < NT; ++q) {
                        if (d.tor_j[q] != at || !a.act_tor[q]) continue;
                        const double* v = a.gtor + 6 * q + 3;
                        x += v[0]; y += v[1]; z += v[2];
                    }
                    long long pb, pe, mb, me2;
                    atom_probe_ranges(d, g, pb, pe, mb, me2);
                    add_probe_range_lanes(d, a, at, pb, pe, 0, 1, x, y, z);
                    add_probe_range_lanes(d, a, at, mb, me2, 0, 1, x, y, z);
                }
            }
            for (long long q = d.tor_off[at] + lane; q < d.tor_off[at + 1] && q < NT; q += 32) {
                if (!a.act_tor[q]) continue;
                const double* v = a.gtor + 6 * q;
                x += v[0]; y += v[1]; z += v[2];
            }
            long long pb, pe, mb, me2;
            atom_probe_ranges(d, at, pb, pe, mb, me2);
            add_probe_range_lanes(d, a, at, pb, pe, lane, 32, x, y, z);
            add_probe_range_lanes(d, a, at, mb, me2, lane, 32, x, y, z);
            for (int o = 16; o > 0; o >>= 1) {
                x += __shfl_xor_sync(0xffffffffu, x, o);
                y += __shfl_xor_sync(0xffffffffu, y, o);
                z += __shfl_xor_sync(0xffffffffu, z, o);
            }
            if (lane == 0) { grad[3LL * at] = x; grad[3LL * at + 1] = y; grad[3LL * at + 2] = z; }
        }
    }
}

void launch_adjoint(const Dev& d, const Rd& r, const AdjBuf& a, const NNTask* cms_task, int side, double* grad,
                    long long* scan_tmp, cudaStream_t s)
{
    const long long D = d.dot_cap;
    k_adj_zero<<<grid_adj(std::max(D, (long long)d.N + d.tor_cap + d.probe_cap), 256), 256, 0, s>>>(d, r, a, D);
    k_adj_queries<<<grid_adj(D, 256), 256, 0, s>>>(d, r, a, cms_task, side);
    k_adj_ref_count<<<grid_adj(D, 256), 256, 0, s>>>(d, r, a);
    scan_counts(a.rcnt, a.roff, D, scan_tmp, s);
    k_adj_ref_fill<<<grid_adj(D, 256), 256, 0, s>>>(d, r, a);
    k_adj_ref_sum<<<grid_adj(D, 256), 256, 0, s>>>(d, r, a);
    k_adj_collect<<<grid_adj((long long)d.N + d.tor_cap + d.probe_cap, 256), 256, 0, s>>>(d, a);
    cudaMemsetAsync(a.skey, 0, sizeof(int) * 3 * ADJ_KEYS, s);
    k_adj_key_count<<<grid_adj((long long)d.N + d.tor_cap + d.probe_cap, 256), 256, 0, s>>>(d, a);
    k_adj_key_scan<<<1, 96, 0, s>>>(d, a);
    k_adj_key_scatter<<<grid_adj((long long)d.N + d.tor_cap + d.probe_cap, 256), 256, 0, s>>>(d, a);
    // convex and concave units: one lane per atom (3 tangents); toroidal units: one lane per coordinate
    k_adj_units<0, 3><<<grid_adj(d.N, 128), 128, 0, s>>>(d, a);
    k_adj_units<1, 1><<<grid_adj(d.tor_cap, 128), 128, 0, s>>>(d, a);
    k_adj_units<2, 3><<<grid_adj(d.probe_cap, 128), 128, 0, s>>>(d, a);
    k_adj_gather_w<<<grid_adj(d.N, 128), 128, 0, s>>>(d, a, grad);
}

}  // namespace cms
