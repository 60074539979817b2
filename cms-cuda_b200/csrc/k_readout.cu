// Readouts of a generated surface: CMS (both sides), maximum possible CMS and
// Lawrence & Colman shape complementarity.
//
// Reference behaviour (cms-cuda/_core.py):
//   calc_contact_molecular_surface                 _core.py:946-1004
//   calc_max_possible_contact_molecular_surface    _core.py:1007-1034
//   trim_peripheral_band_vectorized                _core.py:1037-1077
//   _binned_median                                 _core.py:1080-1104
//   calc_neighbor_distance_vectorized              _core.py:1107-1147
//   CalcLoadedSC                                   _core.py:807-863
//
// The nearest-dot search is brute force over every (query, reference) pair.
// Coordinates relative to the complex centre are staged in FP32; the FP32
// squared distance filters candidates and every reference whose FP32 value is
// within a proven error bound of the running FP32 minimum is re-evaluated in
// FP64 in the reference's (cdist) order, so the minimum and the first index
// attaining it are exactly those of the FP64 search.
#include "cms_readout.cuh"

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

// dot offset per complex & molecule, clamped to the dot capacity (a run past
// the capacity is flagged and redone, but must not read out of bounds)
__device__ __forceinline__ long long doff(const Dev& d, long long i) { return min(d.dot_off[i], d.dot_cap); }

// ---------------------------------------------------------------------------
// compaction of buried / accessible dots, FP32 packing
// ---------------------------------------------------------------------------
__global__ void k_flag_buried(Dev d, Rd r, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long D = doff(d, 2LL * d.B);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap; i += (long long)gridDim.x * blockDim.x)
        r.flag[i] = (i < D && d.dbur[i]) ? 1 : 0;
}

__device__ __forceinline__ float4 pack_f4(const Dev& d, long long dot, int c)
{
    const Cplx& C = d.cx[c];
    const double* p = d.dxyz + 3 * dot;
    return make_float4((float)(p[0] - C.ctr[0]), (float)(p[1] - C.ctr[1]), (float)(p[2] - C.ctr[2]), 0.f);
}

// dot -> complex * 2 + molecule, from its owner atom (every dot lies in its owner's segment)
__device__ __forceinline__ int dot_cm(const Dev& d, long long dot)
{
    const int a = d.datom[dot];
    return 2 * d.cplx[a] + d.mol[a];
}

__global__ void k_split_buried(Dev d, Rd r, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long D = doff(d, 2LL * d.B);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap && i < D; i += (long long)gridDim.x * blockDim.x) {
        const int cm = dot_cm(d, i);
        const float4 f = pack_f4(d, i, cm >> 1);
        if (r.flag[i]) {
            long long k = r.bur_scan[i];
            r.bur_idx[k] = (int)i;
            r.bur_f4[k] = f;
            r.bur_cm[k] = cm;
        } else {
            long long k = i - r.bur_scan[i];
            r.acc_idx[k] = (int)i;
            r.acc_f4[k] = f;
        }
    }
}

void launch_split_buried(const Dev& d, const Rd& r, long long dot_cap, long long* scan_tmp, cudaStream_t s)
{
    k_flag_buried<<<grid_for(dot_cap, 256), 256, 0, s>>>(d, r, dot_cap);
    scan_counts(r.flag, r.bur_scan, dot_cap, scan_tmp, s);
    k_split_buried<<<grid_for(dot_cap, 256), 256, 0, s>>>(d, r, dot_cap);
}

// ---------------------------------------------------------------------------
// brute-force nearest-dot search, FP32 filter + FP64 recheck
// ---------------------------------------------------------------------------
// Formulation.  Each tile of queries is staged relative to its own centre c
// (FP32): q' = q - c, r' = r - c, with rho bounding |q'| over the tile.  The
// search minimises s(r) = |r'|^2 - 2 q'.r' (three FMAs per pair) and
// d32 = s + |q'|^2 approximates the squared distance.  Error bound
// (u = 2^-24; d the distance, so |r'| <= rho + d):
//   FMA chain and |r'|^2      <= 5u((rho+d)^2 + 2 rho (rho+d))
//   |q'|^2 and the final add  <= 3u rho^2 + u d^2-scale terms
//   shifting by c in FP32     moves the distance by <= 2u(2 rho + d)
//   the points' FP32 rounding relative to the task centre moves it by <= E0
// so with t = rho + sqrt(D) + 1 the absolute error of d32 is at most
//   eps(D) = 20 u t^2 + 2 (sqrt(D) + 1)(E0 + 4 u t) + (E0 + 4 u t)^2.
// A reference attaining the FP64 minimum has d32 <= m + 2 eps(m) (m = the
// smallest d32 seen); one within the band has d32 <= band^2 + eps(band^2).
// Every reference under those thresholds is rechecked in FP64 in cdist order.
__device__ __forceinline__ double nn_eps(double m, double rho, double E0)
{
    const double u = 5.9604644775390625e-08;
    const double sm = sqrt(fmax(m, 0.0));
    const double t = rho + sm + 1.0;
    const double e = E0 + 4.0 * u * t;
    return 20.0 * u * t * t + 2.0 * (sm + 1.0) * e + e * e;
}

__device__ __forceinline__ double exact_d2(const double* a, const double* b)
{
    // cdist(ref, query, 'sqeuclidean') order: (d0*d0 + d1*d1) + d2*d2
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return (dx * dx + dy * dy) + dz * dz;
}

// original list position of a (possibly spatially ordered) entry, and its point index
__device__ __forceinline__ long long nn_qpos(const NNArgs& a, long long k) { return a.q_perm ? (long long)a.q_perm[k] : k; }
__device__ __forceinline__ long long nn_rpos(const NNArgs& a, long long k) { return a.r_perm ? (long long)a.r_perm[k] : k; }
__device__ __forceinline__ long long nn_rpt(const NNArgs& a, long long k)
{
    const long long o = nn_rpos(a, k);
    return a.r_idx ? (long long)a.r_idx[o] : o;
}

// Packed FP32 pairs (Blackwell f32x2 arithmetic): one instruction does the
// same IEEE round-to-nearest operation on two lanes, so packed results equal
// the scalar ones bit for bit.
typedef unsigned long long f2_t;
__device__ __forceinline__ f2_t pk2(float a, float b) { f2_t r; asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b)); return r; }
__device__ __forceinline__ void upk2(f2_t v, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ f2_t fma2(f2_t a, f2_t b, f2_t c) { f2_t r; asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c)); return r; }

// s(r) for one query: |r|^2 - 2 q.r as three FMAs (the packed loop's order)
__device__ __forceinline__ float nn_s(float qx2, float qy2, float qz2, float rx, float ry, float rz, float rr)
{
    return __fmaf_rn(qz2, rz, __fmaf_rn(qy2, ry, __fmaf_rn(qx2, rx, rr)));
}

__device__ __forceinline__ float nn_rr(float rx, float ry, float rz)
{
    return __fmaf_rn(rz, rz, __fmaf_rn(ry, ry, rx * rx));
}

static constexpr int NN_T = 128;              // threads per tile
static constexpr int NN_W = NN_T / 32;        // warps per tile
static constexpr int NN_BLK = 32;             // references per block (one bounding box)
static constexpr int NN_SR = NN_ROUND;        // references per sub-round (one bounding box)
static constexpr int NN_SRB = NN_SR / NN_BLK; // blocks per sub-round
static constexpr int NN_SORT = 512;           // rounds of a task visited nearest first (more: index order)
static constexpr int NN_TILE = NN_T * 4;      // queries per tile of the default variant (standalone searches)

// Tunable shapes: queries per thread Q (2 or 4: tiles of 256 or 512 queries),
// and either k_nn_w (variants 0 and 2: each warp stages its own blocks in
// reach) or k_nn with 512-reference rounds staged by the whole CTA (variants 1
// and 3; k_nn's 1024-reference rounds, nn_var_sub 2, remain for the standalone
// searches).  Every variant computes the same exact result; the autotuner
// picks per stage.
__host__ __device__ constexpr int nn_var_q(int v) { return (v & 2) ? 2 : 4; }
__host__ __device__ constexpr int nn_var_sub(int v) { return (v & 1) ? 1 : 2; }

// one query's state
struct NNQ {
    float qx2, qy2, qz2;  // -2 q'
    double qq;            // |q'|^2 (FP32 value, held in FP64)
    int dot;              // index of the query point (FP64 coordinates read on recheck)
    float ms, ms2;        // smallest block minimum of s; smallest among the other blocks
    int mb;               // block holding ms
    float ts;             // s threshold: candidates have s <= ts
    float tslo;           // band: s at or below this is a hit for certain (d32 + eps <= band^2)
    float cth;            // cull threshold on the squared box distance
    double best;
    int bidx;
    bool live, done;
};

// Per-tile constants.  Box culling: a reference at squared distance L from
// the query in the staged FP32 frame has d32 >= L - eps(L) >= L (1 - B) - A,
// with eps(D) <= A + B D from the bound above (expand t^2 and sqrt(D)).
// A block whose box lies farther than (th + A) / (1 - B) from a query holds
// no candidate for a d32 threshold th.
struct NNTile {
    float cx, cy, cz;     // tile centre
    double rho, E0;       // bound on |q'|, FP32 rounding of the staged points
    double A, cull;       // cull threshold = (th + A) * cull
};

__device__ __forceinline__ NNTile nn_tile(float cx, float cy, float cz, double half_diag, double E0)
{
    const double u = 5.9604644775390625e-08;
    NNTile t;
    t.cx = cx; t.cy = cy; t.cz = cz;
    // |q - c| <= half diagonal of the box, plus the rounding of c and of q - c
    const double cn = fabs((double)cx) + fabs((double)cy) + fabs((double)cz);
    t.rho = (half_diag + 1e-6 * (cn + 1.0)) * (1.0 + 1e-6);
    t.E0 = E0;
    const double e0 = E0 + 4.0 * u * (t.rho + 1.0);
    t.A = 40.0 * u * (t.rho + 1.0) * (t.rho + 1.0) + 3.0 * e0 + 4.0 * u + 2.0 * e0 * e0;
    const double B = 52.0 * u + e0 + 32.0 * u * u;
    t.cull = (1.0 + 1e-6) / (1.0 - B);
    return t;
}

// d32 threshold for the minimum searches: m + 2 eps(m), m = smallest d32 seen
__device__ __forceinline__ double nn_min_th(float ms, double qq, const NNTile& t)
{
    const double m = (double)ms + qq;
    return m + 2.0 * nn_eps(m, t.rho, t.E0) * 1.01;
}

__device__ __forceinline__ float nn_cull_th(double th, const NNTile& t)
{
    return __double2float_ru((th + t.A) * t.cull);
}

// squared distance between two boxes (0 when they overlap); an empty box
// (lo = +inf, hi = -inf) is infinitely far from everything
__device__ __forceinline__ float box_gap2(float lx, float ly, float lz, float hx, float hy, float hz, float4 blo, float4 bhi)
{
    const float gx = fmaxf(fmaxf(blo.x - hx, lx - bhi.x), 0.f);
    const float gy = fmaxf(fmaxf(blo.y - hy, ly - bhi.y), 0.f);
    const float gz = fmaxf(fmaxf(blo.z - hz, lz - bhi.z), 0.f);
    return gx * gx + gy * gy + gz * gz;
}

// the FP32 box distance is within a few ulps of the exact one: scale it down
// before comparing against a cull threshold
__device__ __forceinline__ bool box_far(float g2, float cth) { return g2 * 0.999999f > cth; }

// BAND mode: re-examine a block of n (<= 32) staged references [k0, k0+n) for
// every (lane, query) of the warp whose block minimum fell under its
// threshold.  The warp takes the flagged lanes one at a time and checks the
// block in parallel, one reference per lane, FP32 filter then FP64 test.
__device__ __forceinline__ void nn_band_warp(const NNArgs& a, const NNTask& T, NNQ& q, unsigned need,
                                             const float4* sA, const float4* sB, int k0, int n, long long rb)
{
    const int lane = threadIdx.x & 31;
    while (need) {
        const int L = __ffs(need) - 1;
        need &= need - 1;
        const float qx2 = __shfl_sync(0xffffffffu, q.qx2, L);
        const float qy2 = __shfl_sync(0xffffffffu, q.qy2, L);
        const float qz2 = __shfl_sync(0xffffffffu, q.qz2, L);
        const float ts = __shfl_sync(0xffffffffu, q.ts, L);
        const int qdot = __shfl_sync(0xffffffffu, q.dot, L);
        bool hit = false, tested = false;
        if (lane < n) {
            const int k = k0 + lane;
            const float v = nn_s(qx2, qy2, qz2, sA[k].x, sA[k].z, sB[k].x, sB[k].z);
            if (v <= ts) {
                const double* rp = a.r_xyz + 3LL * nn_rpt(a, T.r0 + rb + k);
                hit = exact_d2(rp, a.q_xyz + 3LL * qdot) <= a.band_thr64;
                tested = true;
            }
        }
        if (a.recheck_count) {
            const unsigned t = __ballot_sync(0xffffffffu, tested);
            if (lane == 0 && t) atomicAdd(a.recheck_count, (unsigned long long)__popc(t));
        }
        if (__any_sync(0xffffffffu, hit) && lane == L) q.done = true;
    }
}

// FP32 filter + FP64 recheck of one reference for a minimum search
__device__ __forceinline__ void nn_recheck(const NNArgs& a, const NNTask& T, const NNTile& tl, float qx2, float qy2,
                                           float qz2, float ts, int qdot, long long k, double& best, int& bidx)
{
    const float4 r = a.r_f4[T.r0 + k];
    const float rx = r.x - tl.cx, ry = r.y - tl.cy, rz = r.z - tl.cz;
    const float v = nn_s(qx2, qy2, qz2, rx, ry, rz, nn_rr(rx, ry, rz));
    if (v <= ts) {
        const long long rk = T.r0 + k;
        if (a.recheck_count) atomicAdd(a.recheck_count, 1ull);
        const double e = exact_d2(a.r_xyz + 3LL * nn_rpt(a, rk), a.q_xyz + 3LL * qdot);
        const int ko = (int)(nn_rpos(a, rk) - T.r0);     // original position: first index on ties
        if (e < best || (e == best && ko < bidx)) { best = e; bidx = ko; }
    }
}

// nn_recheck over one block [k0, k1) (at most NN_BLK references): the FP32
// filter first for all of them (independent loads), then the FP64 test for
// the few under the threshold; ties resolve by original index in any order
__device__ __forceinline__ void nn_recheck_block(const NNArgs& a, const NNTask& T, const NNTile& tl, float qx2,
                                                 float qy2, float qz2, float ts, int qdot, long long k0, long long k1,
                                                 double& best, int& bidx)
{
    unsigned cand = 0u;
#pragma unroll 8
    for (int t = 0; t < NN_BLK; ++t) {
        const long long k = k0 + t;
        if (k < k1) {
            const float4 r = a.r_f4[T.r0 + k];
            const float rx = r.x - tl.cx, ry = r.y - tl.cy, rz = r.z - tl.cz;
            if (nn_s(qx2, qy2, qz2, rx, ry, rz, nn_rr(rx, ry, rz)) <= ts) cand |= 1u << t;
        }
    }
    if (a.recheck_count && cand) atomicAdd(a.recheck_count, (unsigned long long)__popc(cand));
    while (cand) {
        const int t = __ffs(cand) - 1;
        cand &= cand - 1;
        const long long rk = T.r0 + k0 + t;
        const double e = exact_d2(a.r_xyz + 3LL * nn_rpt(a, rk), a.q_xyz + 3LL * qdot);
        const int ko = (int)(nn_rpos(a, rk) - T.r0);     // original position: first index on ties
        if (e < best || (e == best && ko < bidx)) { best = e; bidx = ko; }
    }
}

// Minimum searches, rare case: candidates may sit in more than one block.
// The warp rechecks every reference of the task for each flagged lane,
// skipping blocks whose box is beyond the lane's cull threshold, and keeps
// the smallest FP64 value with the smallest index.
__device__ __forceinline__ void nn_full_warp(const NNArgs& a, const NNTask& T, const NNTile& tl, long long ro, int nsr,
                                             NNQ& q, unsigned need, long long qbase)
{
    const int lane = threadIdx.x & 31;
    const long long nblk = (long long)nsr * NN_SRB;
    while (need) {
        const int L = __ffs(need) - 1;
        need &= need - 1;
        const float qx2 = __shfl_sync(0xffffffffu, q.qx2, L);
        const float qy2 = __shfl_sync(0xffffffffu, q.qy2, L);
        const float qz2 = __shfl_sync(0xffffffffu, q.qz2, L);
        const float ts = __shfl_sync(0xffffffffu, q.ts, L);
        const float cth = __shfl_sync(0xffffffffu, q.cth, L);
        const int qdot = __shfl_sync(0xffffffffu, q.dot, L);
        const float4 qf = a.q_f4[qbase + L];
        double best = INFINITY;
        int bidx = 0x7fffffff;
        for (long long blk0 = 0; blk0 < nblk; blk0 += 32) {
            const long long blk = blk0 + lane;
            bool want = false;
            if (blk < nblk) {
                const float4 lo = a.box_blk[2 * (ro * NN_SRB + blk)], hi = a.box_blk[2 * (ro * NN_SRB + blk) + 1];
                want = !box_far(box_gap2(qf.x, qf.y, qf.z, qf.x, qf.y, qf.z, lo, hi), cth);
            }
            unsigned wb = __ballot_sync(0xffffffffu, want);
            while (wb) {
                const int b = __ffs(wb) - 1;
                wb &= wb - 1;
                const long long k = (blk0 + b) * NN_BLK + lane;
                if (k < T.rn) nn_recheck(a, T, tl, qx2, qy2, qz2, ts, qdot, k, best, bidx);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double e2 = __shfl_xor_sync(0xffffffffu, best, o);
            const int i2 = __shfl_xor_sync(0xffffffffu, bidx, o);
            if (e2 < best || (e2 == best && i2 < bidx)) { best = e2; bidx = i2; }
        }
        if (lane == L) { q.best = best; q.bidx = bidx; }
    }
}

// box of round i (SUB sub-rounds) of a task whose sub-rounds start at ro
template <int SUB>
__device__ __forceinline__ void nn_round_box(const NNArgs& a, long long ro, int nsr, int i, float4& lo, float4& hi)
{
    lo = a.box_round[2 * (ro + (long long)i * SUB)];
    hi = a.box_round[2 * (ro + (long long)i * SUB) + 1];
#pragma unroll
    for (int s = 1; s < SUB; ++s) {
        if ((long long)i * SUB + s >= nsr) break;
        const float4 l2 = a.box_round[2 * (ro + (long long)i * SUB + s)], h2 = a.box_round[2 * (ro + (long long)i * SUB + s) + 1];
        lo = make_float4(fminf(lo.x, l2.x), fminf(lo.y, l2.y), fminf(lo.z, l2.z), 0.f);
        hi = make_float4(fmaxf(hi.x, h2.x), fmaxf(hi.y, h2.y), fmaxf(hi.z, h2.z), 0.f);
    }
}

// Nearest-dot search over tiles of 128 * Q queries.  Each warp owns 32 * Q
// consecutive queries (Q per lane, Q / 2 packed pairs).  The task's references
// come in rounds of SUB * 512, visited in order of their box distance to the
// tile's box; a round is staged in shared memory only when some warp's query
// box is within its cull threshold, and each warp skips the 32-reference
// blocks whose box is beyond it.  The minimum searches keep, per query, the
// smallest block minimum of s, the block holding it and the smallest minimum
// of the other blocks; after the scan, the FP64 recheck covers that one block
// when no other block can hold a candidate (the usual case) and every block
// otherwise.  The band search stops a query at its first FP64 hit and a tile
// once every query has one or no round is left within reach.
template <int MODE, int Q, int SUB>
__global__ void __launch_bounds__(NN_T, MODE == NN_BAND ? 10 : 8) k_nn(NNArgs a)
{
    if (a.ovf && *a.ovf) return;
    constexpr int P = Q / 2;                  // packed query pairs per lane
    constexpr int WQ = 32 * Q;                // queries per warp
    constexpr int TILE = NN_T * Q;            // queries per tile
    constexpr int RR = SUB * NN_SR;           // references per round
    constexpr int RB = RR / NN_BLK;           // blocks per round
    __shared__ float4 sA[RR];     // (x, x, y, y)
    __shared__ float4 sB[RR];     // (z, z, |r|^2, |r|^2)
    __shared__ float4 sBox[2 * RB];
    __shared__ float sKey[NN_SORT];
    __shared__ short sOrd[NN_SORT];
    __shared__ float sWbox[6][NN_W];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long long ntiles = a.tile_off[a.ntask];
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int lo = 0, hi = a.ntask - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (a.tile_off[mid] <= tile) lo = mid; else hi = mid - 1;
        }
        const NNTask T = a.task[lo];
        const long long ro = a.round_off[lo];     // first sub-round of the task
        const int nsr = a.round_cnt[lo];          // sub-rounds of the task
        if (ro + nsr > a.round_cap) continue;     // over capacity: the run is flagged and redone
        const int nrt = (nsr + SUB - 1) / SUB;    // rounds
        const long long qw = (tile - a.tile_off[lo]) * TILE + (long long)wid * WQ;

        // queries and the warp's box
        NNQ q[Q];
        float qpx[Q], qpy[Q], qpz[Q];
        float wl[3] = {INFINITY, INFINITY, INFINITY}, wh[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
        for (int j = 0; j < Q; ++j) {
            const long long qi = qw + j * 32 + lane;
            q[j].live = qi < T.qn;
            qpx[j] = qpy[j] = qpz[j] = 0.f;
            q[j].dot = 0;
            if (q[j].live) {
                const float4 f = a.q_f4[T.q0 + qi];
                qpx[j] = f.x; qpy[j] = f.y; qpz[j] = f.z;
                const long long qo = nn_qpos(a, T.q0 + qi);
                q[j].dot = a.q_idx ? a.q_idx[qo] : (int)qo;
                wl[0] = fminf(wl[0], f.x); wl[1] = fminf(wl[1], f.y); wl[2] = fminf(wl[2], f.z);
                wh[0] = fmaxf(wh[0], f.x); wh[1] = fmaxf(wh[1], f.y); wh[2] = fmaxf(wh[2], f.z);
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            for (int o = 16; o > 0; o >>= 1) {
                wl[k] = fminf(wl[k], __shfl_xor_sync(0xffffffffu, wl[k], o));
                wh[k] = fmaxf(wh[k], __shfl_xor_sync(0xffffffffu, wh[k], o));
            }
        }
        if (lane == 0) for (int k = 0; k < 3; ++k) { sWbox[k][wid] = wl[k]; sWbox[3 + k][wid] = wh[k]; }
        __syncthreads();
        // the tile's box, centre and constants
        float tb[6];
        for (int k = 0; k < 3; ++k) {
            float l = sWbox[k][0], h = sWbox[3 + k][0];
            for (int w = 1; w < NN_W; ++w) { l = fminf(l, sWbox[k][w]); h = fmaxf(h, sWbox[3 + k][w]); }
            tb[k] = l; tb[3 + k] = h;
        }
        NNTile tl;
        {
            const float cx = 0.5f * (tb[0] + tb[3]), cy = 0.5f * (tb[1] + tb[4]), cz = 0.5f * (tb[2] + tb[5]);
            const double ex = (double)tb[3] - tb[0], ey = (double)tb[4] - tb[1], ez = (double)tb[5] - tb[2];
            tl = nn_tile(cx, cy, cz, 0.5 * sqrt(ex * ex + ey * ey + ez * ez), T.E);
        }
        const double band_th = MODE == NN_BAND ? a.band_thr64 + nn_eps(a.band_thr64, tl.rho, tl.E0) * 1.01 : 0.0;
        const double band_lo = MODE == NN_BAND ? a.band_thr64 - nn_eps(a.band_thr64, tl.rho, tl.E0) * 1.01 : 0.0;
        const float band_cth = MODE == NN_BAND ? nn_cull_th(band_th, tl) : 0.f;
        float cthw = -INFINITY;        // warp cull threshold: max over its open queries
#pragma unroll
        for (int j = 0; j < Q; ++j) {
            const float x = qpx[j] - tl.cx, y = qpy[j] - tl.cy, z = qpz[j] - tl.cz;
            q[j].qx2 = -2.0f * x; q[j].qy2 = -2.0f * y; q[j].qz2 = -2.0f * z;
            q[j].qq = (double)nn_rr(x, y, z);
            q[j].ms = INFINITY; q[j].ms2 = INFINITY; q[j].mb = -1;
            q[j].best = INFINITY; q[j].bidx = -1;
            q[j].done = !q[j].live;
            if (MODE == NN_BAND) {
                q[j].ts = __double2float_ru(band_th - q[j].qq);
                q[j].tslo = __double2float_rd(band_lo - q[j].qq);
                q[j].cth = band_cth;
            } else {
                q[j].ts = INFINITY;
                q[j].cth = INFINITY;
            }
            if (!q[j].done) cthw = fmaxf(cthw, q[j].cth);
        }
        for (int o = 16; o > 0; o >>= 1) cthw = fmaxf(cthw, __shfl_xor_sync(0xffffffffu, cthw, o));
        f2_t qxp[P], qyp[P], qzp[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            qxp[p] = pk2(q[2 * p].qx2, q[2 * p + 1].qx2);
            qyp[p] = pk2(q[2 * p].qy2, q[2 * p + 1].qy2);
            qzp[p] = pk2(q[2 * p].qz2, q[2 * p + 1].qz2);
        }

        // visiting order of the rounds: nearest to the tile's box first
        const bool sorted = nrt <= NN_SORT;
        if (sorted) {
            for (int i = threadIdx.x; i < nrt; i += NN_T) {
                float4 rlo, rhi;
                nn_round_box<SUB>(a, ro, nsr, i, rlo, rhi);
                sKey[i] = box_gap2(tb[0], tb[1], tb[2], tb[3], tb[4], tb[5], rlo, rhi);
            }
            __syncthreads();
            for (int i = threadIdx.x; i < nrt; i += NN_T) {
                const float ki = sKey[i];
                int rank = 0;
                for (int j2 = 0; j2 < nrt; ++j2) {
                    const float kj = sKey[j2];
                    rank += (kj < ki || (kj == ki && j2 < i)) ? 1 : 0;
                }
                sOrd[rank] = (short)i;
            }
            __syncthreads();
        }

        for (int kr = 0; kr < nrt; ++kr) {
            const int i = sorted ? sOrd[kr] : kr;
            float4 rlo, rhi;
            nn_round_box<SUB>(a, ro, nsr, i, rlo, rhi);
            const bool open = cthw > -INFINITY;
            const bool need = open && !box_far(box_gap2(wl[0], wl[1], wl[2], wh[0], wh[1], wh[2], rlo, rhi), cthw);
            if (!__syncthreads_or(need)) {
                // every later round is at least as far from the tile's box
                if (sorted && !__syncthreads_or(open && !box_far(sKey[i], cthw))) break;
                continue;
            }
            const long long rb = (long long)i * RR;
            const int nr = (int)min((long long)RR, T.rn - rb);
            for (int k = threadIdx.x; k < nr; k += NN_T) {
                const float4 r = a.r_f4[T.r0 + rb + k];
                const float rx = r.x - tl.cx, ry = r.y - tl.cy, rz = r.z - tl.cz;
                const float rr = nn_rr(rx, ry, rz);
                sA[k] = make_float4(rx, rx, ry, ry);
                sB[k] = make_float4(rz, rz, rr, rr);
            }
            for (int k = threadIdx.x; k < 2 * RB; k += NN_T) {
                // blocks of a missing second sub-round (odd sub-round count) are never reached: nr stops first
                const bool have = (long long)i * SUB + k / (2 * NN_SRB) < nsr;
                sBox[k] = have ? a.box_blk[2 * (ro + (long long)i * SUB) * NN_SRB + k]
                               : make_float4(INFINITY, INFINITY, INFINITY, 0.f);
            }
            __syncthreads();
            if (need) {
                for (int b = 0; b < RB; ++b) {
                    const int sb = b * NN_BLK;
                    if (sb >= nr) break;
                    const float4 blo = sBox[2 * b], bhi = sBox[2 * b + 1];
                    if (box_far(box_gap2(wl[0], wl[1], wl[2], wh[0], wh[1], wh[2], blo, bhi), cthw)) continue;
                    // each lane's open queries against the block's box
                    bool lane_need = false;
#pragma unroll
                    for (int j = 0; j < Q; ++j)
                        lane_need |= !q[j].done &&
                                     !box_far(box_gap2(qpx[j], qpy[j], qpz[j], qpx[j], qpy[j], qpz[j], blo, bhi), q[j].cth);
                    if (!__any_sync(0xffffffffu, lane_need)) continue;
                    const int n = min(NN_BLK, nr - sb);
                    if (a.pair_count && lane == 0) atomicAdd(a.pair_count, (unsigned long long)n * WQ);
                    float mv[Q];
#pragma unroll
                    for (int j = 0; j < Q; ++j) mv[j] = INFINITY;
#pragma unroll 4
                    for (int k = sb; k < sb + n; ++k) {
                        const float4 ra = sA[k];
                        const float4 rb4 = sB[k];
                        const f2_t rxx = pk2(ra.x, ra.y), ryy = pk2(ra.z, ra.w);
                        const f2_t rzz = pk2(rb4.x, rb4.y), rrr = pk2(rb4.z, rb4.w);
#pragma unroll
                        for (int p = 0; p < P; ++p) {
                            const f2_t sv = fma2(qzp[p], rzz, fma2(qyp[p], ryy, fma2(qxp[p], rxx, rrr)));
                            float a0, a1;
                            upk2(sv, a0, a1);
                            mv[2 * p] = fminf(mv[2 * p], a0);
                            mv[2 * p + 1] = fminf(mv[2 * p + 1], a1);
                        }
                    }
                    if (MODE == NN_BAND) {
#pragma unroll
                        for (int j = 0; j < Q; ++j) {
                            // a block minimum within band^2 - eps is a hit without the FP64 recheck;
                            // only minima in the uncertain strip go to it
                            if (!q[j].done && mv[j] <= q[j].tslo) q[j].done = true;
                            const unsigned nj = __ballot_sync(0xffffffffu, !q[j].done && mv[j] <= q[j].ts);
                            if (nj) nn_band_warp(a, T, q[j], nj, sA, sB, sb, n, rb);
                        }
                    } else {
                        const int blk = i * RB + b;
#pragma unroll
                        for (int j = 0; j < Q; ++j) {
                            if (mv[j] < q[j].ms) { q[j].ms2 = q[j].ms; q[j].ms = mv[j]; q[j].mb = blk; }
                            else q[j].ms2 = fminf(q[j].ms2, mv[j]);
                        }
                    }
                }
                // thresholds for the next rounds
                float c = -INFINITY;
#pragma unroll
                for (int j = 0; j < Q; ++j) {
                    if (MODE != NN_BAND && q[j].live && q[j].ms < INFINITY)
                        q[j].cth = nn_cull_th(nn_min_th(q[j].ms, q[j].qq, tl), tl);
                    if (!q[j].done) c = fmaxf(c, q[j].cth);
                }
                for (int o = 16; o > 0; o >>= 1) c = fmaxf(c, __shfl_xor_sync(0xffffffffu, c, o));
                cthw = c;
                if (MODE == NN_BAND) {
                    // the warp's box shrinks to its open queries
                    float l3[3] = {INFINITY, INFINITY, INFINITY}, h3[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
                    for (int j = 0; j < Q; ++j) {
                        if (q[j].done) continue;
                        l3[0] = fminf(l3[0], qpx[j]); l3[1] = fminf(l3[1], qpy[j]); l3[2] = fminf(l3[2], qpz[j]);
                        h3[0] = fmaxf(h3[0], qpx[j]); h3[1] = fmaxf(h3[1], qpy[j]); h3[2] = fmaxf(h3[2], qpz[j]);
                    }
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        for (int o = 16; o > 0; o >>= 1) {
                            l3[k] = fminf(l3[k], __shfl_xor_sync(0xffffffffu, l3[k], o));
                            h3[k] = fmaxf(h3[k], __shfl_xor_sync(0xffffffffu, h3[k], o));
                        }
                        wl[k] = l3[k]; wh[k] = h3[k];
                    }
                }
            }
        }

        if (MODE != NN_BAND) {
            // FP64 recheck: the best block alone when no other block can hold a candidate
            bool full[Q];
#pragma unroll
            for (int j = 0; j < Q; ++j) {
                full[j] = false;
                if (!q[j].live || !(q[j].ms < INFINITY)) continue;
                const double th = nn_min_th(q[j].ms, q[j].qq, tl);
                q[j].ts = __double2float_ru(th - q[j].qq);
                q[j].cth = nn_cull_th(th, tl);
                if (q[j].ms2 > q[j].ts) {
                    const long long k0 = (long long)q[j].mb * NN_BLK;
                    const long long k1 = min(k0 + NN_BLK, T.rn);
                    double best = INFINITY;
                    int bidx = 0x7fffffff;
                    nn_recheck_block(a, T, tl, q[j].qx2, q[j].qy2, q[j].qz2, q[j].ts, q[j].dot, k0, k1, best, bidx);
                    q[j].best = best; q[j].bidx = bidx;
                } else {
                    full[j] = true;
                }
            }
#pragma unroll
            for (int j = 0; j < Q; ++j) {
                const unsigned nf = __ballot_sync(0xffffffffu, full[j]);
                if (nf) nn_full_warp(a, T, tl, ro, nsr, q[j], nf, T.q0 + qw + j * 32);
            }
        }
#pragma unroll
        for (int j = 0; j < Q; ++j) {
            if (!q[j].live) continue;
            const long long o = nn_qpos(a, T.q0 + qw + j * 32 + lane);
            if (MODE == NN_BAND) a.out_flag[o] = q[j].done ? 0 : 1;     // keep iff no reference within the band
            else {
                a.out_d2[o] = q[j].best;
                if (MODE == NN_ARGMIN) a.out_idx[o] = q[j].bidx;
            }
        }
        __syncthreads();
    }
}

// Nearest-dot search with the warps of a tile independent of each other: a
// warp stages, one 32-reference block at a time in its own shared memory,
// only the blocks whose box lies within reach of its queries' box (the cull
// threshold of its open queries), in the FP32 frame of its own queries (the
// centre of their box).  A CTA-wide staging of whole rounds in reach of the
// tile's box brings in many references out of reach of a given warp, most of
// all for the band search's reach of the band width.  The minimum searches
// visit the sub-round nearest to the warp's box first (its minima set the
// threshold), then the others in order.  Same FP32 filter, FP64 recheck and
// error bounds as k_nn (any frame centre bounds |q'| by the box's half
// diagonal), so the same exact results.
template <int MODE, int Q>
__global__ void __launch_bounds__(NN_T, MODE == NN_BAND ? 10 : 8) k_nn_w(NNArgs a)
{
    if (a.ovf && *a.ovf) return;
    constexpr int P = Q / 2;
    constexpr int WQ = 32 * Q;
    constexpr int TILE = NN_T * Q;
    __shared__ float4 wA[NN_W][NN_BLK];       // (x, x, y, y) of the warp's staged block
    __shared__ float4 wB[NN_W][NN_BLK];       // (z, z, |r|^2, |r|^2)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float4* const sA = wA[wid];
    float4* const sB = wB[wid];
    const long long ntiles = a.tile_off[a.ntask];
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int lo = 0, hi = a.ntask - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (a.tile_off[mid] <= tile) lo = mid; else hi = mid - 1;
        }
        const NNTask T = a.task[lo];
        const long long ro = a.round_off[lo];
        const int nsr = a.round_cnt[lo];
        if (ro + nsr > a.round_cap) continue;     // over capacity: the run is flagged and redone
        const long long qw = (tile - a.tile_off[lo]) * TILE + (long long)wid * WQ;
        if (qw >= T.qn) continue;

        NNQ q[Q];
        float qpx[Q], qpy[Q], qpz[Q];
        float wl[3] = {INFINITY, INFINITY, INFINITY}, wh[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
        for (int j = 0; j < Q; ++j) {
            const long long qi = qw + j * 32 + lane;
            q[j].live = qi < T.qn;
            qpx[j] = qpy[j] = qpz[j] = 0.f;
            q[j].dot = 0;
            if (q[j].live) {
                const float4 f = a.q_f4[T.q0 + qi];
                qpx[j] = f.x; qpy[j] = f.y; qpz[j] = f.z;
                const long long qo = nn_qpos(a, T.q0 + qi);
                q[j].dot = a.q_idx ? a.q_idx[qo] : (int)qo;
                wl[0] = fminf(wl[0], f.x); wl[1] = fminf(wl[1], f.y); wl[2] = fminf(wl[2], f.z);
                wh[0] = fmaxf(wh[0], f.x); wh[1] = fmaxf(wh[1], f.y); wh[2] = fmaxf(wh[2], f.z);
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            for (int o = 16; o > 0; o >>= 1) {
                wl[k] = fminf(wl[k], __shfl_xor_sync(0xffffffffu, wl[k], o));
                wh[k] = fmaxf(wh[k], __shfl_xor_sync(0xffffffffu, wh[k], o));
            }
        }
        NNTile tl;
        {
            const float cx = 0.5f * (wl[0] + wh[0]), cy = 0.5f * (wl[1] + wh[1]), cz = 0.5f * (wl[2] + wh[2]);
            const double ex = (double)wh[0] - wl[0], ey = (double)wh[1] - wl[1], ez = (double)wh[2] - wl[2];
            tl = nn_tile(cx, cy, cz, 0.5 * sqrt(ex * ex + ey * ey + ez * ez), T.E);
        }
        const double band_th = MODE == NN_BAND ? a.band_thr64 + nn_eps(a.band_thr64, tl.rho, tl.E0) * 1.01 : 0.0;
        const double band_lo = MODE == NN_BAND ? a.band_thr64 - nn_eps(a.band_thr64, tl.rho, tl.E0) * 1.01 : 0.0;
        const float band_cth = MODE == NN_BAND ? nn_cull_th(band_th, tl) : 0.f;
#pragma unroll
        for (int j = 0; j < Q; ++j) {
            const float x = qpx[j] - tl.cx, y = qpy[j] - tl.cy, z = qpz[j] - tl.cz;
            q[j].qx2 = -2.0f * x; q[j].qy2 = -2.0f * y; q[j].qz2 = -2.0f * z;
            q[j].qq = (double)nn_rr(x, y, z);
            q[j].ms = INFINITY; q[j].ms2 = INFINITY; q[j].mb = -1;
            q[j].best = INFINITY; q[j].bidx = -1;
            q[j].done = !q[j].live;
            if (MODE == NN_BAND) {
                q[j].ts = __double2float_ru(band_th - q[j].qq);
                q[j].tslo = __double2float_rd(band_lo - q[j].qq);
                q[j].cth = band_cth;
            } else {
                q[j].ts = INFINITY;
                q[j].cth = INFINITY;
            }
        }
        f2_t qxp[P], qyp[P], qzp[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            qxp[p] = pk2(q[2 * p].qx2, q[2 * p + 1].qx2);
            qyp[p] = pk2(q[2 * p].qy2, q[2 * p + 1].qy2);
            qzp[p] = pk2(q[2 * p].qz2, q[2 * p + 1].qz2);
        }
        // warp cull threshold: the largest over its open queries (-inf: none open)
        auto warp_cth = [&]() {
            float c = -INFINITY;
#pragma unroll
            for (int j = 0; j < Q; ++j)
                if (!q[j].done) c = fmaxf(c, q[j].cth);
            for (int o = 16; o > 0; o >>= 1) c = fmaxf(c, __shfl_xor_sync(0xffffffffu, c, o));
            return c;
        };
        float cthw = warp_cth();

        // one sub-round: its blocks in reach, each staged and scanned
        auto visit = [&](int g) {
            const long long rb0 = (long long)g * NN_SR;
            const int nr = (int)min((long long)NN_SR, T.rn - rb0);
            bool bn = false;
            if (lane < NN_SRB && lane * NN_BLK < nr) {
                const float4 blo = a.box_blk[2 * ((ro + g) * NN_SRB + lane)];
                const float4 bhi = a.box_blk[2 * ((ro + g) * NN_SRB + lane) + 1];
                bn = !box_far(box_gap2(wl[0], wl[1], wl[2], wh[0], wh[1], wh[2], blo, bhi), cthw);
            }
            unsigned bm = __ballot_sync(0xffffffffu, bn);
            while (bm && cthw > -INFINITY) {
                const int b = __ffs(bm) - 1;
                bm &= bm - 1;
                const int sb = b * NN_BLK;
                const int n = min(NN_BLK, nr - sb);
                const float4 blo = a.box_blk[2 * ((ro + g) * NN_SRB + b)];
                const float4 bhi = a.box_blk[2 * ((ro + g) * NN_SRB + b) + 1];
                bool lane_need = false;
#pragma unroll
                for (int j = 0; j < Q; ++j)
                    lane_need |= !q[j].done &&
                                 !box_far(box_gap2(qpx[j], qpy[j], qpz[j], qpx[j], qpy[j], qpz[j], blo, bhi), q[j].cth);
                if (!__any_sync(0xffffffffu, lane_need)) continue;
                __syncwarp();
                if (lane < n) {
                    const float4 r = a.r_f4[T.r0 + rb0 + sb + lane];
                    const float rx = r.x - tl.cx, ry = r.y - tl.cy, rz = r.z - tl.cz;
                    const float rr = nn_rr(rx, ry, rz);
                    sA[lane] = make_float4(rx, rx, ry, ry);
                    sB[lane] = make_float4(rz, rz, rr, rr);
                }
                __syncwarp();
                if (a.pair_count && lane == 0) atomicAdd(a.pair_count, (unsigned long long)n * WQ);
                float mv[Q];
#pragma unroll
                for (int j = 0; j < Q; ++j) mv[j] = INFINITY;
#pragma unroll 4
                for (int k = 0; k < n; ++k) {
                    const float4 ra = sA[k];
                    const float4 rb4 = sB[k];
                    const f2_t rxx = pk2(ra.x, ra.y), ryy = pk2(ra.z, ra.w);
                    const f2_t rzz = pk2(rb4.x, rb4.y), rrr = pk2(rb4.z, rb4.w);
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        const f2_t sv = fma2(qzp[p], rzz, fma2(qyp[p], ryy, fma2(qxp[p], rxx, rrr)));
                        float a0, a1;
                        upk2(sv, a0, a1);
                        mv[2 * p] = fminf(mv[2 * p], a0);
                        mv[2 * p + 1] = fminf(mv[2 * p + 1], a1);
                    }
                }
                if (MODE == NN_BAND) {
#pragma unroll
                    for (int j = 0; j < Q; ++j) {
                        // a block minimum within band^2 - eps is a hit without the FP64 recheck
                        if (!q[j].done && mv[j] <= q[j].tslo) q[j].done = true;
                        const unsigned nj = __ballot_sync(0xffffffffu, !q[j].done && mv[j] <= q[j].ts);
                        if (nj) nn_band_warp(a, T, q[j], nj, sA, sB, 0, n, rb0 + sb);
                    }
                    cthw = warp_cth();
                } else {
                    const int blk = g * NN_SRB + b;
#pragma unroll
                    for (int j = 0; j < Q; ++j) {
                        if (mv[j] < q[j].ms) { q[j].ms2 = q[j].ms; q[j].ms = mv[j]; q[j].mb = blk; }
                        else q[j].ms2 = fminf(q[j].ms2, mv[j]);
                    }
                }
            }
            if (MODE != NN_BAND) {
                // thresholds for the next sub-rounds
#pragma unroll
                for (int j = 0; j < Q; ++j)
                    if (q[j].live && q[j].ms < INFINITY) q[j].cth = nn_cull_th(nn_min_th(q[j].ms, q[j].qq, tl), tl);
                cthw = warp_cth();
            }
        };

        if (nsr > 0 && cthw > -INFINITY) {
            int gfirst = -1;
            if (MODE != NN_BAND) {
                // the sub-round nearest to the warp's box first (smallest gap, then smallest index)
                float bg = INFINITY;
                int bi = 0x7fffffff;
                for (int g0 = 0; g0 < nsr; g0 += 32) {
                    const int gi = g0 + lane;
                    if (gi < nsr) {
                        const float gap = box_gap2(wl[0], wl[1], wl[2], wh[0], wh[1], wh[2], a.box_round[2 * (ro + gi)],
                                                   a.box_round[2 * (ro + gi) + 1]);
                        if (gap < bg) { bg = gap; bi = gi; }
                    }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const float g2 = __shfl_xor_sync(0xffffffffu, bg, o);
                    const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (g2 < bg || (g2 == bg && i2 < bi)) { bg = g2; bi = i2; }
                }
                gfirst = bi < nsr ? bi : 0;
                visit(gfirst);
            }
            for (int g0 = 0; g0 < nsr && cthw > -INFINITY; g0 += 32) {
                const int gi = g0 + lane;
                bool near = false;
                if (gi < nsr && gi != gfirst) {
                    const float4 rlo = a.box_round[2 * (ro + gi)], rhi = a.box_round[2 * (ro + gi) + 1];
                    near = !box_far(box_gap2(wl[0], wl[1], wl[2], wh[0], wh[1], wh[2], rlo, rhi), cthw);
                }
                unsigned rm = __ballot_sync(0xffffffffu, near);
                while (rm && cthw > -INFINITY) {
                    const int g = g0 + __ffs(rm) - 1;
                    rm &= rm - 1;
                    if (MODE != NN_BAND) {
                        // the threshold may have shrunk since the chunk's test
                        const float gap = box_gap2(wl[0], wl[1], wl[2], wh[0], wh[1], wh[2], a.box_round[2 * (ro + g)],
                                                   a.box_round[2 * (ro + g) + 1]);
                        if (box_far(gap, cthw)) continue;
                    }
                    visit(g);
                }
            }
        }

        if (MODE != NN_BAND) {
            // FP64 recheck: the best block alone when no other block can hold a candidate
            bool full[Q];
#pragma unroll
            for (int j = 0; j < Q; ++j) {
                full[j] = false;
                if (!q[j].live || !(q[j].ms < INFINITY)) continue;
                const double th = nn_min_th(q[j].ms, q[j].qq, tl);
                q[j].ts = __double2float_ru(th - q[j].qq);
                q[j].cth = nn_cull_th(th, tl);
                if (q[j].ms2 > q[j].ts) {
                    const long long k0 = (long long)q[j].mb * NN_BLK;
                    const long long k1 = min(k0 + NN_BLK, T.rn);
                    double best = INFINITY;
                    int bidx = 0x7fffffff;
                    nn_recheck_block(a, T, tl, q[j].qx2, q[j].qy2, q[j].qz2, q[j].ts, q[j].dot, k0, k1, best, bidx);
                    q[j].best = best; q[j].bidx = bidx;
                } else {
                    full[j] = true;
                }
            }
#pragma unroll
            for (int j = 0; j < Q; ++j) {
                const unsigned nf = __ballot_sync(0xffffffffu, full[j]);
                if (nf) nn_full_warp(a, T, tl, ro, nsr, q[j], nf, T.q0 + qw + j * 32);
            }
        }
#pragma unroll
        for (int j = 0; j < Q; ++j) {
            if (!q[j].live) continue;
            const long long o = nn_qpos(a, T.q0 + qw + j * 32 + lane);
            if (MODE == NN_BAND) a.out_flag[o] = q[j].done ? 0 : 1;     // keep iff no reference within the band
            else {
                a.out_d2[o] = q[j].best;
                if (MODE == NN_ARGMIN) a.out_idx[o] = q[j].bidx;
            }
        }
    }
}

__global__ void k_nn_tiles(NNArgs a)
{
    if (a.ovf && *a.ovf) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < a.ntask; t += gridDim.x * blockDim.x) {
        const NNTask T = a.task[t];
        const bool on = T.qn > 0 && (T.rn > 0 || a.band_mode);
        a.tile_cnt[t] = on ? (int)((T.qn + a.tile_q - 1) / a.tile_q) : 0;
        a.round_cnt[t] = on ? (int)((T.rn + NN_SR - 1) / NN_SR) : 0;
    }
}

// one warp per sub-round: the box of each 32-reference block (lane b < 16) and of the sub-round
__global__ void k_nn_boxes(NNArgs a)
{
    if (a.ovf && *a.ovf) return;
    const long long nround = min(a.round_off[a.ntask], a.round_cap);
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long g = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; g < nround; g += nw) {
        int lo = 0, hi = a.ntask - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (a.round_off[mid] <= g) lo = mid; else hi = mid - 1;
        }
        const NNTask T = a.task[lo];
        const long long k0 = (g - a.round_off[lo]) * NN_SR + (long long)lane * NN_BLK;
        const long long k1 = lane < NN_SRB ? min(k0 + NN_BLK, T.rn) : k0;
        float l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (long long k = k0; k < k1; ++k) {
            const float4 p = a.r_f4[T.r0 + k];
            l[0] = fminf(l[0], p.x); l[1] = fminf(l[1], p.y); l[2] = fminf(l[2], p.z);
            h[0] = fmaxf(h[0], p.x); h[1] = fmaxf(h[1], p.y); h[2] = fmaxf(h[2], p.z);
        }
        if (lane < NN_SRB) {
            a.box_blk[2 * (g * NN_SRB + lane)] = make_float4(l[0], l[1], l[2], 0.f);
            a.box_blk[2 * (g * NN_SRB + lane) + 1] = make_float4(h[0], h[1], h[2], 0.f);
        }
        for (int k = 0; k < 3; ++k) {
            for (int o = 16; o > 0; o >>= 1) {
                l[k] = fminf(l[k], __shfl_xor_sync(0xffffffffu, l[k], o));
                h[k] = fmaxf(h[k], __shfl_xor_sync(0xffffffffu, h[k], o));
            }
        }
        if (lane == 0) {
            a.box_round[2 * g] = make_float4(l[0], l[1], l[2], 0.f);
            a.box_round[2 * g + 1] = make_float4(h[0], h[1], h[2], 0.f);
        }
    }
}

void launch_nn_tiles(NNArgs a, int mode, int variant, long long* scan_tmp, cudaStream_t s)
{
    a.band_mode = mode == NN_BAND;
    a.tile_q = NN_T * nn_var_q(variant);
    k_nn_tiles<<<grid_for(a.ntask, 128), 128, 0, s>>>(a);
    scan_counts(a.tile_cnt, a.tile_off, a.ntask, scan_tmp, s);
    scan_counts(a.round_cnt, a.round_off, a.ntask, scan_tmp, s);
}

template <int MODE>
static void nn_dispatch(const NNArgs& a, int variant, unsigned grid, cudaStream_t s)
{
    switch (variant) {
    case 1: k_nn<MODE, 4, 1><<<grid, NN_T, 0, s>>>(a); break;
    case 2: k_nn_w<MODE, 2><<<grid, NN_T, 0, s>>>(a); break;
    case 3: k_nn<MODE, 2, 1><<<grid, NN_T, 0, s>>>(a); break;
    default: k_nn_w<MODE, 4><<<grid, NN_T, 0, s>>>(a); break;
    }
}

void launch_nn_kernel(NNArgs a, int mode, int variant, long long tile_cap, cudaStream_t s)
{
    a.band_mode = mode == NN_BAND;
    a.tile_q = NN_T * nn_var_q(variant);
    k_nn_boxes<<<grid_for(a.round_cap * 32, 256), 256, 0, s>>>(a);
    // one tile per CTA (tile_cap bounds the tile count of the largest tiles'
    // variant times 2); CTAs past the tile count exit at once
    if (nn_var_q(variant) == 2) tile_cap *= 2;
    const unsigned grid = (unsigned)(tile_cap < 1 ? 1 : (tile_cap > 0x7fffffffLL ? 0x7fffffffLL : tile_cap));
    if (mode == NN_MIN) k_nn<NN_MIN, 4, 2><<<grid, NN_T, 0, s>>>(a);      // standalone searches only
    else if (mode == NN_ARGMIN) nn_dispatch<NN_ARGMIN>(a, variant, grid, s);
    else nn_dispatch<NN_BAND>(a, variant, grid, s);
}

// CTAs a standalone search launches: one per tile of the default shape (k_points_task makes the tiles), plus one
long long nn_standalone_tile_cap(long long n_query) { return (n_query + NN_TILE - 1) / NN_TILE + 1; }

void launch_nn(NNArgs a, int mode, int variant, long long tile_cap, long long* scan_tmp, cudaStream_t s)
{
    launch_nn_tiles(a, mode, variant, scan_tmp, s);
    launch_nn_kernel(a, mode, variant, tile_cap, s);
}

// ---------------------------------------------------------------------------
// standalone nearest-dot search of two point sets (no batch state)
// ---------------------------------------------------------------------------
__global__ void k_points_bbox(const double* q, long long nq, const double* r, long long nr, double* partials)
{
    __shared__ double sh[6][32];
    double v[6] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY};   // min xyz, -max xyz
    const long long n = nq + nr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double* p = i < nq ? q + 3 * i : r + 3 * (i - nq);
        for (int k = 0; k < 3; ++k) { v[k] = fmin(v[k], p[k]); v[3 + k] = fmin(v[3 + k], -p[k]); }
    }
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] = fmin(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) for (int k = 0; k < 6; ++k) sh[k][w] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 6; ++k) {
            double m = sh[k][0];
            for (int i = 1; i < nw; ++i) m = fmin(m, sh[k][i]);
            partials[6 * blockIdx.x + k] = m;
        }
    }
}

// reduce the partial boxes, then the single task covering both sets
__global__ void k_points_task(const double* partials, int nblocks, long long nq, long long nr, double* bbox,
                              NNTask* task, int* tile_cnt, long long* tile_off, int* round_cnt, long long* round_off)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double v[6];
    for (int k = 0; k < 6; ++k) {
        double m = INFINITY;
        for (int b = 0; b < nblocks; ++b) m = fmin(m, partials[6 * b + k]);
        v[k] = m;
    }
    double half = 0.0;
    for (int k = 0; k < 3; ++k) {
        const double lo = v[k], hi = -v[3 + k];
        bbox[k] = 0.5 * (lo + hi);
        half = fmax(half, 0.5 * (hi - lo));
    }
    NNTask T;
    T.q0 = 0; T.qn = nq; T.r0 = 0; T.rn = nr; T.c = 0;
    T.E = 2.5e-7 * (half + 1.0);
    task[0] = T;
    const long long nt = (nq > 0 && nr > 0) ? (nq + NN_TILE - 1) / NN_TILE : 0;
    tile_cnt[0] = (int)nt;
    tile_off[0] = 0;
    tile_off[1] = nt;
    const long long nrd = nt > 0 ? (nr + NN_SR - 1) / NN_SR : 0;
    round_cnt[0] = (int)nrd;
    round_off[0] = 0;
    round_off[1] = nrd;
}

__global__ void k_points_pack(const double* q, long long nq, const double* r, long long nr, const double* bbox,
                              float4* q_f4, float4* r_f4)
{
    const long long n = nq + nr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double* p = i < nq ? q + 3 * i : r + 3 * (i - nq);
        const float4 f = make_float4((float)(p[0] - bbox[0]), (float)(p[1] - bbox[1]), (float)(p[2] - bbox[2]), 0.f);
        if (i < nq) q_f4[i] = f; else r_f4[i - nq] = f;
    }
}

void launch_points_setup(const double* q, long long nq, const double* r, long long nr, double* partials,
                         int partial_blocks, double* bbox, float4* q_f4, float4* r_f4, NNTask* task, int* tile_cnt,
                         long long* tile_off, int* round_cnt, long long* round_off, cudaStream_t s)
{
    k_points_bbox<<<partial_blocks, 256, 0, s>>>(q, nq, r, nr, partials);
    k_points_task<<<1, 32, 0, s>>>(partials, partial_blocks, nq, nr, bbox, task, tile_cnt, tile_off, round_cnt,
                                   round_off);
    k_points_pack<<<grid_for(nq + nr, 256), 256, 0, s>>>(q, nq, r, nr, bbox, q_f4, r_f4);
}

// ---------------------------------------------------------------------------
// task tables
// ---------------------------------------------------------------------------
// CMS: queries = buried dots of molecule m, references = buried dots of 1-m
__global__ void k_tasks_cms(Dev d, Rd r, NNTask* task)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * d.B; t += gridDim.x * blockDim.x) {
        const int c = t >> 1, m = t & 1, o = (c * 2) + (1 - m);
        NNTask T;
        T.c = c;
        T.E = 2.5e-7 * d.cx[c].R;
        T.q0 = r.bur_scan[doff(d, t)];
        T.qn = r.bur_scan[doff(d, t + 1)] - T.q0;
        T.r0 = r.bur_scan[doff(d, o)];
        T.rn = r.bur_scan[doff(d, o + 1)] - T.r0;
        task[t] = T;
    }
}

// SC trim: queries = buried dots of molecule m, references = accessible dots of m
__global__ void k_tasks_trim(Dev d, Rd r, NNTask* task)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * d.B; t += gridDim.x * blockDim.x) {
        const long long ds = doff(d, t), de = doff(d, t + 1);
        NNTask T;
        T.c = t >> 1;
        T.E = 2.5e-7 * d.cx[T.c].R;
        T.q0 = r.bur_scan[ds];
        T.qn = r.bur_scan[de] - T.q0;
        T.r0 = ds - r.bur_scan[ds];
        T.rn = (de - r.bur_scan[de]) - T.r0;
        task[t] = T;
    }
}

// SC neighbour distance: queries = trimmed dots of m, references = trimmed dots of 1-m
__global__ void k_tasks_sc(Dev d, Rd r, NNTask* task)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * d.B; t += gridDim.x * blockDim.x) {
        const int c = t >> 1, m = t & 1, o = (c * 2) + (1 - m);
        NNTask T;
        T.c = c;
        T.E = 2.5e-7 * d.cx[c].R;
        T.q0 = r.trim_scan[r.bur_scan[doff(d, t)]];
        T.qn = r.trim_scan[r.bur_scan[doff(d, t + 1)]] - T.q0;
        T.r0 = r.trim_scan[r.bur_scan[doff(d, o)]];
        T.rn = r.trim_scan[r.bur_scan[doff(d, o + 1)]] - T.r0;
        if (T.rn == 0) T.qn = 0;
        task[t] = T;
    }
}

void launch_tasks(const Dev& d, const Rd& r, int kind, NNTask* task, cudaStream_t s)
{
    const unsigned g = grid_for(2LL * d.B, 128);
    if (kind == 0) k_tasks_cms<<<g, 128, 0, s>>>(d, r, task);
    else if (kind == 1) k_tasks_trim<<<g, 128, 0, s>>>(d, r, task);
    else k_tasks_sc<<<g, 128, 0, s>>>(d, r, task);
}

// ---------------------------------------------------------------------------
// Spatial order of the packed lists.  Each complex & molecule range of a list
// is reordered by the Morton code of a 16^3 grid over its bounding box,
// stably (list order inside a cell), so 32-entry blocks and 512-entry rounds
// of the nearest-dot search are compact boxes.  The searches return the same
// results in any order: ties go to the smallest original position.
// ---------------------------------------------------------------------------
static constexpr int SO_GRID = 8;                     // cells per axis (a range holds a few thousand entries)
static constexpr int SO_CELLS = SO_GRID * SO_GRID * SO_GRID;

__device__ __forceinline__ int so_pad(int b) { return b + (b >> 7); }   // 128 buckets per lane, skewed banks

__device__ __forceinline__ unsigned so_spread4(unsigned v)      // up to 4 bits -> every third bit
{
    v &= 0xfu;
    v = (v | (v << 4)) & 0x0c3u;
    v = (v | (v << 2)) & 0x249u;
    return v;
}
static_assert(SO_GRID <= 16 && (SO_GRID & (SO_GRID - 1)) == 0, "Morton cells of up to 4 bits per axis");

__device__ __forceinline__ void so_range(const Dev& d, const Rd& r, int list, long long t, long long& s, long long& e)
{
    const long long ds = doff(d, t), de = doff(d, t + 1);
    if (list == SO_BUR) { s = r.bur_scan[ds]; e = r.bur_scan[de]; }
    else if (list == SO_ACC) { s = ds - r.bur_scan[ds]; e = de - r.bur_scan[de]; }
    else { s = r.trim_scan[r.bur_scan[ds]]; e = r.trim_scan[r.bur_scan[de]]; }
}

static constexpr int SO_W = 4;                               // warps per range
static constexpr int SO_STRIDE = SO_CELLS + SO_CELLS / 128;   // padded cell counters of one warp

// One CTA per range: the warps take a quarter of the range each, count its
// cells, and after a scan over (cell, warp) place its entries in list order,
// so the order is stable across the whole range.
__global__ void __launch_bounds__(SO_W * 32) k_spatial_order(Dev d, Rd r, int list, int set)
{
    CMS_EXIT_ON_OVERFLOW(d);
    extern __shared__ int so_cnt[];            // SO_W x SO_STRIDE cell counters
    __shared__ float sbox[SO_W][6];
    __shared__ int swarp[SO_W];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, tid = threadIdx.x;
    const unsigned lt = (1u << lane) - 1u;
    int* cnt = so_cnt + w * SO_STRIDE;
    const float4* f4 = list == SO_BUR ? r.bur_f4 : (list == SO_ACC ? r.acc_f4 : r.trim_f4);
    float4* of4 = r.so_f4[set];
    int* operm = r.so_perm[set];
    for (long long t = blockIdx.x; t < 2LL * d.B; t += gridDim.x) {
        long long s, e;
        so_range(d, r, list, t, s, e);
        const long long n = e - s;
        if (n <= 0) continue;
        // bounding box of the range
        float l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (long long i = tid; i < n; i += SO_W * 32) {
            const float4 p = f4[s + i];
            l[0] = fminf(l[0], p.x); l[1] = fminf(l[1], p.y); l[2] = fminf(l[2], p.z);
            h[0] = fmaxf(h[0], p.x); h[1] = fmaxf(h[1], p.y); h[2] = fmaxf(h[2], p.z);
        }
        for (int k = 0; k < 3; ++k) {
            for (int o = 16; o > 0; o >>= 1) {
                l[k] = fminf(l[k], __shfl_xor_sync(0xffffffffu, l[k], o));
                h[k] = fmaxf(h[k], __shfl_xor_sync(0xffffffffu, h[k], o));
            }
            if (lane == 0) { sbox[w][k] = l[k]; sbox[w][3 + k] = h[k]; }
        }
        __syncthreads();
        float sc[3];
        for (int k = 0; k < 3; ++k) {
            l[k] = sbox[0][k]; h[k] = sbox[0][3 + k];
            for (int v = 1; v < SO_W; ++v) { l[k] = fminf(l[k], sbox[v][k]); h[k] = fmaxf(h[k], sbox[v][3 + k]); }
            sc[k] = (float)SO_GRID / fmaxf(h[k] - l[k], 1e-3f);
        }
        auto cell = [&](float4 p) -> int {
            const int ix = min(SO_GRID - 1, max(0, (int)((p.x - l[0]) * sc[0])));
            const int iy = min(SO_GRID - 1, max(0, (int)((p.y - l[1]) * sc[1])));
            const int iz = min(SO_GRID - 1, max(0, (int)((p.z - l[2]) * sc[2])));
            return (int)(so_spread4(ix) | (so_spread4(iy) << 1) | (so_spread4(iz) << 2));
        };
        // this warp's quarter of the range and its cell counts
        const long long c0 = n * w / SO_W, c1 = n * (w + 1) / SO_W;
        for (int b = lane; b < SO_CELLS; b += 32) cnt[so_pad(b)] = 0;
        __syncwarp();
        for (long long i = c0 + lane; i < c1; i += 32) atomicAdd(&cnt[so_pad(cell(f4[s + i]))], 1);
        __syncthreads();
        // exclusive scan in (cell, warp) order: thread T owns cells [32 T, 32 T + 32)
        constexpr int PER = SO_CELLS / (SO_W * 32);
        int sum = 0;
        for (int k = 0; k < PER; ++k)
            for (int v = 0; v < SO_W; ++v) sum += so_cnt[v * SO_STRIDE + so_pad(tid * PER + k)];
        int x = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) swarp[w] = x;
        __syncthreads();
        int run = x - sum;
        for (int v = 0; v < w; ++v) run += swarp[v];
        for (int k = 0; k < PER; ++k) {
            for (int v = 0; v < SO_W; ++v) {
                int* c = &so_cnt[v * SO_STRIDE + so_pad(tid * PER + k)];
                const int cv = *c;
                *c = run;
                run += cv;
            }
        }
        __syncthreads();
        // stable scatter of this warp's quarter, 32 entries at a time in list order
        for (long long i0 = c0; i0 < c1; i0 += 32) {
            const long long i = i0 + lane;
            const bool on = i < c1;
            float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
            int b = SO_CELLS;
            if (on) { p = f4[s + i]; b = cell(p); }
            const unsigned peers = __match_any_sync(0xffffffffu, b);
            const int base = on ? cnt[so_pad(b)] : 0;
            __syncwarp();
            if (on && (peers & lt) == 0) cnt[so_pad(b)] = base + __popc(peers);
            __syncwarp();
            if (on) {
                const long long o = s + base + __popc(peers & lt);
                of4[o] = p;
                operm[o] = (int)(s + i);
            }
        }
        __syncthreads();
    }
}

void launch_spatial_order(const Dev& d, const Rd& r, int list, int set, cudaStream_t s)
{
    const int smem = SO_W * SO_STRIDE * (int)sizeof(int);
    cudaFuncSetAttribute(k_spatial_order, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_spatial_order<<<grid_for(2LL * d.B, 1, 12), SO_W * 32, smem, s>>>(d, r, list, set);
}

// ---------------------------------------------------------------------------
// per-dot CMS weights and deterministic per-atom sums (np.bincount order)
// ---------------------------------------------------------------------------
// per buried dot: area * exp(-d2 * weight) against the other molecule's buried dots
__global__ void k_cms_weights(Dev d, Rd r, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NB = r.bur_scan[doff(d, 2LL * d.B)];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cap; k += (long long)gridDim.x * blockDim.x) {
        if (k < NB) {
            const int dot = r.bur_idx[k];
            r.val[k] = d.darea[dot] * exp((-r.nn_d2[k]) * d.st.weight);
            r.own[k] = d.datom[dot];
        } else {
            r.own[k] = -1;
        }
    }
}

// values of every dot of molecule 0 (maximum possible CMS): own = owner or -1
__global__ void k_area_values(Dev d, Rd r, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long D = doff(d, 2LL * d.B);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap; i += (long long)gridDim.x * blockDim.x) {
        if (i < D) {
            const int cm = dot_cm(d, i);
            r.val[i] = d.darea[i];
            r.own[i] = (cm & 1) == 0 ? d.datom[i] : -1;
        } else {
            r.own[i] = -1;
        }
    }
}

// Per-atom sums in entry order, as np.bincount adds them: one warp per
// complex & molecule segment walks its entries 32 at a time (every atom's
// entries lie in one segment, so no other warp touches its sum).  Lanes that
// hold the same owner fold their values in lane order, starting from the
// atom's running sum; the group's first lane stores it back.
template <bool DOTS>
__global__ void k_own_fold(Dev d, Rd r, double* out)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const int lane = threadIdx.x & 31;
    const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long t = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); t < 2LL * d.B; t += nw) {
        long long s = doff(d, t), e = doff(d, t + 1);
        if (!DOTS) { s = r.bur_scan[s]; e = r.bur_scan[e]; }
        for (long long b = s; b < e; b += 32) {
            const long long k = b + lane;
            const int a = k < e ? r.own[k] : -1;
            const double v = k < e ? r.val[k] : 0.0;
            const unsigned peers = __match_any_sync(0xffffffffu, a);
            if (a >= 0) {
                double acc = out[a];
                for (unsigned m = peers; m; m &= m - 1) acc += __shfl_sync(peers, v, __ffs(m) - 1);
                if (lane == __ffs(peers) - 1) out[a] = acc;
            }
            __syncwarp();
        }
    }
}

void launch_per_atom_sum(const Dev& d, const Rd& r, bool dots, double* out, cudaStream_t s)
{
    cudaMemsetAsync(out, 0, sizeof(double) * d.N, s);
    const unsigned g = grid_for(2LL * d.B, 4);
    if (dots) k_own_fold<true><<<g, 128, 0, s>>>(d, r, out);
    else k_own_fold<false><<<g, 128, 0, s>>>(d, r, out);
}

void launch_cms_weights(const Dev& d, const Rd& r, long long cap, cudaStream_t s)
{
    k_cms_weights<<<grid_for(cap, 256), 256, 0, s>>>(d, r, cap);
}

void launch_area_values(const Dev& d, const Rd& r, long long cap, cudaStream_t s)
{
    k_area_values<<<grid_for(cap, 256), 256, 0, s>>>(d, r, cap);
}

// per complex & molecule: total of per-atom values (deterministic block tree)
__device__ __forceinline__ double block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0) for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
    __syncthreads();
    return t;
}

__global__ void k_atom_totals(Dev d, const double* per_atom, double* tot)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ double sh[32];
    const int t = blockIdx.x;                      // complex * 2 + molecule
    const int c = t >> 1, m = t & 1;
    const Cplx C = d.cx[c];
    const int s = C.a0 + (m ? C.n0 : 0), e = m ? C.a0 + C.n : C.a0 + C.n0;
    double v = 0.0;
    for (int a = s + threadIdx.x; a < e; a += blockDim.x) v += per_atom[a];
    double total = block_sum(v, sh);
    if (threadIdx.x == 0) tot[t] = total;
}

void launch_atom_totals(const Dev& d, const double* per_atom, double* tot, cudaStream_t s)
{
    k_atom_totals<<<2 * d.B, 256, 0, s>>>(d, per_atom, tot);
}

// ---------------------------------------------------------------------------
// shape complementarity
// ---------------------------------------------------------------------------
__global__ void k_trim_compact_flags(Dev d, Rd r, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NB = r.bur_scan[doff(d, 2LL * d.B)];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cap; k += (long long)gridDim.x * blockDim.x)
        if (k >= NB) r.keep[k] = 0;
}

__global__ void k_trim_fill(Dev d, Rd r, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NB = r.bur_scan[doff(d, 2LL * d.B)];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cap && k < NB; k += (long long)gridDim.x * blockDim.x) {
        if (r.keep[k]) {
            long long t = r.trim_scan[k];
            r.trim_idx[t] = r.bur_idx[k];
            r.trim_f4[t] = r.bur_f4[k];
        }
    }
}

void launch_trim_compact(const Dev& d, const Rd& r, long long cap, long long* scan_tmp, cudaStream_t s)
{
    k_trim_compact_flags<<<grid_for(cap, 256), 256, 0, s>>>(d, r, cap);
    scan_counts(r.keep, r.trim_scan, cap, scan_tmp, s);
    k_trim_fill<<<grid_for(cap, 256), 256, 0, s>>>(d, r, cap);
}

// grouped-data median (_core.py:1080-1104) of n values produced by `get`
template <class G>
__device__ double binned_median(long long n, double w, G&& get, long long* shl)
{
    if (n == 0) return 0.0;
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    for (long long k = threadIdx.x; k < n; k += blockDim.x) {
        long long b = (long long)floor(get(k) / w);
        lo = min(lo, b); hi = max(hi, b);
    }
    // block min / max
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) { shl[wp] = lo; shl[32 + wp] = hi; }
    __syncthreads();
    lo = shl[0]; hi = shl[32];
    for (int i = 1; i < nw; ++i) { lo = min(lo, shl[i]); hi = max(hi, shl[32 + i]); }
    __syncthreads();
    const double pct = 100.0 / (double)n;
    // count of values with bin <= t
    auto count_le = [&](long long t) -> long long {
        long long c = 0;
        for (long long k = threadIdx.x; k < n; k += blockDim.x)
            c += ((long long)floor(get(k) / w) <= t) ? 1 : 0;
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        __syncthreads();
        if (lane == 0) shl[wp] = c;
        __syncthreads();
        long long s = 0;
        for (int i = 0; i < nw; ++i) s += shl[i];
        __syncthreads();
        return s;
    };
    // smallest bin t with cumulative percentage >= 50 (np.searchsorted 'left')
    // (bins of non-finite values can span the whole int64 range: the midpoint is
    // taken on the unsigned difference, so every step narrows [a, b])
    long long a = lo, b = hi;
    while (a < b) {
        const long long mid = a + (long long)(((unsigned long long)b - (unsigned long long)a) >> 1);
        if ((double)count_le(mid) * pct >= 50.0) b = mid; else a = mid + 1;
    }
    const long long cum = count_le(a);
    const long long cnt = cum - (a == LLONG_MIN ? 0 : count_le(a - 1));
    const double cumperc = (double)cum * pct;
    const double before = cumperc - (double)cnt * pct;
    const double bin_perc = (double)cnt * pct;
    return (double)a * w + (50.0 - before) * w / bin_perc;
}

// one block per (complex, molecule): trimmed area, neighbour statistics
__global__ void k_sc_stats(Dev d, Rd r, const NNTask* task, double* out)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ double sh[32];
    __shared__ long long shl[64];
    const int t = blockIdx.x;
    const long long ds = doff(d, t), de = doff(d, t + 1);
    const long long bs = r.bur_scan[ds], be = r.bur_scan[de];
    // trimmed area: sum of areas of kept buried dots
    double v = 0.0;
    for (long long k = bs + threadIdx.x; k < be; k += blockDim.x)
        if (r.keep[k]) v += d.darea[r.bur_idx[k]];
    const double area = block_sum(v, sh);
    const long long ntrim = r.trim_scan[be] - r.trim_scan[bs];
    const NNTask T = task[t];
    double dmean = 0.0, dmed = 0.0, smean = 0.0, smed = 0.0;
    if (T.qn > 0 && T.rn > 0) {
        const long long q0 = T.q0, n = T.qn;
        const double weight = d.st.weight;
        auto distk = [&](long long k) -> double { return sqrt(r.nn_d2[q0 + k]); };
        auto rk = [&](long long k) -> double {
            const long long o = q0 + k;
            const V3 nm = ld3(d.dnml + 3LL * r.trim_idx[o]);
            const V3 nt = ld3(d.dnml + 3LL * r.trim_idx[T.r0 + r.nn_idx[o]]);
            const double dist = sqrt(r.nn_d2[o]);
            double rv = dot_alt(nm, nt);
            rv = rv * exp((-(dist * dist)) * weight);
            return rv < -0.999 ? -0.999 : (rv > 0.999 ? 0.999 : rv);
        };
        double sd = 0.0, sr = 0.0;
        for (long long k = threadIdx.x; k < n; k += blockDim.x) { sd += distk(k); sr += rk(k); }
        const double tot_d = block_sum(sd, sh);
        const double tot_r = block_sum(sr, sh);
        dmed = binned_median(n, d.st.bw_dist, distk, shl);
        const double rmed = binned_median(n, d.st.bw_norm, rk, shl);
        dmean = tot_d / (double)n;
        smean = -(tot_r / (double)n);
        smed = -rmed;
    }
    if (threadIdx.x == 0) {
        double* o = out + (long long)t * SC_SIDE_FIELDS;
        o[0] = dmean; o[1] = dmed; o[2] = smean; o[3] = smed; o[4] = area;
        o[5] = (double)ntrim; o[6] = (double)(de - ds);
    }
}

__global__ void k_sc_final(Dev d, const double* side, double* out)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.B; c += gridDim.x * blockDim.x) {
        const double* s0 = side + (long long)(2 * c) * SC_SIDE_FIELDS;
        const double* s1 = side + (long long)(2 * c + 1) * SC_SIDE_FIELDS;
        double* o = out + (long long)c * SC_FIELDS;
        const double dmean = (s0[0] + s1[0]) / 2, dmed = (s0[1] + s1[1]) / 2;
        const double smean = (s0[2] + s1[2]) / 2, smed = (s0[3] + s1[3]) / 2;
        o[0] = smed;                 // sc
        o[1] = s0[4] + s1[4];        // trimmed interface area
        o[2] = dmed;                 // median distance
        o[3] = dmean; o[4] = smean;
    }
}

void launch_sc_stats(const Dev& d, const Rd& r, const NNTask* task, double* side, double* out, cudaStream_t s)
{
    k_sc_stats<<<2 * d.B, 256, 0, s>>>(d, r, task, side);
    k_sc_final<<<grid_for(d.B, 128), 128, 0, s>>>(d, side, out);
}

}  // namespace cms
