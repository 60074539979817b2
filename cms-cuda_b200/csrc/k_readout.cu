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

// dot -> complex via binary search of dot_off (per complex & molecule)
__device__ __forceinline__ int dot_cm(const Dev& d, long long dot)
{
    int lo = 0, hi = 2 * d.B - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (doff(d, mid) <= dot) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_split_buried(Dev d, Rd r, long long cap)
{
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
static constexpr int NN_Q = 4;                // queries per thread (two packed pairs)
static constexpr int NN_TILE = NN_T * NN_Q;   // queries per tile
static constexpr int NN_R = 1024;             // references staged per round
static constexpr int NN_SUB = 32;             // references per threshold check

// one query's state
struct NNQ {
    float qx2, qy2, qz2;  // -2 q
    double qq;            // |q|^2 (FP32 value, held in FP64)
    int dot;              // index of the query point (FP64 coordinates read on recheck)
    float ms;             // smallest s seen
    float ts;             // s threshold: candidates have s <= ts (tile-relative)
    double best;
    int bidx;
    bool live, done;
};

struct NNTile {
    float cx, cy, cz;     // tile centre
    double rho, E0;       // bound on |q'|, FP32 rounding of the staged points
};

__device__ __forceinline__ float nn_s_threshold(const NNQ& q, const NNTile& t)
{
    if (!(q.ms < INFINITY)) return INFINITY;
    const double m = (double)q.ms + q.qq;
    const double th = m + 2.0 * nn_eps(m, t.rho, t.E0) * 1.01;
    return __double2float_ru(th - q.qq);
}

// Re-examine a block of n (<= 32) staged references [k0, k0+n) for every
// (lane, query) of the warp whose block minimum fell under its threshold.
// The warp takes the flagged lanes one at a time and checks the block in
// parallel, one reference per lane: FP32 filter against the lane's threshold
// at block start (a superset of what a sequential scan would recheck), FP64
// recheck in cdist order, then a warp reduction to the smallest FP64 value
// and, on ties, the smallest reference index -- what an in-order scan keeps.
template <int MODE>
__device__ __forceinline__ void nn_rescan_warp(const NNArgs& a, const NNTask& T, NNQ& q, unsigned need,
                                               const float4* sA, const float4* sB, int k0, int n, long long rb,
                                               const NNTile& tl)
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
        double e = INFINITY;
        float sv = INFINITY;
        int idx = 0x7fffffff;
        if (lane < n) {
            const int k = k0 + lane;
            const float v = nn_s(qx2, qy2, qz2, sA[k].x, sA[k].z, sB[k].x, sB[k].z);
            if (v <= ts) {
                const long long rk = T.r0 + rb + k;
                const double* rp = a.r_xyz + 3LL * (a.r_idx ? a.r_idx[rk] : rk);
                e = exact_d2(rp, a.q_xyz + 3LL * qdot);
                sv = v;
                idx = (int)(rb + k);
            }
        }
        if (MODE == NN_BAND) {
            const bool hit = __any_sync(0xffffffffu, e <= a.band_thr64);
            if (lane == L && hit) q.done = true;
        } else {
            for (int o = 16; o > 0; o >>= 1) {
                const double e2 = __shfl_xor_sync(0xffffffffu, e, o);
                const int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
                const float v2 = __shfl_xor_sync(0xffffffffu, sv, o);
                if (e2 < e || (e2 == e && i2 < idx)) { e = e2; idx = i2; }
                sv = fminf(sv, v2);
            }
            if (lane == L) {
                if (e < q.best) { q.best = e; q.bidx = idx; }
                if (sv < q.ms) { q.ms = sv; q.ts = nn_s_threshold(q, tl); }
            }
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(NN_T) k_nn(NNArgs a)
{
    __shared__ float4 sA[NN_R];   // (x, x, y, y)
    __shared__ float4 sB[NN_R];   // (z, z, |r|^2, |r|^2)
    const int lane = threadIdx.x & 31;
    const long long ntiles = a.tile_off[a.ntask];
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int lo = 0, hi = a.ntask - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (a.tile_off[mid] <= tile) lo = mid; else hi = mid - 1;
        }
        const NNTask T = a.task[lo];
        const long long qb = (tile - a.tile_off[lo]) * NN_TILE + threadIdx.x;
        // queries of the tile, then the tile centre and radius
        NNQ q[NN_Q];
        float qx[NN_Q], qy[NN_Q], qz[NN_Q];
        float lo3[3] = {INFINITY, INFINITY, INFINITY}, hi3[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
        for (int j = 0; j < NN_Q; ++j) {
            const long long qi = qb + (long long)j * NN_T;
            q[j].live = qi < T.qn;
            qx[j] = qy[j] = qz[j] = 0.f;
            q[j].dot = 0;
            if (q[j].live) {
                const float4 f = a.q_f4[T.q0 + qi];
                qx[j] = f.x; qy[j] = f.y; qz[j] = f.z;
                q[j].dot = a.q_idx ? a.q_idx[T.q0 + qi] : (int)(T.q0 + qi);
                lo3[0] = fminf(lo3[0], f.x); lo3[1] = fminf(lo3[1], f.y); lo3[2] = fminf(lo3[2], f.z);
                hi3[0] = fmaxf(hi3[0], f.x); hi3[1] = fmaxf(hi3[1], f.y); hi3[2] = fmaxf(hi3[2], f.z);
            }
        }
        __shared__ float sbox[6][NN_T / 32];
        __shared__ double srho[NN_T / 32];
        for (int k = 0; k < 3; ++k) {
            for (int o = 16; o > 0; o >>= 1) {
                lo3[k] = fminf(lo3[k], __shfl_xor_sync(0xffffffffu, lo3[k], o));
                hi3[k] = fmaxf(hi3[k], __shfl_xor_sync(0xffffffffu, hi3[k], o));
            }
        }
        if (lane == 0) for (int k = 0; k < 3; ++k) { sbox[k][threadIdx.x >> 5] = lo3[k]; sbox[3 + k][threadIdx.x >> 5] = hi3[k]; }
        __syncthreads();
        NNTile tl;
        {
            float c3[3];
            for (int k = 0; k < 3; ++k) {
                float l = sbox[k][0], h = sbox[3 + k][0];
                for (int w = 1; w < NN_T / 32; ++w) { l = fminf(l, sbox[k][w]); h = fmaxf(h, sbox[3 + k][w]); }
                c3[k] = (l <= h) ? 0.5f * (l + h) : 0.f;
            }
            tl.cx = c3[0]; tl.cy = c3[1]; tl.cz = c3[2];
        }
        double rho = 0.0;
#pragma unroll
        for (int j = 0; j < NN_Q; ++j) {
            qx[j] -= tl.cx; qy[j] -= tl.cy; qz[j] -= tl.cz;
            if (q[j].live) rho = fmax(rho, sqrt((double)qx[j] * qx[j] + (double)qy[j] * qy[j] + (double)qz[j] * qz[j]));
        }
        for (int o = 16; o > 0; o >>= 1) rho = fmax(rho, __shfl_xor_sync(0xffffffffu, rho, o));
        if (lane == 0) srho[threadIdx.x >> 5] = rho;
        __syncthreads();
        for (int w = 0; w < NN_T / 32; ++w) rho = fmax(rho, srho[w]);
        __syncthreads();
        tl.rho = rho * (1.0 + 1e-6) + 1e-6;
        tl.E0 = T.E;
#pragma unroll
        for (int j = 0; j < NN_Q; ++j) {
            q[j].qx2 = -2.0f * qx[j]; q[j].qy2 = -2.0f * qy[j]; q[j].qz2 = -2.0f * qz[j];
            q[j].qq = (double)nn_rr(qx[j], qy[j], qz[j]);
            q[j].ms = INFINITY;
            q[j].best = INFINITY;
            q[j].bidx = -1;
            q[j].done = !q[j].live;
            if (MODE == NN_BAND) {
                const double t = a.band_thr64 + nn_eps(a.band_thr64, tl.rho, tl.E0) * 1.01;
                q[j].ts = __double2float_ru(t - q[j].qq);
            } else {
                q[j].ts = INFINITY;
                if (q[j].live && T.rn > 0) {
                    // seed with reference 0 (the first index, so ties keep it)
                    const long long r0 = a.r_idx ? a.r_idx[T.r0] : T.r0;
                    const float4 f = a.r_f4[T.r0];
                    const float rx = f.x - tl.cx, ry = f.y - tl.cy, rz = f.z - tl.cz;
                    q[j].best = exact_d2(a.r_xyz + 3LL * r0, a.q_xyz + 3LL * q[j].dot);
                    q[j].bidx = 0;
                    q[j].ms = nn_s(q[j].qx2, q[j].qy2, q[j].qz2, rx, ry, rz, nn_rr(rx, ry, rz));
                    q[j].ts = nn_s_threshold(q[j], tl);
                }
            }
        }
        const f2_t qx01 = pk2(q[0].qx2, q[1].qx2), qy01 = pk2(q[0].qy2, q[1].qy2), qz01 = pk2(q[0].qz2, q[1].qz2);
        const f2_t qx23 = pk2(q[2].qx2, q[3].qx2), qy23 = pk2(q[2].qy2, q[3].qy2), qz23 = pk2(q[2].qz2, q[3].qz2);
        // Order of the reference rounds.  The minimum searches go in index order
        // (first index wins ties).  The band test only asks whether ANY reference
        // is within the band, so it starts at the references that sit next to the
        // tile's first query in dot order (usually its own surface patch) and
        // wraps around: every pair is still examined unless a hit ends the scan.
        long long rb_start = 0;
        if (MODE == NN_BAND && a.hint_scan && T.rn > NN_R) {
            const long long first = T.q0 + (tile - a.tile_off[lo]) * NN_TILE;
            const long long dot = a.q_idx ? a.q_idx[first] : first;
            const long long pos = (dot - a.hint_scan[dot]) - T.r0 - NN_R / 2;
            rb_start = pos < 0 ? 0 : (pos >= T.rn ? T.rn - 1 : pos);
        }
        for (long long seen = 0; seen < T.rn;) {
            const long long rb = (rb_start + seen) % T.rn;
            const int nr = (int)min(min((long long)NN_R, T.rn - seen), T.rn - rb);
            seen += nr;
            __syncthreads();
            for (int k = threadIdx.x; k < nr; k += NN_T) {
                const float4 r = a.r_f4[T.r0 + rb + k];
                const float rx = r.x - tl.cx, ry = r.y - tl.cy, rz = r.z - tl.cz;
                const float rr = nn_rr(rx, ry, rz);
                sA[k] = make_float4(rx, rx, ry, ry);
                sB[k] = make_float4(rz, rz, rr, rr);
            }
            __syncthreads();
            // warp-uniform: the block loop below uses full-warp ballots and shuffles
            const bool all_done = __all_sync(0xffffffffu, q[0].done && q[1].done && q[2].done && q[3].done);
            if (!all_done) {
                for (int sb = 0; sb < nr; sb += NN_SUB) {
                    const int n = min(NN_SUB, nr - sb);
                    float m0 = INFINITY, m1 = INFINITY, m2 = INFINITY, m3 = INFINITY;
#pragma unroll 4
                    for (int k = sb; k < sb + n; ++k) {
                        const float4 ra = sA[k];
                        const float4 rb4 = sB[k];
                        const f2_t rxx = pk2(ra.x, ra.y), ryy = pk2(ra.z, ra.w);
                        const f2_t rzz = pk2(rb4.x, rb4.y), rrr = pk2(rb4.z, rb4.w);
                        const f2_t s01 = fma2(qz01, rzz, fma2(qy01, ryy, fma2(qx01, rxx, rrr)));
                        const f2_t s23 = fma2(qz23, rzz, fma2(qy23, ryy, fma2(qx23, rxx, rrr)));
                        float a0, a1, a2, a3;
                        upk2(s01, a0, a1);
                        upk2(s23, a2, a3);
                        m0 = fminf(m0, a0); m1 = fminf(m1, a1); m2 = fminf(m2, a2); m3 = fminf(m3, a3);
                    }
                    const unsigned n0 = __ballot_sync(0xffffffffu, !q[0].done && m0 <= q[0].ts);
                    const unsigned n1 = __ballot_sync(0xffffffffu, !q[1].done && m1 <= q[1].ts);
                    const unsigned n2 = __ballot_sync(0xffffffffu, !q[2].done && m2 <= q[2].ts);
                    const unsigned n3 = __ballot_sync(0xffffffffu, !q[3].done && m3 <= q[3].ts);
                    if (n0) nn_rescan_warp<MODE>(a, T, q[0], n0, sA, sB, sb, n, rb, tl);
                    if (n1) nn_rescan_warp<MODE>(a, T, q[1], n1, sA, sB, sb, n, rb, tl);
                    if (n2) nn_rescan_warp<MODE>(a, T, q[2], n2, sA, sB, sb, n, rb, tl);
                    if (n3) nn_rescan_warp<MODE>(a, T, q[3], n3, sA, sB, sb, n, rb, tl);
                }
            }
            if (MODE == NN_BAND) {
                if (__syncthreads_and(q[0].done && q[1].done && q[2].done && q[3].done)) break;
            }
        }
        (void)lane;
#pragma unroll
        for (int j = 0; j < NN_Q; ++j) {
            if (!q[j].live) continue;
            const long long o = T.q0 + qb + (long long)j * NN_T;
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
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < a.ntask; t += gridDim.x * blockDim.x) {
        const NNTask T = a.task[t];
        a.tile_cnt[t] = (T.qn > 0 && (T.rn > 0 || a.band_mode)) ? (int)((T.qn + NN_TILE - 1) / NN_TILE) : 0;
    }
}

void launch_nn_tiles(NNArgs a, int mode, long long* scan_tmp, cudaStream_t s)
{
    a.band_mode = mode == NN_BAND;
    k_nn_tiles<<<grid_for(a.ntask, 128), 128, 0, s>>>(a);
    scan_counts(a.tile_cnt, a.tile_off, a.ntask, scan_tmp, s);
}

void launch_nn_kernel(NNArgs a, int mode, long long tile_cap, cudaStream_t s)
{
    a.band_mode = mode == NN_BAND;
    const unsigned grid = grid_for(tile_cap, 1, 8);   // persistent: at most 8 tiles in flight per SM
    if (mode == NN_MIN) k_nn<NN_MIN><<<grid, NN_T, 0, s>>>(a);
    else if (mode == NN_ARGMIN) k_nn<NN_ARGMIN><<<grid, NN_T, 0, s>>>(a);
    else k_nn<NN_BAND><<<grid, NN_T, 0, s>>>(a);
}

void launch_nn(NNArgs a, int mode, long long tile_cap, long long* scan_tmp, cudaStream_t s)
{
    launch_nn_tiles(a, mode, scan_tmp, s);
    launch_nn_kernel(a, mode, tile_cap, s);
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
                              NNTask* task, int* tile_cnt, long long* tile_off)
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
                         long long* tile_off, cudaStream_t s)
{
    k_points_bbox<<<partial_blocks, 256, 0, s>>>(q, nq, r, nr, partials);
    k_points_task<<<1, 32, 0, s>>>(partials, partial_blocks, nq, nr, bbox, task, tile_cnt, tile_off);
    k_points_pack<<<grid_for(nq + nr, 256), 256, 0, s>>>(q, nq, r, nr, bbox, q_f4, r_f4);
}

// ---------------------------------------------------------------------------
// task tables
// ---------------------------------------------------------------------------
// CMS: queries = buried dots of molecule m, references = buried dots of 1-m
__global__ void k_tasks_cms(Dev d, Rd r, NNTask* task)
{
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
// per-dot CMS weights and deterministic per-atom sums (np.bincount order)
// ---------------------------------------------------------------------------
// per buried dot: area * exp(-d2 * weight) against the other molecule's buried dots
__global__ void k_cms_weights(Dev d, Rd r, long long cap)
{
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

__global__ void k_own_count(Rd r, long long cap, int* cnt)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cap; k += (long long)gridDim.x * blockDim.x) {
        int a = r.own[k];
        if (a >= 0) atomicAdd(&cnt[a], 1);
    }
}

__global__ void k_own_scatter(Rd r, long long cap, const long long* off, int* fill, int* slot)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cap; k += (long long)gridDim.x * blockDim.x) {
        int a = r.own[k];
        if (a >= 0) slot[off[a] + atomicAdd(&fill[a], 1)] = (int)k;
    }
}

__global__ void k_own_sum(long long N, const long long* off, int* slot, const double* val, double* out)
{
    for (long long a = blockIdx.x * (long long)blockDim.x + threadIdx.x; a < N; a += (long long)gridDim.x * blockDim.x) {
        const long long s = off[a], e = off[a + 1];
        for (long long i = s + 1; i < e; ++i) {           // entries in increasing dot order
            int v = slot[i];
            long long k = i - 1;
            while (k >= s && slot[k] > v) { slot[k + 1] = slot[k]; --k; }
            slot[k + 1] = v;
        }
        double acc = 0.0;
        for (long long i = s; i < e; ++i) acc += val[slot[i]];
        out[a] = acc;
    }
}

void launch_per_atom_sum(const Dev& d, const Rd& r, long long cap, double* out, long long* scan_tmp, cudaStream_t s)
{
    cudaMemsetAsync(r.acnt, 0, sizeof(int) * d.N, s);
    cudaMemsetAsync(r.afill, 0, sizeof(int) * d.N, s);
    k_own_count<<<grid_for(cap, 256), 256, 0, s>>>(r, cap, r.acnt);
    scan_counts(r.acnt, r.aoff, d.N, scan_tmp, s);
    k_own_scatter<<<grid_for(cap, 256), 256, 0, s>>>(r, cap, r.aoff, r.afill, r.aslot);
    k_own_sum<<<grid_for(d.N, 128), 128, 0, s>>>(d.N, r.aoff, r.aslot, r.val, out);
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
    const long long NB = r.bur_scan[doff(d, 2LL * d.B)];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cap; k += (long long)gridDim.x * blockDim.x)
        if (k >= NB) r.keep[k] = 0;
}

__global__ void k_trim_fill(Dev d, Rd r, long long cap)
{
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
    long long a = lo, b = hi;
    while (a < b) {
        long long mid = a + ((b - a) >> 1);
        if ((double)count_le(mid) * pct >= 50.0) b = mid; else a = mid + 1;
    }
    const long long cum = count_le(a);
    const long long cnt = cum - count_le(a - 1);
    const double cumperc = (double)cum * pct;
    const double before = cumperc - (double)cnt * pct;
    const double bin_perc = (double)cnt * pct;
    return (double)a * w + (50.0 - before) * w / bin_perc;
}

// one block per (complex, molecule): trimmed area, neighbour statistics
__global__ void k_sc_stats(Dev d, Rd r, const NNTask* task, double* out)
{
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
