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
// Error model (u = 2^-24): coordinates relative to the centre are within R of
// it per axis.  For any pair, |sqrt(D32) - sqrt(D)| <= E + rho*sqrt(D) with
// E = 3.53 u R and rho = 2.7 u (input rounding of both points, the rounded
// difference and the three-term FP32 sum).  A reference that attains the
// FP64 minimum therefore has sqrt(D32) <= (sqrt(m) + E)(1 + 3 rho) + E,
// m = smallest D32 seen; the kernel rechecks everything under that bound.
__device__ __forceinline__ float nn_threshold(float m, double E)
{
    if (!(m < INFINITY)) return INFINITY;
    double t = (sqrt((double)m) + E) * (1.0 + 1e-6) + E;
    return __double2float_ru(t * t * (1.0 + 1e-6));
}

__device__ __forceinline__ double exact_d2(const double* a, const double* b)
{
    // cdist(ref, query, 'sqeuclidean') order: (d0*d0 + d1*d1) + d2*d2
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return (dx * dx + dy * dy) + dz * dz;
}

// Packed FP32 pairs (Blackwell f32x2 arithmetic): one instruction does the
// same IEEE round-to-nearest operation on two lanes, so the packed distances
// equal the scalar ones bit for bit.
typedef unsigned long long f2_t;
__device__ __forceinline__ f2_t pk2(float a, float b) { f2_t r; asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b)); return r; }
__device__ __forceinline__ void upk2(f2_t v, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ f2_t sub2(f2_t a, f2_t b) { f2_t r; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b)); return r; }
__device__ __forceinline__ f2_t mul2(f2_t a, f2_t b) { f2_t r; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b)); return r; }
__device__ __forceinline__ f2_t fma2(f2_t a, f2_t b, f2_t c) { f2_t r; asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c)); return r; }

__device__ __forceinline__ float d2_f32(float rx, float ry, float rz, float qx, float qy, float qz)
{
    const float dx = rx - qx, dy = ry - qy, dz = rz - qz;
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, dx * dx));
}

static constexpr int NN_T = 128;              // threads per tile
static constexpr int NN_Q = 4;                // queries per thread (two packed pairs)
static constexpr int NN_TILE = NN_T * NN_Q;   // queries per tile
static constexpr int NN_R = 1024;             // references staged per round
static constexpr int NN_SUB = 32;             // references per threshold check

// one query's state
struct NNQ {
    float qx, qy, qz;
    int dot;            // dot index of the query (its FP64 coordinates are read on recheck)
    float mf, thr;
    double best;
    int bidx;
    bool live, done;
};

// re-examine references [k0, k0+n) of the staged round for one query whose
// block minimum fell under its threshold: FP32 filter, FP64 recheck in order
template <int MODE>
__device__ __forceinline__ void nn_rescan(const NNArgs& a, const NNTask& T, NNQ& q, const float4* sA,
                                          const float2* sB, int k0, int n, long long rb, double E)
{
    for (int k = k0; k < k0 + n; ++k) {
        const float d2 = d2_f32(sA[k].x, sA[k].z, sB[k].x, q.qx, q.qy, q.qz);
        if (d2 <= q.thr) {
            const long long rk = T.r0 + rb + k;
            const double* rp = a.r_xyz + 3LL * (a.r_idx ? a.r_idx[rk] : rk);
            const double e = exact_d2(rp, a.q_xyz + 3LL * q.dot);
            if (MODE == NN_BAND) {
                if (e <= a.band_thr64) { q.done = true; q.best = e; return; }
            } else {
                if (e < q.best) { q.best = e; q.bidx = (int)(rb + k); }
                if (d2 < q.mf) { q.mf = d2; q.thr = nn_threshold(q.mf, E); }
            }
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(NN_T) k_nn(NNArgs a)
{
    __shared__ float4 sA[NN_R];   // (x, x, y, y)
    __shared__ float2 sB[NN_R];   // (z, z)
    const long long ntiles = a.tile_off[a.ntask];
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int lo = 0, hi = a.ntask - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (a.tile_off[mid] <= tile) lo = mid; else hi = mid - 1;
        }
        const NNTask T = a.task[lo];
        const long long qb = (tile - a.tile_off[lo]) * NN_TILE + threadIdx.x;
        const double E = T.E;
        float band_thr = INFINITY;
        if (MODE == NN_BAND) {
            double t = (sqrt(a.band_thr64) * (1.0 + 1e-6)) + E;
            band_thr = __double2float_ru(t * t * (1.0 + 1e-6));
        }
        NNQ q[NN_Q];
#pragma unroll
        for (int j = 0; j < NN_Q; ++j) {
            const long long qi = qb + (long long)j * NN_T;
            q[j].live = qi < T.qn;
            q[j].qx = q[j].qy = q[j].qz = 0.f;
            q[j].dot = 0;
            if (q[j].live) {
                const float4 f = a.q_f4[T.q0 + qi];
                q[j].qx = f.x; q[j].qy = f.y; q[j].qz = f.z;
                q[j].dot = a.q_idx ? a.q_idx[T.q0 + qi] : (int)(T.q0 + qi);
            }
            q[j].mf = INFINITY;
            q[j].thr = MODE == NN_BAND ? band_thr : INFINITY;
            q[j].best = INFINITY;
            q[j].bidx = -1;
            q[j].done = !q[j].live;
        }
        const f2_t qx01 = pk2(q[0].qx, q[1].qx), qy01 = pk2(q[0].qy, q[1].qy), qz01 = pk2(q[0].qz, q[1].qz);
        const f2_t qx23 = pk2(q[2].qx, q[3].qx), qy23 = pk2(q[2].qy, q[3].qy), qz23 = pk2(q[2].qz, q[3].qz);
        for (long long rb = 0; rb < T.rn; rb += NN_R) {
            const int nr = (int)min((long long)NN_R, T.rn - rb);
            __syncthreads();
            for (int k = threadIdx.x; k < nr; k += NN_T) {
                const float4 r = a.r_f4[T.r0 + rb + k];
                sA[k] = make_float4(r.x, r.x, r.y, r.y);
                sB[k] = make_float2(r.z, r.z);
            }
            __syncthreads();
            const bool all_done = q[0].done && q[1].done && q[2].done && q[3].done;
            if (!all_done) {
                for (int sb = 0; sb < nr; sb += NN_SUB) {
                    const int n = min(NN_SUB, nr - sb);
                    float m0 = INFINITY, m1 = INFINITY, m2 = INFINITY, m3 = INFINITY;
#pragma unroll 4
                    for (int k = sb; k < sb + n; ++k) {
                        const float4 ra = sA[k];
                        const float2 rz = sB[k];
                        const f2_t rxx = pk2(ra.x, ra.y), ryy = pk2(ra.z, ra.w), rzz = pk2(rz.x, rz.y);
                        f2_t dx = sub2(rxx, qx01), dy = sub2(ryy, qy01), dz = sub2(rzz, qz01);
                        f2_t s01 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
                        dx = sub2(rxx, qx23); dy = sub2(ryy, qy23); dz = sub2(rzz, qz23);
                        f2_t s23 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
                        float a0, a1, a2, a3;
                        upk2(s01, a0, a1);
                        upk2(s23, a2, a3);
                        m0 = fminf(m0, a0); m1 = fminf(m1, a1); m2 = fminf(m2, a2); m3 = fminf(m3, a3);
                    }
                    if (!q[0].done && m0 <= q[0].thr) nn_rescan<MODE>(a, T, q[0], sA, sB, sb, n, rb, E);
                    if (!q[1].done && m1 <= q[1].thr) nn_rescan<MODE>(a, T, q[1], sA, sB, sb, n, rb, E);
                    if (!q[2].done && m2 <= q[2].thr) nn_rescan<MODE>(a, T, q[2], sA, sB, sb, n, rb, E);
                    if (!q[3].done && m3 <= q[3].thr) nn_rescan<MODE>(a, T, q[3], sA, sB, sb, n, rb, E);
                }
            }
            if (MODE == NN_BAND) {
                if (__syncthreads_and(q[0].done && q[1].done && q[2].done && q[3].done)) break;
            }
        }
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
    const int c = t >> 1, m = t & 1;
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
