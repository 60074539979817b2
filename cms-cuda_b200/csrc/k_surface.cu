// Surface pipeline, front half: per-complex setup, cell lists, attention
// numbers, neighbour / buried-partner lists, the pair loop and the triple
// (probe placement) loop.
//
// Reference behaviour (cms-cuda/_core.py):
//   assign_attention_numbers   _core.py:1150-1195
//   build_neighbor_arrays      _core.py:1251-1349
//   second_loop                _core.py:1351-1442
//   vec_third_loop             _core.py:1445-1643
// Every distance test keeps the reference's summation order (dot_seq for
// cdist / np.sum / norm, dot_alt for einsum) and strictness.
#include <type_traits>

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

// ---------------------------------------------------------------------------
// per-complex setup: bounding box, radmax, cell grid
// ---------------------------------------------------------------------------
static constexpr long long MAX_CELLS_PER_COMPLEX = 1ll << 21;

__global__ void k_setup(Dev d, int* ncell)
{
    const int c = blockIdx.x;
    const int a0 = d.atom_off[c], a1 = d.atom_off[c + 1];
    // per molecule: min xyz, -max xyz; then -max radius over both
    double v[13];
    for (int k = 0; k < 13; ++k) v[k] = INFINITY;
    for (int g = a0 + threadIdx.x; g < a1; g += blockDim.x) {
        double4 a = d.xyzr[g];
        const int m = (g - a0) < d.n0[c] ? 0 : 1;
        double* b = v + 6 * m;
        b[0] = fmin(b[0], a.x); b[1] = fmin(b[1], a.y); b[2] = fmin(b[2], a.z);
        b[3] = fmin(b[3], -a.x); b[4] = fmin(b[4], -a.y); b[5] = fmin(b[5], -a.z);
        v[12] = fmin(v[12], -a.w);
        d.cplx[g] = c;
        d.mol[g] = (int8_t)m;
    }
    __shared__ double sh[13][32];
    for (int k = 0; k < 13; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] = fmin(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) for (int k = 0; k < 13; ++k) sh[k][w] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 13; ++k) { double m = sh[k][0]; for (int i = 1; i < nw; ++i) m = fmin(m, sh[k][i]); v[k] = m; }
        Cplx C;
        for (int m = 0; m < 2; ++m)
            for (int k = 0; k < 3; ++k) { C.mlo[m][k] = v[6 * m + k]; C.mhi[m][k] = -v[6 * m + 3 + k]; }
        // whole-complex box and radius in the layout used below
        double u[7];
        for (int k = 0; k < 3; ++k) { u[k] = fmin(v[k], v[6 + k]); u[3 + k] = fmin(v[3 + k], v[9 + k]); }
        u[6] = v[12];
        for (int k = 0; k < 7; ++k) v[k] = u[k];
        C.a0 = a0; C.n = a1 - a0; C.n0 = d.n0[c];
        const double rp = d.st.rp;
        if (C.n <= 0) {
            C.radmax = 0; C.h = 1; C.R = 1;
            for (int k = 0; k < 3; ++k) { C.dims[k] = 1; C.org[k] = 0; C.ctr[k] = 0; }
            d.status[c] |= ST_EMPTY;
            ncell[c] = 0;
        } else {
            double lo[3] = {v[0], v[1], v[2]}, hi[3] = {-v[3], -v[4], -v[5]};
            C.radmax = -v[6];
            // cells of half the longest neighbour bridge (2 radmax + 2 rp); the
            // scans below visit every cell that meets their search ball
            const double cut = 2.0 * fmax(C.radmax, 0.0) + 2.0 * fmax(rp, 0.0);
            double h = fmax(fmax(0.5 * cut, d.all_atoms ? 0.0 : d.st.sep / 6.0), 0.1) * (1.0 + 1e-6) + 1e-6;
            long long nc;
            for (;;) {
                nc = 1;
                for (int k = 0; k < 3; ++k) {
                    C.dims[k] = (int)floor((hi[k] - lo[k]) / h) + 1;
                    nc *= C.dims[k];
                }
                if (nc <= MAX_CELLS_PER_COMPLEX) break;
                h *= 1.25;
            }
            C.h = h;
            double half = 0.0;
            for (int k = 0; k < 3; ++k) {
                C.org[k] = lo[k];
                C.ctr[k] = 0.5 * (lo[k] + hi[k]);
                half = fmax(half, 0.5 * (hi[k] - lo[k]));
            }
            C.R = half + fmax(C.radmax, 0.0) + 2.0 * fmax(rp, 0.0) + 1.0;
            ncell[c] = (int)nc;
        }
        C.cell0 = 0;
        d.cx[c] = C;
        d.coin[c] = ~0ull;
    }
}

void launch_setup(const Dev& d, cudaStream_t s)
{
    k_setup<<<d.B, 256, 0, s>>>(d, d.ncell);
}

// ---------------------------------------------------------------------------
// cell lists (counting sort of atoms by cell, then each cell sorted by atom id)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atom_cell(const Dev& d, int g, int c, int& cx, int& cy, int& cz)
{
    const Cplx& C = d.cx[c];
    double4 a = d.xyzr[g];
    cx = cell_coord(a.x, C.org[0], C.h, C.dims[0]);
    cy = cell_coord(a.y, C.org[1], C.h, C.dims[1]);
    cz = cell_coord(a.z, C.org[2], C.h, C.dims[2]);
}

__global__ void k_cell_count(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < d.N; g += (long long)gridDim.x * blockDim.x) {
        int c = d.cplx[g];
        int x, y, z;
        atom_cell(d, (int)g, c, x, y, z);
        const Cplx& C = d.cx[c];
        long long cell = d.ncell_scan[c] + ((long long)x * C.dims[1] + y) * C.dims[2] + z;
        if (cell >= d.cells_cap) { atomicOr(&d.status[c], ST_OVERFLOW); cell = -1; }
        d.cell_of[g] = (int)cell;
        if (cell >= 0) atomicAdd(&d.cell_cnt[cell], 1);
    }
}

__global__ void k_cell_fill(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < d.N; g += (long long)gridDim.x * blockDim.x) {
        int cell = d.cell_of[g];
        if (cell < 0) continue;
        int pos = atomicAdd(&d.cell_fill[cell], 1);
        d.cell_atom[d.cell_start[cell] + pos] = (int)g;
    }
}

__global__ void k_cell_sort(Dev d, long long ncells_cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long ncells = d.ncell_scan[d.B];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells && c < ncells_cap;
         c += (long long)gridDim.x * blockDim.x) {
        long long s = d.cell_start[c], e = d.cell_start[c + 1];
        for (long long i = s + 1; i < e; ++i) {
            int v = d.cell_atom[i];
            long long k = i - 1;
            while (k >= s && d.cell_atom[k] > v) { d.cell_atom[k + 1] = d.cell_atom[k]; --k; }
            d.cell_atom[k + 1] = v;
        }
    }
}

__global__ void k_zero_int(int* p, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = 0;
}

// d.ncell_scan must already hold the exclusive scan of d.ncell
void launch_cells(const Dev& d, long long n_cells, long long* scan_tmp, cudaStream_t s)
{
    k_zero_int<<<grid_for(n_cells, 256), 256, 0, s>>>(d.cell_cnt, n_cells);
    k_zero_int<<<grid_for(n_cells, 256), 256, 0, s>>>(d.cell_fill, n_cells);
    k_cell_count<<<grid_for(d.N, 256), 256, 0, s>>>(d);
    scan_counts(d.cell_cnt, d.cell_start, n_cells, scan_tmp, s);
    k_cell_fill<<<grid_for(d.N, 256), 256, 0, s>>>(d);
    k_cell_sort<<<grid_for(n_cells, 128), 128, 0, s>>>(d, n_cells);
}

// ---------------------------------------------------------------------------
// Ball scan: a warp visits every atom in the cells that meet the ball of
// radius `range` around atom g (a superset of the atoms within range).  The
// cells of one (x, y) column that meet the ball are contiguous in cell_atom,
// so the warp lays the columns end to end and hands one atom to each lane;
// f(j) is called by all 32 lanes together, j = -1 past the end; when f
// returns bool, the scan stops after the first call where any lane returned
// true.  Cell bounds get a 1e-9 A margin over the rounding of the cell
// assignment.
// ---------------------------------------------------------------------------
static constexpr int NB_WARPS = 4;

__device__ __forceinline__ double slab_gap(double x, double lo, double hi)
{
    return fmax(fmax(lo - x, x - hi), 0.0);
}

__device__ __forceinline__ int warp_scan_excl(int v, int& total)
{
    const int lane = threadIdx.x & 31;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

struct BallScratch {
    int pre[33];
    long long beg[32];
};

template <class F>
__device__ __forceinline__ void scan_ball(const Dev& d, int g, int c, double range, BallScratch& S, F&& f)
{
    const int lane = threadIdx.x & 31;
    const Cplx& C = d.cx[c];
    const double4 a = d.xyzr[g];
    int x, y, z;
    atom_cell(d, g, c, x, y, z);
    const double re = range * (1.0 + 1e-9) + 1e-9;
    const double rc = fmin(ceil(re / C.h), 1e6);
    const int R = (int)rc;
    const int x0 = max(x - R, 0), x1 = min(x + R, C.dims[0] - 1);
    const int y0 = max(y - R, 0), y1 = min(y + R, C.dims[1] - 1);
    const int ny = y1 - y0 + 1;
    const int ncol = (x1 - x0 + 1) * ny;
    const long long c0 = d.ncell_scan[c];
    for (int cb = 0; cb < ncol; cb += 32) {
        const int col = cb + lane;
        long long s = 0;
        int len = 0;
        if (col < ncol) {
            const int ix = x0 + col / ny, iy = y0 + col % ny;
            const double gx = slab_gap(a.x, C.org[0] + ix * C.h, C.org[0] + (ix + 1) * C.h) - 1e-9;
            const double gy = slab_gap(a.y, C.org[1] + iy * C.h, C.org[1] + (iy + 1) * C.h) - 1e-9;
            const double gx2 = gx > 0.0 ? gx * gx : 0.0, gy2 = gy > 0.0 ? gy * gy : 0.0;
            const double rem = re * re - (gx2 + gy2);
            if (rem >= 0.0) {
                const double dz = sqrt(rem) + 1e-9;
                const int z0 = cell_coord(a.z - dz, C.org[2], C.h, C.dims[2]);
                const int z1 = cell_coord(a.z + dz, C.org[2], C.h, C.dims[2]);
                const long long base = c0 + ((long long)ix * C.dims[1] + iy) * C.dims[2];
                s = d.cell_start[base + z0];
                len = (int)(d.cell_start[base + z1 + 1] - s);
            }
        }
        int tot;
        const int ex = warp_scan_excl(len, tot);
        __syncwarp();
        S.pre[lane] = ex;
        S.beg[lane] = s;
        if (lane == 31) S.pre[32] = tot;
        __syncwarp();
        for (int b = 0; b < tot; b += 32) {
            const int i = b + lane;
            int j = -1;
            if (i < tot) {
                int lo = 0, hi = 31;          // column holding i: largest k with pre[k] <= i
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S.pre[mid] <= i) lo = mid; else hi = mid - 1;
                }
                j = d.cell_atom[S.beg[lo] + (i - S.pre[lo])];
            }
            if constexpr (std::is_same<decltype(f(j)), bool>::value) {
                if (__any_sync(0xffffffffu, f(j))) {
                    __syncwarp();
                    return;
                }
            } else {
                f(j);
            }
        }
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// attention numbers: blocker (1) when the closest atom of the other molecule
// is at least `sep` away, else 5; every atom gets 5 in all-atoms mode
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NB_WARPS * 32) k_attention(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ BallScratch sc[NB_WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long wid = blockIdx.x * (long long)NB_WARPS + w;
    const long long nw = (long long)gridDim.x * NB_WARPS;
    for (long long gg = wid; gg < d.N; gg += nw) {
        const int g = (int)gg;
        if (d.all_atoms) { if (lane == 0) d.atten[g] = 5; continue; }
        const int c = d.cplx[g];
        const V3 xi = atom_xyz(d, g);
        const int8_t mi = d.mol[g];
        // farther than sep (plus a margin) from the other molecule's box: no atom within sep
        {
            const Cplx& C = d.cx[c];
            const int o = 1 - mi;
            const double gx = slab_gap(xi.x, C.mlo[o][0], C.mhi[o][0]);
            const double gy = slab_gap(xi.y, C.mlo[o][1], C.mhi[o][1]);
            const double gz = slab_gap(xi.z, C.mlo[o][2], C.mhi[o][2]);
            const double se = d.st.sep * (1.0 + 1e-9) + 1e-9;
            if (gx * gx + gy * gy + gz * gz > se * se) { if (lane == 0) d.atten[g] = 1; continue; }
        }
        // the reference's min over the other molecule of cdist >= sep fails as soon as one distance is
        // below sep (sqrt is monotone): stop the scan at the first such atom
        bool near = false;
        scan_ball(d, g, c, d.st.sep, sc[w], [&](int j) -> bool {
            const bool hit = j >= 0 && d.mol[j] != mi && !(sqrt(sq_seq(xi - atom_xyz(d, j))) >= d.st.sep);
            near |= hit;
            return hit;
        });
        near = __any_sync(0xffffffffu, near);
        if (lane == 0) d.atten[g] = near ? 5 : 1;
    }
}

void launch_attention(const Dev& d, cudaStream_t s)
{
    k_attention<<<grid_for(d.N, NB_WARPS), NB_WARPS * 32, 0, s>>>(d);
}

// ---------------------------------------------------------------------------
// neighbour / buried-partner lists
//   neighbour:  same molecule, j != i, d2 < ((ri + rj) + 2 rp)^2
//   buried:     other molecule, atten_j >= 5, same bridge test
//   coincident: same molecule, j != i, d2 <= 1e-4 (first pair reported)
// rows sorted by (d2, j) (neighbours) and by j (buried partners)
// ---------------------------------------------------------------------------
static constexpr int NB_CAP = 256;

// Warp bitonic sort of 32 * E (key, val) pairs into ascending (key, val)
// order; element i is held by lane i % 32 as its (i / 32)-th entry.  Strides
// under 32 exchange through shuffles, the others within a lane.  The vals of
// the real entries are distinct (atom ids or slots); padding is (~0, INT_MAX).
template <int E>
__device__ __forceinline__ void warp_bitonic(unsigned long long (&key)[E], int (&val)[E])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32 * E; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int pe = e ^ (j >> 5);
                    if (pe > e) {
                        const bool up = ((e * 32 + lane) & k) == 0;
                        const bool gt = key[e] > key[pe] || (key[e] == key[pe] && val[e] > val[pe]);
                        if (gt == up) {
                            const unsigned long long tk = key[e]; key[e] = key[pe]; key[pe] = tk;
                            const int tv = val[e]; val[e] = val[pe]; val[pe] = tv;
                        }
                    }
                }
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const unsigned long long ok = __shfl_xor_sync(0xffffffffu, key[e], j);
                    const int ov = __shfl_xor_sync(0xffffffffu, val[e], j);
                    const bool up = ((e * 32 + lane) & k) == 0;
                    const bool lower = (lane & j) == 0;
                    const bool other_less = ok < key[e] || (ok == key[e] && ov < val[e]);
                    if (lower == up ? other_less : !other_less) { key[e] = ok; val[e] = ov; }
                }
            }
        }
    }
}

// write row[i] = the val of rank i for the K (<= 32 * E) entries in sd2 / sid, ranked by (d2, id); d2 >= 0,
// so its bit pattern orders like the value
template <int E>
__device__ __forceinline__ void sort_row(const double* sd2, const int* sid, int K, int* row)
{
    const int lane = threadIdx.x & 31;
    unsigned long long key[E];
    int val[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = e * 32 + lane;
        key[e] = i < K ? (unsigned long long)__double_as_longlong(sd2[i]) : ~0ULL;
        val[e] = i < K ? sid[i] : 0x7fffffff;
    }
    warp_bitonic<E>(key, val);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = e * 32 + lane;
        if (i < K) row[i] = val[e];
    }
}

// every partner of atom g lies within ri + radmax + 2 rp
__device__ __forceinline__ double nb_range(const Dev& d, int c, double ri)
{
    return ri + fmax(d.cx[c].radmax, 0.0) + 2.0 * d.st.rp;
}

__device__ __forceinline__ void classify(const Dev& d, int g, V3 xi, double ri, int8_t mi, int j,
                                         bool& is_nb, bool& is_bur, bool& coin, double& d2)
{
    is_nb = is_bur = coin = false;
    d2 = 0;
    if (j < 0 || j == g) return;
    double4 aj = d.xyzr[j];
    d2 = sq_seq(xi - v3(aj.x, aj.y, aj.z));
    double rs = ri + aj.w;
    double t = rs + 2.0 * d.st.rp;
    double b2 = t * t;
    if (d.mol[j] == mi) {
        coin = d2 <= 0.0001;
        is_nb = d2 < b2;
    } else {
        is_bur = d.atten[j] >= 5 && d2 < b2;
    }
}

__global__ void __launch_bounds__(NB_WARPS * 32, 8) k_nb_count(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ BallScratch sc[NB_WARPS];
    __shared__ int sid[NB_WARPS][NB_CAP];
    __shared__ int sbid[NB_WARPS][NB_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const long long wid = blockIdx.x * (long long)NB_WARPS + w;
    const long long nw = (long long)gridDim.x * NB_WARPS;
    StashCursor ncur{0, 0};
    for (long long gg = wid; gg < d.N; gg += nw) {
        const int g = (int)gg;
        const int c = d.cplx[g];
        double4 ai = d.xyzr[g];
        const V3 xi = v3(ai.x, ai.y, ai.z);
        const int8_t mi = d.mol[g];
        int nn = 0, nb = 0;
        scan_ball(d, g, c, nb_range(d, c, ai.w), sc[w], [&](int j) {
            bool is_nb, is_bur, coin; double d2;
            classify(d, g, xi, ai.w, mi, j, is_nb, is_bur, coin, d2);
            const unsigned m = __ballot_sync(0xffffffffu, is_nb);
            if (is_nb && nn + __popc(m & lt) < NB_CAP) sid[w][nn + __popc(m & lt)] = j;
            nn += __popc(m);
            const unsigned mb = __ballot_sync(0xffffffffu, is_bur);
            if (is_bur && nb + __popc(mb & lt) < NB_CAP) sbid[w][nb + __popc(mb & lt)] = j;
            nb += __popc(mb);
            if (coin) {
                const int a0 = d.cx[c].a0;
                unsigned long long key = ((unsigned long long)(g - a0) << 32) | (unsigned)(j - a0);
                atomicMin(&d.coin[c], key);
            }
        });
        __syncwarp();
        // keep the rows (unsorted) for the emit pass
        long long so = -1;
        if (nn <= NB_CAP && nb <= NB_CAP && nn + nb > 0) {
            so = stash_take(d.nbs_top, d.nbs_cap, ncur, nn + nb);
            if (so >= 0) {
                for (int e = lane; e < nn; e += 32) d.nbs_buf[so + e] = sid[w][e];
                for (int e = lane; e < nb; e += 32) d.nbs_buf[so + nn + e] = sbid[w][e];
            }
        }
        if (lane == 0) {
            d.nnb[g] = nn;
            d.nbur[g] = nb;
            d.access[g] = nn == 0 ? 1 : 0;
            d.nb_soff[g] = so;
        }
        __syncwarp();
    }
}

void launch_neighbor_count(const Dev& d, cudaStream_t s)
{
    k_nb_count<<<grid_for(d.N, NB_WARPS), NB_WARPS * 32, 0, s>>>(d);
}

// one scan gathers both lists unsorted; neighbours are then placed by their
// (d2, j) rank and buried partners by their atom index
__global__ void __launch_bounds__(NB_WARPS * 32) k_nb_emit(Dev d, int* __restrict__ tmp_id)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ BallScratch sc[NB_WARPS];
    __shared__ double sd2[NB_WARPS][NB_CAP];
    __shared__ int sid[NB_WARPS][NB_CAP];
    __shared__ int sbid[NB_WARPS][NB_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const long long wid = blockIdx.x * (long long)NB_WARPS + w;
    const long long nw = (long long)gridDim.x * NB_WARPS;
    for (long long gg = wid; gg < d.N; gg += nw) {
        const int g = (int)gg;
        const int c = d.cplx[g];
        double4 ai = d.xyzr[g];
        const V3 xi = v3(ai.x, ai.y, ai.z);
        const int8_t mi = d.mol[g];
        const int K = d.nnb[g];
        const long long off = d.nb_off[g];
        const int KB = d.nbur[g];
        const long long boff = d.bu_off[g];
        if (off + K > d.nb_cap || boff + KB > d.bu_cap) {
            if (lane == 0) atomicOr(&d.status[c], ST_OVERFLOW);
            continue;
        }
        const bool in_sh = K <= NB_CAP, b_sh = KB <= NB_CAP;
        const long long so = d.nb_soff[g];
        if (so >= 0) {
            // the count pass's rows (both fit the shared arrays); d2 as classify computes it
            for (int e = lane; e < K; e += 32) {
                const int j = d.nbs_buf[so + e];
                const double4 aj = d.xyzr[j];
                sd2[w][e] = sq_seq(xi - v3(aj.x, aj.y, aj.z));
                sid[w][e] = j;
            }
            for (int e = lane; e < KB; e += 32) sbid[w][e] = d.nbs_buf[so + K + e];
        } else {
            int cnt = 0, bcnt = 0;
            scan_ball(d, g, c, nb_range(d, c, ai.w), sc[w], [&](int j) {
                bool is_nb, is_bur, coin; double d2;
                classify(d, g, xi, ai.w, mi, j, is_nb, is_bur, coin, d2);
                const unsigned m = __ballot_sync(0xffffffffu, is_nb);
                if (is_nb) {
                    const int pos = cnt + __popc(m & lt);
                    if (pos < K) {
                        if (in_sh) { sd2[w][pos] = d2; sid[w][pos] = j; }
                        else { d.nb_d2[off + pos] = d2; tmp_id[off + pos] = j; }
                    }
                }
                cnt += __popc(m);
                const unsigned mb = __ballot_sync(0xffffffffu, is_bur);
                if (is_bur) {
                    const int pos = bcnt + __popc(mb & lt);
                    if (pos < KB) {
                        if (b_sh) sbid[w][pos] = j;
                        else d.bu_id[boff + pos] = j;
                    }
                }
                bcnt += __popc(mb);
            });
        }
        __syncwarp();
        if (K <= 32) sort_row<1>(sd2[w], sid[w], K, d.nb_id + off);
        else if (K <= 64) sort_row<2>(sd2[w], sid[w], K, d.nb_id + off);
        else if (K <= 128) sort_row<4>(sd2[w], sid[w], K, d.nb_id + off);
        else for (int e = lane; e < K; e += 32) {
            const double ke = in_sh ? sd2[w][e] : d.nb_d2[off + e];
            const int je = in_sh ? sid[w][e] : tmp_id[off + e];
            int rank = 0;
            for (int f = 0; f < K; ++f) {
                const double kf = in_sh ? sd2[w][f] : d.nb_d2[off + f];
                const int jf = in_sh ? sid[w][f] : tmp_id[off + f];
                rank += (kf < ke || (kf == ke && jf < je)) ? 1 : 0;
            }
            d.nb_id[off + rank] = je;
        }
        if (b_sh) {
            for (int e = lane; e < KB; e += 32) {
                const int je = sbid[w][e];
                int rank = 0;
                for (int f = 0; f < KB; ++f) rank += sbid[w][f] < je ? 1 : 0;
                d.bu_id[boff + rank] = je;
            }
        } else if (lane == 0) {
            for (long long i = boff + 1; i < boff + KB; ++i) {
                int v = d.bu_id[i];
                long long k = i - 1;
                while (k >= boff && d.bu_id[k] > v) { d.bu_id[k + 1] = d.bu_id[k]; --k; }
                d.bu_id[k + 1] = v;
            }
        }
        __syncwarp();
    }
}

void launch_neighbor_emit(const Dev& d, cudaStream_t s)
{
    k_nb_emit<<<grid_for(d.N, NB_WARPS), NB_WARPS * 32, 0, s>>>(d, d.nb_tmp);
}

// ---------------------------------------------------------------------------
// pair geometry (second_loop, _core.py:1372-1416)
// ---------------------------------------------------------------------------
struct PairGeo {
    V3 uij, tij;
    double dij, rij;
    bool between, ok;
};

__device__ __forceinline__ PairGeo pair_geo(V3 xi, double ri, V3 xj, double rj, double rp)
{
    PairGeo p;
    V3 diff = xj - xi;
    double dij_sq = sq_alt(diff);
    p.dij = sqrt(dij_sq);
    double eri = ri + rp, erj = rj + rp;
    double asymm = (eri * eri - erj * erj) / p.dij;
    p.between = fabs(asymm) < p.dij;
    p.uij = diff / p.dij;
    p.tij = ((xi + xj) * 0.5) + p.uij * (asymm * 0.5);
    double far_sq = (eri + erj) * (eri + erj) - dij_sq;
    double rd = ri - rj;
    double cont_sq = dij_sq - rd * rd;
    p.ok = far_sq > 0.0 && cont_sq > 0.0;
    p.rij = ((0.5 * sqrt(far_sq)) * sqrt(cont_sq)) / p.dij;
    return p;
}

// ---------------------------------------------------------------------------
// pair loop: single-neighbour shortcut, toroid queue
// ---------------------------------------------------------------------------
template <bool EMIT>
__global__ void k_pairs(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const double rp = d.st.rp;
    for (long long gg = blockIdx.x * (long long)blockDim.x + threadIdx.x; gg < d.N; gg += (long long)gridDim.x * blockDim.x) {
        const int g = (int)gg;
        const int K = d.nnb[g];
        int ntor = 0;
        if (K > 0) {
            double4 ai = d.xyzr[g];
            const V3 xi = v3(ai.x, ai.y, ai.z);
            const long long off = d.nb_off[g];
            const int8_t ati = d.atten[g];
            if (K <= 1) {
                // shortcut: a single forward, well-formed neighbour marks both atoms
                // accessible and the atom contributes no pairs (_core.py:1393-1400)
                int j = d.nb_id[off];
                if (!EMIT && j > g) {
                    double4 aj = d.xyzr[j];
                    PairGeo p = pair_geo(xi, ai.w, v3(aj.x, aj.y, aj.z), aj.w, rp);
                    if (p.ok) { d.access[g] = 1; d.access[j] = 1; }
                }
            } else {
                const long long base = EMIT ? d.tor_off[g] : 0;
                for (int k = 0; k < K; ++k) {
                    int j = d.nb_id[off + k];
                    if (j <= g) continue;
                    double4 aj = d.xyzr[j];
                    PairGeo p = pair_geo(xi, ai.w, v3(aj.x, aj.y, aj.z), aj.w, rp);
                    if (!p.ok) continue;
                    bool need = ati > 1 || (d.atten[j] > 1 && rp > 0.0);
                    if (need) {
                        if (EMIT && base + ntor < d.tor_cap) { d.tor_i[base + ntor] = g; d.tor_j[base + ntor] = j; }
                        ++ntor;
                    }
                }
            }
        }
        if (!EMIT) d.ntor[g] = ntor;
    }
}

// each toroid's circle, one thread per toroid, for the toroidal count and emit passes
__global__ void k_tor_geo(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NT = min(d.tor_off[d.N], d.tor_cap);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < NT; q += (long long)gridDim.x * blockDim.x)
        tor_geo_store(d, q, tor_pair_of(d, d.tor_i[q], d.tor_j[q]));
}

void launch_pairs(const Dev& d, bool emit, cudaStream_t s)
{
    if (emit) {
        k_pairs<true><<<grid_for(d.N, 128), 128, 0, s>>>(d);
        k_tor_geo<<<grid_for(d.tor_cap, 128), 128, 0, s>>>(d);
    } else {
        k_pairs<false><<<grid_for(d.N, 128), 128, 0, s>>>(d);
    }
}

// ---------------------------------------------------------------------------
// triple loop: probe placement over (i, j, k) with j, k neighbours of i,
// natom_k > natom_j; probes ordered as all "+" then all "-" per complex
// ---------------------------------------------------------------------------
// probe collision against atom1's neighbours except atom2 and atom3 (alt, <=)
__device__ __forceinline__ bool probe_collides(const Dev& d, V3 pt, long long off, int K, int j, int k, double rp)
{
    for (int s = 0; s < K; ++s) {
        int n = d.nb_id[off + s];
        if (n == j || n == k) continue;
        double4 an = d.xyzr[n];
        double t = an.w + rp;
        if (sq_alt(pt - v3(an.x, an.y, an.z)) <= t * t) return true;
    }
    return false;
}

// Triple (i, j, k) validity of vec_third_loop (_core.py:1472-1494), cheapest
// tests first: k after j, not all three blockers, then the two distance tests.
struct TripleBase {
    bool valid;
    int k;
    V3 xk; double erk, dik;
};

__device__ __forceinline__ TripleBase triple_base(const Dev& d, V3 xi, double eri, int j, V3 xj, double erj,
                                                  int8_t ati, int8_t atj, int k)
{
    TripleBase t;
    t.valid = false;
    t.k = k;
    if (k <= j) return t;
    if (ati <= 1 && atj <= 1 && d.atten[k] <= 1) return t;
    double4 ak = d.xyzr[k];
    t.xk = v3(ak.x, ak.y, ak.z);
    t.erk = ak.w + d.st.rp;
    double djk = norm3(t.xk - xj);
    if (!(djk < erj + t.erk)) return t;
    t.dik = norm3(t.xk - xi);
    if (!(t.dik < eri + t.erk)) return t;
    t.valid = true;
    return t;
}

static constexpr int TR_WARPS = 2;
static constexpr int TR_QCAP = 256;   // queued (pair slot, k slot) triples per warp
static constexpr int TR_HEAD = 8;     // row slots each lane tests for its own probes before the shared scan

__device__ __forceinline__ void stash_one(const Dev& d, long long e, int a0, int a1, int a2, double h, V3 pt, V3 alt,
                                          int g, unsigned ord)
{
    d.sp_a[3 * e] = a0; d.sp_a[3 * e + 1] = a1; d.sp_a[3 * e + 2] = a2;
    d.sp_h[e] = h;
    st3(d.sp_xyz + 3 * e, pt);
    st3(d.sp_alt + 3 * e, alt);
    d.sp_g[e] = g;
    d.sp_ord[e] = ord;
}

// Count pass: the chunk's probes go to the stash (one reservation per chunk)
// with their final slot, so the probe arrays are filled by a scatter instead
// of a second pass over the triples.  The fields are the emit pass's.
__device__ __forceinline__ void probe_stash(const Dev& d, int g, int j, int k, double h, V3 pp, V3 pm, V3 up,
                                            bool okp, bool okm, unsigned bp, unsigned bm, int nplus, int nminus)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int np = __popc(bp), nm = __popc(bm);
    if (np + nm == 0) return;                     // warp-uniform
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(d.ptop, (unsigned long long)(np + nm));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (okp) {
        const long long e = (long long)base + __popc(bp & lt);
        if (e < d.probe_cap) stash_one(d, e, g, j, k, h, pp, up * 1.0, g, (unsigned)(nplus + __popc(bp & lt)));
    }
    if (okm) {
        const long long e = (long long)base + np + __popc(bm & lt);
        if (e < d.probe_cap)
            stash_one(d, e, j, g, k, h, pm, up * -1.0, g, 0x80000000u | (unsigned)(nminus + __popc(bm & lt)));
    }
}

// first "+" and "-" probe slot of atom g: per complex [+mol0 | -mol0 | +mol1 | -mol1]
__device__ __forceinline__ void probe_bases(const Dev& d, int g, long long& pbase, long long& mbase)
{
    const int c = d.cplx[g];
    const Cplx C = d.cx[c];
    const int s0 = C.a0, s1 = C.a0 + C.n0, e1 = C.a0 + C.n;
    const int ms = d.mol[g] == 0 ? s0 : s1, me = d.mol[g] == 0 ? s1 : e1;
    const long long cbase = d.plus_off[s0] + d.minus_off[s0];
    const long long m0 = (d.plus_off[s1] - d.plus_off[s0]) + (d.minus_off[s1] - d.minus_off[s0]);
    const long long mb = cbase + (d.mol[g] == 0 ? 0 : m0);
    pbase = mb + (d.plus_off[g] - d.plus_off[ms]);
    mbase = mb + (d.plus_off[me] - d.plus_off[ms]) + (d.minus_off[g] - d.minus_off[ms]);
}

__global__ void k_probe_scatter(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long n = min((long long)*d.ptop, d.probe_cap);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int g = d.sp_g[e];
        const unsigned o = d.sp_ord[e];
        long long pbase, mbase;
        probe_bases(d, g, pbase, mbase);
        const long long q = ((o >> 31) ? mbase : pbase) + (long long)(o & 0x7fffffffu);
        const int a0 = d.sp_a[3 * e], a1 = d.sp_a[3 * e + 1], a2 = d.sp_a[3 * e + 2];
        if (q < d.probe_cap) {
            d.pa0[q] = a0; d.pa1[q] = a1; d.pa2[q] = a2;
            d.ph[q] = d.sp_h[e];
            st3(d.pxyz + 3 * q, ld3(d.sp_xyz + 3 * e));
            st3(d.palt + 3 * q, ld3(d.sp_alt + 3 * e));
        }
        d.access[a0] = 1; d.access[a1] = 1; d.access[a2] = 1;
    }
}

void launch_probe_scatter(const Dev& d, long long probe_grid, cudaStream_t s)
{
    k_probe_scatter<<<grid_for(probe_grid, 256), 256, 0, s>>>(d);
}

// probes of the queued triples, in queue order: "+" and "-" probes are
// ballot-ordered into the atom's two probe ranges
template <bool EMIT>
__device__ __forceinline__ void triples_flush(const Dev& d, int g, V3 xi, double ri, double eri, long long off,
                                              int K, const unsigned* queue, int qn, int& nplus, int& nminus,
                                              long long pbase, long long mbase)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const double rp = d.st.rp;
    for (int e0 = 0; e0 < qn; e0 += 32) {
        const int e = e0 + lane;
        bool okp = false, okm = false;
        V3 pp, pm, up;
        double h = 0.0;
        int j = -1, k = -1;
        if (e < qn) {
            const unsigned ent = queue[e];
            j = d.nb_id[off + (ent >> 16)];
            k = d.nb_id[off + (ent & 0xffffu)];
            const double4 aj = d.xyzr[j], ak = d.xyzr[k];
            const V3 xj = v3(aj.x, aj.y, aj.z), xk = v3(ak.x, ak.y, ak.z);
            const PairGeo p = pair_geo(xi, ri, xj, aj.w, rp);
            const double erk = ak.w + rp;
            const double dik = norm3(xk - xi);
            const V3 uik = (xk - xi) / dik;
            const double dt = dot_alt(p.uij, uik);
            const double wijk = acos(dt < -1.0 ? -1.0 : (dt > 1.0 ? 1.0 : dt));   // np.clip keeps NaN
            const double swijk = sin(wijk);
            if (!((dt >= 1.0) || (dt <= -1.0) || (wijk <= 0.0) || (swijk <= 0.0))) {
                const V3 uijk = cross3(p.uij, uik) / swijk;
                const V3 utb = cross3(uijk, p.uij);
                const double asymm = (eri * eri - erk * erk) / dik;
                const V3 tik = (xi + xk) * 0.5 + uik * (asymm * 0.5);
                const double dtb = dot_alt(uik, tik - p.tij);
                const V3 bijk = p.tij + utb * (dtb / swijk);
                const V3 bma = bijk - xi;
                const double h2 = eri * eri - dot_alt(bma, bma);
                if (h2 > 0.0) {
                    h = sqrt(h2);
                    up = uijk;
                    pp = bijk + uijk * (h * 1.0);
                    pm = bijk + uijk * (h * -1.0);
                    okp = !probe_collides(d, pp, off, K, j, k, rp);
                    okm = !probe_collides(d, pm, off, K, j, k, rp);
                }
            }
        }
        const unsigned bp = __ballot_sync(0xffffffffu, okp);
        const unsigned bm = __ballot_sync(0xffffffffu, okm);
        if (!EMIT) probe_stash(d, g, j, k, h, pp, pm, up, okp, okm, bp, bm, nplus, nminus);
        if (EMIT) {
            if (okp) {
                long long q = pbase + nplus + __popc(bp & lt);
                if (q < d.probe_cap) {
                    d.pa0[q] = g; d.pa1[q] = j; d.pa2[q] = k;
                    d.ph[q] = h; st3(d.pxyz + 3 * q, pp); st3(d.palt + 3 * q, up * 1.0);
                }
            }
            if (okm) {
                long long q = mbase + nminus + __popc(bm & lt);
                if (q < d.probe_cap) {
                    d.pa0[q] = j; d.pa1[q] = g; d.pa2[q] = k;
                    d.ph[q] = h; st3(d.pxyz + 3 * q, pm); st3(d.palt + 3 * q, up * -1.0);
                }
            }
            if (okp || okm) { d.access[g] = 1; d.access[j] = 1; d.access[k] = 1; }
        }
        nplus += __popc(bp);
        nminus += __popc(bm);
    }
}

// Rows of up to KC neighbours run from shared memory: the row's
// coordinates and radii, and per neighbour k the distance dik = |xk - xi| and
// unit vector uik = (xk - xi) / dik, which every pair (i, j) of the row
// reuses.  Queued pairs keep their geometry for the probe pass.
// The row cache holds KC = 128 or 64 neighbours: the smaller cache halves the
// shared memory of a warp, so more warps fit an SM (registers capped to match;
// longer rows take the LONG kernel), picked per batch shape by the autotuner.
static constexpr int TR_PC = 32;      // neighbour slots (pairs) per chunk of the candidate matrix

template <int KC>
struct TrRow {
    double x[KC], y[KC], z[KC], r[KC];
    double ux[KC], uy[KC], uz[KC], dk[KC];
    int id[KC];
    int8_t at[KC];
    unsigned char rk[KC];    // rank of the slot's atom id in the row
    unsigned char ord[KC];   // slot of each id rank
};

struct TrPairC { V3 uij, tij; double rij; int ps; };

// one chunk's pairs (i, j) and their (pair, k) candidate matrix
template <int KC>
struct TrWork {
    TrPairC pr[TR_PC];
    unsigned cb[TR_PC][KC / 32];      // candidate k slots of each pair
    int cpos[TR_PC];                  // first (pair, k) combination of each pair
    unsigned kill;                    // pairs killed by a degenerate triple
};

// norm3(v) < T, skipping the square root when the squared comparison settles
// it: with a 1e-12 relative margin on T^2 the rounded root lies on the same side
__device__ __forceinline__ bool norm_lt(V3 v, double T)
{
    const double s = dot_seq(v, v);
    const double T2 = T * T;
    if (s < T2 * (1.0 - 1e-12)) return true;
    if (s > T2 * (1.0 + 1e-12)) return false;
    return sqrt(s) < T;
}

// triple_base on the cached row: k after j, not all three blockers, the two distance tests
template <int KC>
__device__ __forceinline__ bool triple_ok_c(const TrRow<KC>& R, int ks, int j, V3 xj, double erj, double eri,
                                            int8_t ati, int8_t atj, double rp)
{
    if (R.id[ks] <= j) return false;
    if (ati <= 1 && atj <= 1 && R.at[ks] <= 1) return false;
    const double erk = R.r[ks] + rp;
    if (!norm_lt(v3(R.x[ks], R.y[ks], R.z[ks]) - xj, erj + erk)) return false;
    return R.dk[ks] < eri + erk;
}

template <int KC>
__device__ __forceinline__ bool probe_collides_c(const TrRow<KC>& R, int K, V3 pt, int j, int k, double rp)
{
    for (int s = 0; s < K; ++s) {
        const int n = R.id[s];
        if (n == j || n == k) continue;
        const double t = R.r[s] + rp;
        if (sq_alt(pt - v3(R.x[s], R.y[s], R.z[s])) <= t * t) return true;
    }
    return false;
}

// probe_collides_c for the triple's two probes in one pass over the row (each neighbour read once); the
// loop ends when both have collided
template <int KC>
__device__ __forceinline__ void probe_pair_collides_c(const TrRow<KC>& R, int K, V3 pp, V3 pm, int j, int k, double rp,
                                                      bool& cp, bool& cm)
{
    cp = cm = false;
    for (int s = 0; s < K; ++s) {
        const int n = R.id[s];
        if (n == j || n == k) continue;
        const double t = R.r[s] + rp;
        const double t2 = t * t;
        const V3 x = v3(R.x[s], R.y[s], R.z[s]);
        cp = cp || sq_alt(pp - x) <= t2;
        cm = cm || sq_alt(pm - x) <= t2;
        if (cp && cm) return;
    }
}

template <bool EMIT, int KC>
__device__ __forceinline__ void triples_flush_c(const Dev& d, int g, V3 xi, double eri, const TrRow<KC>& R, int K,
                                                const unsigned* queue, const TrPairC* pq, int qn, int& nplus,
                                                int& nminus, long long pbase, long long mbase)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const double rp = d.st.rp;
    for (int e0 = 0; e0 < qn; e0 += 32) {
        const int e = e0 + lane;
        bool okp = false, okm = false, live = false, cp = false, cm = false;
        V3 pp = v3(0.0, 0.0, 0.0), pm = pp, up;
        double h = 0.0;
        int j = -1, k = -1;
        if (e < qn) {
            const unsigned ent = queue[e];
            const TrPairC& P = pq[ent >> 16];
            const int ks = (int)(ent & 0xffffu);
            j = R.id[P.ps];
            k = R.id[ks];
            const V3 xk = v3(R.x[ks], R.y[ks], R.z[ks]);
            const double erk = R.r[ks] + rp;
            const double dik = R.dk[ks];
            const V3 uik = v3(R.ux[ks], R.uy[ks], R.uz[ks]);
            const double dt = dot_alt(P.uij, uik);
            const double wijk = acos(dt < -1.0 ? -1.0 : (dt > 1.0 ? 1.0 : dt));   // np.clip keeps NaN
            const double swijk = sin(wijk);
            if (!((dt >= 1.0) || (dt <= -1.0) || (wijk <= 0.0) || (swijk <= 0.0))) {
                const V3 uijk = cross3(P.uij, uik) / swijk;
                const V3 utb = cross3(uijk, P.uij);
                const double asymm = (eri * eri - erk * erk) / dik;
                const V3 tik = (xi + xk) * 0.5 + uik * (asymm * 0.5);
                const double dtb = dot_alt(uik, tik - P.tij);
                const V3 bijk = P.tij + utb * (dtb / swijk);
                const V3 bma = bijk - xi;
                const double h2 = eri * eri - dot_alt(bma, bma);
                if (h2 > 0.0) {
                    h = sqrt(h2);
                    up = uijk;
                    pp = bijk + uijk * (h * 1.0);
                    pm = bijk + uijk * (h * -1.0);
                    live = true;
                    probe_pair_collides_c(R, K < TR_HEAD ? K : TR_HEAD, pp, pm, j, k, rp, cp, cm);
                }
            }
        }
        // The rest of the row for the probes still open, one triple at a time with the row over the lanes:
        // most probes collide with one of the nearest neighbours (the row is in distance order), so a lane
        // that must scan the whole row would otherwise hold up the warp alone.
        unsigned open = __ballot_sync(0xffffffffu, live && !(cp && cm));
        while (open) {
            const int src = __ffs(open) - 1;
            open &= open - 1;
            const V3 qp = v3(__shfl_sync(0xffffffffu, pp.x, src), __shfl_sync(0xffffffffu, pp.y, src),
                             __shfl_sync(0xffffffffu, pp.z, src));
            const V3 qm = v3(__shfl_sync(0xffffffffu, pm.x, src), __shfl_sync(0xffffffffu, pm.y, src),
                             __shfl_sync(0xffffffffu, pm.z, src));
            const int qj = __shfl_sync(0xffffffffu, j, src), qk = __shfl_sync(0xffffffffu, k, src);
            bool hp = __shfl_sync(0xffffffffu, cp, src), hm = __shfl_sync(0xffffffffu, cm, src);
            for (int s0 = TR_HEAD; s0 < K && !(hp && hm); s0 += 32) {
                const int sl = s0 + lane;
                bool ap = false, am = false;
                if (sl < K) {
                    const int n = R.id[sl];
                    if (n != qj && n != qk) {
                        const double t = R.r[sl] + rp;
                        const double t2 = t * t;
                        const V3 x = v3(R.x[sl], R.y[sl], R.z[sl]);
                        ap = sq_alt(qp - x) <= t2;
                        am = sq_alt(qm - x) <= t2;
                    }
                }
                hp = __any_sync(0xffffffffu, ap) || hp;
                hm = __any_sync(0xffffffffu, am) || hm;
            }
            if (lane == src) { cp = hp; cm = hm; }
        }
        okp = live && !cp;
        okm = live && !cm;
        const unsigned bp = __ballot_sync(0xffffffffu, okp);
        const unsigned bm = __ballot_sync(0xffffffffu, okm);
        if (!EMIT) probe_stash(d, g, j, k, h, pp, pm, up, okp, okm, bp, bm, nplus, nminus);
        if (EMIT) {
            if (okp) {
                long long q = pbase + nplus + __popc(bp & lt);
                if (q < d.probe_cap) {
                    d.pa0[q] = g; d.pa1[q] = j; d.pa2[q] = k;
                    d.ph[q] = h; st3(d.pxyz + 3 * q, pp); st3(d.palt + 3 * q, up * 1.0);
                }
            }
            if (okm) {
                long long q = mbase + nminus + __popc(bm & lt);
                if (q < d.probe_cap) {
                    d.pa0[q] = j; d.pa1[q] = g; d.pa2[q] = k;
                    d.ph[q] = h; st3(d.pxyz + 3 * q, pm); st3(d.palt + 3 * q, up * -1.0);
                }
            }
            if (okp || okm) { d.access[g] = 1; d.access[j] = 1; d.access[k] = 1; }
        }
        nplus += __popc(bp);
        nminus += __popc(bm);
    }
}

// The triple loop of one atom whose row fits the cache (K <= KC).  The
// row's pairs (i, j) are taken 32 neighbour slots at a time: their geometry
// one pair per lane, then the (pair, k) combinations with k after j (by atom
// id) spread over the lanes, then the queue in (pair, k slot) order -- the
// order of the reference's loops -- one pair per lane, for the probe pass.
template <bool EMIT, int KC>
__device__ __forceinline__ void triples_row_c(const Dev& d, int g, int K, long long off, V3 xi, double ri, double eri,
                                              int8_t ati, TrRow<KC>& R, unsigned* queue, TrWork<KC>& W, int& nplus,
                                              int& nminus, long long pbase, long long mbase)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const double rp = d.st.rp;
    for (int s = lane; s < K; s += 32) {
        const int id = d.nb_id[off + s];
        const double4 a = d.xyzr[id];
        R.x[s] = a.x; R.y[s] = a.y; R.z[s] = a.z; R.r[s] = a.w;
        R.id[s] = id;
        R.at[s] = d.atten[id];
        const V3 v = v3(a.x, a.y, a.z) - xi;
        const double dk = norm3(v);
        const V3 u = v / dk;
        R.dk[s] = dk; R.ux[s] = u.x; R.uy[s] = u.y; R.uz[s] = u.z;
    }
    __syncwarp();
    for (int s = lane; s < K; s += 32) {      // atom ids of a row are distinct
        const int id = R.id[s];
        int r = 0;
        for (int f = 0; f < K; ++f) r += R.id[f] < id ? 1 : 0;
        R.rk[s] = (unsigned char)r;
        R.ord[r] = (unsigned char)s;
    }
    __syncwarp();
    for (int ps0 = 0; ps0 < K; ps0 += TR_PC) {
        // pairs (i, j) of the chunk: j after i and the pair geometry ok
        const int ps = ps0 + lane;
        bool v = false;
        PairGeo p;
        if (ps < K && R.id[ps] > g) {
            p = pair_geo(xi, ri, v3(R.x[ps], R.y[ps], R.z[ps]), R.r[ps], rp);
            v = p.ok;
        }
        const unsigned vm = __ballot_sync(0xffffffffu, v);
        const int np = __popc(vm);
        if (np == 0) continue;
        // combinations of each pair: the slots whose atom id is above j's
        int nk = 0;
        if (v) {
            const int pi = __popc(vm & lt);
            W.pr[pi] = TrPairC{p.uij, p.tij, p.rij, ps};
            nk = K - 1 - (int)R.rk[ps];
        }
        int x = nk;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const int NC = __shfl_sync(0xffffffffu, x, 31);
        if (v) W.cpos[__popc(vm & lt)] = x - nk;
        for (int t = lane; t < np * (KC / 32); t += 32) W.cb[t / (KC / 32)][t % (KC / 32)] = 0u;
        if (lane == 0) W.kill = 0u;
        __syncwarp();
        // candidate matrix: a degenerate triple (|uij.uik| >= 1) inside the
        // torus kills its pair (_core.py:1524-1543)
        for (int c = lane; c < NC; c += 32) {
            int lo = 0, hi = np - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (W.cpos[mid] <= c) lo = mid; else hi = mid - 1;
            }
            const int pi = lo;
            const TrPairC& P = W.pr[pi];
            const int pj = P.ps;
            const int ks = R.ord[(int)R.rk[pj] + 1 + (c - W.cpos[pi])];
            if (!triple_ok_c(R, ks, R.id[pj], v3(R.x[pj], R.y[pj], R.z[pj]), R.r[pj] + rp, eri, ati, R.at[pj], rp))
                continue;
            const double dt = dot_alt(P.uij, v3(R.ux[ks], R.uy[ks], R.uz[ks]));
            if (dt >= 1.0 || dt <= -1.0) {
                const double erk = R.r[ks] + rp;
                const double dtijk2 = sq_seq(P.tij - v3(R.x[ks], R.y[ks], R.z[ks]));
                const double rkp2 = erk * erk - P.rij * P.rij;
                if (dtijk2 < rkp2) atomicOr(&W.kill, 1u << pi);
            } else {
                atomicOr(&W.cb[pi][ks >> 5], 1u << (ks & 31));
            }
        }
        __syncwarp();
        // queue, one pair per lane: candidates of the live pairs in (pair, k
        // slot) order, flushed whenever the next pair would overflow the queue
        int nq = 0;
        if (lane < np && !((W.kill >> lane) & 1u))
            for (int r = 0; r * 32 < K; ++r) nq += __popc(W.cb[lane][r]);
        int qx = nq;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, qx, o);
            if (lane >= o) qx += y;
        }
        const int qtot = __shfl_sync(0xffffffffu, qx, 31);
        const int qpos = qx - nq;                 // this pair's first entry in the chunk
        int base = 0;                             // entries of earlier pairs already flushed
        while (base < qtot) {
            // the pairs that fit: every entry in [base, base + TR_QCAP)
            const bool take = nq > 0 && qpos >= base && qpos + nq <= base + TR_QCAP;
            const unsigned tm = __ballot_sync(0xffffffffu, take);
            if (tm == 0u) break;                  // cannot happen: the first pending pair always fits
            const int last = 31 - __clz(tm);
            const int end = __shfl_sync(0xffffffffu, qpos + nq, last);
            if (take) {
                int t = qpos - base;
                for (int r = 0; r * 32 < K; ++r) {
                    unsigned m = W.cb[lane][r];
                    while (m) {
                        const int b = __ffs(m) - 1;
                        m &= m - 1;
                        queue[t++] = ((unsigned)lane << 16) | (unsigned)(r * 32 + b);
                    }
                }
            }
            __syncwarp();
            triples_flush_c<EMIT, KC>(d, g, xi, eri, R, K, queue, W.pr, end - base, nplus, nminus, pbase, mbase);
            __syncwarp();
            base = end;
        }
    }
}

// LONG = false: atoms whose neighbour row fits the cache (KC); true: the others
template <bool EMIT, bool LONG, int KC, int MINB>
__global__ void __launch_bounds__(TR_WARPS * 32, MINB) k_triples(Dev d)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ unsigned queue_s[TR_WARPS][TR_QCAP];
    __shared__ TrRow<KC> rows_s[LONG ? 1 : TR_WARPS];
    __shared__ TrWork<KC> work_s[LONG ? 1 : TR_WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    unsigned* queue = queue_s[w];
    const long long wid = blockIdx.x * (long long)TR_WARPS + w;
    const long long nw = (long long)gridDim.x * TR_WARPS;
    const double rp = d.st.rp;
    for (long long gg = wid; gg < d.N; gg += nw) {
        const int g = (int)gg;
        const int K = d.nnb[g];
        if (LONG != (K > KC)) continue;
        if (EMIT && d.nplus[g] == 0 && d.nminus[g] == 0) continue;    // no probes: nothing to write
        int nplus = 0, nminus = 0;
        const int8_t ati = d.atten[g];
        const long long off = d.nb_off[g];
        bool any_open = ati > 1;
        if (K > 1 && !any_open) {
            // every triple of an all-blocker neighbourhood is skipped (_core.py:1486-1494)
            for (int kb = 0; kb < K && !any_open; kb += 32) {
                const int ks = kb + lane;
                any_open = __any_sync(0xffffffffu, ks < K && d.atten[d.nb_id[off + ks]] > 1);
            }
        }
        if (K > 1 && any_open && K <= 0xffff) {
            const double4 ai = d.xyzr[g];
            const V3 xi = v3(ai.x, ai.y, ai.z);
            const double eri = ai.w + rp;
            long long pbase = 0, mbase = 0;
            if (EMIT) {
                // probe layout per complex: [+mol0 | -mol0 | +mol1 | -mol1]
                probe_bases(d, g, pbase, mbase);
            }
            if (!LONG) {
                triples_row_c<EMIT, KC>(d, g, K, off, xi, ai.w, eri, ati, rows_s[w], queue, work_s[w], nplus, nminus,
                                        pbase, mbase);
                if (!EMIT && lane == 0) { d.nplus[g] = nplus; d.nminus[g] = nminus; }
                continue;
            }
            int qn = 0;
            for (int ps = 0; ps < K; ++ps) {
                const int j = d.nb_id[off + ps];
                if (j <= g) continue;
                const double4 aj = d.xyzr[j];
                const V3 xj = v3(aj.x, aj.y, aj.z);
                const PairGeo p = pair_geo(xi, ai.w, xj, aj.w, rp);
                if (!p.ok) continue;
                const double erj = aj.w + rp;
                const int8_t atj = d.atten[j];
                // a degenerate triple (|uij.uik| >= 1) inside the torus kills the whole pair
                // (_core.py:1524-1543); the others are queued in (pair, k) order
                bool kill = false;
                int nq = 0;
                unsigned cand[4];
                for (int kb = 0, r = 0; kb < K; kb += 32, ++r) {
                    const int ks = kb + lane;
                    bool c = false;
                    if (ks < K) {
                        const TripleBase t = triple_base(d, xi, eri, j, xj, erj, ati, atj, d.nb_id[off + ks]);
                        if (t.valid) {
                            const V3 uik = (t.xk - xi) / t.dik;
                            const double dt = dot_alt(p.uij, uik);
                            if (dt >= 1.0 || dt <= -1.0) {
                                const double dtijk2 = sq_seq(p.tij - t.xk);
                                const double rkp2 = t.erk * t.erk - p.rij * p.rij;
                                kill |= dtijk2 < rkp2;
                            } else {
                                c = true;
                            }
                        }
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, c);
                    if (r < 4) cand[r] = m;
                    nq += __popc(m);
                }
                if (__any_sync(0xffffffffu, kill)) continue;
                if (nq == 0) continue;
                if (qn + nq > TR_QCAP) {
                    __syncwarp();
                    triples_flush<EMIT>(d, g, xi, ai.w, eri, off, K, queue, qn, nplus, nminus, pbase, mbase);
                    __syncwarp();
                    qn = 0;
                }
                if (K <= 128 && nq <= TR_QCAP) {
                    for (int r = 0; r * 32 < K; ++r) {
                        const unsigned m = cand[r];
                        if ((m >> lane) & 1u) queue[qn + __popc(m & lt)] = ((unsigned)ps << 16) | (unsigned)(r * 32 + lane);
                        qn += __popc(m);
                    }
                } else {
                    // long rows: recompute candidacy chunk by chunk, flushing as the queue fills
                    for (int kb = 0; kb < K; kb += 32) {
                        const int ks = kb + lane;
                        bool c = false;
                        if (ks < K) {
                            const TripleBase t = triple_base(d, xi, eri, j, xj, erj, ati, atj, d.nb_id[off + ks]);
                            if (t.valid) {
                                const double dt = dot_alt(p.uij, (t.xk - xi) / t.dik);
                                c = !(dt >= 1.0 || dt <= -1.0);
                            }
                        }
                        const unsigned m = __ballot_sync(0xffffffffu, c);
                        if (qn + 32 > TR_QCAP) {
                            __syncwarp();
                            triples_flush<EMIT>(d, g, xi, ai.w, eri, off, K, queue, qn, nplus, nminus, pbase, mbase);
                            __syncwarp();
                            qn = 0;
                        }
                        if (c) queue[qn + __popc(m & lt)] = ((unsigned)ps << 16) | (unsigned)ks;
                        qn += __popc(m);
                    }
                }
                __syncwarp();
            }
            if (qn > 0) {
                __syncwarp();
                triples_flush<EMIT>(d, g, xi, ai.w, eri, off, K, queue, qn, nplus, nminus, pbase, mbase);
                __syncwarp();
            }
        }
        if (!EMIT && lane == 0) { d.nplus[g] = nplus; d.nminus[g] = nminus; }
    }
}

void launch_triples(const Dev& d, bool emit, int variant, cudaStream_t s)
{
    const unsigned g = grid_for(d.N, TR_WARPS, 32);
    if (variant == 0) {
        if (emit) {
            k_triples<true, false, 128, 8><<<g, TR_WARPS * 32, 0, s>>>(d);
            k_triples<true, true, 128, 8><<<g, TR_WARPS * 32, 0, s>>>(d);
        } else {
            k_triples<false, false, 128, 7><<<g, TR_WARPS * 32, 0, s>>>(d);
            k_triples<false, true, 128, 7><<<g, TR_WARPS * 32, 0, s>>>(d);
        }
    } else if (variant == 1) {
        if (emit) {
            k_triples<true, false, 64, 10><<<g, TR_WARPS * 32, 0, s>>>(d);
            k_triples<true, true, 64, 10><<<g, TR_WARPS * 32, 0, s>>>(d);
        } else {
            k_triples<false, false, 64, 10><<<g, TR_WARPS * 32, 0, s>>>(d);
            k_triples<false, true, 64, 10><<<g, TR_WARPS * 32, 0, s>>>(d);
        }
    } else {
        if (emit) {
            k_triples<true, false, 64, 12><<<g, TR_WARPS * 32, 0, s>>>(d);
            k_triples<true, true, 64, 12><<<g, TR_WARPS * 32, 0, s>>>(d);
        } else {
            k_triples<false, false, 64, 12><<<g, TR_WARPS * 32, 0, s>>>(d);
            k_triples<false, true, 64, 12><<<g, TR_WARPS * 32, 0, s>>>(d);
        }
    }
}

// ---------------------------------------------------------------------------
// low probes (height < rp): flag, scan, compact -- per complex contiguous
// ---------------------------------------------------------------------------
__global__ void k_low_flag(Dev d, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long P = d.plus_off[d.N] + d.minus_off[d.N];
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < cap; p += (long long)gridDim.x * blockDim.x)
        d.plow_flag[p] = (p < P && d.ph[p] < d.st.rp) ? 1 : 0;
}

__global__ void k_low_fill(Dev d, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long P = d.plus_off[d.N] + d.minus_off[d.N];
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < cap && p < P; p += (long long)gridDim.x * blockDim.x)
        if (d.plow_flag[p]) d.plow_list[d.plow_off[p]] = (int)p;
}

// Low probes of the complexes with more than CMS_LOW_CELL_MIN of them, sorted
// by cell of the complex's atom grid, coordinates clamped to the grid (probes
// can lie just outside the atoms' box; clamping is monotone, so a search over
// the clamped cell range of a ball still meets every low probe inside the
// ball).  The concave kernels look up such a complex's nearby low probes there
// instead of scanning all of its low probes (a cost quadratic in their number:
// whole-molecule surfaces); the others keep the plain scan.
__device__ __forceinline__ long long complex_low_count(const Dev& d, int c)
{
    const Cplx& C = d.cx[c];
    const int s0 = C.a0, e1 = C.a0 + C.n;
    const long long pb = min(d.plus_off[s0] + d.minus_off[s0], d.probe_cap);
    const long long pe = min(d.plus_off[e1] + d.minus_off[e1], d.probe_cap);
    return d.plow_off[pe] - d.plow_off[pb];
}

__global__ void k_low_cell_count(Dev d, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NL = d.plow_off[cap];
    for (long long li = blockIdx.x * (long long)blockDim.x + threadIdx.x; li < NL; li += (long long)gridDim.x * blockDim.x) {
        const int p = d.plow_list[li];
        const int c = d.cplx[d.pa0[p]];
        if (complex_low_count(d, c) <= CMS_LOW_CELL_MIN) { d.plc_cell[li] = -1; continue; }
        const Cplx& C = d.cx[c];
        const double* x = d.pxyz + 3LL * p;
        const int cx = cell_coord(x[0], C.org[0], C.h, C.dims[0]);
        const int cy = cell_coord(x[1], C.org[1], C.h, C.dims[1]);
        const int cz = cell_coord(x[2], C.org[2], C.h, C.dims[2]);
        long long cell = d.ncell_scan[c] + ((long long)cx * C.dims[1] + cy) * C.dims[2] + cz;
        if (cell >= d.cells_cap) { atomicOr(&d.status[c], ST_OVERFLOW); cell = -1; }
        d.plc_cell[li] = (int)cell;
        if (cell >= 0) atomicAdd(&d.plc_cnt[cell], 1);
    }
}

__global__ void k_low_cell_fill(Dev d, long long cap)
{
    CMS_EXIT_ON_OVERFLOW(d);
    const long long NL = d.plow_off[cap];
    for (long long li = blockIdx.x * (long long)blockDim.x + threadIdx.x; li < NL; li += (long long)gridDim.x * blockDim.x) {
        const int cell = d.plc_cell[li];
        if (cell < 0) continue;
        const int pos = atomicAdd(&d.plc_fill[cell], 1);
        d.plc_item[d.plc_start[cell] + pos] = d.plow_list[li];
    }
}

void launch_low_probes(const Dev& d, long long probe_cap, long long* scan_tmp, cudaStream_t s)
{
    k_low_flag<<<grid_for(probe_cap, 256), 256, 0, s>>>(d, probe_cap);
    scan_counts(d.plow_flag, d.plow_off, probe_cap, scan_tmp, s);
    k_low_fill<<<grid_for(probe_cap, 256), 256, 0, s>>>(d, probe_cap);
    k_zero_int<<<grid_for(d.cells_cap, 256), 256, 0, s>>>(d.plc_cnt, d.cells_cap);
    k_zero_int<<<grid_for(d.cells_cap, 256), 256, 0, s>>>(d.plc_fill, d.cells_cap);
    k_low_cell_count<<<grid_for(probe_cap, 256), 256, 0, s>>>(d, probe_cap);
    scan_counts(d.plc_cnt, d.plc_start, d.cells_cap, scan_tmp, s);
    k_low_cell_fill<<<grid_for(probe_cap, 256), 256, 0, s>>>(d, probe_cap);
}

}  // namespace cms
