// Internal data layout of a batch on the device, shared by all kernels.
//
// A batch holds B independent complexes.  Atoms of complex c occupy global
// indices [atom_off[c], atom_off[c+1]): binder (molecule 0) first, then
// target (molecule 1) -- the reference's natom numbering (_core.py:372-399)
// shifted by atom_off[c].  Every other per-complex array (neighbour rows,
// toroid pairs, probes, dots) is laid out complex by complex in the same way,
// so a complex is always a contiguous range and per-complex totals are
// differences of exclusive scans.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "cms_math.cuh"

namespace cms {

struct Settings {
    double rp, density, band, sep, weight, bw_dist, bw_norm;
};

// per-complex geometry and bookkeeping, filled by k_complex_setup
struct Cplx {
    int a0, n0, n;              // first global atom, binder atoms, all atoms
    int dims[3];                // cell grid dimensions
    double org[3], h;           // grid origin and cell edge
    double ctr[3], R;           // centre and half-extent bounding every dot
    double radmax;
    long long cell0;            // first global cell
    double mlo[2][3], mhi[2][3];  // bounding box of each molecule's atom centres
};

// dot segment bookkeeping: for complex c, molecule m and dot type t
// (0 convex, 1 toroidal arc 1, 2 toroidal arc 2, 3 concave):
//   seg[(c*2+m)*4+t].dot0   global index of the segment's first dot
//   seg[(c*2+m)*4+t].scan0  value of that type's unit scan at the segment's first unit
struct Seg { long long dot0, scan0; };

enum : int {
    ST_OK = 0,
    ST_COINCIDENT = 1,       // two atoms of one molecule within 0.01 A
    ST_EMPTY = 2,            // complex without atoms
    ST_OVERFLOW = 4,         // a capacity was exceeded (host re-plans)
    ST_NEAR_OVERFLOW = 8,    // more than CMS_NEAR_CAP nearby low probes
};

#define CMS_NEAR_CAP 512
// complexes with more low probes than this find a probe's nearby low probes through cell lists (k_surface.cu)
#define CMS_LOW_CELL_MIN 4096

// Device pointers of one batch (workspace owned by the context).
struct Dev {
    Settings st;
    int B;
    int all_atoms;
    long long N;                       // atoms
    // inputs / per-atom
    const int* atom_off;               // B+1
    const int* n0;                     // B
    double4* xyzr;                     // N  (x, y, z, radius)
    double* dens;                      // N
    int* cplx;                         // N
    int8_t* mol;                       // N
    int8_t* atten;                     // N
    int8_t* access;                    // N
    int* cell_of;                      // N
    // per complex
    Cplx* cx;                          // B
    int* ncell;                        // B  cells per complex
    long long* ncell_scan;             // B+1
    int* status;                       // B
    int* ovf;                          // 1: a capacity of this run was exceeded (set by the check kernels)
    unsigned long long* coin;          // B  first coincident pair (i<<32|j), local
    // cells
    long long cells_cap;
    int* cell_cnt;                     // cells
    long long* cell_start;             // cells+1
    int* cell_fill;                    // cells
    int* cell_atom;                    // N
    // neighbour rows (CSR over atoms)
    int* nnb;  long long* nb_off;      // N, N+1
    int* nbur; long long* bu_off;      // N, N+1
    long long nb_cap, bu_cap;
    int* nb_id;  double* nb_d2;        // nb_cap
    int* nb_tmp;                       // nb_cap (unsorted ids of long rows)
    int* bu_id;                        // bu_cap
    // pairs / toroid queue
    int* ntor; long long* tor_off;     // N, N+1
    long long tor_cap;
    int* tor_i; int* tor_j;            // tor_cap
    struct TorGeo* tor_geo;            // tor_cap: each toroid's circle, made after the pair loop (k_tor_geo)
    // probes: per atom counts of + and - probes, per complex layout
    int* nplus; long long* plus_off;   // N, N+1
    int* nminus; long long* minus_off; // N, N+1
    long long probe_cap;
    int* pa0; int* pa1; int* pa2;      // probe_cap
    double* ph; double* pxyz; double* palt;   // probe_cap, 3*cap, 3*cap
    int* plow_flag; long long* plow_off;      // probe_cap, probe_cap+1
    int* plow_list;                            // probe_cap
    // low probes by cell of their complex's atom grid (clamped to it): counts, scan, probe ids, cell of each
    int* plc_cnt; int* plc_fill;               // cells
    long long* plc_start;                      // cells+1
    int* plc_item; int* plc_cell;              // probe_cap
    // probes stashed by the triple count pass (any order), with their final slot:
    // generating atom and sign bit (31) | rank among that atom's probes of that sign
    unsigned long long* ptop;                  // 1: stash entries taken
    int* sp_a; double* sp_h; double* sp_xyz; double* sp_alt;   // probe_cap (x3, x1, x3, x3)
    int* sp_g; unsigned* sp_ord;               // probe_cap
    // dots
    int* conv_cnt; long long* conv_off;          // N, N+1
    struct CvGeo* cv_geo;                        // N: each convex atom's frame (k_convex_geo)
    int* tor1_cnt; long long* tor1_off;          // tor_cap, +1
    int* tor2_cnt; long long* tor2_off;          // tor_cap, +1
    int8_t* tor_has;                             // tor_cap (toroidal access)
    int* tor_lflag; long long* tor_loff;         // tor_cap, +1: pair has dots, its exclusive scan
    int* tor_list;                               // tor_cap: pairs with dots, in pair order (emit work list)
    int* conc_cnt; long long* conc_off;          // probe_cap, +1
    struct ConcGeo* cc_geo;                      // probe_cap: each probe's spherical-triangle frame (k_probe_geo)
    // kept candidates of the convex and concave count passes: (latitude << 16 | point) in candidate
    // order per unit, so the emit passes write those alone; cv_soff / cc_soff: first entry (-1: none)
    unsigned long long* ks_top;                  // 1: entries taken
    int* ks_buf; long long ks_cap;               // ks_cap (= dot capacity)
    int* cv_soff;                                // N
    int* cc_soff;                                // probe_cap: first of the probe's dots in cs_* (-1: none)
    int* tor_soff; int* tor_sn;                  // tor_cap: kept torus points (those with arc dots) of a pair
    // concave dots made by the count pass (cc_soff indexes these): point, area, owner, sub-index, burial
    unsigned long long* cs_top;                  // 1: entries taken
    double* cs_xyz; double* cs_area; int* cs_own; int* cs_sub; int8_t* cs_bur; long long cs_cap;
    // neighbour rows sorted by the count pass: per atom its neighbours then its buried partners, in
    // the final order; nb_soff: the atom's first entry (-1: not kept, the emit pass gathers them again)
    unsigned long long* nbs_top;                 // 1: entries taken
    int* nbs_buf; long long nbs_cap;             // nbs_cap (= neighbour + buried-partner capacity)
    long long* nb_soff;                          // N
    Seg* seg;                                    // B*8
    long long* dot_off;                          // B*2+1 (per complex & molecule)
    long long dot_cap;
    double* dxyz; double* dnml; double* darea;   // dot_cap (x3, x3, x1)
    int8_t* dbur; int8_t* dtype; int* datom;     // dot_cap
    int* dunit;                                  // dot_cap: generating unit (atom / pair / probe)
    int* dsub;                                   // dot_cap: (lat<<16 | point) or (torus point<<16 | arc point)
    unsigned long long* tor_last1;               // N: last toroid pair with atom1 == a (scatter-max)
    unsigned long long* tor_last2;               // N
};

__device__ __forceinline__ V3 atom_xyz(const Dev& d, int g) { double4 a = d.xyzr[g]; return v3(a.x, a.y, a.z); }

// grid helpers
// Warp-local bump allocation from a buffer shared by all warps: a warp takes
// STASH_CHUNK entries (or more, for one large request) from the global counter
// at a time and hands them out to its successive units, so the counter sees
// one atomic per chunk instead of one per unit.  A chunk's unused tail is left
// empty.  Returns -1 when the entries would pass the buffer's capacity.
static constexpr int STASH_CHUNK = 1024;
struct StashCursor { unsigned long long cur, end; };

__device__ __forceinline__ long long stash_take(unsigned long long* top, long long cap, StashCursor& c, int n)
{
    if (c.cur + (unsigned long long)n > c.end) {
        const unsigned long long want = n > STASH_CHUNK ? (unsigned long long)n : (unsigned long long)STASH_CHUNK;
        unsigned long long o = 0;
        if ((threadIdx.x & 31) == 0) o = atomicAdd(top, want);
        o = __shfl_sync(0xffffffffu, o, 0);
        c.cur = o;
        c.end = o + want;
    }
    const unsigned long long r = c.cur;
    c.cur += (unsigned long long)n;
    return r + (unsigned long long)n <= (unsigned long long)cap ? (long long)r : -1;
}

// Graph-mode runs use fixed capacities; when a stage's total exceeds its
// capacity the run is flagged (and redone by the host), and every later
// pipeline kernel returns at entry so nothing indexes past a capacity.
#define CMS_EXIT_ON_OVERFLOW(d) \
    do {                        \
        if (*(d).ovf) return;   \
    } while (0)

__device__ __forceinline__ int cell_coord(double x, double o, double h, int dim)
{
    int c = (int)floor((x - o) / h);
    return c < 0 ? 0 : (c >= dim ? dim - 1 : c);
}

}  // namespace cms
