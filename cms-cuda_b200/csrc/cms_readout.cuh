// Readout workspace and launchers (k_readout.cu).
#pragma once
#include "cms_kernels.cuh"

namespace cms {

enum { NN_MIN = 0, NN_ARGMIN = 1, NN_BAND = 2 };

// references per sub-round of the nearest-dot search (the granularity of the
// round boxes); a search's box arrays hold ceil(references / NN_ROUND)
// sub-rounds per task
static constexpr int NN_ROUND = 512;
static constexpr int NN_VARIANTS = 4;        // tunable search shapes (k_readout.cu)
static inline long long nn_round_cap(long long refs, long long ntask) { return refs / NN_ROUND + ntask + 1; }

#define SC_SIDE_FIELDS 7   // d_mean, d_median, s_mean, s_median, trimmedArea, nTrimmedDots, nAllDots
#define SC_FIELDS 5        // sc, area, distance, d_mean (surface 2), s_mean (surface 2)

// one nearest-dot task: queries [q0, q0+qn) against references [r0, r0+rn)
// of the same complex, both as positions in packed lists
struct NNTask {
    long long q0, qn, r0, rn;
    double E;       // FP32 error scale: 2.5e-7 x the per-axis half-extent bounding both point sets
    int c;
};

struct NNArgs {
    const NNTask* task;
    int ntask;
    int* tile_cnt;          // ntask
    long long* tile_off;    // ntask + 1
    const float4* q_f4; const int* q_idx;       // packed FP32 points; index into q_xyz (null: identity)
    const float4* r_f4; const int* r_idx;
    const double* q_xyz; const double* r_xyz;   // FP64 coordinates for the recheck
    double* out_d2; int* out_idx; int* out_flag;
    double band_thr64;      // band^2 (BAND mode)
    // rounds of NN_ROUND references per task and their bounding boxes (lo, hi):
    // box_round 2 per round, box_blk 2 per 32-reference block (32 per round)
    int* round_cnt;         // ntask
    long long* round_off;   // ntask + 1
    float4* box_round;
    float4* box_blk;
    long long round_cap;    // rounds the box arrays hold
    int band_mode;
    int tile_q;             // queries per tile of the launched variant
    const int* ovf;         // the batch's overflow flag (null for standalone searches)
    // spatially ordered lists: the original position of each entry (null: lists in their own order);
    // outputs go to the queries' original positions, and reference indices are original positions
    const int* q_perm; const int* r_perm;
    // instrumented runs only (null otherwise): (query, reference) pairs the FP32 filter evaluated in the
    // scan, and references rechecked in FP64
    unsigned long long* pair_count; unsigned long long* recheck_count;
};

// readout workspace, capacity = dot capacity unless noted
struct Rd {
    int* flag; long long* bur_scan;             // D, D+1
    int* bur_idx; float4* bur_f4; int* bur_cm;  // buried dots, in dot order
    int* acc_idx; float4* acc_f4;               // accessible dots, in dot order
    int* keep; long long* trim_scan;            // per buried entry, +1
    int* trim_idx; float4* trim_f4;             // trimmed dots
    double* nn_d2; int* nn_idx;                 // per query entry
    double* val; int* own;                      // per entry value / owner atom (-1: none)
    // spatially ordered copies (k_readout.cu) of the buried list (set 0, made with the lists) and of
    // the accessible, then the trimmed list (set 1): points and each entry's original position
    float4* so_f4[2]; int* so_perm[2];
};

enum { SO_BUR = 0, SO_ACC = 1, SO_TRIM = 2 };

// adjoint of the contact molecular surface (k_adjoint.cu); capacity D = dot
// capacity unless noted
struct AdjBuf {
    double4* A;            // per dot: (dCMS/dp, dCMS/darea)
    int* cms_idx;          // per buried entry: nearest reference position of the CMS search
    int* ref_ent;          // per buried entry: the buried entry of the reference its query picked (-1: none)
    double4* ref_vec;      // per buried entry: contribution to that reference dot's position
    int* rcnt; int* rfill; long long* roff; int* rslot;   // per buried entry (capacity D), roff D + 1
    double* gconv;         // 6 per atom: convex unit contributions (atom, frame atom)
    double* gtor;          // 6 per toroid pair: (atom 1, atom 2)
    double* gconc;         // 9 per probe: (atom 0, atom 1, atom 2)
    int* act_conv; int* act_tor; int* act_conc;   // per unit: its dots given an adjoint (> 0: active unit)
    int8_t* act_atom;      // atoms of active units
    int* list_conv; int* list_tor; int* list_conc;         // active units
    int* skey;             // 3 x ADJ_KEYS: active units per work key, then each key's next slot
    int* slist_conv; int* slist_tor; int* slist_conc;      // active units, largest dot counts first
    int* nact;             // 3 counters
    const double* gtot;    // per complex: upstream gradient of the side's CMS
};

void launch_adjoint(const Dev& d, const Rd& r, const AdjBuf& a, const NNTask* cms_task, int side, double* grad,
                    long long* scan_tmp, cudaStream_t s);
void launch_recompute(const Dev& d, double* xyz, double* area, cudaStream_t s);

// rigid-body pose refinement (k_refine.cu)
struct RefineParams {
    double eta_t, eta_w;    // ascent step per unit gradient: A, radians
    double max_t, max_w;    // step caps: A, radians
};
void launch_pose_apply(const Dev& d, const double* ref, const double* pose, const double* cen, cudaStream_t s);
void launch_pose_update(const Dev& d, const double* grad, const double* ref, double* pose, const double* cen,
                        const double* totals, double* hist, int* step, int hist_steps, const RefineParams& prm,
                        cudaStream_t s);
void launch_track_max(const long long* summary, long long* mx, cudaStream_t s);
void launch_pose_centroid(const Dev& d, const double* ref, double* cen, cudaStream_t s);

void launch_split_buried(const Dev& d, const Rd& r, long long dot_cap, long long* scan_tmp, cudaStream_t s);
void launch_spatial_order(const Dev& d, const Rd& r, int list, int set, cudaStream_t s);
void launch_tasks(const Dev& d, const Rd& r, int kind, NNTask* task, cudaStream_t s);
void launch_nn(NNArgs a, int mode, int variant, long long tile_cap, long long* scan_tmp, cudaStream_t s);
void launch_nn_tiles(NNArgs a, int mode, int variant, long long* scan_tmp, cudaStream_t s);
void launch_nn_kernel(NNArgs a, int mode, int variant, long long tile_cap, cudaStream_t s);
// tile_cap for launch_nn_kernel (variant 0) of a standalone search of n_query points
long long nn_standalone_tile_cap(long long n_query);
// standalone search helpers: bounding box of two point sets, FP32 packing, one task
void launch_points_setup(const double* q, long long nq, const double* r, long long nr, double* partials,
                         int partial_blocks, double* bbox, float4* q_f4, float4* r_f4, NNTask* task, int* tile_cnt,
                         long long* tile_off, int* round_cnt, long long* round_off, cudaStream_t s);
void launch_cms_weights(const Dev& d, const Rd& r, long long cap, cudaStream_t s);
void launch_area_values(const Dev& d, const Rd& r, long long cap, cudaStream_t s);
void launch_per_atom_sum(const Dev& d, const Rd& r, bool dots, double* out, cudaStream_t s);
void launch_atom_totals(const Dev& d, const double* per_atom, double* tot, cudaStream_t s);
void launch_trim_compact(const Dev& d, const Rd& r, long long cap, long long* scan_tmp, cudaStream_t s);
void launch_sc_stats(const Dev& d, const Rd& r, const NNTask* task, double* side, double* out, cudaStream_t s);

}  // namespace cms
