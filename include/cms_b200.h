/*
 * cms_b200.h -- C ABI of the B200 contact-molecular-surface library
 * (libcms_b200.so).
 *
 * The reference package (ullahsamee/cms-cuda) has no native interface: its
 * hot path is the Python class MolecularSurfaceCalculator
 * (cms-cuda/_core.py:762-1147, GPU twin cms-cuda/_gpu.py:310-686).  Each entry
 * point below replaces one method or step of that class; the citation in its
 * comment names it.  A Python binding (ctypes) of exactly these symbols is the
 * package `cms_cuda` next to the CUDA sources.
 *
 * Conventions
 *  - Every function returns cms_status (0 = success).  On failure
 *    cms_last_error() returns a message; no C++ exception crosses the ABI.
 *  - A batch holds B independent complexes.  Complex c owns atoms
 *    [atom_off[c], atom_off[c+1]) of the concatenated arrays, binder
 *    (molecule 0) first: n_binder[c] atoms, then the target (molecule 1).
 *    This is the reference's natom numbering (_core.py:918-943) per complex.
 *  - `where` arguments say whether pointers are host (CMS_HOST) or device
 *    (CMS_DEVICE) memory; host buffers are copied on the context's stream.
 *  - A context is bound to one device and one CUDA stream and is not
 *    thread-safe (one context per host thread, as the reference keeps one
 *    stream per thread, _gpu.py:70-83).
 */
#ifndef CMS_B200_H
#define CMS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cms_ctx cms_ctx;
typedef int32_t cms_status;

enum {
    CMS_OK = 0,
    CMS_ERR_ARG = -1,          /* invalid argument (ValueError in Python) */
    CMS_ERR_CUDA = -2,         /* CUDA runtime error */
    CMS_ERR_STATE = -3,        /* call order (RuntimeError: cache / mode mismatch) */
    CMS_ERR_COINCIDENT = -4,   /* coincident atoms (RuntimeError, _core.py:1286-1293) */
    CMS_ERR_EMPTY = -5,        /* complex without atoms (AssertionError, _core.py:895) */
    CMS_ERR_CAPACITY = -6      /* a fixed capacity was exceeded in graph mode */
};

enum { CMS_HOST = 0, CMS_DEVICE = 1 };

/* Stages that cms_set_concurrency may run as parallel branches. */
enum {
    CMS_CONC_COUNT = 1,        /* the convex, toroidal and concave count passes */
    CMS_CONC_EMIT = 2,         /* the convex, toroidal and concave emit passes */
    CMS_CONC_READOUT = 4       /* the SC searches beside the CMS search and its adjoint */
};

/* Settings of the calculator; defaults of _core.py:766-773. */
typedef struct {
    double rp;             /* probe radius, 1.7 */
    double density;        /* dots per A^2, 15.0 */
    double band;           /* SC peripheral band, 1.5 */
    double sep;            /* attention separation, 8.0 */
    double weight;         /* CMS distance weight, 0.5 */
    double binwidth_dist;  /* SC distance median bin, 0.02 */
    double binwidth_norm;  /* SC normal median bin, 0.02 */
} cms_settings;

/* Per-complex sizes after surface generation (for export buffers). */
typedef struct {
    int64_t n_atoms, n_binder;
    int64_t nb_entries, bu_entries;       /* neighbour / buried-partner list entries */
    int64_t max_nb, max_bu;               /* longest row (>= 1), padded width of the reference */
    int64_t n_toroid;                     /* toroid queue length */
    int64_t n_probes;
    int64_t n_probes_plus[2], n_probes_minus[2];
    int64_t n_dots[2];                    /* dots per molecule */
    int64_t n_trimmed[2];                 /* SC trimmed dots per molecule (after cms_shape_complementarity) */
    int64_t convex, toroidal, concave;    /* results.dots counters */
    int64_t n_blocked[2];                 /* atoms with attention 1 (blockers) per molecule */
    int64_t n_attended[2];                /* atoms with attention 5 per molecule (results nBuriedAtoms) */
    int32_t status;                       /* per-complex status bits */
    int32_t coincident_i, coincident_j;   /* first coincident pair (local indices) or -1 */
    double radmax;
} cms_complex_info;

/* Create a context on `device` using CUDA stream `stream` (NULL: a new
 * non-blocking stream owned by the context).  Replaces the calculator
 * constructor (_core.py:762-775, _gpu.py:312-330). */
cms_status cms_ctx_create(cms_ctx** out, int device, void* stream);
cms_status cms_ctx_destroy(cms_ctx* ctx);

/* Calculator settings (the `settings` object, _core.py:766-773). */
cms_status cms_set_settings(cms_ctx* ctx, const cms_settings* s);
cms_status cms_get_settings(cms_ctx* ctx, cms_settings* s);

/* Load B complexes: atom_off[B+1], n_binder[B] (host int64 arrays), xyz
 * (N x 3, row-major f64), radius (N f64) and optional per-atom density
 * (NULL: settings.density).  Replaces reset + add_binder_and_target /
 * AddMolecule (_core.py:918-943). */
cms_status cms_load_batch(cms_ctx* ctx, int32_t B, const int64_t* atom_off, const int64_t* n_binder,
                          const double* xyz, const double* radius, const double* density, int32_t where);

/* Generate the molecular surfaces of every loaded complex: attention numbers,
 * neighbour lists, pair/triple loops and convex, toroidal and concave dots.
 * all_atoms = 1 is the single-molecule mode of maximum possible CMS.
 * Replaces _ensure_surfaces_generated (_core.py:865-909). */
cms_status cms_generate_surfaces(cms_ctx* ctx, int32_t all_atoms);

/* Contact molecular surface of both sides of every complex.
 * per_atom (N): for a target atom, its target-side CMS; for a binder atom,
 * its binder-side CMS.  totals (2B): totals[2c+1] target side,
 * totals[2c] binder side.  Replaces calc_contact_molecular_surface
 * (_core.py:946-1004) for target_side True and False. */
cms_status cms_contact_ms(cms_ctx* ctx, double* per_atom, double* totals, int32_t where);

/* Gradient of sum_c grad_total[c] * CMS_c (one side: target_side 1 = the
 * target-side CMS, 0 = the binder side) with respect to every atom's
 * coordinates, grad_xyz (N x 3), with the dot topology of the last surface
 * generation held fixed (which dots exist, their burial, subdivision indices,
 * construction branches and each query's nearest dot).  grad_total (B) NULL
 * means all ones.  Runs the CMS readout first when needed.  The reference has
 * no gradient; this is the adjoint of calc_contact_molecular_surface
 * (_core.py:946-1004) through the dot construction (_core.py:1646-2333). */
cms_status cms_contact_ms_backward(cms_ctx* ctx, int32_t target_side, const double* grad_total, double* grad_xyz,
                                   int32_t where);

/* Include the gradient of one side's CMS in the captured pipeline
 * (cms_run_graph / cms_graph_launch); upstream gradients are all ones until
 * cms_set_grad_total (device or host, B values) replaces them, and
 * cms_grad_xyz reads the last result.  No reference counterpart. */
cms_status cms_set_backward(cms_ctx* ctx, int32_t enable, int32_t target_side);
cms_status cms_set_grad_total(cms_ctx* ctx, const double* grad_total, int32_t where);
cms_status cms_grad_xyz(cms_ctx* ctx, double* grad_xyz, int32_t where);

/* Self-check of the adjoint's formula: the positions (n x 3) and areas (n) of
 * complex c's dots of one molecule recomputed from the atoms and the stored
 * dot topology by the adjoint's geometry code on plain doubles, in
 * cms_export_dots order.  Equal bit for bit to the generated dots. */
cms_status cms_recompute_dots(cms_ctx* ctx, int32_t c, int32_t molecule, double* coor, double* area);

/* Maximum possible CMS (per-atom dot area of molecule 0, surface generated
 * with all_atoms = 1).  per_atom (N; molecule-0 atoms), totals (B).
 * Replaces calc_max_possible_contact_molecular_surface (_core.py:1007-1034). */
cms_status cms_max_contact_ms(cms_ctx* ctx, double* per_atom, double* totals, int32_t where);

/* Per-residue sums of a per-atom readout, for the whole batch in one launch:
 * values 0 = the per-atom CMS of cms_contact_ms, 1 = the per-atom maximum
 * CMS of cms_max_contact_ms (either is computed first when needed).  Residue
 * r adds the values of atoms res_atoms[res_off[r] .. res_off[r+1]) (batch
 * atom indices; res_off has n_residues + 1 entries from 0 to n_entries) in
 * that order, starting from 0.0, into sums[r].  Replaces the reference CLI's
 * per_residue loop (examples/calculate_cms_sc.py:105-114).  Offsets or atom
 * indices out of range give CMS_ERR_ARG. */
cms_status cms_residue_sums(cms_ctx* ctx, int32_t values, int64_t n_residues, const int64_t* res_off,
                            int64_t n_entries, const int32_t* res_atoms, double* sums, int32_t where);

/* Shape complementarity.  sc (B x 5): sc, interface area, median distance,
 * mean distance, mean normal score (surface 2).  sides (B x 2 x 7):
 * d_mean, d_median, s_mean, s_median, trimmedArea, nTrimmedDots, nAllDots of
 * each molecule.  Replaces CalcLoadedSC (_core.py:807-863) with
 * trim_peripheral_band_vectorized, calc_neighbor_distance_vectorized and
 * _binned_median (_core.py:1037-1147). */
cms_status cms_shape_complementarity(cms_ctx* ctx, double* sc, double* sides, int32_t where);

/* Sizes and status of complex c (valid after cms_generate_surfaces). */
cms_status cms_complex_info_get(cms_ctx* ctx, int32_t c, cms_complex_info* info);

/* Host copies of complex c's state, the arrays the reference keeps in
 * calc.run (_core.py:777-789); atom indices are local to the complex. */
cms_status cms_export_atoms(cms_ctx* ctx, int32_t c, int8_t* atten, int8_t* access, int32_t* n_neighbors,
                            int32_t* n_buried);
cms_status cms_export_neighbors(cms_ctx* ctx, int32_t c, int64_t* nb_off, int32_t* nb_id, int64_t* bu_off,
                                int32_t* bu_id);
cms_status cms_export_toroid(cms_ctx* ctx, int32_t c, int32_t* atom1, int32_t* atom2, double* uij, double* tij,
                             double* rij, int8_t* between);
cms_status cms_export_probes(cms_ctx* ctx, int32_t c, int32_t* a0, int32_t* a1, int32_t* a2, double* height,
                             double* point, double* alt);
cms_status cms_export_dots(cms_ctx* ctx, int32_t c, int32_t molecule, double* coor, double* outnml, double* area,
                           int8_t* buried, int8_t* type, int32_t* atom_idx);
/* Construction indices of complex c's dots of one molecule, in
 * cms_export_dots order: unit = the generating atom (convex dots), toroid
 * pair (toroidal, cms_export_toroid order) or probe (concave,
 * cms_export_probes order); sub = (latitude << 16) | point for convex and
 * concave dots, (torus point << 16) | (arc 2 ? 1 << 15 : 0) | arc point for
 * toroidal dots.  The reference keeps no such indices; they define the dot
 * topology the gradient holds fixed. */
cms_status cms_export_dot_units(cms_ctx* ctx, int32_t c, int32_t molecule, int32_t* unit, int32_t* sub);

/* local dot indices (within the molecule's dot array) of the SC trimmed dots */
cms_status cms_export_trimmed(cms_ctx* ctx, int32_t c, int32_t molecule, int32_t* dot_index);

/* Brute-force nearest dot: for each query point (n_query x 3 f64) the
 * smallest squared distance to the reference points (n_ref x 3 f64) in
 * scipy cdist 'sqeuclidean' order, and the first reference index attaining
 * it -- cdist(ref, query).min(axis=0) / .argmin(axis=0), the primitive the
 * reference calls min_sqdist (cms-cuda/_gpu_kernels.py:508-566).  FP32
 * filter with an FP64 recheck, so both outputs equal the FP64 search's.
 * out_index may be NULL.  Uses the context's workspace. */
cms_status cms_nearest_dots(cms_ctx* ctx, const double* query_xyz, int64_t n_query, const double* ref_xyz,
                            int64_t n_ref, double* out_d2, int32_t* out_index, int32_t where);

/* Allocation-free variant of cms_nearest_dots, for callers that cannot
 * allocate GPU memory: a framework or application that owns every device
 * allocation through its own pool, plugins it hosts, and real-time loops that
 * must not meet cudaMalloc's implicit synchronisation.  This entry point has
 * no counterpart in the reference.  query_xyz, ref_xyz, out_d2 and out_index
 * (NULL: no indices) must be memory a kernel on the current device can use
 * (its device memory, managed or mapped pinned memory; anything else is
 * CMS_ERR_ARG, nothing launched); the work is enqueued on `stream` (NULL: the
 * default stream) and no memory is allocated: the scratch is one fixed
 * 32 MiB device array per GPU, so n_query + n_ref may not exceed 1,964,032
 * points (CMS_ERR_ARG otherwise, nothing launched).  The first call on a
 * device looks up the scratch address (make it before any stream capture;
 * calls after a cudaDeviceReset are not supported); calls that overlap on the
 * GPU share the scratch and race.  A CUDA error already pending on the
 * calling thread is left in place and the call returns CMS_ERR_CUDA. */
cms_status cms_nearest_dots_noalloc(const double* query_xyz, int64_t n_query, const double* ref_xyz,
                                    int64_t n_ref, double* out_d2, int32_t* out_index, void* stream);

/* Capture the whole pipeline (surfaces + CMS + SC) of the loaded batch shape
 * in a CUDA graph with the current capacities (run it once first), then
 * replay it; later cms_load_batch calls with the same B, N and offsets reuse
 * it.  Falls back to the stage-synchronised path on capacity overflow. */
cms_status cms_run_graph(cms_ctx* ctx);

/* Replay the captured pipeline graph on the context's stream without
 * waiting (capturing it first if needed); results are read by the usual
 * readout calls, which synchronise.  cms_graph_check waits and returns
 * CMS_ERR_CAPACITY if the inputs outgrew the captured capacities (then call
 * cms_run_graph, which re-sizes). */
cms_status cms_graph_launch(cms_ctx* ctx);
cms_status cms_graph_check(cms_ctx* ctx);

/* Rigid-body pose refinement of every complex's binder by gradient ascent on
 * the target-side CMS (no reference counterpart; the objective is
 * calc_contact_molecular_surface, _core.py:946-1004).  cms_refine_begin takes
 * the reference coordinates (N x 3: binders in their starting poses, targets
 * fixed) of the loaded batch and up to max_steps of history; each step of
 * cms_refine_run is one replay of a captured graph -- apply the poses,
 * regenerate the surfaces, CMS, its adjoint, and a clipped ascent step on
 * each binder's rotation (about its reference centroid) and translation.
 * cms_hist (steps x B) receives the CMS of every evaluated pose; the run
 * checks capacities every 25 steps and redoes a chunk that outgrew them.
 * cms_refine_pose returns the current rotations (B x 9), translations (B x 3)
 * and coordinates (N x 3, any may be NULL). */
cms_status cms_refine_begin(cms_ctx* ctx, const double* ref_xyz, int32_t max_steps, int32_t where);
cms_status cms_refine_set_params(cms_ctx* ctx, double eta_t, double eta_w, double max_t, double max_w);
cms_status cms_refine_run(cms_ctx* ctx, int32_t steps, double* cms_hist, int32_t where);
cms_status cms_refine_pose(cms_ctx* ctx, double* rot, double* trans, double* xyz, int32_t where);
cms_status cms_refine_end(cms_ctx* ctx);

/* Search shapes of the batched pipeline's three nearest-dot searches (CMS, SC
 * band trim, SC neighbour argmin): variants[3], each 0..3 = 4 queries per
 * thread with each warp staging its own reference blocks in reach, 4 queries
 * per thread with 512-reference rounds staged by the whole CTA, 2 with
 * per-warp blocks, 2 with 512-reference rounds.  Every shape
 * gives the same results.  By default an autotuner times all shapes on each
 * new batch shape before capturing the graph and keeps the fastest per search
 * (tune_ms[3 x 4]: the times it measured, NULL to skip); cms_set_nn_variants
 * forces shapes and turns the tuner off, cms_set_autotune(1) turns it back on.
 * The reference's CuPy kernels have fixed launch shapes (_gpu_kernels.py). */
cms_status cms_set_nn_variants(cms_ctx* ctx, const int32_t* variants);
cms_status cms_get_nn_variants(cms_ctx* ctx, int32_t* variants, double* tune_ms);
cms_status cms_set_autotune(cms_ctx* ctx, int32_t enable);

/* Shapes of the surface kernels that the autotuner also picks per batch
 * shape, variants[5] for the toroidal count, toroidal emit, concave count,
 * concave emit and triple count passes: toroidal 0 = 16 toroid pairs per warp
 * batch, 4 warps per CTA, 1 = 32 pairs, 2 warps, 2 = 16 pairs, 4 warps,
 * registers for 6 CTAs per SM; concave 0, 1, 2 = registers for 4, 5, 6 CTAs
 * per SM; triples 0 = neighbour rows of up to 128 cached per warp, 1 / 2 =
 * up to 64, registers for 10 / 12 CTAs of 2 warps.  Every shape generates the
 * same surfaces.  cms_get_surface_variants returns the shapes in use and the
 * tuner's measured stage times (tune_ms[5 x 3], NULL to skip);
 * cms_set_surface_variants
 * forces shapes and turns the tuner off (cms_set_autotune(1) turns it back
 * on).  The reference's kernels have fixed launch shapes. */
cms_status cms_set_surface_variants(cms_ctx* ctx, const int32_t* variants);
cms_status cms_get_surface_variants(cms_ctx* ctx, int32_t* variants, double* tune_ms);

/* Nearest-dot search work of the last run: pairs[0..5] = (query x reference
 * pairs, queries) of the CMS search, the SC band (trim) search and the SC
 * neighbour search -- the algorithmic work behind the FP32 roofline. */
cms_status cms_nn_work(cms_ctx* ctx, int64_t* pairs);

/* Run independent stages of the captured pipeline concurrently: mode is an
 * OR of CMS_CONC_* bits (0 = every stage in order).  A set bit runs that
 * group on the context's stream and two side streams -- parallel branches of
 * the graph.  Default: CMS_CONC_EMIT | CMS_CONC_READOUT.  The results are
 * the same for every mode; the sizing run, the stage-synchronised path and
 * cms_profile_stages always run the stages in order.  Modes outside 0..7
 * give CMS_ERR_ARG.  No reference counterpart. */
cms_status cms_set_concurrency(cms_ctx* ctx, int32_t mode);

/* Nearest-dot search work the kernels actually did, counted by the kernels
 * themselves in one extra (eager) run of the CMS and SC readouts on the
 * current surfaces: counts[0..2] = (query, reference) pairs the FP32 filter
 * evaluated in the CMS, SC band and SC argmin searches after the box culling,
 * counts[3..5] = references rechecked in FP64 by each.  The readout results
 * are unchanged.  No reference counterpart (its searches are plain brute
 * force, _gpu_kernels.py:78-117). */
cms_status cms_nn_evaluated(cms_ctx* ctx, int64_t* counts);

/* Measured FP32 FMA throughput of the context's device (TFLOP/s, FMA = 2
 * FLOP): the denominator of the nearest-dot search's roofline. */
cms_status cms_fp32_peak(cms_ctx* ctx, double* tflops);

/* Cumulative host->device and device->host bytes moved by the context's
 * loads, readouts and synchronising bookkeeping (exports excluded). */
cms_status cms_transfer_bytes(cms_ctx* ctx, int64_t* h2d, int64_t* d2h);

/* Number of kernel nodes in the captured pipeline graph (-1 before capture). */
int64_t cms_kernel_launches(cms_ctx* ctx);

/* Run the batched pipeline (surfaces, CMS, SC) once with the current
 * capacities and a CUDA event after every stage; ms[s] receives stage s's
 * milliseconds (s < cap), *n_stages the number of stages.  Diagnostic
 * counterpart of the reference's per-stage NVTX ranges (_gpu.py:30). */
cms_status cms_profile_stages(cms_ctx* ctx, double* ms, int32_t cap, int32_t* n_stages);
const char* cms_stage_name(int32_t stage);

const char* cms_last_error(cms_ctx* ctx);
const char* cms_version(void);

/* Number of visible CUDA devices (0 when none or no driver); replaces the
 * reference's gpu_available() probe (cms-cuda/_api.py:15-22). */
int32_t cms_device_count(void);

#ifdef __cplusplus
}
#endif

#endif /* CMS_B200_H */
