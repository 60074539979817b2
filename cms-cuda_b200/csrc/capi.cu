// C ABI of libcms_b200.so: context, device workspace, pipeline orchestration
// (stage-synchronised sizing path and CUDA-graph path) and exports.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cms_b200.h"
#include "cms_readout.cuh"
#include "cms_circle.cuh"

using namespace cms;

// stage groups run as parallel graph branches unless cms_set_concurrency says otherwise: the emit passes
// and the readouts (on the 4096-complex batch 231.4 ms a step against 235.5 with every stage in order);
// the count passes are not (245.4 ms with them alone as branches)
#define CMS_CONC_DEFAULT (CMS_CONC_EMIT | CMS_CONC_READOUT)

namespace {

struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

__global__ void k_pack_atoms(long long N, const double* xyz, const double* rad, const double* dens_in, double dens,
                             double4* xyzr, double* dens_out)
{
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < N; g += (long long)gridDim.x * blockDim.x) {
        xyzr[g] = make_double4(xyz[3 * g], xyz[3 * g + 1], xyz[3 * g + 2], rad[g]);
        dens_out[g] = dens_in ? dens_in[g] : dens;
    }
}

__global__ void k_fill_d(double* p, long long n, double v)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_fill_i(int* p, long long n, int v)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = v;
}

// Per-residue sums of a per-atom array: residue r adds the values of atoms
// res_atoms[res_off[r] .. res_off[r+1]) in that order, starting from 0.0 --
// the running dictionary sum of the reference CLI's per_residue
// (examples/calculate_cms_sc.py:105-114), one residue per thread.  Offsets
// outside [0, n_entries] or decreasing, and atom indices outside [0, N), set
// *bad and are skipped.
__global__ void k_residue_sums(const double* per_atom, long long N, const long long* res_off, long long n_res,
                               const int* res_atoms, long long n_entries, double* out, int* bad)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n_res; r += (long long)gridDim.x * blockDim.x) {
        long long k0 = res_off[r], k1 = res_off[r + 1];
        if (k0 < 0 || k1 > n_entries || k1 < k0) {
            *bad = 1;
            k0 = k1 = 0;
        }
        double acc = 0.0;
        for (long long k = k0; k < k1; ++k) {
            const int a = res_atoms[k];
            if (a < 0 || a >= N) { *bad = 1; continue; }
            acc += per_atom[a];
        }
        out[r] = acc;
    }
}

// totals the host needs after a run: cells, neighbour / buried entries,
// toroid pairs, probes, dots, buried dots, trimmed dots
// capacity check of a stage total (two totals summed when b is given)
__global__ void k_cap_check(const long long* a, const long long* b, long long cap, int* ovf)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const long long t = *a + (b ? *b : 0);
        if (t > cap) *ovf = 1;
    }
}

__global__ void k_summary(Dev d, Rd r, long long* out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        out[0] = d.ncell_scan[d.B];
        out[1] = d.nb_off[d.N];
        out[2] = d.bu_off[d.N];
        out[3] = d.tor_off[d.N];
        out[4] = d.plus_off[d.N] + d.minus_off[d.N];
        out[5] = d.dot_off[2LL * d.B];
    }
}

// toroid queue geometry for export (second_loop formulas, _core.py:1372-1416)
__global__ void k_export_toroid(Dev d, long long q0, long long n, double* out)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long q = q0 + k;
        const int i = d.tor_i[q], j = d.tor_j[q];
        const double rp = d.st.rp;
        double4 a = d.xyzr[i], b = d.xyzr[j];
        V3 xi = v3(a.x, a.y, a.z), xj = v3(b.x, b.y, b.z);
        V3 diff = xj - xi;
        double dij_sq = sq_alt(diff);
        double dij = sqrt(dij_sq);
        double eri = a.w + rp, erj = b.w + rp;
        double asymm = (eri * eri - erj * erj) / dij;
        V3 uij = diff / dij;
        V3 tij = ((xi + xj) * 0.5) + uij * (asymm * 0.5);
        double far_sq = (eri + erj) * (eri + erj) - dij_sq;
        double rd = a.w - b.w;
        double cont_sq = dij_sq - rd * rd;
        double rij = ((0.5 * sqrt(far_sq)) * sqrt(cont_sq)) / dij;
        double* o = out + 8 * k;
        o[0] = uij.x; o[1] = uij.y; o[2] = uij.z;
        o[3] = tij.x; o[4] = tij.y; o[5] = tij.z;
        o[6] = rij;
        o[7] = fabs(asymm) < dij ? 1.0 : 0.0;
    }
}

// per-complex sizes, counters and status (one block per complex)
__global__ void k_complex_info(Dev d, Rd r, int want_sc, cms_complex_info* out)
{
    __shared__ long long sh[6][32];
    const int c = blockIdx.x;
    const Cplx C = d.cx[c];
    const int a0 = C.a0, s1 = C.a0 + C.n0, a1 = C.a0 + C.n;
    long long v[6] = {1, 1, 0, 0, 0, 0};   // max nb, max bu, blocked0, blocked1, attended0, attended1
    for (int g = a0 + threadIdx.x; g < a1; g += blockDim.x) {
        v[0] = max(v[0], (long long)d.nnb[g]);
        v[1] = max(v[1], (long long)d.nbur[g]);
        const int m = g < s1 ? 0 : 1;
        if (d.atten[g] == 1) ++v[2 + m]; else ++v[4 + m];
    }
    for (int o = 16; o > 0; o >>= 1) {
        v[0] = max(v[0], __shfl_xor_sync(0xffffffffu, v[0], o));
        v[1] = max(v[1], __shfl_xor_sync(0xffffffffu, v[1], o));
        for (int k = 2; k < 6; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) for (int k = 0; k < 6; ++k) sh[k][w] = v[k];
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int i = 1; i < nw; ++i) {
        v[0] = max(v[0], sh[0][i]);
        v[1] = max(v[1], sh[1][i]);
        for (int k = 2; k < 6; ++k) v[k] += sh[k][i];
    }
    cms_complex_info I;
    memset(&I, 0, sizeof(I));
    I.n_atoms = C.n;
    I.n_binder = C.n0;
    I.nb_entries = d.nb_off[a1] - d.nb_off[a0];
    I.bu_entries = d.bu_off[a1] - d.bu_off[a0];
    I.max_nb = v[0];
    I.max_bu = v[1];
    I.n_toroid = d.tor_off[a1] - d.tor_off[a0];
    I.n_probes_plus[0] = d.plus_off[s1] - d.plus_off[a0];
    I.n_probes_plus[1] = d.plus_off[a1] - d.plus_off[s1];
    I.n_probes_minus[0] = d.minus_off[s1] - d.minus_off[a0];
    I.n_probes_minus[1] = d.minus_off[a1] - d.minus_off[s1];
    I.n_probes = I.n_probes_plus[0] + I.n_probes_plus[1] + I.n_probes_minus[0] + I.n_probes_minus[1];
    long long cnt[4] = {0, 0, 0, 0};
    for (int m = 0; m < 2; ++m) {
        const long long ds = d.dot_off[2 * c + m], de = d.dot_off[2 * c + m + 1];
        I.n_dots[m] = de - ds;
        for (int t = 0; t < 4; ++t) {
            const long long e = t < 3 ? d.seg[(c * 2 + m) * 4 + t + 1].dot0 : de;
            cnt[t] += e - d.seg[(c * 2 + m) * 4 + t].dot0;
        }
        if (want_sc) {
            const long long bs = r.bur_scan[ds], be = r.bur_scan[de];
            I.n_trimmed[m] = r.trim_scan[be] - r.trim_scan[bs];
        }
        I.n_blocked[m] = v[2 + m];
        I.n_attended[m] = v[4 + m];
    }
    I.convex = cnt[0];
    I.toroidal = cnt[1] + cnt[2];
    I.concave = cnt[3];
    I.status = d.status[c];
    const unsigned long long k = d.coin[c];
    if (k != ~0ull) {
        I.status |= ST_COINCIDENT;
        I.coincident_i = (int32_t)(k >> 32);
        I.coincident_j = (int32_t)(k & 0xffffffffu);
    } else {
        I.coincident_i = I.coincident_j = -1;
    }
    I.radmax = C.radmax;
    out[c] = I;
}

// FP32 FMA throughput probe: 8 independent FMA chains per thread, the result
// folded into one store so nothing is optimised away
__global__ void __launch_bounds__(256) k_fp32_peak(float* out, int iters, float a, float b)
{
    float x[8];
    for (int k = 0; k < 8; ++k) x[k] = (float)(threadIdx.x + k) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = __fmaf_rn(x[k], a, b);
    }
    float s = 0.f;
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == 12345.678f) out[blockIdx.x] = s;
}

}  // namespace

struct cms_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cms_settings st{1.7, 15.0, 1.5, 8.0, 0.5, 0.02, 0.02};
    int B = 0;
    long long N = 0;
    std::vector<int64_t> h_off, h_n0;
    std::vector<DBuf> bufs;
    Dev d{};
    Rd r{};
    long long cap_cells = 0, cap_nb = 0, cap_bu = 0, cap_tor = 0, cap_probe = 0, cap_dot = 0, cap_conc = 0;
    long long tot[8] = {0};
    bool have_batch = false, surf_ok = false, cms_ok = false, sc_ok = false, max_ok = false;
    int surf_all_atoms = -1;
    long long* pinned = nullptr;
    // per-complex host mirrors (valid after generation)
    std::vector<long long> h_nb_off_b, h_plus, h_minus, h_dot_off, h_tor_off_b;
    std::vector<int> h_status;
    std::vector<unsigned long long> h_coin;
    std::vector<Seg> h_seg;
    std::vector<double> h_radmax;
    std::vector<cms_complex_info> h_info;   // per-complex info table of the last run
    int info_state = 0;                      // 0 stale, 1 computed before SC, 2 with SC counts
    // graph
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    long long graph_key[4] = {-1, -1, -1, -1};
    long long graph_vk = -1;                 // search shapes the graph was captured with
    // gradient of one side's CMS (cms_set_backward / cms_contact_ms_backward)
    int bwd_enabled = 0, bwd_side = 1;
    bool bwd_ok = false;
    // nearest-dot search shapes per stage (CMS, SC band, SC argmin), chosen by
    // the autotuner for each batch shape (or forced by cms_set_nn_variants)
    int nn_var[3] = {0, 0, 0};
    // rigid-body pose refinement (cms_refine_*)
    bool refine = false;
    RefineParams rprm{0.002, 0.0002, 0.05, 0.00872664625997};   // max 0.05 A and 0.5 degree per step
    int hist_cap = 0;
    bool autotune = true;
    long long tune_key[3] = {-1, -1, -1};
    double tune_ms[3][NN_VARIANTS] = {};
    // surface kernel shapes (toroidal count, toroidal emit, concave count, concave emit), tuned with the
    // search shapes (or forced by cms_set_surface_variants)
    int sv[SURF_TUNED] = {0, 0, 0, 0, 0};
    double sv_ms[SURF_TUNED][SURF_VARIANTS] = {};
    long long launches = -1;
    std::string err;
    // stage timing: an event after each pipeline stage when profiling
    bool profiling = false;
    // stages run concurrently (CMS_CONC_* bits; graph and eager runs with the current capacities)
    int conc = CMS_CONC_DEFAULT;
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    bool counting = false;   // readouts run with the nearest-dot work counters (cms_nn_evaluated)
    long long h2d_bytes = 0, d2h_bytes = 0;   // host<->device bytes moved by the hot path
    std::vector<cudaEvent_t> marks;
    std::vector<int> mark_ids;

    // named buffer slots
    enum Slot {
        S_IN_XYZ, S_IN_RAD, S_IN_DENS, S_ATOM_OFF, S_N0, S_XYZR, S_DENS, S_CPLX, S_MOL, S_ATTEN, S_ACCESS, S_CELL_OF,
        S_CX, S_NCELL, S_NCELL_SCAN, S_STATUS, S_COIN, S_CELL_CNT, S_CELL_START, S_CELL_FILL, S_CELL_ATOM,
        S_NNB, S_NB_OFF, S_NBUR, S_BU_OFF, S_NB_ID, S_NB_D2, S_NB_TMP, S_BU_ID,
        S_NTOR, S_TOR_OFF, S_TOR_I, S_TOR_J,
        S_NPLUS, S_PLUS_OFF, S_NMINUS, S_MINUS_OFF, S_PA0, S_PA1, S_PA2, S_PH, S_PXYZ, S_PALT, S_PLOW_FLAG, S_PLOW_OFF,
        S_PLOW_LIST,
        S_CONV_CNT, S_CONV_OFF, S_TOR1_CNT, S_TOR1_OFF, S_TOR2_CNT, S_TOR2_OFF, S_TOR_HAS, S_CONC_CNT, S_CONC_OFF,
        S_SEG, S_DOT_OFF, S_DXYZ, S_DNML, S_DAREA, S_DBUR, S_DTYPE, S_DATOM, S_DUNIT, S_DSUB, S_TOR_LAST1, S_TOR_LAST2,
        S_R_FLAG, S_R_BUR_SCAN, S_R_BUR_IDX, S_R_BUR_F4, S_R_BUR_CM, S_R_ACC_IDX, S_R_ACC_F4, S_R_KEEP, S_R_TRIM_SCAN,
        S_R_TRIM_IDX, S_R_TRIM_F4, S_R_NN_D2, S_R_NN_IDX, S_R_VAL, S_R_OWN,
        S_CM_TMP, S_SCAN_TMP, S_PER_ATOM_CMS, S_TOT_CMS, S_PER_ATOM_MAX, S_TOT_MAX, S_SC_SIDE, S_SC_OUT, S_TASKS,
        S_TILE_CNT, S_TILE_OFF, S_ROUND_CNT, S_ROUND_OFF, S_BOX_ROUND, S_BOX_BLK, S_SUMMARY, S_EXPORT,
        S_NN_Q, S_NN_R, S_NN_QF4, S_NN_RF4, S_NN_PART, S_NN_BBOX, S_NN_TASK, S_NN_TCNT, S_NN_TOFF, S_NN_RCNT, S_NN_ROFF,
        S_NN_BOXR, S_NN_BOXB, S_NN_D2, S_NN_IDX, S_INFO,
        S_CMS_IDX, S_ADJ_A, S_ADJ_REFDOT, S_ADJ_REFVEC, S_ADJ_RCNT, S_ADJ_RFILL, S_ADJ_ROFF, S_ADJ_RSLOT,
        S_ADJ_GCONV, S_ADJ_GTOR, S_ADJ_GCONC, S_ADJ_GTOT, S_ADJ_GRAD, S_RECOMP_XYZ, S_RECOMP_AREA,
        S_ADJ_ACT_CONV, S_ADJ_ACT_TOR, S_ADJ_ACT_CONC, S_ADJ_ACT_ATOM, S_ADJ_LIST_CONV, S_ADJ_LIST_TOR,
        S_ADJ_LIST_CONC, S_ADJ_NACT, S_OVF, S_REF_XYZ, S_POSE, S_POSE_CKPT, S_POSE_CEN, S_HIST, S_STEP, S_MAXSUM,
        S_TOR_LFLAG, S_TOR_LOFF, S_TOR_LIST, S_PTOP, S_SP_A, S_SP_H, S_SP_XYZ, S_SP_ALT, S_SP_G, S_SP_ORD,
        S_SO_F4_0, S_SO_F4_1, S_SO_PERM_0, S_SO_PERM_1, S_KS_TOP, S_KS_BUF, S_CV_SOFF, S_CC_SOFF, S_TOR_SOFF, S_TOR_SN, S_NBS_TOP, S_NBS_BUF, S_NB_SOFF, S_ADJ_SKEY, S_ADJ_SLIST_CONV, S_ADJ_SLIST_TOR, S_ADJ_SLIST_CONC, S_CS_TOP, S_CS_XYZ, S_CS_AREA, S_CS_OWN,
        S_CS_SUB, S_CS_BUR, S_RES_OFF, S_RES_ATOMS, S_RES_SUM, S_RES_FLAG, S_NN_COUNT, S_PLC_CNT, S_PLC_FILL, S_PLC_START,
        S_PLC_ITEM, S_PLC_CELL, S_TILE_CNT2, S_TILE_OFF2, S_ROUND_CNT2, S_ROUND_OFF2, S_BOX_ROUND2,
        S_BOX_BLK2, S_SCAN_TMP2, S_R_SC_D2, S_TOR_GEO, S_CC_GEO, S_CV_GEO,
        S_COUNT
    };

    cms_ctx() : bufs(S_COUNT) {}

    template <class T>
    T* ensure(int slot, long long count)
    {
        size_t need = (size_t)std::max<long long>(count, 1) * sizeof(T);
        DBuf& b = bufs[slot];
        if (b.bytes < need) {
            if (b.p) cudaFree(b.p);
            size_t alloc = need + need / 4;
            b.p = nullptr;
            b.bytes = 0;
            if (cudaMalloc(&b.p, alloc) != cudaSuccess) {
                b.p = nullptr;
                throw std::string("device allocation failed");
            }
            b.bytes = alloc;
        }
        return (T*)b.p;
    }
    template <class T>
    T* get(int slot) { return (T*)bufs[slot].p; }
};

namespace {

struct Fail {
    cms_status code;
    std::string msg;
};

void ck(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw Fail{CMS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

long long read_ll(cms_ctx* x, const long long* dev)
{
    x->d2h_bytes += sizeof(long long);
    ck(cudaMemcpyAsync(x->pinned, dev, sizeof(long long), cudaMemcpyDeviceToHost, x->stream), "readback");
    ck(cudaStreamSynchronize(x->stream), "sync");
    return x->pinned[0];
}

unsigned grid1(long long n) { long long b = (n + 255) / 256; return (unsigned)std::max(1LL, std::min(b, 148LL * 16)); }

// (re)bind every per-atom / per-complex buffer for the current batch
void bind_batch(cms_ctx* x)
{
    const long long N = x->N, B = x->B;
    Dev& d = x->d;
    d.B = x->B;
    d.N = N;
    d.atom_off = x->ensure<int>(cms_ctx::S_ATOM_OFF, B + 1);
    d.n0 = x->ensure<int>(cms_ctx::S_N0, B);
    d.xyzr = x->ensure<double4>(cms_ctx::S_XYZR, N);
    d.dens = x->ensure<double>(cms_ctx::S_DENS, N);
    d.cplx = x->ensure<int>(cms_ctx::S_CPLX, N);
    d.mol = x->ensure<int8_t>(cms_ctx::S_MOL, N);
    d.atten = x->ensure<int8_t>(cms_ctx::S_ATTEN, N);
    d.access = x->ensure<int8_t>(cms_ctx::S_ACCESS, N);
    d.cell_of = x->ensure<int>(cms_ctx::S_CELL_OF, N);
    d.cx = x->ensure<Cplx>(cms_ctx::S_CX, B);
    d.ncell = x->ensure<int>(cms_ctx::S_NCELL, B);
    d.ncell_scan = x->ensure<long long>(cms_ctx::S_NCELL_SCAN, B + 1);
    d.status = x->ensure<int>(cms_ctx::S_STATUS, B);
    d.coin = x->ensure<unsigned long long>(cms_ctx::S_COIN, B);
    d.cell_atom = x->ensure<int>(cms_ctx::S_CELL_ATOM, N);
    d.nnb = x->ensure<int>(cms_ctx::S_NNB, N);
    d.ovf = x->ensure<int>(cms_ctx::S_OVF, 1);
    d.nb_off = x->ensure<long long>(cms_ctx::S_NB_OFF, N + 1);
    d.nb_soff = x->ensure<long long>(cms_ctx::S_NB_SOFF, N);
    d.nbs_top = x->ensure<unsigned long long>(cms_ctx::S_NBS_TOP, 1);
    d.nbur = x->ensure<int>(cms_ctx::S_NBUR, N);
    d.bu_off = x->ensure<long long>(cms_ctx::S_BU_OFF, N + 1);
    d.ntor = x->ensure<int>(cms_ctx::S_NTOR, N);
    d.tor_off = x->ensure<long long>(cms_ctx::S_TOR_OFF, N + 1);
    d.nplus = x->ensure<int>(cms_ctx::S_NPLUS, N);
    d.plus_off = x->ensure<long long>(cms_ctx::S_PLUS_OFF, N + 1);
    d.nminus = x->ensure<int>(cms_ctx::S_NMINUS, N);
    d.minus_off = x->ensure<long long>(cms_ctx::S_MINUS_OFF, N + 1);
    d.conv_cnt = x->ensure<int>(cms_ctx::S_CONV_CNT, N);
    d.cv_geo = x->ensure<CvGeo>(cms_ctx::S_CV_GEO, N);
    d.conv_off = x->ensure<long long>(cms_ctx::S_CONV_OFF, N + 1);
    d.cv_soff = x->ensure<int>(cms_ctx::S_CV_SOFF, N);
    d.ks_top = x->ensure<unsigned long long>(cms_ctx::S_KS_TOP, 1);
    d.seg = x->ensure<Seg>(cms_ctx::S_SEG, 8 * B);
    d.dot_off = x->ensure<long long>(cms_ctx::S_DOT_OFF, 2 * B + 1);
    d.tor_last1 = x->ensure<unsigned long long>(cms_ctx::S_TOR_LAST1, N);
    d.tor_last2 = x->ensure<unsigned long long>(cms_ctx::S_TOR_LAST2, N);
    x->ensure<int>(cms_ctx::S_CM_TMP, 2 * B + 2);
    x->ensure<double>(cms_ctx::S_PER_ATOM_CMS, N);
    x->ensure<double>(cms_ctx::S_TOT_CMS, 2 * B);
    x->ensure<double>(cms_ctx::S_PER_ATOM_MAX, N);
    x->ensure<double>(cms_ctx::S_TOT_MAX, 2 * B);
    x->ensure<double>(cms_ctx::S_SC_SIDE, 2 * B * SC_SIDE_FIELDS);
    x->ensure<double>(cms_ctx::S_SC_OUT, B * SC_FIELDS);
    x->ensure<NNTask>(cms_ctx::S_TASKS, 3 * 2 * B);
    x->ensure<int>(cms_ctx::S_TILE_CNT, 2 * B);
    x->ensure<long long>(cms_ctx::S_TILE_OFF, 2 * B + 1);
    x->ensure<int>(cms_ctx::S_ROUND_CNT, 2 * B);
    x->ensure<long long>(cms_ctx::S_ROUND_OFF, 2 * B + 1);
    // the second set of search scratch, for the SC searches when they run beside the CMS search
    x->ensure<int>(cms_ctx::S_TILE_CNT2, 2 * B);
    x->ensure<long long>(cms_ctx::S_TILE_OFF2, 2 * B + 1);
    x->ensure<int>(cms_ctx::S_ROUND_CNT2, 2 * B);
    x->ensure<long long>(cms_ctx::S_ROUND_OFF2, 2 * B + 1);
    x->ensure<long long>(cms_ctx::S_SUMMARY, 8);
}

void bind_caps(cms_ctx* x)
{
    Dev& d = x->d;
    Rd& r = x->r;
    d.cells_cap = x->cap_cells;
    d.cell_cnt = x->ensure<int>(cms_ctx::S_CELL_CNT, x->cap_cells);
    d.cell_fill = x->ensure<int>(cms_ctx::S_CELL_FILL, x->cap_cells);
    d.cell_start = x->ensure<long long>(cms_ctx::S_CELL_START, x->cap_cells + 1);
    d.nb_cap = x->cap_nb;
    d.bu_cap = x->cap_bu;
    d.nb_id = x->ensure<int>(cms_ctx::S_NB_ID, x->cap_nb);
    d.nb_tmp = x->ensure<int>(cms_ctx::S_NB_TMP, x->cap_nb);
    d.nb_d2 = x->ensure<double>(cms_ctx::S_NB_D2, x->cap_nb);
    d.bu_id = x->ensure<int>(cms_ctx::S_BU_ID, x->cap_bu);
    d.nbs_cap = x->cap_nb + x->cap_bu;
    d.nbs_buf = x->ensure<int>(cms_ctx::S_NBS_BUF, d.nbs_cap);
    d.tor_cap = x->cap_tor;
    d.tor_i = x->ensure<int>(cms_ctx::S_TOR_I, x->cap_tor);
    d.tor_geo = x->ensure<TorGeo>(cms_ctx::S_TOR_GEO, x->cap_tor);
    d.tor_j = x->ensure<int>(cms_ctx::S_TOR_J, x->cap_tor);
    d.tor1_cnt = x->ensure<int>(cms_ctx::S_TOR1_CNT, x->cap_tor);
    d.tor2_cnt = x->ensure<int>(cms_ctx::S_TOR2_CNT, x->cap_tor);
    d.tor1_off = x->ensure<long long>(cms_ctx::S_TOR1_OFF, x->cap_tor + 1);
    d.tor2_off = x->ensure<long long>(cms_ctx::S_TOR2_OFF, x->cap_tor + 1);
    d.tor_has = x->ensure<int8_t>(cms_ctx::S_TOR_HAS, x->cap_tor);
    d.tor_lflag = x->ensure<int>(cms_ctx::S_TOR_LFLAG, x->cap_tor);
    d.tor_soff = x->ensure<int>(cms_ctx::S_TOR_SOFF, x->cap_tor);
    d.tor_sn = x->ensure<int>(cms_ctx::S_TOR_SN, x->cap_tor);
    d.tor_loff = x->ensure<long long>(cms_ctx::S_TOR_LOFF, x->cap_tor + 1);
    d.tor_list = x->ensure<int>(cms_ctx::S_TOR_LIST, x->cap_tor);
    d.probe_cap = x->cap_probe;
    d.pa0 = x->ensure<int>(cms_ctx::S_PA0, x->cap_probe);
    d.pa1 = x->ensure<int>(cms_ctx::S_PA1, x->cap_probe);
    d.pa2 = x->ensure<int>(cms_ctx::S_PA2, x->cap_probe);
    d.ph = x->ensure<double>(cms_ctx::S_PH, x->cap_probe);
    d.pxyz = x->ensure<double>(cms_ctx::S_PXYZ, 3 * x->cap_probe);
    d.palt = x->ensure<double>(cms_ctx::S_PALT, 3 * x->cap_probe);
    d.plow_flag = x->ensure<int>(cms_ctx::S_PLOW_FLAG, x->cap_probe);
    d.plow_off = x->ensure<long long>(cms_ctx::S_PLOW_OFF, x->cap_probe + 1);
    d.plow_list = x->ensure<int>(cms_ctx::S_PLOW_LIST, x->cap_probe);
    d.plc_cnt = x->ensure<int>(cms_ctx::S_PLC_CNT, x->cap_cells);
    d.plc_fill = x->ensure<int>(cms_ctx::S_PLC_FILL, x->cap_cells);
    d.plc_start = x->ensure<long long>(cms_ctx::S_PLC_START, x->cap_cells + 1);
    d.plc_item = x->ensure<int>(cms_ctx::S_PLC_ITEM, x->cap_probe);
    d.plc_cell = x->ensure<int>(cms_ctx::S_PLC_CELL, x->cap_probe);
    d.ptop = x->ensure<unsigned long long>(cms_ctx::S_PTOP, 1);
    d.sp_a = x->ensure<int>(cms_ctx::S_SP_A, 3 * x->cap_probe);
    d.sp_h = x->ensure<double>(cms_ctx::S_SP_H, x->cap_probe);
    d.sp_xyz = x->ensure<double>(cms_ctx::S_SP_XYZ, 3 * x->cap_probe);
    d.sp_alt = x->ensure<double>(cms_ctx::S_SP_ALT, 3 * x->cap_probe);
    d.sp_g = x->ensure<int>(cms_ctx::S_SP_G, x->cap_probe);
    d.sp_ord = x->ensure<unsigned>(cms_ctx::S_SP_ORD, x->cap_probe);
    d.conc_cnt = x->ensure<int>(cms_ctx::S_CONC_CNT, x->cap_probe);
    d.cc_geo = x->ensure<ConcGeo>(cms_ctx::S_CC_GEO, x->cap_probe);
    d.conc_off = x->ensure<long long>(cms_ctx::S_CONC_OFF, x->cap_probe + 1);
    d.cc_soff = x->ensure<int>(cms_ctx::S_CC_SOFF, x->cap_probe);
    d.cs_cap = x->cap_conc;
    d.cs_top = x->ensure<unsigned long long>(cms_ctx::S_CS_TOP, 1);
    d.cs_xyz = x->ensure<double>(cms_ctx::S_CS_XYZ, 3 * x->cap_conc);
    d.cs_area = x->ensure<double>(cms_ctx::S_CS_AREA, x->cap_conc);
    d.cs_own = x->ensure<int>(cms_ctx::S_CS_OWN, x->cap_conc);
    d.cs_sub = x->ensure<int>(cms_ctx::S_CS_SUB, x->cap_conc);
    d.cs_bur = x->ensure<int8_t>(cms_ctx::S_CS_BUR, x->cap_conc);
    d.dot_cap = x->cap_dot;
    const long long D = x->cap_dot;
    d.dxyz = x->ensure<double>(cms_ctx::S_DXYZ, 3 * D);
    d.ks_cap = D;
    d.ks_buf = x->ensure<int>(cms_ctx::S_KS_BUF, D);
    d.dnml = x->ensure<double>(cms_ctx::S_DNML, 3 * D);
    d.darea = x->ensure<double>(cms_ctx::S_DAREA, D);
    d.dbur = x->ensure<int8_t>(cms_ctx::S_DBUR, D);
    d.dtype = x->ensure<int8_t>(cms_ctx::S_DTYPE, D);
    d.datom = x->ensure<int>(cms_ctx::S_DATOM, D);
    d.dunit = x->ensure<int>(cms_ctx::S_DUNIT, D);
    d.dsub = x->ensure<int>(cms_ctx::S_DSUB, D);
    r.flag = x->ensure<int>(cms_ctx::S_R_FLAG, D);
    r.bur_scan = x->ensure<long long>(cms_ctx::S_R_BUR_SCAN, D + 1);
    r.bur_idx = x->ensure<int>(cms_ctx::S_R_BUR_IDX, D);
    r.bur_f4 = x->ensure<float4>(cms_ctx::S_R_BUR_F4, D);
    r.bur_cm = x->ensure<int>(cms_ctx::S_R_BUR_CM, D);
    r.acc_idx = x->ensure<int>(cms_ctx::S_R_ACC_IDX, D);
    r.acc_f4 = x->ensure<float4>(cms_ctx::S_R_ACC_F4, D);
    r.keep = x->ensure<int>(cms_ctx::S_R_KEEP, D);
    r.trim_scan = x->ensure<long long>(cms_ctx::S_R_TRIM_SCAN, D + 1);
    r.trim_idx = x->ensure<int>(cms_ctx::S_R_TRIM_IDX, D);
    r.trim_f4 = x->ensure<float4>(cms_ctx::S_R_TRIM_F4, D);
    r.nn_d2 = x->ensure<double>(cms_ctx::S_R_NN_D2, D);
    r.nn_idx = x->ensure<int>(cms_ctx::S_R_NN_IDX, D);
    x->ensure<int>(cms_ctx::S_CMS_IDX, D);
    r.val = x->ensure<double>(cms_ctx::S_R_VAL, D);
    r.own = x->ensure<int>(cms_ctx::S_R_OWN, D);
    r.so_f4[0] = x->ensure<float4>(cms_ctx::S_SO_F4_0, D);
    r.so_f4[1] = x->ensure<float4>(cms_ctx::S_SO_F4_1, D);
    r.so_perm[0] = x->ensure<int>(cms_ctx::S_SO_PERM_0, D);
    r.so_perm[1] = x->ensure<int>(cms_ctx::S_SO_PERM_1, D);
    // search boxes: every search's references are a subset of the dots
    const long long rounds = nn_round_cap(D, 2LL * x->B);
    x->ensure<float4>(cms_ctx::S_BOX_ROUND, 2 * rounds);
    x->ensure<float4>(cms_ctx::S_BOX_BLK, 2 * rounds * (NN_ROUND / 32));
    long long mx = std::max({x->N + 1, x->cap_cells + 1, x->cap_tor + 1, x->cap_probe + 1, D + 1, 2LL * x->B + 2});
    x->ensure<long long>(cms_ctx::S_SCAN_TMP, scan_tmp_elems(mx) + 8);
}

// Buffers of the SC searches when they run beside the CMS search (graph path):
// their own tile / round / box scratch, scan scratch and neighbour distances.
void bind_sc_side(cms_ctx* x)
{
    const long long D = x->cap_dot;
    const long long rounds = nn_round_cap(D, 2LL * x->B);
    x->ensure<float4>(cms_ctx::S_BOX_ROUND2, 2 * rounds);
    x->ensure<float4>(cms_ctx::S_BOX_BLK2, 2 * rounds * (NN_ROUND / 32));
    x->ensure<long long>(cms_ctx::S_SCAN_TMP2, scan_tmp_elems(D + 1) + 8);
    x->ensure<double>(cms_ctx::S_R_SC_D2, D);
}

void set_settings_dev(cms_ctx* x)
{
    x->d.st.rp = x->st.rp; x->d.st.density = x->st.density; x->d.st.band = x->st.band; x->d.st.sep = x->st.sep;
    x->d.st.weight = x->st.weight; x->d.st.bw_dist = x->st.binwidth_dist; x->d.st.bw_norm = x->st.binwidth_norm;
}

long long* scan_tmp(cms_ctx* x) { return x->get<long long>(cms_ctx::S_SCAN_TMP); }

// pipeline stages, in enqueue order (cms_profile_stages reports one time each)
enum Stage {
    P_CELLS, P_ATTENTION, P_NB_COUNT, P_NB_EMIT, P_PAIRS, P_TRIPLES_COUNT, P_TRIPLES_EMIT, P_CONVEX_COUNT,
    P_TOROIDAL_COUNT, P_CONCAVE_COUNT, P_LAYOUT, P_CONVEX_EMIT, P_TOROIDAL_EMIT, P_CONCAVE_EMIT, P_SPLIT,
    P_CMS_NN, P_CMS_SUM, P_SC_BAND_NN, P_SC_ARGMIN_NN, P_SC_STATS, P_MAX_SUM, P_BACKWARD, P_NSTAGES
};

void mark(cms_ctx* x, int stage)
{
    if (!x->profiling) return;
    cudaEvent_t e;
    ck(cudaEventCreate(&e), "event");
    ck(cudaEventRecord(e, x->stream), "event record");
    x->marks.push_back(e);
    x->mark_ids.push_back(stage);
}

// ---------------------------------------------------------------------------
// the pipeline.  sized = true: read each stage's total back and grow the
// buffers to fit (host syncs between stages); sized = false: enqueue every
// stage with the current capacities (capturable in a CUDA graph).
// ---------------------------------------------------------------------------
// headroom of a grown capacity: need / 8 normally; need / 3 while refining
// poses (the surfaces change from step to step inside one captured graph)
static thread_local int t_growth_div = 8;

void grow(long long& cap, long long need)
{
    if (need > cap) cap = need + need / t_growth_div + 64;
}

// The convex, toroidal and concave passes are independent of each other (each
// reads the neighbour lists, the toroid queue or the probes and writes its own
// counts, stash entries and dot segments; the shared kept-candidate buffer is
// handed out by an atomic cursor, and a unit that does not get room is
// recomputed by its emit pass).  Outside the sizing run and stage profiling
// they run concurrently on the context's stream and two side streams (a
// fork / join by events, which a stream capture records as graph branches),
// so the SMs hold the warps of two or three latency-bound kernels at once.
void ensure_side_streams(cms_ctx* x)
{
    if (x->side[0]) return;
    for (int k = 0; k < 2; ++k) {
        ck(cudaStreamCreateWithFlags(&x->side[k], cudaStreamNonBlocking), "side stream");
        ck(cudaEventCreateWithFlags(&x->ev_join[k], cudaEventDisableTiming), "event");
    }
    ck(cudaEventCreateWithFlags(&x->ev_fork, cudaEventDisableTiming), "event");
}

void fork_side(cms_ctx* x)
{
    ck(cudaEventRecord(x->ev_fork, x->stream), "fork");
    for (int k = 0; k < 2; ++k) ck(cudaStreamWaitEvent(x->side[k], x->ev_fork, 0), "fork");
}

void join_side(cms_ctx* x)
{
    for (int k = 0; k < 2; ++k) {
        ck(cudaEventRecord(x->ev_join[k], x->side[k]), "join");
        ck(cudaStreamWaitEvent(x->stream, x->ev_join[k], 0), "join");
    }
}

void enqueue_surface(cms_ctx* x, bool sized)
{
    const bool par_count = !sized && !x->profiling && (x->conc & CMS_CONC_COUNT);
    const bool par_emit = !sized && !x->profiling && (x->conc & CMS_CONC_EMIT);
    if (par_count || par_emit) ensure_side_streams(x);
    Dev& d = x->d;
    cudaStream_t s = x->stream;
    long long* tmp = scan_tmp(x);
    mark(x, -1);
    ck(cudaMemsetAsync(d.status, 0, sizeof(int) * x->B, s), "memset");
    ck(cudaMemsetAsync(d.ovf, 0, sizeof(int), s), "memset");
    launch_setup(d, s);
    scan_counts(d.ncell, d.ncell_scan, d.B, tmp, s);
    if (sized) {
        long long nc = read_ll(x, d.ncell_scan + d.B);
        grow(x->cap_cells, nc);
        bind_caps(x);
        tmp = scan_tmp(x);
    }
    k_cap_check<<<1, 32, 0, s>>>(d.ncell_scan + d.B, nullptr, x->cap_cells, d.ovf);
    launch_cells(d, x->cap_cells, tmp, s);
    mark(x, P_CELLS);
    launch_attention(d, s);
    mark(x, P_ATTENTION);
    ck(cudaMemsetAsync(d.nbs_top, 0, sizeof(unsigned long long), s), "memset");
    launch_neighbor_count(d, s);
    scan_counts(d.nnb, d.nb_off, d.N, tmp, s);
    scan_counts(d.nbur, d.bu_off, d.N, tmp, s);
    mark(x, P_NB_COUNT);
    if (sized) {
        const long long nb0 = x->cap_nb, bu0 = x->cap_bu;
        grow(x->cap_nb, read_ll(x, d.nb_off + d.N));
        grow(x->cap_bu, read_ll(x, d.bu_off + d.N));
        bind_caps(x);
        tmp = scan_tmp(x);
        // the sorted-row buffer may have moved: the emit pass gathers every row again
        if (x->cap_nb != nb0 || x->cap_bu != bu0)
            ck(cudaMemsetAsync(d.nb_soff, 0xff, sizeof(long long) * d.N, s), "memset");
    }
    k_cap_check<<<1, 32, 0, s>>>(d.nb_off + d.N, nullptr, x->cap_nb, d.ovf);
    k_cap_check<<<1, 32, 0, s>>>(d.bu_off + d.N, nullptr, x->cap_bu, d.ovf);
    launch_neighbor_emit(d, s);
    mark(x, P_NB_EMIT);
    launch_pairs(d, false, s);
    scan_counts(d.ntor, d.tor_off, d.N, tmp, s);
    if (sized) {
        grow(x->cap_tor, read_ll(x, d.tor_off + d.N));
        bind_caps(x);
        tmp = scan_tmp(x);
    }
    k_cap_check<<<1, 32, 0, s>>>(d.tor_off + d.N, nullptr, x->cap_tor, d.ovf);
    launch_pairs(d, true, s);
    mark(x, P_PAIRS);
    ck(cudaMemsetAsync(d.ptop, 0, sizeof(unsigned long long), s), "memset");
    launch_triples(d, false, x->sv[4], s);
    scan_counts(d.nplus, d.plus_off, d.N, tmp, s);
    scan_counts(d.nminus, d.minus_off, d.N, tmp, s);
    mark(x, P_TRIPLES_COUNT);
    // the count pass stashed every probe when they fit the capacity it ran with
    bool stashed = true;
    if (sized) {
        const long long need = read_ll(x, d.plus_off + d.N) + read_ll(x, d.minus_off + d.N);
        stashed = need <= x->cap_probe;
        grow(x->cap_probe, need);
        bind_caps(x);
        tmp = scan_tmp(x);
    }
    k_cap_check<<<1, 32, 0, s>>>(d.plus_off + d.N, d.minus_off + d.N, x->cap_probe, d.ovf);
    if (stashed) launch_probe_scatter(d, x->cap_probe, s);
    else launch_triples(d, true, x->sv[4], s);
    launch_low_probes(d, x->cap_probe, tmp, s);
    launch_probe_geo(d, x->cap_probe, s);
    launch_convex_geo(d, s);
    mark(x, P_TRIPLES_EMIT);
    ck(cudaMemsetAsync(d.tor1_cnt, 0, sizeof(int) * x->cap_tor, s), "memset");
    ck(cudaMemsetAsync(d.tor2_cnt, 0, sizeof(int) * x->cap_tor, s), "memset");
    ck(cudaMemsetAsync(d.conc_cnt, 0, sizeof(int) * x->cap_probe, s), "memset");
    ck(cudaMemsetAsync(d.ks_top, 0, sizeof(unsigned long long), s), "memset");
    ck(cudaMemsetAsync(d.cs_top, 0, sizeof(unsigned long long), s), "memset");
    if (par_count) {
        fork_side(x);
        launch_convex(d, false, s);
        launch_toroidal(d, x->cap_tor, false, x->sv[0], x->side[0]);
        launch_concave(d, x->cap_probe, false, x->sv[2], x->side[1]);
        join_side(x);
    } else {
        launch_convex(d, false, s);
        mark(x, P_CONVEX_COUNT);
        launch_toroidal(d, x->cap_tor, false, x->sv[0], s);
        mark(x, P_TOROIDAL_COUNT);
        launch_concave(d, x->cap_probe, false, x->sv[2], s);
        mark(x, P_CONCAVE_COUNT);
    }
    scan_counts(d.conv_cnt, d.conv_off, d.N, tmp, s);
    scan_counts(d.tor1_cnt, d.tor1_off, x->cap_tor, tmp, s);
    scan_counts(d.tor2_cnt, d.tor2_off, x->cap_tor, tmp, s);
    scan_counts(d.conc_cnt, d.conc_off, x->cap_probe, tmp, s);
    launch_layout(d, (long long*)x->get<int>(cms_ctx::S_CM_TMP), tmp, s);
    mark(x, P_LAYOUT);
    if (sized) {
        const long long cap0 = x->cap_dot, conc0 = x->cap_conc;
        grow(x->cap_dot, read_ll(x, d.dot_off + 2LL * d.B));
        grow(x->cap_conc, read_ll(x, d.conc_off + x->cap_probe));
        bind_caps(x);
        tmp = scan_tmp(x);
        if (x->cap_dot != cap0 || x->cap_conc != conc0) {
            // the kept-candidate buffers may have moved: the emit passes recompute every unit
            ck(cudaMemsetAsync(d.cv_soff, 0xff, sizeof(int) * d.N, s), "memset");
            ck(cudaMemsetAsync(d.cc_soff, 0xff, sizeof(int) * x->cap_probe, s), "memset");
            ck(cudaMemsetAsync(d.tor_soff, 0xff, sizeof(int) * x->cap_tor, s), "memset");
        }
    }
    k_cap_check<<<1, 32, 0, s>>>(d.dot_off + 2LL * d.B, nullptr, x->cap_dot, d.ovf);
    if (par_emit) {
        // the toroidal work list's scan is the only user of the scan scratch in this phase
        fork_side(x);
        launch_convex(d, true, s);
        launch_tor_list(d, x->cap_tor, tmp, x->side[0]);
        launch_toroidal(d, x->cap_tor, true, x->sv[1], x->side[0]);
        launch_concave(d, x->cap_probe, true, x->sv[3], x->side[1]);
        join_side(x);
    } else {
        launch_convex(d, true, s);
        mark(x, P_CONVEX_EMIT);
        launch_tor_list(d, x->cap_tor, tmp, s);
        launch_toroidal(d, x->cap_tor, true, x->sv[1], s);
        mark(x, P_TOROIDAL_EMIT);
        launch_concave(d, x->cap_probe, true, x->sv[3], s);
        mark(x, P_CONCAVE_EMIT);
    }
    launch_tor_access(d, x->cap_tor, s);
}

void enqueue_split(cms_ctx* x)
{
    launch_split_buried(x->d, x->r, x->cap_dot, scan_tmp(x), x->stream);
    launch_spatial_order(x->d, x->r, SO_BUR, 0, x->stream);   // the CMS and band searches' lists
    mark(x, P_SPLIT);
}

NNArgs nn_args(cms_ctx* x, int kind, int set = 0)
{
    NNArgs a{};
    a.task = x->get<NNTask>(cms_ctx::S_TASKS) + kind * 2 * x->B;
    a.ntask = 2 * x->B;
    a.tile_cnt = x->get<int>(set ? cms_ctx::S_TILE_CNT2 : cms_ctx::S_TILE_CNT);
    a.tile_off = x->get<long long>(set ? cms_ctx::S_TILE_OFF2 : cms_ctx::S_TILE_OFF);
    a.round_cnt = x->get<int>(set ? cms_ctx::S_ROUND_CNT2 : cms_ctx::S_ROUND_CNT);
    a.round_off = x->get<long long>(set ? cms_ctx::S_ROUND_OFF2 : cms_ctx::S_ROUND_OFF);
    a.box_round = x->get<float4>(set ? cms_ctx::S_BOX_ROUND2 : cms_ctx::S_BOX_ROUND);
    a.box_blk = x->get<float4>(set ? cms_ctx::S_BOX_BLK2 : cms_ctx::S_BOX_BLK);
    a.round_cap = nn_round_cap(x->cap_dot, 2LL * x->B);
    a.ovf = x->d.ovf;
    if (x->counting) {
        unsigned long long* c = x->get<unsigned long long>(cms_ctx::S_NN_COUNT);
        a.pair_count = c + kind;
        a.recheck_count = c + 3 + kind;
    }
    return a;
}

long long tile_cap(cms_ctx* x) { return x->cap_dot / 256 + 2LL * x->B + 1; }

void enqueue_cms(cms_ctx* x)
{
    Dev& d = x->d;
    Rd& r = x->r;
    cudaStream_t s = x->stream;
    long long* tmp = scan_tmp(x);
    NNTask* task = x->get<NNTask>(cms_ctx::S_TASKS);
    launch_tasks(d, r, 0, task, s);
    k_fill_d<<<grid1(x->cap_dot), 256, 0, s>>>(r.nn_d2, x->cap_dot, INFINITY);
    NNArgs a = nn_args(x, 0);
    a.q_f4 = r.so_f4[0]; a.q_perm = r.so_perm[0]; a.q_idx = r.bur_idx;
    a.r_f4 = r.so_f4[0]; a.r_perm = r.so_perm[0]; a.r_idx = r.bur_idx;
    a.q_xyz = a.r_xyz = d.dxyz;
    a.out_d2 = r.nn_d2;
    a.out_idx = x->get<int>(cms_ctx::S_CMS_IDX);       // kept for the adjoint
    launch_nn(a, NN_ARGMIN, x->nn_var[0], tile_cap(x), tmp, s);
    mark(x, P_CMS_NN);
    launch_cms_weights(d, r, x->cap_dot, s);
    launch_per_atom_sum(d, r, false, x->get<double>(cms_ctx::S_PER_ATOM_CMS), s);
    launch_atom_totals(d, x->get<double>(cms_ctx::S_PER_ATOM_CMS), x->get<double>(cms_ctx::S_TOT_CMS), s);
    mark(x, P_CMS_SUM);
}

// SC readout; side = true: on the first side stream with the second set of
// search scratch and its own neighbour distances (beside the CMS search, which
// writes r.nn_d2)
void enqueue_sc(cms_ctx* x, bool side = false)
{
    Dev& d = x->d;
    Rd r = x->r;
    const cudaStream_t s = side ? x->side[0] : x->stream;
    long long* tmp = side ? x->get<long long>(cms_ctx::S_SCAN_TMP2) : scan_tmp(x);
    if (side) r.nn_d2 = x->get<double>(cms_ctx::S_R_SC_D2);
    const int set = side ? 1 : 0;
    NNTask* task = x->get<NNTask>(cms_ctx::S_TASKS);
    launch_tasks(d, r, 1, task + 2 * x->B, s);
    launch_spatial_order(d, r, SO_ACC, 1, s);
    NNArgs a = nn_args(x, 1, set);
    a.q_f4 = r.so_f4[0]; a.q_perm = r.so_perm[0]; a.q_idx = r.bur_idx;
    a.r_f4 = r.so_f4[1]; a.r_perm = r.so_perm[1]; a.r_idx = r.acc_idx;
    a.q_xyz = a.r_xyz = d.dxyz;
    a.out_flag = r.keep;
    a.band_thr64 = x->st.band * x->st.band;
    launch_nn(a, NN_BAND, x->nn_var[1], tile_cap(x), tmp, s);
    mark(x, P_SC_BAND_NN);
    launch_trim_compact(d, r, x->cap_dot, tmp, s);
    launch_tasks(d, r, 2, task + 4 * x->B, s);
    k_fill_d<<<grid1(x->cap_dot), 256, 0, s>>>(r.nn_d2, x->cap_dot, INFINITY);
    k_fill_i<<<grid1(x->cap_dot), 256, 0, s>>>(r.nn_idx, x->cap_dot, -1);
    launch_spatial_order(d, r, SO_TRIM, 1, s);        // the accessible list is no longer needed
    NNArgs b = nn_args(x, 2, set);
    b.q_f4 = r.so_f4[1]; b.q_perm = r.so_perm[1]; b.q_idx = r.trim_idx;
    b.r_f4 = r.so_f4[1]; b.r_perm = r.so_perm[1]; b.r_idx = r.trim_idx;
    b.q_xyz = b.r_xyz = d.dxyz;
    b.out_d2 = r.nn_d2; b.out_idx = r.nn_idx;
    launch_nn(b, NN_ARGMIN, x->nn_var[2], tile_cap(x), tmp, s);
    mark(x, P_SC_ARGMIN_NN);
    launch_sc_stats(d, r, task + 4 * x->B, x->get<double>(cms_ctx::S_SC_SIDE), x->get<double>(cms_ctx::S_SC_OUT), s);
    mark(x, P_SC_STATS);
}

void enqueue_max(cms_ctx* x)
{
    Dev& d = x->d;
    Rd& r = x->r;
    cudaStream_t s = x->stream;
    launch_area_values(d, r, x->cap_dot, s);
    launch_per_atom_sum(d, r, true, x->get<double>(cms_ctx::S_PER_ATOM_MAX), s);
    launch_atom_totals(d, x->get<double>(cms_ctx::S_PER_ATOM_MAX), x->get<double>(cms_ctx::S_TOT_MAX), s);
}

// adjoint buffers, sized to the current capacities
AdjBuf bind_adj(cms_ctx* x)
{
    const long long D = x->cap_dot;
    AdjBuf a{};
    a.A = x->ensure<double4>(cms_ctx::S_ADJ_A, D);
    a.cms_idx = x->get<int>(cms_ctx::S_CMS_IDX);
    a.ref_ent = x->ensure<int>(cms_ctx::S_ADJ_REFDOT, D);
    a.ref_vec = x->ensure<double4>(cms_ctx::S_ADJ_REFVEC, D);
    a.rcnt = x->ensure<int>(cms_ctx::S_ADJ_RCNT, D);
    a.rfill = x->ensure<int>(cms_ctx::S_ADJ_RFILL, D);
    a.roff = x->ensure<long long>(cms_ctx::S_ADJ_ROFF, D + 1);
    a.rslot = x->ensure<int>(cms_ctx::S_ADJ_RSLOT, D);
    a.gconv = x->ensure<double>(cms_ctx::S_ADJ_GCONV, 6 * x->N);
    a.gtor = x->ensure<double>(cms_ctx::S_ADJ_GTOR, 6 * std::max(x->cap_tor, 1LL));
    a.gconc = x->ensure<double>(cms_ctx::S_ADJ_GCONC, 9 * std::max(x->cap_probe, 1LL));
    a.gtot = x->ensure<double>(cms_ctx::S_ADJ_GTOT, x->B);
    const long long T = std::max(x->cap_tor, 1LL), P = std::max(x->cap_probe, 1LL);
    a.act_conv = x->ensure<int>(cms_ctx::S_ADJ_ACT_CONV, x->N);
    a.act_tor = x->ensure<int>(cms_ctx::S_ADJ_ACT_TOR, T);
    a.act_conc = x->ensure<int>(cms_ctx::S_ADJ_ACT_CONC, P);
    a.act_atom = x->ensure<int8_t>(cms_ctx::S_ADJ_ACT_ATOM, x->N);
    a.list_conv = x->ensure<int>(cms_ctx::S_ADJ_LIST_CONV, x->N);
    a.list_tor = x->ensure<int>(cms_ctx::S_ADJ_LIST_TOR, T);
    a.list_conc = x->ensure<int>(cms_ctx::S_ADJ_LIST_CONC, P);
    a.nact = x->ensure<int>(cms_ctx::S_ADJ_NACT, 4);
    a.skey = x->ensure<int>(cms_ctx::S_ADJ_SKEY, 3 * 256);
    a.slist_conv = x->ensure<int>(cms_ctx::S_ADJ_SLIST_CONV, x->N);
    a.slist_tor = x->ensure<int>(cms_ctx::S_ADJ_SLIST_TOR, T);
    a.slist_conc = x->ensure<int>(cms_ctx::S_ADJ_SLIST_CONC, P);
    x->ensure<double>(cms_ctx::S_ADJ_GRAD, 3 * x->N);
    return a;
}

void enqueue_backward(cms_ctx* x)
{
    const AdjBuf a = bind_adj(x);
    launch_adjoint(x->d, x->r, a, x->get<NNTask>(cms_ctx::S_TASKS), x->bwd_side,
                   x->get<double>(cms_ctx::S_ADJ_GRAD), scan_tmp(x), x->stream);
    mark(x, P_BACKWARD);
}

void fill_gtot(cms_ctx* x, const double* g, int where)
{
    double* dst = x->ensure<double>(cms_ctx::S_ADJ_GTOT, x->B);
    if (g) {
        if (where == CMS_HOST) x->h2d_bytes += 8LL * x->B;
        ck(cudaMemcpyAsync(dst, g, sizeof(double) * x->B,
                           where == CMS_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, x->stream), "grad");
    } else {
        k_fill_d<<<grid1(x->B), 256, 0, x->stream>>>(dst, x->B, 1.0);
    }
}

void enqueue_pose_apply(cms_ctx* x)
{
    launch_pose_apply(x->d, x->get<double>(cms_ctx::S_REF_XYZ), x->get<double>(cms_ctx::S_POSE),
                      x->get<double>(cms_ctx::S_POSE_CEN), x->stream);
}

void enqueue_pose_update(cms_ctx* x)
{
    launch_pose_update(x->d, x->get<double>(cms_ctx::S_ADJ_GRAD), x->get<double>(cms_ctx::S_REF_XYZ),
                       x->get<double>(cms_ctx::S_POSE), x->get<double>(cms_ctx::S_POSE_CEN),
                       x->get<double>(cms_ctx::S_TOT_CMS), x->get<double>(cms_ctx::S_HIST),
                       x->get<int>(cms_ctx::S_STEP), x->hist_cap, x->rprm, x->stream);
}

void enqueue_summary(cms_ctx* x)
{
    k_summary<<<1, 32, 0, x->stream>>>(x->d, x->r, x->get<long long>(cms_ctx::S_SUMMARY));
}

// host mirrors of per-complex offsets, status and coincident pairs
void pull_host_state(cms_ctx* x)
{
    const int B = x->B;
    const long long N = x->N;
    cudaStream_t s = x->stream;
    ck(cudaMemcpyAsync(x->pinned, x->get<long long>(cms_ctx::S_SUMMARY), 8 * sizeof(long long),
                       cudaMemcpyDeviceToHost, s), "summary");
    x->h_status.resize(B);
    x->h_coin.resize(B);
    x->h_dot_off.resize(2 * B + 1);
    x->h_seg.resize(8 * B);
    std::vector<Cplx> cx(B);
    ck(cudaMemcpyAsync(x->h_status.data(), x->d.status, sizeof(int) * B, cudaMemcpyDeviceToHost, s), "status");
    ck(cudaMemcpyAsync(x->h_coin.data(), x->d.coin, sizeof(unsigned long long) * B, cudaMemcpyDeviceToHost, s), "coin");
    ck(cudaMemcpyAsync(x->h_dot_off.data(), x->d.dot_off, sizeof(long long) * (2 * B + 1), cudaMemcpyDeviceToHost, s), "dot_off");
    ck(cudaMemcpyAsync(x->h_seg.data(), x->d.seg, sizeof(Seg) * 8 * B, cudaMemcpyDeviceToHost, s), "seg");
    ck(cudaMemcpyAsync(cx.data(), x->d.cx, sizeof(Cplx) * B, cudaMemcpyDeviceToHost, s), "cx");
    ck(cudaStreamSynchronize(s), "sync");
    x->d2h_bytes += 8 * (long long)sizeof(long long) + (long long)B * (sizeof(int) + sizeof(unsigned long long) +
                    8 * sizeof(Seg) + sizeof(Cplx)) + (2LL * B + 1) * (long long)sizeof(long long);
    for (int k = 0; k < 6; ++k) x->tot[k] = x->pinned[k];
    x->info_state = 0;
    x->h_radmax.resize(B);
    for (int c = 0; c < B; ++c) x->h_radmax[c] = cx[c].radmax;
    (void)N;
}

bool over_capacity(cms_ctx* x)
{
    return x->tot[0] > x->cap_cells || x->tot[1] > x->cap_nb || x->tot[2] > x->cap_bu || x->tot[3] > x->cap_tor ||
           x->tot[4] > x->cap_probe || x->tot[5] > x->cap_dot;
}

void run_sized_surface(cms_ctx* x, int all_atoms)
{
    x->d.all_atoms = all_atoms;
    set_settings_dev(x);
    bind_caps(x);
    enqueue_surface(x, true);
    enqueue_split(x);
    enqueue_summary(x);
    pull_host_state(x);
    x->surf_ok = true;
    x->surf_all_atoms = all_atoms;
    x->cms_ok = x->sc_ok = x->max_ok = false;
}

long long host_ll(cms_ctx* x, const long long* dev_ptr)
{
    long long v = 0;
    ck(cudaMemcpy(&v, dev_ptr, sizeof(long long), cudaMemcpyDeviceToHost), "readback");
    return v;
}

cms_status fail(cms_ctx* x, cms_status code, const std::string& m)
{
    if (x) x->err = m;
    return code;
}

#define API_BEGIN try {
#define API_END                                                    \
    }                                                              \
    catch (const Fail& f) { return fail(x, f.code, f.msg); }      \
    catch (const std::string& m) { return fail(x, CMS_ERR_CUDA, m); } \
    catch (...) { return fail(x, CMS_ERR_CUDA, "unknown error"); } \
    return CMS_OK;

void copy_out(cms_ctx* x, void* dst, const void* src, size_t bytes, int where)
{
    if (where == CMS_HOST) x->d2h_bytes += (long long)bytes;
    ck(cudaMemcpyAsync(dst, src, bytes, where == CMS_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                       x->stream), "copy out");
    ck(cudaStreamSynchronize(x->stream), "sync");
}

void need_surface(cms_ctx* x)
{
    if (!x->have_batch) throw Fail{CMS_ERR_STATE, "no batch loaded"};
    if (!x->surf_ok) throw Fail{CMS_ERR_STATE, "surfaces not generated"};
}

void check_complex(cms_ctx* x, int c)
{
    need_surface(x);
    if (c < 0 || c >= x->B) throw Fail{CMS_ERR_ARG, "complex index out of range"};
}

}  // namespace

extern "C" {

const char* cms_version(void) { return "cms_b200 0.1.0 (sm_100a)"; }

int32_t cms_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

const char* cms_last_error(cms_ctx* x) { return x ? x->err.c_str() : "null context"; }

cms_status cms_ctx_create(cms_ctx** out, int device, void* stream)
{
    cms_ctx* x = nullptr;
    if (!out) return CMS_ERR_ARG;
    try {
        x = new cms_ctx();
        x->device = device;
        ck(cudaSetDevice(device), "cudaSetDevice");
        if (stream) {
            x->stream = (cudaStream_t)stream;
        } else {
            ck(cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking), "stream");
            x->own_stream = true;
        }
        ck(cudaMallocHost(&x->pinned, 64 * sizeof(long long)), "pinned");
    } catch (const Fail& f) {
        *out = x;
        return fail(x, f.code, f.msg);
    }
    *out = x;
    return CMS_OK;
}

cms_status cms_ctx_destroy(cms_ctx* x)
{
    if (!x) return CMS_OK;
    cudaSetDevice(x->device);
    if (x->stream) cudaStreamSynchronize(x->stream);
    if (x->gexec) cudaGraphExecDestroy(x->gexec);
    if (x->graph) cudaGraphDestroy(x->graph);
    for (auto& b : x->bufs) if (b.p) cudaFree(b.p);
    if (x->pinned) cudaFreeHost(x->pinned);
    if (x->own_stream && x->stream) cudaStreamDestroy(x->stream);
    for (int k = 0; k < 2; ++k) {
        if (x->side[k]) cudaStreamDestroy(x->side[k]);
        if (x->ev_join[k]) cudaEventDestroy(x->ev_join[k]);
    }
    if (x->ev_fork) cudaEventDestroy(x->ev_fork);
    delete x;
    return CMS_OK;
}

cms_status cms_set_settings(cms_ctx* x, const cms_settings* s)
{
    if (!x || !s) return fail(x, CMS_ERR_ARG, "null argument");
    x->st = *s;
    x->surf_ok = false;
    return CMS_OK;
}

cms_status cms_get_settings(cms_ctx* x, cms_settings* s)
{
    if (!x || !s) return fail(x, CMS_ERR_ARG, "null argument");
    *s = x->st;
    return CMS_OK;
}

cms_status cms_load_batch(cms_ctx* x, int32_t B, const int64_t* atom_off, const int64_t* n_binder, const double* xyz,
                          const double* radius, const double* density, int32_t where)
{
    if (!x) return CMS_ERR_ARG;
    if (B <= 0 || !atom_off || !n_binder || !xyz || !radius) return fail(x, CMS_ERR_ARG, "invalid batch arguments");
    API_BEGIN
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    x->h_off.assign(atom_off, atom_off + B + 1);
    x->h_n0.assign(n_binder, n_binder + B);
    if (x->h_off[0] != 0) throw Fail{CMS_ERR_ARG, "atom_off[0] must be 0"};
    for (int c = 0; c < B; ++c) {
        long long n = x->h_off[c + 1] - x->h_off[c];
        if (n < 0) throw Fail{CMS_ERR_ARG, "atom_off must be non-decreasing"};
        if (n == 0) throw Fail{CMS_ERR_EMPTY, "complex without atoms"};
        if (x->h_n0[c] < 0 || x->h_n0[c] > n) throw Fail{CMS_ERR_ARG, "n_binder out of range"};
    }
    const long long N = x->h_off[B];
    if (N >= (1LL << 31)) throw Fail{CMS_ERR_ARG, "too many atoms in one batch"};
    const bool same_shape = x->have_batch && x->B == B && x->N == N;
    x->B = B;
    x->N = N;
    bind_batch(x);
    cudaStream_t s = x->stream;
    std::vector<int> off32(B + 1), n032(B);
    for (int c = 0; c <= B; ++c) off32[c] = (int)x->h_off[c];
    for (int c = 0; c < B; ++c) n032[c] = (int)x->h_n0[c];
    ck(cudaMemcpyAsync((void*)x->d.atom_off, off32.data(), sizeof(int) * (B + 1), cudaMemcpyHostToDevice, s), "upload");
    ck(cudaMemcpyAsync((void*)x->d.n0, n032.data(), sizeof(int) * B, cudaMemcpyHostToDevice, s), "upload");
    x->h2d_bytes += (long long)sizeof(int) * (2LL * B + 1);
    const double* dxyz = xyz;
    const double* drad = radius;
    const double* ddens = density;
    if (where == CMS_HOST) {
        double* bx = x->ensure<double>(cms_ctx::S_IN_XYZ, 3 * N);
        double* br = x->ensure<double>(cms_ctx::S_IN_RAD, N);
        ck(cudaMemcpyAsync(bx, xyz, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s), "upload xyz");
        ck(cudaMemcpyAsync(br, radius, sizeof(double) * N, cudaMemcpyHostToDevice, s), "upload radius");
        dxyz = bx;
        drad = br;
        x->h2d_bytes += (long long)sizeof(double) * 4 * N;
        if (density) {
            double* bd = x->ensure<double>(cms_ctx::S_IN_DENS, N);
            ck(cudaMemcpyAsync(bd, density, sizeof(double) * N, cudaMemcpyHostToDevice, s), "upload density");
            ddens = bd;
            x->h2d_bytes += (long long)sizeof(double) * N;
        }
    }
    k_pack_atoms<<<grid1(N), 256, 0, s>>>(N, dxyz, drad, ddens, x->st.density, x->d.xyzr, x->d.dens);
    ck(cudaGetLastError(), "pack");
    if (where == CMS_HOST) ck(cudaStreamSynchronize(s), "sync");   // host buffers may be released after return
    x->have_batch = true;
    x->surf_ok = x->cms_ok = x->sc_ok = x->max_ok = x->bwd_ok = false;
    if (!same_shape) {
        x->graph_key[0] = -1;
        if (x->bwd_enabled) fill_gtot(x, nullptr, CMS_DEVICE);    // upstream gradients of ones
    }
    API_END
}

cms_status cms_generate_surfaces(cms_ctx* x, int32_t all_atoms)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    if (!x->have_batch) throw Fail{CMS_ERR_STATE, "no batch loaded"};
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    run_sized_surface(x, all_atoms ? 1 : 0);
    ck(cudaGetLastError(), "surface kernels");
    API_END
}

cms_status cms_contact_ms(cms_ctx* x, double* per_atom, double* totals, int32_t where)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    need_surface(x);
    if (!x->cms_ok) {
        enqueue_cms(x);
        ck(cudaGetLastError(), "cms kernels");
        x->cms_ok = true;
    }
    if (per_atom) copy_out(x, per_atom, x->get<double>(cms_ctx::S_PER_ATOM_CMS), sizeof(double) * x->N, where);
    if (totals) copy_out(x, totals, x->get<double>(cms_ctx::S_TOT_CMS), sizeof(double) * 2 * x->B, where);
    API_END
}

cms_status cms_residue_sums(cms_ctx* x, int32_t values, int64_t n_residues, const int64_t* res_off,
                            int64_t n_entries, const int32_t* res_atoms, double* sums, int32_t where)
{
    if (!x) return CMS_ERR_ARG;
    if (n_residues < 0 || n_entries < 0 || (values != 0 && values != 1) || (n_residues > 0 && (!res_off || !sums)) ||
        (n_entries > 0 && !res_atoms))
        return fail(x, CMS_ERR_ARG, "cms_residue_sums: bad arguments");
    API_BEGIN
    need_surface(x);
    if (values == 0 && !x->cms_ok) {
        enqueue_cms(x);
        ck(cudaGetLastError(), "cms kernels");
        x->cms_ok = true;
    }
    if (values == 1 && !x->max_ok) {
        enqueue_max(x);
        ck(cudaGetLastError(), "max cms kernels");
        x->max_ok = true;
    }
    if (n_residues == 0) return CMS_OK;
    cudaStream_t s = x->stream;
    const long long* doff = (const long long*)res_off;
    const int* datoms = res_atoms;
    double* dsum = sums;
    if (where == CMS_HOST) {
        if (res_off[0] != 0 || res_off[n_residues] != n_entries)
            throw Fail{CMS_ERR_ARG, "cms_residue_sums: offsets must run from 0 to n_entries"};
        long long* o = x->ensure<long long>(cms_ctx::S_RES_OFF, n_residues + 1);
        int* a = x->ensure<int>(cms_ctx::S_RES_ATOMS, n_entries);
        x->h2d_bytes += (long long)(sizeof(long long) * (n_residues + 1) + sizeof(int) * n_entries);
        ck(cudaMemcpyAsync(o, res_off, sizeof(long long) * (n_residues + 1), cudaMemcpyHostToDevice, s), "upload");
        if (n_entries > 0)
            ck(cudaMemcpyAsync(a, res_atoms, sizeof(int) * n_entries, cudaMemcpyHostToDevice, s), "upload");
        doff = o;
        datoms = a;
        dsum = x->ensure<double>(cms_ctx::S_RES_SUM, n_residues);
    }
    int* flag = (int*)(x->pinned + 32);
    int* dflag = x->ensure<int>(cms_ctx::S_RES_FLAG, 1);
    ck(cudaMemsetAsync(dflag, 0, sizeof(int), s), "clear flag");
    const double* vals = x->get<double>(values == 0 ? cms_ctx::S_PER_ATOM_CMS : cms_ctx::S_PER_ATOM_MAX);
    k_residue_sums<<<grid1(n_residues), 256, 0, s>>>(vals, x->N, doff, n_residues, datoms, n_entries, dsum, dflag);
    ck(cudaGetLastError(), "residue sums");
    ck(cudaMemcpyAsync(flag, dflag, sizeof(int), cudaMemcpyDeviceToHost, s), "readback");
    ck(cudaStreamSynchronize(s), "sync");
    if (*flag) throw Fail{CMS_ERR_ARG, "cms_residue_sums: residue offsets or atom indices out of range"};
    if (where == CMS_HOST) copy_out(x, sums, dsum, sizeof(double) * n_residues, CMS_HOST);
    API_END
}

cms_status cms_max_contact_ms(cms_ctx* x, double* per_atom, double* totals, int32_t where)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    need_surface(x);
    if (!x->max_ok) {
        enqueue_max(x);
        ck(cudaGetLastError(), "max cms kernels");
        x->max_ok = true;
    }
    if (per_atom) copy_out(x, per_atom, x->get<double>(cms_ctx::S_PER_ATOM_MAX), sizeof(double) * x->N, where);
    if (totals) {
        std::vector<double> t(2 * x->B), o(x->B);
        copy_out(x, t.data(), x->get<double>(cms_ctx::S_TOT_MAX), sizeof(double) * 2 * x->B, CMS_HOST);
        for (int c = 0; c < x->B; ++c) o[c] = t[2 * c];
        if (where == CMS_HOST) std::memcpy(totals, o.data(), sizeof(double) * x->B);
        else ck(cudaMemcpy(totals, o.data(), sizeof(double) * x->B, cudaMemcpyHostToDevice), "copy");
    }
    API_END
}

cms_status cms_shape_complementarity(cms_ctx* x, double* sc, double* sides, int32_t where)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    need_surface(x);
    if (!x->sc_ok) {
        enqueue_sc(x);
        ck(cudaGetLastError(), "sc kernels");
        x->sc_ok = true;
    }
    if (sc) copy_out(x, sc, x->get<double>(cms_ctx::S_SC_OUT), sizeof(double) * SC_FIELDS * x->B, where);
    if (sides) copy_out(x, sides, x->get<double>(cms_ctx::S_SC_SIDE), sizeof(double) * SC_SIDE_FIELDS * 2 * x->B, where);
    API_END
}

cms_status cms_complex_info_get(cms_ctx* x, int32_t c, cms_complex_info* info)
{
    if (!x || !info) return fail(x, CMS_ERR_ARG, "null argument");
    API_BEGIN
    check_complex(x, c);
    // the whole table is computed on the device once per run (one kernel, one copy)
    const int want_sc = x->sc_ok ? 1 : 0;
    if (x->info_state != (x->sc_ok ? 2 : 1)) {
        cms_complex_info* dinfo = x->ensure<cms_complex_info>(cms_ctx::S_INFO, x->B);
        k_complex_info<<<x->B, 256, 0, x->stream>>>(x->d, x->r, want_sc, dinfo);
        x->h_info.resize(x->B);
        ck(cudaMemcpyAsync(x->h_info.data(), dinfo, sizeof(cms_complex_info) * x->B, cudaMemcpyDeviceToHost,
                           x->stream), "info");
        ck(cudaStreamSynchronize(x->stream), "sync");
        x->info_state = x->sc_ok ? 2 : 1;
    }
    *info = x->h_info[c];
    API_END
}

cms_status cms_export_atoms(cms_ctx* x, int32_t c, int8_t* atten, int8_t* access, int32_t* n_neighbors, int32_t* n_buried)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    check_complex(x, c);
    const long long a0 = x->h_off[c], n = x->h_off[c + 1] - a0;
    if (atten) ck(cudaMemcpy(atten, x->d.atten + a0, n, cudaMemcpyDeviceToHost), "copy");
    if (access) ck(cudaMemcpy(access, x->d.access + a0, n, cudaMemcpyDeviceToHost), "copy");
    if (n_neighbors) ck(cudaMemcpy(n_neighbors, x->d.nnb + a0, 4 * n, cudaMemcpyDeviceToHost), "copy");
    if (n_buried) ck(cudaMemcpy(n_buried, x->d.nbur + a0, 4 * n, cudaMemcpyDeviceToHost), "copy");
    API_END
}

cms_status cms_export_neighbors(cms_ctx* x, int32_t c, int64_t* nb_off, int32_t* nb_id, int64_t* bu_off, int32_t* bu_id)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    check_complex(x, c);
    const long long a0 = x->h_off[c], n = x->h_off[c + 1] - a0;
    std::vector<long long> off(n + 1);
    for (int pass = 0; pass < 2; ++pass) {
        const long long* doff = pass == 0 ? x->d.nb_off : x->d.bu_off;
        const int* did = pass == 0 ? x->d.nb_id : x->d.bu_id;
        int64_t* ooff = pass == 0 ? nb_off : bu_off;
        int32_t* oid = pass == 0 ? nb_id : bu_id;
        ck(cudaMemcpy(off.data(), doff + a0, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost), "copy");
        const long long base = off[0], cnt = off[n] - off[0];
        if (ooff) for (long long i = 0; i <= n; ++i) ooff[i] = off[i] - base;
        if (oid && cnt > 0) {
            ck(cudaMemcpy(oid, did + base, sizeof(int) * cnt, cudaMemcpyDeviceToHost), "copy");
            for (long long i = 0; i < cnt; ++i) oid[i] -= (int32_t)a0;
        }
    }
    API_END
}

cms_status cms_export_toroid(cms_ctx* x, int32_t c, int32_t* atom1, int32_t* atom2, double* uij, double* tij, double* rij,
                             int8_t* between)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    check_complex(x, c);
    const long long a0 = x->h_off[c], a1 = x->h_off[c + 1];
    const long long q0 = host_ll(x, x->d.tor_off + a0), n = host_ll(x, x->d.tor_off + a1) - q0;
    if (n > 0) {
        std::vector<int> ti(n), tj(n);
        ck(cudaMemcpy(ti.data(), x->d.tor_i + q0, sizeof(int) * n, cudaMemcpyDeviceToHost), "copy");
        ck(cudaMemcpy(tj.data(), x->d.tor_j + q0, sizeof(int) * n, cudaMemcpyDeviceToHost), "copy");
        for (long long k = 0; k < n; ++k) {
            if (atom1) atom1[k] = ti[k] - (int)a0;
            if (atom2) atom2[k] = tj[k] - (int)a0;
        }
        double* buf = x->ensure<double>(cms_ctx::S_EXPORT, 8 * n);
        k_export_toroid<<<grid1(n), 256, 0, x->stream>>>(x->d, q0, n, buf);
        std::vector<double> h(8 * n);
        ck(cudaMemcpyAsync(h.data(), buf, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost, x->stream), "copy");
        ck(cudaStreamSynchronize(x->stream), "sync");
        for (long long k = 0; k < n; ++k) {
            const double* o = &h[8 * k];
            if (uij) { uij[3 * k] = o[0]; uij[3 * k + 1] = o[1]; uij[3 * k + 2] = o[2]; }
            if (tij) { tij[3 * k] = o[3]; tij[3 * k + 1] = o[4]; tij[3 * k + 2] = o[5]; }
            if (rij) rij[k] = o[6];
            if (between) between[k] = o[7] != 0.0;
        }
    }
    API_END
}

cms_status cms_export_probes(cms_ctx* x, int32_t c, int32_t* a0, int32_t* a1, int32_t* a2, double* height, double* point,
                             double* alt)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    check_complex(x, c);
    cms_complex_info I;
    cms_status st = cms_complex_info_get(x, c, &I);
    if (st != CMS_OK) return st;
    const long long at0 = x->h_off[c];
    const long long base = host_ll(x, x->d.plus_off + at0) + host_ll(x, x->d.minus_off + at0);
    // device layout [+mol0 | -mol0 | +mol1 | -mol1]; reference order [+mol0 | +mol1 | -mol0 | -mol1]
    const long long pp0 = I.n_probes_plus[0], pm0 = I.n_probes_minus[0], pp1 = I.n_probes_plus[1], pm1 = I.n_probes_minus[1];
    const long long src[4] = {0, pp0 + pm0, pp0, pp0 + pm0 + pp1};
    const long long len[4] = {pp0, pp1, pm0, pm1};
    long long dst = 0;
    for (int b = 0; b < 4; ++b) {
        const long long n = len[b], q = base + src[b];
        if (n > 0) {
            std::vector<int> t(n);
            int32_t* outs[3] = {a0, a1, a2};
            const int* ins[3] = {x->d.pa0, x->d.pa1, x->d.pa2};
            for (int k = 0; k < 3; ++k) {
                if (!outs[k]) continue;
                ck(cudaMemcpy(t.data(), ins[k] + q, sizeof(int) * n, cudaMemcpyDeviceToHost), "copy");
                for (long long i = 0; i < n; ++i) outs[k][dst + i] = t[i] - (int)at0;
            }
            if (height) ck(cudaMemcpy(height + dst, x->d.ph + q, sizeof(double) * n, cudaMemcpyDeviceToHost), "copy");
            if (point) ck(cudaMemcpy(point + 3 * dst, x->d.pxyz + 3 * q, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost), "copy");
            if (alt) ck(cudaMemcpy(alt + 3 * dst, x->d.palt + 3 * q, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost), "copy");
        }
        dst += n;
    }
    API_END
}

cms_status cms_export_dots(cms_ctx* x, int32_t c, int32_t molecule, double* coor, double* outnml, double* area,
                           int8_t* buried, int8_t* type, int32_t* atom_idx)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    check_complex(x, c);
    if (molecule != 0 && molecule != 1) throw Fail{CMS_ERR_ARG, "molecule must be 0 or 1"};
    const long long ds = x->h_dot_off[2 * c + molecule], n = x->h_dot_off[2 * c + molecule + 1] - ds;
    if (n > 0) {
        if (coor) ck(cudaMemcpy(coor, x->d.dxyz + 3 * ds, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost), "copy");
        if (outnml) ck(cudaMemcpy(outnml, x->d.dnml + 3 * ds, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost), "copy");
        if (area) ck(cudaMemcpy(area, x->d.darea + ds, sizeof(double) * n, cudaMemcpyDeviceToHost), "copy");
        if (buried) ck(cudaMemcpy(buried, x->d.dbur + ds, n, cudaMemcpyDeviceToHost), "copy");
        if (type) ck(cudaMemcpy(type, x->d.dtype + ds, n, cudaMemcpyDeviceToHost), "copy");
        if (atom_idx) {
            ck(cudaMemcpy(atom_idx, x->d.datom + ds, sizeof(int) * n, cudaMemcpyDeviceToHost), "copy");
            const int a0 = (int)x->h_off[c];
            for (long long i = 0; i < n; ++i) atom_idx[i] -= a0;
        }
    }
    API_END
}

cms_status cms_export_dot_units(cms_ctx* x, int32_t c, int32_t molecule, int32_t* unit, int32_t* sub)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    check_complex(x, c);
    if (molecule != 0 && molecule != 1) throw Fail{CMS_ERR_ARG, "molecule must be 0 or 1"};
    const long long ds = x->h_dot_off[2 * c + molecule], n = x->h_dot_off[2 * c + molecule + 1] - ds;
    if (n <= 0) return CMS_OK;
    std::vector<int> u(n), sb(n);
    std::vector<int8_t> ty(n);
    ck(cudaMemcpy(u.data(), x->d.dunit + ds, sizeof(int) * n, cudaMemcpyDeviceToHost), "copy");
    ck(cudaMemcpy(sb.data(), x->d.dsub + ds, sizeof(int) * n, cudaMemcpyDeviceToHost), "copy");
    ck(cudaMemcpy(ty.data(), x->d.dtype + ds, n, cudaMemcpyDeviceToHost), "copy");
    cms_complex_info I;
    cms_status st = cms_complex_info_get(x, c, &I);
    if (st != CMS_OK) return st;
    const long long at0 = x->h_off[c];
    const long long q0 = host_ll(x, x->d.tor_off + at0);
    const long long p0 = host_ll(x, x->d.plus_off + at0) + host_ll(x, x->d.minus_off + at0);
    // probes: device blocks [+mol0 | -mol0 | +mol1 | -mol1] -> cms_export_probes order [+mol0 | +mol1 | -mol0 | -mol1]
    const long long pp0 = I.n_probes_plus[0], pm0 = I.n_probes_minus[0], pp1 = I.n_probes_plus[1];
    const long long dev_start[4] = {0, pp0, pp0 + pm0, pp0 + pm0 + pp1};
    const long long ref_start[4] = {0, pp0 + pp1, pp0, pp0 + pp1 + pm0};
    for (long long i = 0; i < n; ++i) {
        long long v = u[i];
        if (ty[i] == 1) v -= at0;
        else if (ty[i] == 2) v -= q0;
        else {
            const long long pl = v - p0;
            int b = 3;
            while (b > 0 && pl < dev_start[b]) --b;
            v = ref_start[b] + (pl - dev_start[b]);
        }
        if (unit) unit[i] = (int32_t)v;
        if (sub) sub[i] = sb[i];
    }
    API_END
}

cms_status cms_export_trimmed(cms_ctx* x, int32_t c, int32_t molecule, int32_t* dot_index)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    check_complex(x, c);
    if (!x->sc_ok) throw Fail{CMS_ERR_STATE, "shape complementarity not computed"};
    const long long ds = x->h_dot_off[2 * c + molecule], de = x->h_dot_off[2 * c + molecule + 1];
    const long long bs = host_ll(x, x->r.bur_scan + ds), be = host_ll(x, x->r.bur_scan + de);
    const long long ts = host_ll(x, x->r.trim_scan + bs), te = host_ll(x, x->r.trim_scan + be);
    if (te > ts && dot_index) {
        ck(cudaMemcpy(dot_index, x->r.trim_idx + ts, sizeof(int) * (te - ts), cudaMemcpyDeviceToHost), "copy");
        for (long long i = 0; i < te - ts; ++i) dot_index[i] -= (int32_t)ds;
    }
    API_END
}

}  // extern "C"

namespace {

// milliseconds per stage from the profiling marks (the events are released)
void take_stage_times(cms_ctx* x, double* ms, int cap)
{
    ck(cudaStreamSynchronize(x->stream), "sync");
    for (int i = 0; i < cap; ++i) ms[i] = 0.0;
    for (size_t k = 1; k < x->marks.size(); ++k) {
        float t = 0.f;
        ck(cudaEventElapsedTime(&t, x->marks[k - 1], x->marks[k]), "elapsed");
        const int id = x->mark_ids[k];
        if (id >= 0 && id < cap) ms[id] += t;
    }
    for (auto e : x->marks) cudaEventDestroy(e);
    x->marks.clear();
    x->mark_ids.clear();
}

// Autotuner: with the surfaces of the loaded batch in place, run the CMS and
// SC readouts once per search shape (each stage timed with events), twice
// over, and keep the fastest shape per stage.  All shapes give the same
// results, so the choice only changes speed.
void autotune_nn(cms_ctx* x)
{
    const long long key[3] = {x->B, x->N, x->cap_dot};
    if (!x->autotune || std::memcmp(key, x->tune_key, sizeof(key)) == 0) return;
    static const int stage[3] = {P_CMS_NN, P_SC_BAND_NN, P_SC_ARGMIN_NN};
    for (int k = 0; k < 3; ++k)
        for (int v = 0; v < NN_VARIANTS; ++v) x->tune_ms[k][v] = INFINITY;
    double ms[P_NSTAGES];
    for (int rep = 0; rep < 2; ++rep) {
        for (int v = 0; v < NN_VARIANTS; ++v) {
            for (int k = 0; k < 3; ++k) x->nn_var[k] = v;
            x->profiling = true;
            try {
                mark(x, -1);
                enqueue_cms(x);
                enqueue_sc(x);
            } catch (...) {
                x->profiling = false;
                throw;
            }
            x->profiling = false;
            take_stage_times(x, ms, P_NSTAGES);
            for (int k = 0; k < 3; ++k) x->tune_ms[k][v] = std::min(x->tune_ms[k][v], ms[stage[k]]);
        }
    }
    for (int k = 0; k < 3; ++k) {
        int best = 0;
        for (int v = 1; v < NN_VARIANTS; ++v)
            if (x->tune_ms[k][v] < x->tune_ms[k][best]) best = v;
        x->nn_var[k] = best;
    }
    std::memcpy(x->tune_key, key, sizeof(key));
    x->cms_ok = x->sc_ok = true;
}

// Autotuner of the surface kernels' shapes: with the buffers sized for the
// loaded batch, generate the surfaces once per shape (every tunable stage
// timed with events), twice over, and keep the fastest shape per stage.
// Every shape generates the same surfaces.
void autotune_surface(cms_ctx* x)
{
    const long long key[3] = {x->B, x->N, x->cap_dot};
    if (!x->autotune || std::memcmp(key, x->tune_key, sizeof(key)) == 0) return;
    static const int stage[SURF_TUNED] = {P_TOROIDAL_COUNT, P_TOROIDAL_EMIT, P_CONCAVE_COUNT, P_CONCAVE_EMIT,
                                          P_TRIPLES_COUNT};
    for (int k = 0; k < SURF_TUNED; ++k)
        for (int v = 0; v < SURF_VARIANTS; ++v) x->sv_ms[k][v] = INFINITY;
    double ms[P_NSTAGES];
    for (int rep = 0; rep < 2; ++rep) {
        for (int v = 0; v < SURF_VARIANTS; ++v) {
            for (int k = 0; k < SURF_TUNED; ++k) x->sv[k] = v;
            x->profiling = true;
            try {
                mark(x, -1);
                enqueue_surface(x, false);
            } catch (...) {
                x->profiling = false;
                throw;
            }
            x->profiling = false;
            take_stage_times(x, ms, P_NSTAGES);
            for (int k = 0; k < SURF_TUNED; ++k) x->sv_ms[k][v] = std::min(x->sv_ms[k][v], ms[stage[k]]);
        }
    }
    for (int k = 0; k < SURF_TUNED; ++k) {
        int best = 0;
        for (int v = 1; v < SURF_VARIANTS; ++v)
            if (x->sv_ms[k][v] < x->sv_ms[k][best]) best = v;
        x->sv[k] = best;
    }
}

// capture the whole batched pipeline into a CUDA graph for the current shape
void capture_graph(cms_ctx* x)
{
    const long long shape[2] = {x->B, x->N};
    const bool new_shape = x->cap_dot == 0 || std::memcmp(shape, x->tune_key, sizeof(shape)) != 0;
    if (new_shape && (x->cap_dot == 0 || x->autotune)) {
        if (x->refine) enqueue_pose_apply(x);
        run_sized_surface(x, 0);                         // size every buffer for this batch
        autotune_surface(x);                             // pick the surface kernels' shapes on it
        autotune_nn(x);                                  // and the search shapes
    }
    const long long key[4] = {x->B, x->N, x->cap_dot, x->refine ? 100 : (x->bwd_enabled ? 1 + x->bwd_side : 0)};
    const long long vk = (x->nn_var[0] << 8) | (x->nn_var[1] << 4) | x->nn_var[2] |
                         ((long long)(x->sv[0] | (x->sv[1] << 2) | (x->sv[2] << 4) | (x->sv[3] << 6) | (x->sv[4] << 8)) << 12);
    if (x->gexec && std::memcmp(key, x->graph_key, sizeof(key)) == 0 && vk == x->graph_vk) return;
    if (x->gexec) { cudaGraphExecDestroy(x->gexec); x->gexec = nullptr; }
    if (x->graph) { cudaGraphDestroy(x->graph); x->graph = nullptr; }
    x->d.all_atoms = 0;
    set_settings_dev(x);
    bind_caps(x);
    if (x->bwd_enabled) bind_adj(x);                    // allocate before capture
    if (x->conc) ensure_side_streams(x);
    if (x->conc & CMS_CONC_READOUT) bind_sc_side(x);
    ck(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        if (x->refine) {
            // one refinement step: pose -> surfaces -> CMS -> gradient -> pose step
            enqueue_pose_apply(x);
            enqueue_surface(x, false);
            enqueue_split(x);
            enqueue_cms(x);
            enqueue_backward(x);
            enqueue_pose_update(x);
            enqueue_summary(x);
            launch_track_max(x->get<long long>(cms_ctx::S_SUMMARY), x->get<long long>(cms_ctx::S_MAXSUM), x->stream);
        } else {
            enqueue_surface(x, false);
            enqueue_split(x);
            if (x->conc & CMS_CONC_READOUT) {
                // the SC searches beside the CMS search and its adjoint
                fork_side(x);
                enqueue_sc(x, true);
                enqueue_cms(x);
                if (x->bwd_enabled) enqueue_backward(x);
                join_side(x);
            } else {
                enqueue_cms(x);
                enqueue_sc(x);
                if (x->bwd_enabled) enqueue_backward(x);
            }
            enqueue_summary(x);
        }
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(x->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    ck(cudaStreamEndCapture(x->stream, &x->graph), "end capture");
    ck(cudaGraphInstantiate(&x->gexec, x->graph, 0), "instantiate");
    size_t nn = 0;
    ck(cudaGraphGetNodes(x->graph, nullptr, &nn), "nodes");
    std::vector<cudaGraphNode_t> nodes(nn);
    ck(cudaGraphGetNodes(x->graph, nodes.data(), &nn), "nodes");
    long long kernels = 0;
    for (auto& n : nodes) {
        cudaGraphNodeType t;
        cudaGraphNodeGetType(n, &t);
        if (t == cudaGraphNodeTypeKernel) ++kernels;
    }
    x->launches = kernels;
    std::memcpy(x->graph_key, key, sizeof(key));
    x->graph_vk = vk;
}

void mark_graph_results(cms_ctx* x)
{
    x->surf_ok = true;
    x->surf_all_atoms = 0;
    x->cms_ok = x->sc_ok = true;
    x->bwd_ok = x->bwd_enabled != 0;
    x->max_ok = false;
}

}  // namespace

extern "C" {

cms_status cms_run_graph(cms_ctx* x)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    if (!x->have_batch) throw Fail{CMS_ERR_STATE, "no batch loaded"};
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    capture_graph(x);
    ck(cudaGraphLaunch(x->gexec, x->stream), "graph launch");
    pull_host_state(x);
    if (over_capacity(x)) {
        // a capacity was exceeded: size again and rerun without the graph
        run_sized_surface(x, 0);
        enqueue_cms(x);
        enqueue_sc(x);
        if (x->bwd_enabled) enqueue_backward(x);
        enqueue_summary(x);
        pull_host_state(x);
        x->graph_key[0] = -1;
    }
    mark_graph_results(x);
    API_END
}

cms_status cms_graph_launch(cms_ctx* x)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    if (!x->have_batch) throw Fail{CMS_ERR_STATE, "no batch loaded"};
    capture_graph(x);
    ck(cudaGraphLaunch(x->gexec, x->stream), "graph launch");
    mark_graph_results(x);
    API_END
}

cms_status cms_graph_check(cms_ctx* x)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    pull_host_state(x);
    if (over_capacity(x)) throw Fail{CMS_ERR_CAPACITY, "a workspace capacity was exceeded; rerun cms_run_graph"};
    API_END
}

cms_status cms_nn_work(cms_ctx* x, int64_t* pairs)
{
    if (!x || !pairs) return fail(x, CMS_ERR_ARG, "null argument");
    API_BEGIN
    need_surface(x);
    std::vector<NNTask> t(6 * (size_t)x->B);
    ck(cudaMemcpy(t.data(), x->get<NNTask>(cms_ctx::S_TASKS), sizeof(NNTask) * t.size(), cudaMemcpyDeviceToHost), "copy");
    for (int k = 0; k < 3; ++k) {
        long long s = 0, q = 0;
        for (int i = 0; i < 2 * x->B; ++i) {
            const NNTask& T = t[(size_t)k * 2 * x->B + i];
            s += T.qn * T.rn;
            q += T.qn;
        }
        pairs[2 * k] = s;
        pairs[2 * k + 1] = q;
    }
    API_END
}

cms_status cms_nn_evaluated(cms_ctx* x, int64_t* counts)
{
    if (!x || !counts) return fail(x, CMS_ERR_ARG, "null argument");
    struct Off {
        cms_ctx* x;
        ~Off() { x->counting = false; }
    } off{x};
    API_BEGIN
    need_surface(x);
    unsigned long long* c = x->ensure<unsigned long long>(cms_ctx::S_NN_COUNT, 6);
    ck(cudaMemsetAsync(c, 0, 6 * sizeof(unsigned long long), x->stream), "memset");
    x->counting = true;
    enqueue_cms(x);
    enqueue_sc(x);
    x->counting = false;
    ck(cudaGetLastError(), "counted readouts");
    unsigned long long h[6];
    ck(cudaMemcpyAsync(h, c, sizeof(h), cudaMemcpyDeviceToHost, x->stream), "copy");
    ck(cudaStreamSynchronize(x->stream), "sync");
    for (int k = 0; k < 6; ++k) counts[k] = (int64_t)h[k];
    x->cms_ok = x->sc_ok = true;
    API_END
}

int64_t cms_kernel_launches(cms_ctx* x) { return x ? x->launches : -1; }

cms_status cms_nearest_dots(cms_ctx* x, const double* query_xyz, int64_t n_query, const double* ref_xyz,
                            int64_t n_ref, double* out_d2, int32_t* out_index, int32_t where)
{
    if (!x) return CMS_ERR_ARG;
    if (n_query < 0 || n_ref <= 0 || (n_query > 0 && (!query_xyz || !out_d2)) || !ref_xyz)
        return fail(x, CMS_ERR_ARG, "cms_nearest_dots: need n_ref > 0 and non-null point / output arrays");
    if (n_query + n_ref >= (1LL << 31)) return fail(x, CMS_ERR_ARG, "cms_nearest_dots: too many points");
    API_BEGIN
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    if (n_query == 0) return CMS_OK;
    cudaStream_t s = x->stream;
    const double* q = query_xyz;
    const double* r = ref_xyz;
    if (where == CMS_HOST) {
        double* dq = x->ensure<double>(cms_ctx::S_NN_Q, 3 * n_query);
        double* dr = x->ensure<double>(cms_ctx::S_NN_R, 3 * n_ref);
        ck(cudaMemcpyAsync(dq, query_xyz, sizeof(double) * 3 * n_query, cudaMemcpyHostToDevice, s), "upload");
        ck(cudaMemcpyAsync(dr, ref_xyz, sizeof(double) * 3 * n_ref, cudaMemcpyHostToDevice, s), "upload");
        q = dq;
        r = dr;
    }
    const int pblocks = 256;
    double* part = x->ensure<double>(cms_ctx::S_NN_PART, 6 * pblocks);
    double* bbox = x->ensure<double>(cms_ctx::S_NN_BBOX, 8);
    float4* qf = x->ensure<float4>(cms_ctx::S_NN_QF4, n_query);
    float4* rf = x->ensure<float4>(cms_ctx::S_NN_RF4, n_ref);
    NNTask* task = x->ensure<NNTask>(cms_ctx::S_NN_TASK, 1);
    int* tcnt = x->ensure<int>(cms_ctx::S_NN_TCNT, 1);
    long long* toff = x->ensure<long long>(cms_ctx::S_NN_TOFF, 2);
    int* rcnt = x->ensure<int>(cms_ctx::S_NN_RCNT, 1);
    long long* roff = x->ensure<long long>(cms_ctx::S_NN_ROFF, 2);
    const long long rounds = nn_round_cap(n_ref, 1);
    float4* boxr = x->ensure<float4>(cms_ctx::S_NN_BOXR, 2 * rounds);
    float4* boxb = x->ensure<float4>(cms_ctx::S_NN_BOXB, 2 * rounds * (NN_ROUND / 32));
    double* d2 = where == CMS_HOST ? x->ensure<double>(cms_ctx::S_NN_D2, n_query) : out_d2;
    int* idx = where == CMS_HOST ? x->ensure<int>(cms_ctx::S_NN_IDX, n_query) : out_index;
    if (!idx) idx = x->ensure<int>(cms_ctx::S_NN_IDX, n_query);
    launch_points_setup(q, n_query, r, n_ref, part, pblocks, bbox, qf, rf, task, tcnt, toff, rcnt, roff, s);
    NNArgs a{};
    a.task = task; a.ntask = 1; a.tile_cnt = tcnt; a.tile_off = toff;
    a.round_cnt = rcnt; a.round_off = roff; a.box_round = boxr; a.box_blk = boxb; a.round_cap = rounds;
    a.q_f4 = qf; a.q_idx = nullptr; a.r_f4 = rf; a.r_idx = nullptr;
    a.q_xyz = q; a.r_xyz = r;
    a.out_d2 = d2; a.out_idx = idx;
    launch_nn_kernel(a, NN_ARGMIN, 0, nn_standalone_tile_cap(n_query), s);
    ck(cudaGetLastError(), "nearest-dot kernels");
    if (where == CMS_HOST) {
        ck(cudaMemcpyAsync(out_d2, d2, sizeof(double) * n_query, cudaMemcpyDeviceToHost, s), "copy out");
        if (out_index) ck(cudaMemcpyAsync(out_index, idx, sizeof(int) * n_query, cudaMemcpyDeviceToHost, s), "copy out");
        ck(cudaStreamSynchronize(s), "sync");
    }
    API_END
}

cms_status cms_fp32_peak(cms_ctx* x, double* tflops)
{
    if (!x || !tflops) return fail(x, CMS_ERR_ARG, "null argument");
    API_BEGIN
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    int sms = 0;
    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, x->device), "attribute");
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    float* out = x->ensure<float>(cms_ctx::S_EXPORT, blocks);
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    k_fp32_peak<<<blocks, threads, 0, x->stream>>>(out, 256, 0.999f, 1e-3f);     // warm-up
    ck(cudaEventRecord(e0, x->stream), "event");
    k_fp32_peak<<<blocks, threads, 0, x->stream>>>(out, iters, 0.999f, 1e-3f);
    ck(cudaEventRecord(e1, x->stream), "event");
    ck(cudaEventSynchronize(e1), "sync");
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
    *tflops = flops / (ms * 1e-3) / 1e12;
    API_END
}

cms_status cms_transfer_bytes(cms_ctx* x, int64_t* h2d, int64_t* d2h)
{
    if (!x) return CMS_ERR_ARG;
    if (h2d) *h2d = x->h2d_bytes;
    if (d2h) *d2h = x->d2h_bytes;
    return CMS_OK;
}

static const char* k_stage_names[P_NSTAGES] = {
    "cells", "attention", "neighbor_count", "neighbor_emit", "pairs", "triples_count", "triples_emit",
    "convex_count", "toroidal_count", "concave_count", "layout", "convex_emit", "toroidal_emit", "concave_emit",
    "split_buried", "cms_nn", "cms_sum", "sc_band_nn", "sc_argmin_nn", "sc_stats", "max_sum", "cms_backward"};

const char* cms_stage_name(int32_t stage)
{
    return (stage >= 0 && stage < P_NSTAGES) ? k_stage_names[stage] : "";
}

cms_status cms_profile_stages(cms_ctx* x, double* ms, int32_t cap, int32_t* n_stages)
{
    if (!x || !ms) return fail(x, CMS_ERR_ARG, "null argument");
    API_BEGIN
    if (!x->have_batch) throw Fail{CMS_ERR_STATE, "no batch loaded"};
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    if (x->cap_dot == 0) run_sized_surface(x, 0);
    x->d.all_atoms = 0;
    set_settings_dev(x);
    bind_caps(x);
    if (x->bwd_enabled) bind_adj(x);
    x->profiling = true;
    try {
        enqueue_surface(x, false);
        enqueue_split(x);
        enqueue_cms(x);
        enqueue_sc(x);
        if (x->bwd_enabled) enqueue_backward(x);
        enqueue_summary(x);
    } catch (...) {
        x->profiling = false;
        throw;
    }
    x->profiling = false;
    take_stage_times(x, ms, cap);
    if (n_stages) *n_stages = P_NSTAGES;
    pull_host_state(x);
    x->surf_ok = x->cms_ok = x->sc_ok = true;
    x->bwd_ok = x->bwd_enabled != 0;
    x->max_ok = false;
    API_END
}

cms_status cms_refine_begin(cms_ctx* x, const double* ref_xyz, int32_t max_steps, int32_t where)
{
    if (!x || !ref_xyz || max_steps < 0) return fail(x, CMS_ERR_ARG, "bad argument");
    API_BEGIN
    if (!x->have_batch) throw Fail{CMS_ERR_STATE, "no batch loaded"};
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    cudaStream_t s = x->stream;
    double* ref = x->ensure<double>(cms_ctx::S_REF_XYZ, 3 * x->N);
    if (where == CMS_HOST) x->h2d_bytes += 24LL * x->N;
    ck(cudaMemcpyAsync(ref, ref_xyz, sizeof(double) * 3 * x->N,
                       where == CMS_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s), "reference pose");
    double* cen = x->ensure<double>(cms_ctx::S_POSE_CEN, 3 * x->B);
    launch_pose_centroid(x->d, ref, cen, s);
    std::vector<double> id(12 * (size_t)x->B, 0.0);
    for (int c = 0; c < x->B; ++c) id[12 * c] = id[12 * c + 4] = id[12 * c + 8] = 1.0;
    double* pose = x->ensure<double>(cms_ctx::S_POSE, 12 * x->B);
    x->ensure<double>(cms_ctx::S_POSE_CKPT, 12 * x->B);
    ck(cudaMemcpyAsync(pose, id.data(), sizeof(double) * id.size(), cudaMemcpyHostToDevice, s), "pose");
    x->hist_cap = max_steps;
    x->ensure<double>(cms_ctx::S_HIST, std::max(1LL, (long long)max_steps * x->B));
    ck(cudaMemsetAsync(x->ensure<int>(cms_ctx::S_STEP, 1), 0, sizeof(int), s), "step");
    x->ensure<long long>(cms_ctx::S_MAXSUM, 8);
    ck(cudaStreamSynchronize(s), "sync");
    x->refine = true;
    x->bwd_enabled = 1;
    x->bwd_side = 1;
    fill_gtot(x, nullptr, CMS_DEVICE);
    x->graph_key[0] = -1;
    x->tune_key[0] = -1;
    x->cap_dot = 0;                                      // size again with refinement headroom
    API_END
}

cms_status cms_refine_set_params(cms_ctx* x, double eta_t, double eta_w, double max_t, double max_w)
{
    if (!x || !(eta_t >= 0) || !(eta_w >= 0) || !(max_t >= 0) || !(max_w >= 0))
        return fail(x, CMS_ERR_ARG, "step sizes must be non-negative");
    x->rprm = RefineParams{eta_t, eta_w, max_t, max_w};
    x->graph_key[0] = -1;                                // parameters are baked into the captured graph
    return CMS_OK;
}

cms_status cms_refine_run(cms_ctx* x, int32_t steps, double* cms_hist, int32_t where)
{
    if (!x || steps < 0) return fail(x, CMS_ERR_ARG, "bad argument");
    API_BEGIN
    if (!x->refine) throw Fail{CMS_ERR_STATE, "cms_refine_begin first"};
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    cudaStream_t s = x->stream;
    const int B = x->B;
    int* step = x->get<int>(cms_ctx::S_STEP);
    int step0 = 0;
    ck(cudaMemcpy(&step0, step, sizeof(int), cudaMemcpyDeviceToHost), "step");
    if (step0 + steps > x->hist_cap) throw Fail{CMS_ERR_ARG, "more steps than cms_refine_begin's max_steps"};
    const int chunk = 25;
    int done = 0, retries = 0;
    t_growth_div = 3;
    try {
        capture_graph(x);                                // size, tune and capture (also for steps = 0)
        while (done < steps) {
            const int n = std::min(chunk, steps - done);
            capture_graph(x);
            // checkpoint: pose and step counter; the chunk's largest stage totals
            ck(cudaMemcpyAsync(x->get<double>(cms_ctx::S_POSE_CKPT), x->get<double>(cms_ctx::S_POSE),
                               sizeof(double) * 12 * B, cudaMemcpyDeviceToDevice, s), "checkpoint");
            ck(cudaMemsetAsync(x->get<long long>(cms_ctx::S_MAXSUM), 0, 8 * sizeof(long long), s), "max");
            int ck_step = 0;
            ck(cudaMemcpyAsync(&ck_step, step, sizeof(int), cudaMemcpyDeviceToHost, s), "step");
            for (int i = 0; i < n; ++i) ck(cudaGraphLaunch(x->gexec, s), "graph launch");
            long long mx[8];
            ck(cudaMemcpyAsync(mx, x->get<long long>(cms_ctx::S_MAXSUM), sizeof(mx), cudaMemcpyDeviceToHost, s), "max");
            ck(cudaStreamSynchronize(s), "sync");
            const bool over = mx[0] > x->cap_cells || mx[1] > x->cap_nb || mx[2] > x->cap_bu || mx[3] > x->cap_tor ||
                              mx[4] > x->cap_probe || mx[5] > x->cap_dot;
            if (over) {
                // a step outgrew the workspace: back to the checkpoint, size for it with headroom, redo
                if (++retries > 8) {
                    char m[256];
                    std::snprintf(m, sizeof(m), "refinement keeps outgrowing its workspace (need/capacity: cells "
                                  "%lld/%lld, neighbours %lld/%lld, buried %lld/%lld, pairs %lld/%lld, probes %lld/%lld, "
                                  "dots %lld/%lld)", mx[0], x->cap_cells, mx[1], x->cap_nb, mx[2], x->cap_bu, mx[3],
                                  x->cap_tor, mx[4], x->cap_probe, mx[5], x->cap_dot);
                    throw Fail{CMS_ERR_CAPACITY, m};
                }
                ck(cudaMemcpyAsync(x->get<double>(cms_ctx::S_POSE), x->get<double>(cms_ctx::S_POSE_CKPT),
                                   sizeof(double) * 12 * B, cudaMemcpyDeviceToDevice, s), "restore");
                ck(cudaMemcpyAsync(step, &ck_step, sizeof(int), cudaMemcpyHostToDevice, s), "restore step");
                x->cap_cells = std::max(x->cap_cells, mx[0]); x->cap_nb = std::max(x->cap_nb, mx[1]);
                x->cap_bu = std::max(x->cap_bu, mx[2]); x->cap_tor = std::max(x->cap_tor, mx[3]);
                x->cap_probe = std::max(x->cap_probe, mx[4]); x->cap_dot = std::max(x->cap_dot, mx[5]);
                grow(x->cap_cells, mx[0] + 1); grow(x->cap_nb, mx[1] + 1); grow(x->cap_bu, mx[2] + 1);
                grow(x->cap_tor, mx[3] + 1); grow(x->cap_probe, mx[4] + 1); grow(x->cap_dot, mx[5] + 1);
                x->graph_key[0] = -1;
                continue;
            }
            done += n;
            retries = 0;
        }
    } catch (...) {
        t_growth_div = 8;
        throw;
    }
    t_growth_div = 8;
    pull_host_state(x);
    x->surf_ok = true;
    x->surf_all_atoms = 0;
    x->cms_ok = x->bwd_ok = true;
    x->sc_ok = x->max_ok = false;
    if (cms_hist && steps > 0) {
        std::vector<double> h((size_t)steps * B);
        ck(cudaMemcpy(h.data(), x->get<double>(cms_ctx::S_HIST) + (long long)step0 * B, sizeof(double) * h.size(),
                      cudaMemcpyDeviceToHost), "history");
        if (where == CMS_HOST) std::memcpy(cms_hist, h.data(), sizeof(double) * h.size());
        else ck(cudaMemcpy(cms_hist, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice), "history");
    }
    API_END
}

cms_status cms_refine_pose(cms_ctx* x, double* rot, double* trans, double* xyz, int32_t where)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    if (!x->refine) throw Fail{CMS_ERR_STATE, "cms_refine_begin first"};
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    const int B = x->B;
    std::vector<double> P(12 * (size_t)B);
    ck(cudaMemcpy(P.data(), x->get<double>(cms_ctx::S_POSE), sizeof(double) * P.size(), cudaMemcpyDeviceToHost), "pose");
    std::vector<double> R(9 * (size_t)B), T(3 * (size_t)B);
    for (int c = 0; c < B; ++c) {
        for (int k = 0; k < 9; ++k) R[9 * c + k] = P[12 * c + k];
        for (int k = 0; k < 3; ++k) T[3 * c + k] = P[12 * c + 9 + k];
    }
    auto put = [&](double* dst, const std::vector<double>& v) {
        if (!dst) return;
        if (where == CMS_HOST) std::memcpy(dst, v.data(), sizeof(double) * v.size());
        else ck(cudaMemcpy(dst, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice), "copy");
    };
    put(rot, R);
    put(trans, T);
    if (xyz) {
        // coordinates of the current poses (the surfaces of the last step are no longer current)
        enqueue_pose_apply(x);
        std::vector<double4> a(x->N);
        ck(cudaMemcpyAsync(a.data(), x->d.xyzr, sizeof(double4) * x->N, cudaMemcpyDeviceToHost, x->stream), "xyz");
        ck(cudaStreamSynchronize(x->stream), "sync");
        std::vector<double> v(3 * (size_t)x->N);
        for (long long g = 0; g < x->N; ++g) { v[3 * g] = a[g].x; v[3 * g + 1] = a[g].y; v[3 * g + 2] = a[g].z; }
        put(xyz, v);
        x->surf_ok = x->cms_ok = x->sc_ok = x->bwd_ok = x->max_ok = false;
    }
    API_END
}

cms_status cms_refine_end(cms_ctx* x)
{
    if (!x) return CMS_ERR_ARG;
    x->refine = false;
    x->bwd_enabled = 0;
    x->graph_key[0] = -1;
    return CMS_OK;
}

cms_status cms_set_nn_variants(cms_ctx* x, const int32_t* variants)
{
    if (!x || !variants) return fail(x, CMS_ERR_ARG, "null argument");
    for (int k = 0; k < 3; ++k)
        if (variants[k] < 0 || variants[k] >= NN_VARIANTS) return fail(x, CMS_ERR_ARG, "search shape out of range");
    for (int k = 0; k < 3; ++k) x->nn_var[k] = variants[k];
    x->autotune = false;
    x->cms_ok = x->sc_ok = false;
    return CMS_OK;
}

cms_status cms_set_surface_variants(cms_ctx* x, const int32_t* variants)
{
    if (!x || !variants) return fail(x, CMS_ERR_ARG, "null argument");
    for (int k = 0; k < SURF_TUNED; ++k)
        if (variants[k] < 0 || variants[k] >= SURF_VARIANTS) return fail(x, CMS_ERR_ARG, "surface shape out of range");
    for (int k = 0; k < SURF_TUNED; ++k) x->sv[k] = variants[k];
    x->autotune = false;
    return CMS_OK;
}

cms_status cms_get_surface_variants(cms_ctx* x, int32_t* variants, double* tune_ms)
{
    if (!x || !variants) return fail(x, CMS_ERR_ARG, "null argument");
    for (int k = 0; k < SURF_TUNED; ++k) variants[k] = x->sv[k];
    if (tune_ms)
        for (int k = 0; k < SURF_TUNED; ++k)
            for (int v = 0; v < SURF_VARIANTS; ++v) tune_ms[k * SURF_VARIANTS + v] = x->sv_ms[k][v];
    return CMS_OK;
}

cms_status cms_set_concurrency(cms_ctx* x, int32_t mode)
{
    if (!x) return CMS_ERR_ARG;
    if (mode < 0 || mode > (CMS_CONC_COUNT | CMS_CONC_EMIT | CMS_CONC_READOUT))
        return fail(x, CMS_ERR_ARG, "concurrency mode outside 0..7");
    x->conc = mode;
    x->graph_key[0] = -1;            // recapture with the new stream layout
    return CMS_OK;
}

cms_status cms_set_autotune(cms_ctx* x, int32_t enable)
{
    if (!x) return CMS_ERR_ARG;
    x->autotune = enable != 0;
    if (x->autotune) x->tune_key[0] = -1;
    return CMS_OK;
}

cms_status cms_get_nn_variants(cms_ctx* x, int32_t* variants, double* tune_ms)
{
    if (!x || !variants) return fail(x, CMS_ERR_ARG, "null argument");
    for (int k = 0; k < 3; ++k) variants[k] = x->nn_var[k];
    if (tune_ms)
        for (int k = 0; k < 3; ++k)
            for (int v = 0; v < NN_VARIANTS; ++v) tune_ms[k * NN_VARIANTS + v] = x->tune_ms[k][v];
    return CMS_OK;
}

cms_status cms_set_backward(cms_ctx* x, int32_t enable, int32_t target_side)
{
    if (!x) return CMS_ERR_ARG;
    API_BEGIN
    x->bwd_enabled = enable ? 1 : 0;
    x->bwd_side = target_side ? 1 : 0;
    x->bwd_ok = false;
    if (x->have_batch) {
        ck(cudaSetDevice(x->device), "cudaSetDevice");
        fill_gtot(x, nullptr, CMS_DEVICE);
    }
    API_END
}

cms_status cms_set_grad_total(cms_ctx* x, const double* grad_total, int32_t where)
{
    if (!x || !grad_total) return fail(x, CMS_ERR_ARG, "null argument");
    API_BEGIN
    if (!x->have_batch) throw Fail{CMS_ERR_STATE, "no batch loaded"};
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    fill_gtot(x, grad_total, where);
    API_END
}

cms_status cms_contact_ms_backward(cms_ctx* x, int32_t target_side, const double* grad_total, double* grad_xyz,
                                   int32_t where)
{
    if (!x || !grad_xyz) return fail(x, CMS_ERR_ARG, "null argument");
    API_BEGIN
    need_surface(x);
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    if (!x->cms_ok) {
        enqueue_cms(x);
        ck(cudaGetLastError(), "cms kernels");
        x->cms_ok = true;
    }
    x->bwd_side = target_side ? 1 : 0;
    fill_gtot(x, grad_total, where);
    enqueue_backward(x);
    ck(cudaGetLastError(), "adjoint kernels");
    x->bwd_ok = true;
    copy_out(x, grad_xyz, x->get<double>(cms_ctx::S_ADJ_GRAD), sizeof(double) * 3 * x->N, where);
    API_END
}

cms_status cms_grad_xyz(cms_ctx* x, double* grad_xyz, int32_t where)
{
    if (!x || !grad_xyz) return fail(x, CMS_ERR_ARG, "null argument");
    API_BEGIN
    if (!x->bwd_ok) throw Fail{CMS_ERR_STATE, "no gradient computed (enable cms_set_backward before the run)"};
    copy_out(x, grad_xyz, x->get<double>(cms_ctx::S_ADJ_GRAD), sizeof(double) * 3 * x->N, where);
    API_END
}

cms_status cms_recompute_dots(cms_ctx* x, int32_t c, int32_t molecule, double* coor, double* area)
{
    if (!x || !coor || !area || molecule < 0 || molecule > 1) return fail(x, CMS_ERR_ARG, "bad argument");
    API_BEGIN
    check_complex(x, c);
    ck(cudaSetDevice(x->device), "cudaSetDevice");
    double* rx = x->ensure<double>(cms_ctx::S_RECOMP_XYZ, 3 * x->cap_dot);
    double* ra = x->ensure<double>(cms_ctx::S_RECOMP_AREA, x->cap_dot);
    launch_recompute(x->d, rx, ra, x->stream);
    ck(cudaGetLastError(), "recompute");
    const long long b = x->h_dot_off[2 * c + molecule], e = x->h_dot_off[2 * c + molecule + 1];
    if (e > b) {
        copy_out(x, coor, rx + 3 * b, sizeof(double) * 3 * (e - b), CMS_HOST);
        copy_out(x, area, ra + b, sizeof(double) * (e - b), CMS_HOST);
    }
    API_END
}

}  // extern "C"
