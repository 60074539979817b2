// Rigid-body pose refinement of the binders: the device side of the
// gradient-ascent driver (cms_refine_*).
//
// Per complex the pose is a rotation R (row-major 3x3) and a translation t
// applied to the binder's reference coordinates about their centroid c:
//   x = R (x_ref - c) + c + t, evaluated as x_ref + (R - I)(x_ref - c) + t.
// One refinement step is one captured graph: apply the poses, regenerate the
// surfaces, CMS and its adjoint, then per complex reduce the atom gradients
// to the pose gradient
//   dCMS/dt = sum_i g_i,   dCMS/dw = sum_i (R (x_ref_i - c)) x g_i
// (w: a rotation vector applied on the left, R <- Rot(dw) R) and take a
// clipped ascent step: dt = eta_t g_t, dw = eta_w g_w, each scaled down to at
// most max_t A / max_w radians.  Reductions are fixed-order block trees.
// The reference has no pose driver; the CMS it maximises is
// calc_contact_molecular_surface (cms-cuda/_core.py:946-1004).
#include "cms_readout.cuh"

namespace cms {

static constexpr int RF_T = 256;

// x = R (ref - c) + c + t for binder atoms; target atoms copy their reference
__global__ void k_pose_apply(Dev d, const double* ref, const double* pose, const double* cen)
{
    const int c = blockIdx.x;
    const long long a0 = d.atom_off[c], a1 = d.atom_off[c + 1], nb = a0 + d.n0[c];
    const double* P = pose + 12 * c;
    const double* C = cen + 3 * c;
    for (long long g = a0 + threadIdx.x; g < a1; g += blockDim.x) {
        const double* r = ref + 3 * g;
        double4 x = d.xyzr[g];
        if (g < nb) {
            // x_ref + (R - I)(x_ref - c) + t: exactly x_ref at the identity pose
            const double u = r[0] - C[0], v = r[1] - C[1], w = r[2] - C[2];
            x.x = (r[0] + (((P[0] - 1.0) * u + P[1] * v) + P[2] * w)) + P[9];
            x.y = (r[1] + ((P[3] * u + (P[4] - 1.0) * v) + P[5] * w)) + P[10];
            x.z = (r[2] + ((P[6] * u + P[7] * v) + (P[8] - 1.0) * w)) + P[11];
        } else {
            x.x = r[0]; x.y = r[1]; x.z = r[2];
        }
        d.xyzr[g] = x;
    }
}

__device__ __forceinline__ double rf_block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i];
    return s;
}

// rotation matrix of rotation vector w (Rodrigues)
__device__ __forceinline__ void rot_of(const double* w, double* Rm)
{
    const double th = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    double k[3] = {0.0, 0.0, 0.0};
    if (th > 0.0) { k[0] = w[0] / th; k[1] = w[1] / th; k[2] = w[2] / th; }
    const double s = sin(th), c = cos(th), v = 1.0 - c;
    Rm[0] = c + k[0] * k[0] * v;        Rm[1] = k[0] * k[1] * v - k[2] * s; Rm[2] = k[0] * k[2] * v + k[1] * s;
    Rm[3] = k[1] * k[0] * v + k[2] * s; Rm[4] = c + k[1] * k[1] * v;        Rm[5] = k[1] * k[2] * v - k[0] * s;
    Rm[6] = k[2] * k[0] * v - k[1] * s; Rm[7] = k[2] * k[1] * v + k[0] * s; Rm[8] = c + k[2] * k[2] * v;
}

// pose gradient of the target-side CMS, history entry, ascent step
__global__ void k_pose_update(Dev d, const double* grad, const double* ref, double* pose, const double* cen,
                              const double* totals, double* hist, const int* step, int hist_steps, RefineParams prm)
{
    CMS_EXIT_ON_OVERFLOW(d);
    __shared__ double sh[32];
    const int c = blockIdx.x;
    const long long a0 = d.atom_off[c], nb = a0 + d.n0[c];
    double* P = pose + 12 * c;
    const double* C = cen + 3 * c;
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (long long g = a0 + threadIdx.x; g < nb; g += blockDim.x) {
        const double* r = ref + 3 * g;
        const double u = r[0] - C[0], v = r[1] - C[1], w = r[2] - C[2];
        const double ox = (P[0] * u + P[1] * v) + P[2] * w;
        const double oy = (P[3] * u + P[4] * v) + P[5] * w;
        const double oz = (P[6] * u + P[7] * v) + P[8] * w;
        const double* gg = grad + 3 * g;
        acc[0] += gg[0]; acc[1] += gg[1]; acc[2] += gg[2];
        acc[3] += oy * gg[2] - oz * gg[1];
        acc[4] += oz * gg[0] - ox * gg[2];
        acc[5] += ox * gg[1] - oy * gg[0];
    }
    double tot[6];
    for (int k = 0; k < 6; ++k) tot[k] = rf_block_sum(acc[k], sh);
    if (threadIdx.x != 0) return;
    const int st = *step;
    if (hist && st < hist_steps) hist[(long long)st * d.B + c] = totals[2 * c + 1];
    double dt[3] = {prm.eta_t * tot[0], prm.eta_t * tot[1], prm.eta_t * tot[2]};
    double dw[3] = {prm.eta_w * tot[3], prm.eta_w * tot[4], prm.eta_w * tot[5]};
    const double nt = sqrt(dt[0] * dt[0] + dt[1] * dt[1] + dt[2] * dt[2]);
    const double nw = sqrt(dw[0] * dw[0] + dw[1] * dw[1] + dw[2] * dw[2]);
    if (nt > prm.max_t) for (int k = 0; k < 3; ++k) dt[k] *= prm.max_t / nt;
    if (nw > prm.max_w) for (int k = 0; k < 3; ++k) dw[k] *= prm.max_w / nw;
    if (!(nt == nt) || !(nw == nw)) return;              // a NaN gradient leaves the pose unchanged
    double D[9], Rn[9];
    rot_of(dw, D);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rn[3 * i + j] = (D[3 * i] * P[j] + D[3 * i + 1] * P[3 + j]) + D[3 * i + 2] * P[6 + j];
    for (int k = 0; k < 9; ++k) P[k] = Rn[k];
    for (int k = 0; k < 3; ++k) P[9 + k] += dt[k];
}

__global__ void k_step_inc(int* step) { if (threadIdx.x == 0) *step += 1; }

// running maximum of the stage totals over a chunk of steps (capacity check)
__global__ void k_track_max(const long long* summary, long long* mx)
{
    if (threadIdx.x < 8) mx[threadIdx.x] = max(mx[threadIdx.x], summary[threadIdx.x]);
}

// binder centroids of the reference pose (fixed-order block sum)
__global__ void k_pose_centroid(Dev d, const double* ref, double* cen)
{
    __shared__ double sh[32];
    const int c = blockIdx.x;
    const long long a0 = d.atom_off[c], nb = a0 + d.n0[c];
    double acc[3] = {0.0, 0.0, 0.0};
    for (long long g = a0 + threadIdx.x; g < nb; g += blockDim.x)
        for (int k = 0; k < 3; ++k) acc[k] += ref[3 * g + k];
    for (int k = 0; k < 3; ++k) {
        const double s = rf_block_sum(acc[k], sh);
        if (threadIdx.x == 0) cen[3 * c + k] = nb > a0 ? s / (double)(nb - a0) : 0.0;
    }
}

void launch_pose_apply(const Dev& d, const double* ref, const double* pose, const double* cen, cudaStream_t s)
{
    k_pose_apply<<<d.B, RF_T, 0, s>>>(d, ref, pose, cen);
}

void launch_pose_update(const Dev& d, const double* grad, const double* ref, double* pose, const double* cen,
                        const double* totals, double* hist, int* step, int hist_steps, const RefineParams& prm,
                        cudaStream_t s)
{
    k_pose_update<<<d.B, RF_T, 0, s>>>(d, grad, ref, pose, cen, totals, hist, step, hist_steps, prm);
    k_step_inc<<<1, 32, 0, s>>>(step);
}

void launch_track_max(const long long* summary, long long* mx, cudaStream_t s)
{
    k_track_max<<<1, 32, 0, s>>>(summary, mx);
}

void launch_pose_centroid(const Dev& d, const double* ref, double* cen, cudaStream_t s)
{
    k_pose_centroid<<<d.B, RF_T, 0, s>>>(d, ref, cen);
}

}  // namespace cms
