// Host-side launchers of every kernel of the surface pipeline and the readouts.
#pragma once
#include "cms_internal.cuh"

namespace cms {

// scans (k_scan.cu)
long long scan_tmp_elems(long long n);
void scan_counts(const int* in, long long* out, long long n, long long* tmp, cudaStream_t s);

// surface front half (k_surface.cu)
void launch_setup(const Dev& d, cudaStream_t s);
void launch_cells(const Dev& d, long long n_cells, long long* scan_tmp, cudaStream_t s);
void launch_attention(const Dev& d, cudaStream_t s);
void launch_neighbor_count(const Dev& d, cudaStream_t s);
void launch_neighbor_emit(const Dev& d, cudaStream_t s);
void launch_pairs(const Dev& d, bool emit, cudaStream_t s);
// variant: the autotuned shape: 0 = rows of up to 128 neighbours cached, 1 / 2 = up to 64, registers for 10 / 12 CTAs
void launch_triples(const Dev& d, bool emit, int variant, cudaStream_t s);
void launch_low_probes(const Dev& d, long long probe_cap, long long* scan_tmp, cudaStream_t s);

// dots (k_dots.cu)
void launch_convex(const Dev& d, bool emit, cudaStream_t s);
void launch_probe_geo(const Dev& d, long long probe_grid, cudaStream_t s);
void launch_convex_geo(const Dev& d, cudaStream_t s);
// variant: the autotuned shape (toroidal: 0 = 16 pairs x 4 warps, 1 = 32 pairs x 2 warps per batch / CTA,
// 2 = 16 x 4 with registers for 6 CTAs per SM; concave: registers for 4, 5 or 6 CTAs per SM)
static constexpr int SURF_VARIANTS = 3;
static constexpr int SURF_TUNED = 5;    // toroidal count / emit, concave count / emit, triple count
void launch_toroidal(const Dev& d, long long tor_grid, bool emit, int variant, cudaStream_t s);
void launch_concave(const Dev& d, long long probe_grid, bool emit, int variant, cudaStream_t s);
void launch_layout(const Dev& d, long long* cm_count_tmp, long long* scan_tmp, cudaStream_t s);
void launch_tor_access(const Dev& d, long long tor_grid, cudaStream_t s);
void launch_probe_scatter(const Dev& d, long long probe_grid, cudaStream_t s);
void launch_tor_list(const Dev& d, long long tor_grid, long long* scan_tmp, cudaStream_t s);

}  // namespace cms
