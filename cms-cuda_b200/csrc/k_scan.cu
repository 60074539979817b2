// Device-wide exclusive scan of int32 counts into int64 offsets.
//
// out[i] = sum(in[0..i)), out[n] = total.  Three passes: per-tile sums,
// a single-block scan of the tile sums, and a per-tile rescan that adds the
// tile's offset.  Tiles are 2048 items (256 threads x 8).  Entries past the
// live count must be zero (callers memset capacity-sized count arrays), so
// the scan length can be a capacity known when the work is enqueued.
#include "cms_kernels.cuh"

namespace cms {

static constexpr int SCAN_T = 256;
static constexpr int SCAN_V = 8;
static constexpr int SCAN_TILE = SCAN_T * SCAN_V;

__device__ __forceinline__ long long block_excl_scan(long long v, long long* sh, long long& total)
{
    // warp inclusive scan
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        long long s = lane < (SCAN_T / 32) ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < SCAN_T / 32) sh[lane] = s;
    }
    __syncthreads();
    long long before = (w > 0 ? sh[w - 1] : 0) + x - v;
    total = sh[SCAN_T / 32 - 1];
    __syncthreads();
    return before;
}

__global__ void k_scan_tiles(const int* __restrict__ in, long long n, long long* __restrict__ tile_sum)
{
    __shared__ long long sh[32];
    long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_V;
    long long s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k) {
        long long i = base + k;
        if (i < n) s += in[i];
    }
    long long total;
    block_excl_scan(s, sh, total);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// one block: thread t owns a contiguous run of tile sums, so a single block
// scan covers any tile count
__global__ void k_scan_top(long long* __restrict__ tile_sum, long long ntiles, long long* __restrict__ out_total)
{
    __shared__ long long sh[32];
    const long long per = (ntiles + SCAN_T - 1) / SCAN_T;
    const long long b = (long long)threadIdx.x * per, e = min(b + per, ntiles);
    long long s = 0;
    for (long long i = b; i < e; ++i) s += tile_sum[i];
    long long total;
    long long run = block_excl_scan(s, sh, total);
    for (long long i = b; i < e; ++i) {
        const long long v = tile_sum[i];
        tile_sum[i] = run;
        run += v;
    }
    if (threadIdx.x == 0) *out_total = total;
}

__global__ void k_scan_apply(const int* __restrict__ in, long long n, const long long* __restrict__ tile_off,
                             long long* __restrict__ out)
{
    __shared__ long long sh[32];
    long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_V;
    int v[SCAN_V];
    long long s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k) {
        long long i = base + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    long long total;
    long long ex = block_excl_scan(s, sh, total) + tile_off[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k) {
        long long i = base + k;
        if (i < n) out[i] = ex;
        ex += v[k];
    }
}

long long scan_tmp_elems(long long n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

void scan_counts(const int* in, long long* out, long long n, long long* tmp, cudaStream_t s)
{
    long long ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (ntiles == 0) {
        cudaMemsetAsync(out, 0, sizeof(long long), s);
        return;
    }
    k_scan_tiles<<<(unsigned)ntiles, SCAN_T, 0, s>>>(in, n, tmp);
    k_scan_top<<<1, SCAN_T, 0, s>>>(tmp, ntiles, out + n);
    k_scan_apply<<<(unsigned)ntiles, SCAN_T, 0, s>>>(in, n, tmp, out);
}

}  // namespace cms
