// cms_nearest_dots_noalloc: the brute-force nearest-dot search for callers
// that cannot allocate GPU memory.
//
// Some callers cannot call cudaMalloc: a framework or application that owns
// every device allocation through its own pool (an allocation behind its back
// would bypass its accounting and limits), plugins hosted by such an
// application, and real-time loops that must never meet the allocator's
// implicit device synchronisation.  This entry point gives them the same
// search as cms_nearest_dots without any allocation: the caller passes device
// pointers for inputs and outputs, and the search's scratch (the
// bounding-box partials, the search task, the FP32-packed copies of both
// point sets and the boxes of the reference blocks) lives in one fixed
// file-scope device array.
//
// Contract:
//  - scratch is CMS_NOALLOC_SCRATCH_BYTES (32 MiB) per device, allocated when
//    the library is loaded and held until the process exits; it fits at most
//    CMS_NOALLOC_MAX_POINTS query + reference points per call -- larger
//    inputs are rejected with CMS_ERR_ARG before anything is launched;
//  - the four pointers must be memory a kernel on the current device can
//    read or write: device memory of that device, managed memory, or mapped
//    pinned host memory; anything else (plain pageable host memory, another
//    device's memory) is rejected with CMS_ERR_ARG before anything is
//    launched;
//  - the first call on a device (with that device current) looks up the
//    array's device address once and caches it; make that first call before
//    any stream capture.  The cached address belongs to the device's primary
//    context: calls after a cudaDeviceReset of that device are not supported;
//  - every call on a device shares the one array, and the array keeps the
//    previous call's contents (everything a call reads is written earlier in
//    the same call); calls that overlap on the GPU -- on different streams
//    without ordering between them -- race on it and must be serialised by
//    the caller;
//  - a CUDA error already pending on the calling thread when the call starts
//    is left in place for its owner and the call returns CMS_ERR_CUDA without
//    launching; otherwise CMS_ERR_CUDA reports this call's own launches;
//  - no cudaMalloc, cudaFree or allocating library routine is called.
#include <mutex>

#include "../../include/cms_b200.h"
#include "cms_readout.cuh"

using namespace cms;

#define CMS_NOALLOC_SCRATCH_BYTES (32u << 20)
#define CMS_NOALLOC_HEADER_BYTES (16u << 10)
// 3836 x 512 points: 16 bytes each when packed, plus the reference boxes
// (34 float4 per sub-round of NN_ROUND references, at most MAX/NN_ROUND + 2 sub-rounds)
#define CMS_NOALLOC_MAX_POINTS (3836u * 512u)
#define CMS_NOALLOC_MAX_ROUNDS (CMS_NOALLOC_MAX_POINTS / NN_ROUND + 2u)
#define CMS_NOALLOC_BOX_F4 (2u + 2u * (NN_ROUND / 32))
#define CMS_NOALLOC_PARTIAL_BLOCKS 256
#define CMS_NOALLOC_MAX_DEVICES 64

static_assert(CMS_NOALLOC_HEADER_BYTES + 16ull * CMS_NOALLOC_BOX_F4 * CMS_NOALLOC_MAX_ROUNDS +
                  16ull * CMS_NOALLOC_MAX_POINTS <= CMS_NOALLOC_SCRATCH_BYTES,
              "no-alloc scratch layout exceeds the array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[CMS_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[CMS_NOALLOC_MAX_DEVICES] = {nullptr};

// device address of the scratch array on the current device (looked up once)
cms_status noalloc_scratch(unsigned char** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CMS_ERR_CUDA;
    if (dev < 0 || dev >= CMS_NOALLOC_MAX_DEVICES) return CMS_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CMS_ERR_CUDA;
        g_noalloc_addr[dev] = (unsigned char*)p;
    }
    *out = g_noalloc_addr[dev];
    return CMS_OK;
}

// a kernel on the current device can access p (device memory of this device, managed or mapped pinned memory)
bool noalloc_device_accessible(const void* p)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();          // the query's own error (an unknown pointer), not a launch error
        return false;
    }
    switch (at.type) {
    case cudaMemoryTypeDevice: return at.device == dev;
    case cudaMemoryTypeManaged: return true;
    case cudaMemoryTypeHost: return at.devicePointer == p;
    default: return false;
    }
}

}  // namespace

extern "C" cms_status cms_nearest_dots_noalloc(const double* query_xyz, int64_t n_query, const double* ref_xyz,
                                               int64_t n_ref, double* out_d2, int32_t* out_index, void* stream)
{
    if (n_query < 0 || n_ref <= 0 || !ref_xyz || (n_query > 0 && (!query_xyz || !out_d2))) return CMS_ERR_ARG;
    if ((unsigned long long)n_query + (unsigned long long)n_ref > CMS_NOALLOC_MAX_POINTS) return CMS_ERR_ARG;
    if (n_query == 0) return CMS_OK;
    if (cudaPeekAtLastError() != cudaSuccess) return CMS_ERR_CUDA;
    if (!noalloc_device_accessible(query_xyz) || !noalloc_device_accessible(ref_xyz) ||
        !noalloc_device_accessible(out_d2) || (out_index && !noalloc_device_accessible(out_index)))
        return CMS_ERR_ARG;
    unsigned char* base = nullptr;
    cms_status st = noalloc_scratch(&base);
    if (st != CMS_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    // header: bounding-box partials, box, task, tile count and offsets; then the packed points
    double* partials = (double*)base;
    double* bbox = partials + 6 * CMS_NOALLOC_PARTIAL_BLOCKS;
    NNTask* task = (NNTask*)(bbox + 8);
    int* tile_cnt = (int*)(task + 1);
    long long* tile_off = (long long*)(tile_cnt + 4);
    int* round_cnt = (int*)(tile_off + 2);
    long long* round_off = (long long*)(round_cnt + 4);
    // after the header: the round boxes, the block boxes, then the packed points
    float4* box_round = (float4*)(base + CMS_NOALLOC_HEADER_BYTES);
    float4* box_blk = box_round + 2u * CMS_NOALLOC_MAX_ROUNDS;
    float4* q_f4 = box_round + CMS_NOALLOC_BOX_F4 * CMS_NOALLOC_MAX_ROUNDS;
    float4* r_f4 = q_f4 + n_query;
    launch_points_setup(query_xyz, n_query, ref_xyz, n_ref, partials, CMS_NOALLOC_PARTIAL_BLOCKS, bbox, q_f4, r_f4,
                        task, tile_cnt, tile_off, round_cnt, round_off, s);
    NNArgs a{};
    a.task = task; a.ntask = 1; a.tile_cnt = tile_cnt; a.tile_off = tile_off;
    a.round_cnt = round_cnt; a.round_off = round_off; a.box_round = box_round; a.box_blk = box_blk;
    a.round_cap = CMS_NOALLOC_MAX_ROUNDS;
    a.q_f4 = q_f4; a.q_idx = nullptr; a.r_f4 = r_f4; a.r_idx = nullptr;
    a.q_xyz = query_xyz; a.r_xyz = ref_xyz;
    a.out_d2 = out_d2; a.out_idx = out_index;
    launch_nn_kernel(a, out_index ? NN_ARGMIN : NN_MIN, 0, nn_standalone_tile_cap(n_query), s);
    return cudaGetLastError() == cudaSuccess ? CMS_OK : CMS_ERR_CUDA;
}
