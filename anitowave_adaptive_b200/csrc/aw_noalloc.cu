// aw_noalloc.cu — G2P entry point that allocates no device memory.
//
// aw_g2p stages both grid velocities as ghosted per-block tiles in scratch buffers that the grid
// allocates (cudaMalloc) on first use.  Some callers cannot let a library allocate device memory:
// hosts whose allocator owns every byte of the GPU (a pre-sized pool or a fixed budget checked by
// the caller), code that runs inside a region where cudaMalloc's implicit device-wide
// synchronisation would stall other streams or is not allowed, and callers that must know the
// library's device footprint before the first call.  aw_g2p_noalloc serves them: its scratch is
// one file-scope __device__ array of fixed size, allocated when this module is loaded on a device
// and held by every device that loads it until the process exits.
//
// Limits: at most kMaxBlocks blocks and kMaxTileFloats tile floats per velocity field (the sum over
// active blocks of 3 (r+1) (r+2)^2 rounded up to a multiple of 4); larger grids are rejected with
// AW_ERR_INVALID_ARGUMENT before any work is queued.
//
// Every call shares the array and it keeps the last call's contents.  Nothing in it has to start at
// zero: every word a call reads (tile offsets, tiles of active blocks) is written earlier in the
// same call, in stream order.  Calls that overlap on the GPU (on different streams, or from several
// host threads without ordering) race on the array and give undefined results.
//
// The first call on a device, with that device current, looks up the array's device address
// (cudaGetSymbolAddress, which loads this module on that device) and loads the three kernels the
// call launches; it does so even when it has no particles to transfer.  After it, a call neither
// loads code nor takes device memory.  That first call should come before any stream capture on the
// device.

#include <mutex>

#include "aw_internal.cuh"

namespace {

constexpr uint32_t kMaxBlocks = 1u << 16;      // 65,536 blocks
constexpr uint32_t kMaxTileFloats = 1u << 21;  // 2,097,152 floats (8 MiB) per velocity field

// [0, kMaxBlocks): tile offsets; then the tiles of VELOCITY_* and of VELOCITY_OLD_* (16.25 MiB).
// On the host this name only stands for the array; its device address comes from
// cudaGetSymbolAddress.
__device__ __align__(256) uint32_t g_g2p_scratch[kMaxBlocks + 2 * (size_t)kMaxTileFloats];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
uint32_t* g_scratch_dev[kMaxDevices] = {};

aw_status scratch_on_current_device(uint32_t** out) {
    int dev = 0;
    AW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return aw::set_error(AW_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_g2p_scratch);
        if (e != cudaSuccess || !p)
            return aw::set_error(AW_ERR_CUDA, "cudaGetSymbolAddress of the G2P scratch array failed on device %d: %s",
                                 dev, cudaGetErrorString(e));
        // CUDA loads kernels at their first launch unless asked earlier: load them now, so that no
        // later call loads code or takes device memory
        AW_TRY(aw::preload_g2p_with_tiles());
        g_scratch_dev[dev] = (uint32_t*)p;
    }
    *out = g_scratch_dev[dev];
    return AW_OK;
}

}  // namespace

extern "C" aw_status aw_g2p_noalloc(aw_msbg* g, float* d_vel, const float* d_pos, int64_t n, float alpha,
                                    aw_stream s_) {
    using namespace aw;
    AW_CHECK_ARG(g && ((d_pos && d_vel) || n == 0) && n >= 0, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    MsbgState& G = g->st;
    if ((uint32_t)G.nb > kMaxBlocks)
        return set_error(AW_ERR_INVALID_ARGUMENT, "aw_g2p_noalloc: grid has %d blocks, the static scratch holds %u",
                         G.nb, kMaxBlocks);
    const uint64_t tiles = tile_total(G.h_res);
    if (tiles > kMaxTileFloats)
        return set_error(AW_ERR_INVALID_ARGUMENT,
                         "aw_g2p_noalloc: grid needs %llu tile floats per field, the static scratch holds %u",
                         (unsigned long long)tiles, kMaxTileFloats);
    uint32_t* base = nullptr;
    AW_TRY(scratch_on_current_device(&base));
    if (n == 0) return AW_OK;
    uint32_t* toff = base;
    float* tn = (float*)(base + kMaxBlocks);
    float* to = tn + kMaxTileFloats;
    return g2p_with_tiles(G, d_vel, d_pos, n, alpha, toff, tn, to, (cudaStream_t)s_);
}
