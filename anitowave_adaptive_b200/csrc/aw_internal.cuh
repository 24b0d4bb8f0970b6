// aw_internal.cuh — internal types and device helpers of the sm_100a FLIP-on-MSBG library.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "anitowave.h"

namespace aw {

// ------------------------------------------------------------------------------------------------
// Errors
// ------------------------------------------------------------------------------------------------
aw_status set_error(aw_status s, const char* fmt, ...);

#define AW_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return ::aw::set_error(AW_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                   __FILE__, __LINE__);                                                \
    } while (0)
// every kernel launch site is followed by AW_LAUNCH(), which also counts the launch
extern unsigned long long g_launches;
#define AW_LAUNCH()                \
    do {                           \
        ++::aw::g_launches;        \
        AW_CUDA(cudaGetLastError()); \
    } while (0)
#define AW_TRY(expr)                     \
    do {                                 \
        aw_status aw_st_ = (expr);        \
        if (aw_st_ != AW_OK) return aw_st_; \
    } while (0)
#define AW_CHECK_ARG(cond, msg)                                             \
    do {                                                                    \
        if (!(cond)) return ::aw::set_error(AW_ERR_INVALID_ARGUMENT, "%s", msg); \
    } while (0)

// ------------------------------------------------------------------------------------------------
// Device buffers
// ------------------------------------------------------------------------------------------------
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    aw_status alloc(size_t count) {
        free();
        if (count == 0) return AW_OK;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return set_error(e == cudaErrorMemoryAllocation ? AW_ERR_OUT_OF_MEMORY : AW_ERR_CUDA,
                             "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
        }
        n = count;
        return AW_OK;
    }
    // Grow-only storage.  A buffer that has to grow again takes a quarter more than asked for: a level
    // map that keeps changing (a spreading liquid) then reallocates a few times instead of at every
    // new layout (each cudaFree synchronises the device).  A first allocation is exact.
    aw_status ensure(size_t count) { return count <= n ? AW_OK : alloc(n == 0 ? count : count + count / 4); }
    void free() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DBuf() { free(); }
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            free();
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
};

// ------------------------------------------------------------------------------------------------
// Kernel-side views
// ------------------------------------------------------------------------------------------------
// Geometry shared by every level.
struct Geo {
    int D[3];
    float bs;
    float dmin[3];
    int R0;
    int L;
    int nb;
};

// One block-structured MG level: per-block resolution and offsets (MSBG.cuh:86-89 layout).
struct LevelView {
    Geo g;
    const int* res;          // cells per edge (0 = block owns nothing at this level)
    const uint32_t* off[4];  // cells, faces x, y, z
};

struct DenseView {
    int D[3];
};

__host__ __device__ inline int bidx(const Geo& g, int x, int y, int z) { return x + g.D[0] * (y + g.D[1] * z); }
__host__ __device__ inline void bcoord(const Geo& g, int b, int c[3]) {
    c[0] = b % g.D[0];
    c[1] = (b / g.D[0]) % g.D[1];
    c[2] = b / (g.D[0] * g.D[1]);
}
__host__ __device__ inline bool inside(const Geo& g, const int c[3]) {
    return c[0] >= 0 && c[1] >= 0 && c[2] >= 0 && c[0] < g.D[0] && c[1] < g.D[1] && c[2] < g.D[2];
}
__host__ __device__ inline uint32_t cidx(int x, int y, int z, int r) { return (uint32_t)(x + r * (y + r * z)); }
// face index maps (MSBG.cuh:169-179)
__host__ __device__ inline uint32_t fidx(int a, int x, int y, int z, int r) {
    return a == 0 ? (uint32_t)(x + (r + 1) * (y + r * z))
                  : (a == 1 ? (uint32_t)(x + r * (y + (r + 1) * z)) : (uint32_t)(x + r * (y + r * z)));
}
__host__ __device__ inline uint32_t didx(const DenseView& d, int i, int j, int k) {
    return (uint32_t)(i + d.D[0] * (j + d.D[1] * k));
}
__host__ __device__ inline uint32_t dfidx(const DenseView& d, int a, int i, int j, int k) {
    return a == 0 ? (uint32_t)(i + (d.D[0] + 1) * (j + d.D[1] * k))
                  : (a == 1 ? (uint32_t)(i + d.D[0] * (j + (d.D[1] + 1) * k)) : (uint32_t)(i + d.D[0] * (j + d.D[1] * k)));
}

// Single-precision block origin and cell size, with the rounding the oracle reproduces.
__device__ inline float forigin(const Geo& g, int a, int c) { return __fadd_rn(g.dmin[a], __fmul_rn((float)c, g.bs)); }
__device__ inline float fcell(const Geo& g, int r) { return __fdiv_rn(g.bs, (float)r); }

// Block of a point (worldToBlockCoord, MSBG.cuh:151-159), clamped into the domain.
__device__ inline void point_block(const Geo& g, const float p[3], int c[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float rel = __fsub_rn(p[a], g.dmin[a]);
        int v = (int)floorf(__fdiv_rn(rel, g.bs));
        c[a] = min(max(v, 0), g.D[a] - 1);
    }
}

// x of one MG level stored either as float or as FP16 with a per-block float scale.
struct XStore {
    float* f = nullptr;        // FP32 storage
    __half* h = nullptr;       // FP16 storage (mixed precision, MG level >= 1)
    float* scale = nullptr;    // per-block scale (FP16 storage)
    __device__ inline float get(uint32_t i, int b) const { return f ? f[i] : __half2float(h[i]) * scale[b]; }
};

// Warp / block reductions
__device__ inline float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ inline double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------------------------------------
// Host-side objects
// ------------------------------------------------------------------------------------------------
// Floats allocated past the six arrays of every SoA particle buffer: G2P's bulk copies round each
// array segment up to 16 bytes and may read up to 3 floats past the last array's end.
constexpr size_t kSoaPad = 16;

struct ParticleWork {
    DBuf<uint32_t> keys, keys2, keys3, perm, perm2, cell_start, cell_fill, tmp, hist, hscan;
    uint32_t* sorted = nullptr;  // sorted slot -> input index (perm or perm2)
    DBuf<float> soa, soa2;  // 6 SoA arrays: px py pz vx vy vz
    int64_t n = 0;
    // The particle arrays the last aw_p2g sorted (caller pointers and count) and 64-bit hashes of
    // their contents then: hash[0] positions, hash[1] velocities; hash[2..3] receive the hashes of
    // the arrays at a later drop-in G2P or advection, which reuses this sort when they match;
    // hash[4..] holds the partial sums of the hashing kernels.
    const float* src_pos = nullptr;
    const float* src_vel = nullptr;
    int64_t src_n = -1;
    bool src_valid = false;
    DBuf<unsigned long long> hash;
    aw_status ensure(int64_t np, uint32_t ncell);
};

struct MsbgState;
// Work buffers of one FLIP step / projection: pressure (FP32 or FP64), right-hand side, fluid
// flags, max |div u| before and after.
struct FlipBufs {
    DBuf<float> p32, rhs, divmax;
    DBuf<double> p64;
    DBuf<uint8_t> fluid;
    bool p_warm = false;  // p32/p64 hold the last step's pressure on the current layout
    aw_status ensure(const MsbgState& G);
};

struct MsbgState {
    aw_grid_desc desc;
    Geo geo;
    int nb = 0;
    DBuf<uint32_t> level;       // refinement map
    DBuf<uint32_t> level_prev;  // the map before a re-derivation (aw_flip_rebuild_levels)
    DBuf<int> res;              // native res per block (0 inactive), after allocate
    DBuf<uint32_t> off[4];      // level-0 offsets
    bool allocated = false;
    uint32_t tot[4] = {0, 0, 0, 0};
    std::vector<uint32_t> h_level;
    std::vector<int> h_res;
    std::vector<uint32_t> h_off[4];
    DBuf<float> slab;                       // all channels in one allocation
    float* ch[AW_NUM_CHANNELS_EXT] = {};    // channel pointers into the slab
    uint32_t ch_count[AW_NUM_CHANNELS_EXT] = {};
    DBuf<uint32_t> scratch_u32;
    DBuf<uint32_t> scratch_scan, scratch_scan_tmp, scratch_off4;  // level_offsets / aw_msbg_allocate
    // ghosted face tiles (per block: 3 axes x (r+1)(r+2)^2, padded to 16 bytes)
    DBuf<uint32_t> tile_off;
    std::vector<uint32_t> h_tile_off;
    uint32_t tile_tot = 0;
    DBuf<float> tiles_new, tiles_old;
    // per block: holds particles (written by P2G), and its u_new tile was written by this step's G2P
    DBuf<uint8_t> blk_busy, tile_ok;
    DBuf<int> blk_order;  // blocks by descending particle count (the per-block kernels' CTA order)
    bool blk_order_on = false;  // blk_order holds this step's order (small grids only)
    DBuf<float> tiles_bar_new, tiles_bar_old;  // adjoint tiles (VJP kernels)
    DBuf<float> adj_u[3], adj_m[3];             // forward P2G recomputed by aw_vjp_p2g
    DBuf<float> p2g_P[3];                       // P2G momentum accumulator when MOMENTUM_* is not asked for
    DBuf<float> p2g_Phi[3];                     // P2G phase accumulator (two-phase P2G)
    DBuf<int> lattice_tab;                      // per-axis lookup tables of aw_resample_cells
    FlipBufs proj;                              // aw_project / aw_vjp_project work buffers
    DBuf<int> err;  // device error flags: [1] bulk-copy wait timeout in G2P / advection ([0] unused)
    bool test_copy_timeout = false;  // next G2P arms its first copy barrier without issuing the copy
    DBuf<uint8_t> occ;
    DBuf<int> flag;
    ParticleWork pw;
    LevelView view0() const {
        LevelView v;
        v.g = geo;
        v.res = res.p;
        for (int k = 0; k < 4; ++k) v.off[k] = off[k].p;
        return v;
    }
};

// Level map from particle positions (element (i, a) at pos[i * si + a * sa]) into G.level; marks the
// grid unallocated.
aw_status levels_from_positions(MsbgState& G, const float* d_pos, int64_t si, int64_t sa, int64_t n,
                                const int32_t* thresholds, cudaStream_t s);

// Re-derives the level map from particle positions and grades it on the device; *changed receives
// the number of blocks whose level differs from the map before (one small read-back, no per-pass
// host synchronisation).  Marks the grid unallocated.
aw_status relevel_on_device(MsbgState& G, const float* d_pos, int64_t si, int64_t sa, int64_t n,
                            const int32_t* thresholds, int* changed, int* passes, cudaStream_t s);

// Rebuilds a solver's multigrid hierarchy for the grid's new layout (after aw_msbg_allocate), in
// the storage it already holds where the new levels fit, and sets it up with every cell fluid.
aw_status solver_relayout(aw_solver* S);

// Exclusive scan of n u32 values into out[0..n] (out[n] = total).  tmp: scan scratch.
aw_status exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, DBuf<uint32_t>& tmp, cudaStream_t s);

// Particle pipeline (aw_particles.cu)
// record: remember the arrays and their hashes for the drop-in G2P / advection (aw_p2g)
aw_status sort_particles_soa(MsbgState& G, const float* pos_aos, const float* vel_aos, int64_t n, cudaStream_t s,
                             bool record = false);
// Two-phase input of P2G: sorted particle i has phase phase[pid[i]] in [0,1]; the face phase goes to
// phi[3] and 1 / ((1 - phi) rho0 + phi rho1) to beta[3].
struct PhaseIn {
    const uint32_t* pid;
    const float* phase;
    float rho0, rho1;
    float* phi[3];
    float* beta[3];
};
aw_status p2g_sorted(MsbgState& G, const float* soa, int64_t n, const uint32_t* cell_start, float* u[3], float* m[3],
                     float* mom[3], float* cell_count, cudaStream_t s, const PhaseIn* ph = nullptr);
// beta at T-junctions: the coarse face and the 4 fine faces it covers all take the mean of the
// 4 fine values, which keeps the finite-volume operator symmetric for variable coefficients
aw_status beta_sync(MsbgState& G, float* beta[3], cudaStream_t s);
aw_status g2p_launch(MsbgState& G, const float* pos, int pos_stride_soa, float* vel, int vel_soa, int64_t n,
                     float alpha, const float* un[3], const float* uo[3], cudaStream_t s);
aw_status g2p_sorted(MsbgState& G, float* soa, int64_t n, const uint32_t* cs, float alpha, const float* un[3],
                     const float* uo[3], cudaStream_t s);
aw_status build_tiles(MsbgState& G, const float* u[3], float* tiles, cudaStream_t s);
aw_status ensure_tiles(MsbgState& G);
aw_status advect_tiles(MsbgState& G, float* pos, int pos_soa, int64_t n, float dt, const float* tiles, cudaStream_t s);
// RK3 of cell-sorted SoA particles through G.tiles_new (built for G2P), one CTA per block; un: the
// face arrays, sampled where G2P wrote no tile (G.tile_ok)
aw_status advect_sorted(MsbgState& G, float* soa, int64_t n, const uint32_t* cs, float dt, const float* un[3],
                        cudaStream_t s);
aw_status check_device_errors(MsbgState& G, cudaStream_t s);
aw_status sort_core_soa(MsbgState& G, const float* soa_pos, int64_t n, cudaStream_t s);
aw_status gather_soa(MsbgState& G, const float* in_soa, int64_t n, float* out_soa, const uint32_t* ids_in,
                     uint32_t* ids_out, cudaStream_t s);
aw_status advect_launch(MsbgState& G, float* pos, int pos_soa, int64_t n, float dt, const float* u[3], cudaStream_t s);
// G2P (same arithmetic as aw_g2p) through caller-provided tile storage: toff holds nb offsets
// (written here), tn and to at least the grid's total tile size in floats each.
aw_status g2p_with_tiles(MsbgState& G, float* d_vel, const float* d_pos, int64_t n, float alpha, uint32_t* toff,
                         float* tn, float* to, cudaStream_t s);
// loads g2p_with_tiles' kernels on the current device ahead of their first launch
aw_status preload_g2p_with_tiles();
// total tile floats of a grid whose blocks have resolutions h_res (one velocity field)
uint64_t tile_total(const std::vector<int>& h_res);
aw_status build_tiles2(MsbgState& G, const float* un[3], const float* uo[3], cudaStream_t s);

// Adjoint of the particle side (aw_particles.cu).  Particle arrays are AoS (soa = 0) or SoA over n.
aw_status ensure_adjoint_tiles(MsbgState& G);
aw_status tile_fold(MsbgState& G, const float* tb, float* ubar[3], cudaStream_t s);
// RK3 (when do_advect) and the FLIP blend of one step: xbar/vbar in -> out; unbar/uobar += (uobar may be null)
aw_status step_particles_vjp(MsbgState& G, const float* pos, int pos_soa, int64_t n, float alpha, float dt,
                             const float* un[3], const float* uo[3], float* xbar, float* vbar, int bar_soa,
                             int do_advect, float* unbar[3], float* uobar[3], cudaStream_t s);
// y = sample(u, pts): ubar += I^T ybar; xbar += (dI/dx)^T ybar when xbar is given
aw_status sample_vjp(MsbgState& G, const float* pts, int pts_soa, int64_t n, const float* u[3], const float* ybar,
                     int ybar_soa, float* ubar[3], float* xbar, cudaStream_t s);
// P2G + normalisation: xbar, vbar += given ubar and the forward u, m
aw_status p2g_vjp(MsbgState& G, const float* pos, const float* vel, int soa, int64_t n, const float* u[3],
                  const float* m[3], const float* ubar[3], float* xbar, float* vbar, cudaStream_t s);
aw_status unsort6(const uint32_t* perm, int64_t n, const float* in, float* out, cudaStream_t s);
// MAC sample of u at SoA points into SoA out
aw_status sample_soa(MsbgState& G, const float* pts_soa, int64_t n, const float* u[3], float* out_soa, cudaStream_t s);
// Grid side (aw_flip.cu).  project_forward: VELOCITY_* <- Wall(Sync(Grad(u, A^-1 Div u))) with the
// solver set up for `fluid`; project_vjp: ubar (in place) from the adjoint of the projected
// velocity to the adjoint of its input, one more solve with the same operator.
aw_status face_sync(MsbgState& G, float* u[3], cudaStream_t s);
aw_status wall_bc(MsbgState& G, float* u[3], cudaStream_t s);
aw_status face_sync_vjp(MsbgState& G, float* ubar[3], cudaStream_t s);
aw_status project_forward(MsbgState& G, aw_solver* sv, const uint8_t* fluid, float dt, int precision, FlipBufs& B,
                          cudaStream_t s);
aw_status project_vjp(MsbgState& G, aw_solver* sv, const uint8_t* fluid, float dt, int precision, float* ubar[3],
                      FlipBufs& B, cudaStream_t s);

// ------------------------------------------------------------------------------------------------
// FLIP step on SoA particle state (aw_flip.cu), shared by aw_flip_step and the differentiable
// rollout (aw_adjoint.cu).
// ------------------------------------------------------------------------------------------------

// What the adjoint of one step needs, all in the step's sorted particle order.
struct StepRecord {
    DBuf<uint32_t> perm;  // sorted slot -> slot of the step's input state
    DBuf<float> soa;      // x, v at the start of the step (6 n, SoA)
    DBuf<float> u1[3];    // P2G velocity before the T-junction sync
    DBuf<float> m[3];     // P2G mass
    DBuf<float> uo[3];    // backup velocity (G2P's u_old)
    DBuf<float> u6[3];    // projected velocity (G2P's u_new, the advection field)
    DBuf<uint8_t> fluid;  // fluid flags of the projection
    aw_status ensure(const MsbgState& G, int64_t n);
};

// soa_in/ids_in: state in any order; soa_out/ids_out: the stepped state, sorted by cell.
// fluid_in (optional) replaces the fluid flags derived from the particle counts.  ev (optional,
// 8 events) and st (optional) receive phase timings and solver statistics; st syncs the stream.
// Two-phase state of a simulation: phase in [0,1] indexed by particle id, and the two densities.
struct FlipPhase {
    const float* phase;
    float rho0, rho1;
};
// fp (optional, needs ids): P2G also writes PHASE_FIELD_* and BETA_COEFF_*, and the solver's
// coefficients are rebuilt from them before the projection.
// warm_start: the projection starts from the previous step's pressure (B.p_warm), with air cells
// zeroed, instead of from zero.
aw_status flip_step_soa(MsbgState& G, aw_solver* solver, const aw_flip_desc& d, FlipBufs& B, const float* soa_in,
                        const uint32_t* ids_in, float* soa_out, uint32_t* ids_out, int64_t n, const uint8_t* fluid_in,
                        StepRecord* rec, cudaEvent_t* ev, aw_flip_stats* st, cudaStream_t s,
                        const FlipPhase* fp = nullptr, bool warm_start = false);

}  // namespace aw

struct aw_msbg {
    aw::MsbgState st;
};
