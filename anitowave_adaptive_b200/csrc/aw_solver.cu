// aw_solver.cu — multigrid pressure solver on the MSBG: block red-black smoother, residual,
// restriction/prolongation, uniform coarse levels, FP64 coarsest solve, FP32 and mixed solves.
//
// Reference behaviour followed (paths within the reference project):
//   Smoother.cuh:23-94    ghost values across blocks (getPressureLevel; T-junction rule D8 fixed)
//   Smoother.cuh:105-202  smoothActiveBlocks: block parity colouring, <= MAX_BLOCK_ITER block-local
//                         red-black GS sweeps, early exit at TARGET_RESIDUAL_REDUCTION, activation
//   Smoother.cuh:249-291  solveLevel: active set per iteration (here device flags, no host sync)
//   VCycle.cuh:81-131     computeExplicitResidual
//   MultigridTransfer.cuh:9-102 restriction (8-child sum) / prolongation (injection add)
//   VCycle.cuh:177-304    init (coarse offsets, Galerkin) and recursive runCycle
//
// B200 design: every block-structured kernel is one CTA per block with the block and a one-cell
// halo staged in shared memory; the smoother runs all its block-local sweeps out of shared
// memory and touches HBM once per launch.  Uniform coarse levels continue below one cell per
// block and end in an FP64 dense solve (Cholesky inverse built on the device each setup).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "aw_internal.cuh"

namespace aw {

static inline unsigned nblk(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }
aw_status level_offsets(MsbgState& G, int m, int vanish, uint32_t* d_off4, int* d_res, uint32_t tot[4], cudaStream_t s);
__global__ void k_galerkin_ref(Geo g, const uint32_t* __restrict__ level, int axis, int dest,
                               const float* __restrict__ fine, float* __restrict__ coarse,
                               const uint32_t* __restrict__ foff, const uint32_t* __restrict__ coff);

constexpr int EXACT_CAP = 512;       // largest coarsest system factorised densely
constexpr int EXACT_POS_CAP = 32768; // largest coarsest grid scanned by the factor kernel

struct MGLevel {
    bool dense = false;
    int D[3] = {0, 0, 0};
    float H = 0.f;
    bool half = false;  // x stored as FP16 + per-block scale
    DBuf<int> res;
    std::vector<int> h_res;
    DBuf<uint32_t> off[4];
    uint32_t tot[4] = {0, 0, 0, 0};
    // CTA batches: [0]/[1] blocks of one colour, [2] all blocks; each entry {first, count, res, 0}
    DBuf<int4> desc[3];
    std::vector<int> h_blocks[3];  // block of every slot, batch order
    DBuf<int> meta[3];             // slot metadata (NMETA fields x slots, field-major)
    DBuf<int> blk[3];              // block of every slot, batch order, on the device
    int ndesc[3] = {0, 0, 0};
    // dynamic shared memory of the batched kernels on this level
    size_t smem_smooth = 0, smem_x64 = 0, smem_prolong = 0, smem_meta = 0;
    int maxres = 0;
    DBuf<float> W[3], bbar[3];
    DBuf<uint8_t> fluid;
    DBuf<float> x, b, r;
    DBuf<__half> xh;
    DBuf<float> xscale;
    DBuf<uint8_t> status[2];
    size_t ncell() const { return dense ? (size_t)D[0] * D[1] * D[2] : tot[0]; }
    size_t nface(int a) const {
        return dense ? (size_t)(D[0] + (a == 0)) * (D[1] + (a == 1)) * (D[2] + (a == 2)) : tot[1 + a];
    }
};

}  // namespace aw

struct aw_solver {
    aw_msbg* g = nullptr;
    aw_solver_desc d{};
    std::vector<aw::MGLevel> lv;
    int nmsbg = 0;
    // coarsest exact solve
    bool exact = false;
    aw::DBuf<double> M, Minv;
    aw::DBuf<int> ex_idx, ex_n, ex_pos;
    aw::DBuf<uint8_t> ex_prev;  // coarsest fluid flags of the last factorisation (per position)
    bool coef_dirty = true;     // coefficients changed since the last factorisation
    // level-0 bindings for the current solve
    float* x0 = nullptr;
    const float* b0 = nullptr;
    // mixed precision: FP64 vectors of the conjugate-gradient outer loop (residual, direction,
    // -A d), its scalars {rho, rho_old, d.(-A d)} and a zero right-hand side for applying A
    aw::DBuf<double> p64tmp;
    aw::DBuf<double> cg_r, cg_d, cg_q, cg_sc;
    aw::DBuf<float> cg_zero;
    // FP32 conjugate gradients: direction, -A d, scalars {rho, rho_old, d.(-A d)}, partial sums
    aw::DBuf<float> cg32_d, cg32_q, cg32_sc, partials32;
    aw::DBuf<double> partials, norm;
    size_t smem_max = 0, smem_max64 = 0;
    // the whole V-cycle as a CUDA graph, captured once per (x0, b0) binding
    cudaStream_t cap = nullptr;
    cudaGraphExec_t cycle = nullptr;
    const void* cycle_x0 = nullptr;
    const void* cycle_b0 = nullptr;
    unsigned long long cycle_kernels = 0;
    // the mixed-precision CG iterations as one graph with a device-side while loop, per pressure
    // array; cgst = {iterations, restart flag, iteration limit}, cgprm = {||b||, tolerance}
    cudaGraphExec_t cgloop = nullptr;
    const void* cgloop_p = nullptr;
    unsigned long long cgloop_kernels = 0;
    bool use_devloop = true;
    aw::DBuf<int> cgst;
    aw::DBuf<double> cgprm;
    bool use_graph = true;
    bool use_pdl = true;  // V-cycle kernels as programmatic dependent launches
    int tail = 0;         // first level of the uniform tail run as one k_dense_tail launch (0: none)
    double* h_norm = nullptr;  // pinned host word for the per-iteration residual norm
    double* h_cg = nullptr;    // pinned host words of the device-loop state
    ~aw_solver() {
        if (cycle) cudaGraphExecDestroy(cycle);
        if (cgloop) cudaGraphExecDestroy(cgloop);
        if (cap) cudaStreamDestroy(cap);
        if (h_norm) cudaFreeHost(h_norm);
        if (h_cg) cudaFreeHost(h_cg);
    }
};

namespace aw {

struct SmoothParams {
    float omega, target, theta;
    int iters;
    int check_fluid;
    int reverse;  // visit the cell colours black, red (the adjoint order of red, black)
};

__host__ __device__ inline int xi3(int x, int y, int z, int R2) { return (x + 1) + R2 * ((y + 1) + R2 * (z + 1)); }

__device__ inline float block_max(float v, float* red) {
    v = warp_max(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        float t = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.f;
        t = warp_max(t);
        if (lane == 0) red[32] = t;
    }
    __syncthreads();
    float out = red[32];
    __syncthreads();
    return out;
}

__device__ inline double block_sum(double v, double* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = v;
    __syncthreads();
    double out = 0.0;
    if (w == 0) {
        double t = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        out = warp_sum(t);
    }
    __syncthreads();
    return out;  // valid in thread 0
}

struct Coef3 {
    const float* w[3];
};

// ------------------------------------------------------------------------------------------------
// Batched block kernels.  A CTA serves `count` blocks ("slots") of one resolution r, listed
// contiguously: 1 block of 8^3 or 16^3 cells, 4 of 4^3, 16 of 2^3, 64 of 1^3.  Every slot keeps
// its block and a one-cell halo in shared memory; slots never interact (same colour = no shared
// faces), so each slot's arithmetic, early exit and activation are exactly those of a CTA that
// owns one block.
// ------------------------------------------------------------------------------------------------
struct Batch {
    const int4* desc;  // {first slot, count, res, 0}
    const int* meta;   // batch-ordered slot metadata, NMETA fields x nslots (field-major)
    int nslots;
};

// Slot metadata fields.  The host lays them out in batch order when the solver is created, so a CTA
// reads its slots' block ids, offsets and face neighbours with one coalesced round trip after the
// descriptor instead of chasing block id -> offsets -> neighbour offsets.
enum {
    MF_BLOCK = 0,        // block id
    MF_OFF = 1,          // 4 fields: cells, faces x, y, z of this level
    MF_NB = 5,           // 6 directions (2a + (s > 0)) x {neighbour cell offset, kind, neighbour block}
    MF_FINE_OFF = 23,    // cell offset and resolution of the block on the next finer level
    MF_FINE_RES = 24,
    MF_COARSE_OFF = 25,  // ... and on the next coarser level
    MF_COARSE_RES = 26,
    NMETA = 27
};

// Face-neighbour kinds: 0 = outside the domain or absent (ghost 0), 2 = same resolution,
// 3 = coarser neighbour (parent cell), 4 = finer neighbour (mean of the 4 touching cells).
enum { NB_NONE = 0, NB_SAME = 2, NB_COARSE = 3, NB_FINE = 4 };

// Every thread of a batched CTA only ever touches cells of one slot (G * r^3 <= 256, or G == 1).
// Reduce a per-thread non-negative value over the threads of each slot: shuffle within aligned
// groups of min(r^3, 32) lanes, then one shared atomicMax per group.
__device__ inline void slot_max(int* dst, int n3, float v) {
    const int grp = n3 < 32 ? n3 : 32;
    int iv = __float_as_int(v);
    for (int o = 1; o < grp; o <<= 1) iv = max(iv, __shfl_xor_sync(0xffffffffu, iv, o));
    if ((threadIdx.x & (grp - 1)) == 0 && iv > 0) atomicMax(dst, iv);
}

// ---- asynchronous global -> shared copies (completion via cp.async.wait_all) ----
__device__ inline uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ inline void cp_async4(void* s, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ inline void cp_async8(void* s, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ inline void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// Programmatic dependent launch: the V-cycle's kernels are launched so that each may start while its
// predecessor drains.  A kernel reads what its predecessor wrote only after pdl_wait() (which returns
// once the predecessor grid has completed and its memory is visible; at once for a kernel launched
// without the attribute), and lets its successor start with pdl_trigger() once its own main work is
// issued.  Descriptors and slot metadata (fixed at solver build) are staged before the wait.
__device__ inline void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ inline void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// Sources of x for staging: FP32 (copied asynchronously), FP16 + per-block scale (decoded in
// registers), FP64 (copied asynchronously).
struct SrcX {
    XStore x;
    using T = float;
    __device__ bool async() const { return x.f != nullptr; }
    __device__ float get(uint32_t i, int b) const { return x.get(i, b); }
    __device__ void copy(float* dst, uint32_t i) const { cp_async4(dst, x.f + i); }
};
struct SrcD {
    const double* p;
    using T = double;
    __device__ bool async() const { return true; }
    __device__ double get(uint32_t i, int) const { return p[i]; }
    __device__ void copy(double* dst, uint32_t i) const { cp_async8(dst, p + i); }
};

// (p0, p1, p2) given along the axes (a, a+1, a+2) mod 3 -> (x, y, z)
__device__ inline void rot3(int a, int p0, int p1, int p2, int& x, int& y, int& z) {
    x = a == 0 ? p0 : (a == 1 ? p2 : p1);
    y = a == 0 ? p1 : (a == 1 ? p0 : p2);
    z = a == 0 ? p2 : (a == 1 ? p1 : p0);
}

// Every batched CTA runs NT threads over G slots of one resolution R (a power of two, 1..16), so
// that G * R^3 <= NT or G == 1.  The kernels switch on R once per CTA and run a body compiled for
// that R: every index split is then a shift, a mask or a multiply by a constant, and every loop
// has a fixed trip count.
constexpr int NT = 256;
// CTAs per SM the batched block kernels are compiled for (registers per thread <= 64K / (NT x this))
#ifndef AW_BLOCK_CTAS_PER_SM
#define AW_BLOCK_CTAS_PER_SM 6
#endif
// loads in flight per thread when staging decoded or averaged halo values
#ifndef AW_STAGE_BATCH
#define AW_STAGE_BATCH 2
#endif

template <int R>
struct Geom {
    static constexpr int n3 = R * R * R, rr = R * R, nf = (R + 1) * R * R, R2 = R + 2, X3 = R2 * R2 * R2;
    static constexpr int FS = n3 + 3 * nf;  // b, then the three face-coefficient arrays
    static constexpr int FW = n3 / 4 + 2;   // 32-bit words that cover a block's fluid bytes
    static constexpr int GMAX = n3 >= NT ? 1 : NT / n3;
};

#define AW_SWITCH_RES(r, BODY) \
    switch (r) {               \
        case 1: BODY(1); break;  \
        case 2: BODY(2); break;  \
        case 4: BODY(4); break;  \
        case 8: BODY(8); break;  \
        default: BODY(16); break; \
    }

// Shared-memory image of a batched CTA: per slot x with a one-cell halo (xs, (R+2)^3 values of
// type T), b and the face coefficients (fs), the fluid words (fw) and the slot metadata.
template <class T, int R>
struct SlotImage {
    using Gm = Geom<R>;
    T* xs;
    int* meta;
    float* fs;
    uint32_t* fw;
    int G;
    __device__ SlotImage(void* base, int G_) : G(G_) {
        xs = (T*)base;
        meta = (int*)(xs + G * Gm::X3);
        fs = (float*)(meta + NMETA * G);
        fw = (uint32_t*)(fs + G * Gm::FS);
    }
    __device__ int m(int f, int sl) const { return meta[f * G + sl]; }
    __device__ uint32_t off(int k, int sl) const { return (uint32_t)meta[(MF_OFF + k) * G + sl]; }
    __device__ bool fluid(int sl, int i) const {
        return ((const uint8_t*)(fw + sl * Gm::FW))[(off(0, sl) & 3u) + i] != 0;
    }
};

__host__ __device__ inline size_t slot_image_bytes(int G, int r, size_t tsize) {
    const size_t n3 = (size_t)r * r * r, nf = (size_t)(r + 1) * r * r, X3 = (size_t)(r + 2) * (r + 2) * (r + 2);
    return (size_t)G * (X3 * tsize + NMETA * 4 + (n3 + 3 * nf) * 4 + (n3 / 4 + 2) * 4) + 16;
}

// Stage the metadata of a CTA's G slots into meta[NMETA * G] (one round trip); slots whose block is
// inactive (status[b] == 0) get block id -1.
template <int R>
__device__ inline void stage_meta(int* meta, int G, const Batch& B, int first, const uint8_t* __restrict__ status) {
    constexpr int GM = Geom<R>::GMAX;
    const int t = threadIdx.x % GM;
    if (t < G)
        for (int f = threadIdx.x / GM; f < NMETA; f += NT / GM)
            cp_async4(meta + f * G + t, B.meta + (size_t)f * B.nslots + first + t);
    cp_async_wait_all();
    __syncthreads();
    if (status) {
        for (int s = threadIdx.x; s < G; s += NT)
            if (!status[meta[s]]) meta[s] = -1;
        __syncthreads();
    }
}

struct MetaView {
    const int* p;
    int G;
    __device__ int m(int f, int sl) const { return p[f * G + sl]; }
    __device__ uint32_t off(int k, int sl) const { return (uint32_t)p[(MF_OFF + k) * G + sl]; }
};

// Register-batched staging of values that need a decode or a mean: the FP16 interior cells and the
// halo cells (0, 1 or 4 sources each).  K items per thread are addressed, then loaded, then
// stored, so that their loads are in flight together.
template <int R, class Src, bool HALO>
__device__ inline void stage_items(SlotImage<typename Src::T, R>& S, const Src& x) {
    using T = typename Src::T;
    using Gm = Geom<R>;
    constexpr int GM = Gm::GMAX, n3 = Gm::n3, rr = Gm::rr, K = AW_STAGE_BATCH;
    constexpr int NI = HALO ? GM * 6 * rr : GM * n3;
#pragma unroll
    for (int base = 0; base < NI; base += K * NT) {
        uint32_t src[K][4];
        int ns[K], blk[K], dst[K];
        T raw[K][4];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int t = base + k * NT + threadIdx.x;
            ns[k] = 0;
            dst[k] = -1;
            blk[k] = 0;
            if (t >= NI) continue;
            if (!HALO) {
                const int sl = t / n3, i = t % n3;
                if (sl >= S.G) continue;
                const int b = S.m(MF_BLOCK, sl);
                if (b < 0) continue;
                ns[k] = 1;
                src[k][0] = S.off(0, sl) + i;
                blk[k] = b;
                dst[k] = sl * Gm::X3 + xi3(i % R, (i / R) % R, i / rr, Gm::R2);
                continue;
            }
            const int sl = t / (6 * rr), rem0 = t % (6 * rr);
            if (sl >= S.G || S.m(MF_BLOCK, sl) < 0) continue;
            const int face = rem0 / rr, rem = rem0 % rr;
            const int a = face >> 1, sd = (face & 1) ? 1 : -1;
            const int u = rem % R, v = rem / R;  // coordinates along the axes a+1 and a+2
            const int kind = S.m(MF_NB + 3 * face + 1, sl);
            if (kind != NB_NONE) {
                const uint32_t o = (uint32_t)S.m(MF_NB + 3 * face, sl);
                blk[k] = S.m(MF_NB + 3 * face + 2, sl);
                const int rn = kind == NB_SAME ? R : (kind == NB_COARSE ? R / 2 : 2 * R);
                const int qa = sd > 0 ? 0 : rn - 1;
                int qx, qy, qz;
                if (kind != NB_FINE) {
                    const int sh = kind == NB_SAME ? 0 : 1;
                    rot3(a, qa, u >> sh, v >> sh, qx, qy, qz);
                    ns[k] = 1;
                    src[k][0] = o + cidx(qx, qy, qz, rn);
                } else {
                    ns[k] = 4;
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        rot3(a, qa, 2 * u + (e >> 1), 2 * v + (e & 1), qx, qy, qz);
                        src[k][e] = o + cidx(qx, qy, qz, rn);
                    }
                }
            }
            int hx, hy, hz;
            rot3(a, sd > 0 ? R : -1, u, v, hx, hy, hz);
            dst[k] = sl * Gm::X3 + xi3(hx, hy, hz, Gm::R2);
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int e = 0; e < 4; ++e) raw[k][e] = e < ns[k] ? x.get(src[k][e], blk[k]) : T(0);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (dst[k] < 0) continue;
            T v;
            if (ns[k] == 4) {
                T sum = T(0);
#pragma unroll
                for (int e = 0; e < 4; ++e) sum += raw[k][e];
                v = T(0.25) * sum;
            } else {
                v = raw[k][0];
            }
            S.xs[dst[k]] = v;
        }
    }
}

// Stage x (interior + halo), b, the face coefficients and the fluid flags of every live slot.
// Every global load is issued before the first wait: plain copies go through cp.async, decoded
// and averaged values through register batches, so that a CTA pays about one memory round trip.
template <int R, class Src>
__device__ inline void stage_data(SlotImage<typename Src::T, R>& S, const Src& x, const float* __restrict__ bvec, Coef3 W,
                                  const uint8_t* __restrict__ fluid) {
    using Gm = Geom<R>;
    constexpr int GM = Gm::GMAX, n3 = Gm::n3, nf = Gm::nf;
    const bool xa = x.async();
#pragma unroll
    for (int t0 = 0; t0 < GM * n3; t0 += NT) {
        const int t = t0 + threadIdx.x, sl = t / n3, i = t % n3;
        if (sl >= S.G || S.m(MF_BLOCK, sl) < 0) continue;
        const uint32_t oc = S.off(0, sl);
        if (xa) x.copy(S.xs + sl * Gm::X3 + xi3(i % R, (i / R) % R, i / Gm::rr, Gm::R2), oc + i);
        cp_async4(S.fs + sl * Gm::FS + i, bvec + oc + i);
    }
#pragma unroll 4
    for (int t0 = 0; t0 < GM * 3 * nf; t0 += NT) {
        const int t = t0 + threadIdx.x;
        if (t >= GM * 3 * nf) break;
        const int sl = t / (3 * nf), j = t % (3 * nf);
        if (sl >= S.G || S.m(MF_BLOCK, sl) < 0) continue;
        const int a = j / nf;
        const float* wa = a == 0 ? W.w[0] : (a == 1 ? W.w[1] : W.w[2]);
        cp_async4(S.fs + sl * Gm::FS + n3 + j, wa + S.off(1 + a, sl) + (j - a * nf));
    }
    if (fluid) {
        const uint32_t* fwg = (const uint32_t*)fluid;
#pragma unroll
        for (int t0 = 0; t0 < GM * Gm::FW; t0 += NT) {
            const int t = t0 + threadIdx.x;
            if (t >= GM * Gm::FW) break;
            const int sl = t / Gm::FW, w = t % Gm::FW;
            if (sl >= S.G || S.m(MF_BLOCK, sl) < 0) continue;
            const uint32_t oc = S.off(0, sl);
            if (w * 4 < (int)(oc & 3u) + n3) cp_async4(S.fw + sl * Gm::FW + w, fwg + (oc >> 2) + w);
        }
    }
    if (!xa) stage_items<R, Src, false>(S, x);
    stage_items<R, Src, true>(S, x);
    cp_async_wait_all();
}

// Write every slot's x back: FP32, or FP16 with a fresh per-block scale.  sb/off0 are per-slot
// block ids (-1 = skip) and cell offsets in shared memory.
template <int R>
__device__ inline void store_slots(const XStore& x, const int* sb, const int* off0, int G, const float* xs, int* smax) {
    using Gm = Geom<R>;
    constexpr int GM = Gm::GMAX, n3 = Gm::n3;
    if (x.f) {
#pragma unroll
        for (int t0 = 0; t0 < GM * n3; t0 += NT) {
            const int t = t0 + threadIdx.x, sl = t / n3, i = t % n3;
            if (sl >= G || sb[sl] < 0) continue;
            x.f[(uint32_t)off0[sl] + i] = xs[sl * Gm::X3 + xi3(i % R, (i / R) % R, i / Gm::rr, Gm::R2)];
        }
        return;
    }
    for (int t = threadIdx.x; t < G; t += NT) smax[t] = 0;
    __syncthreads();
    {
        float m = 0.f;
#pragma unroll
        for (int t0 = 0; t0 < GM * n3; t0 += NT) {
            const int t = t0 + threadIdx.x, sl = t / n3, i = t % n3;
            if (sl >= G || sb[sl] < 0) continue;
            m = fmaxf(m, fabsf(xs[sl * Gm::X3 + xi3(i % R, (i / R) % R, i / Gm::rr, Gm::R2)]));
        }
        const int sl = GM == 1 ? 0 : min((int)threadIdx.x / n3, G - 1);
        slot_max(&smax[sl], n3, m);
    }
    __syncthreads();
#pragma unroll
    for (int t0 = 0; t0 < GM * n3; t0 += NT) {
        const int t = t0 + threadIdx.x, sl = t / n3, i = t % n3;
        if (sl >= G || sb[sl] < 0) continue;
        const float m = __int_as_float(smax[sl]);
        const float inv = m > 0.f ? 32768.f / m : 0.f;
        x.h[(uint32_t)off0[sl] + i] = __float2half_rn(xs[sl * Gm::X3 + xi3(i % R, (i / R) % R, i / Gm::rr, Gm::R2)] * inv);
    }
    for (int t = threadIdx.x; t < G; t += NT)
        if (sb[t] >= 0) {
            const float m = __int_as_float(smax[t]);
            x.scale[sb[t]] = m > 0.f ? m * (1.f / 32768.f) : 0.f;
        }
}

// Shared smoother state of one CTA (one entry per slot).
struct SmoothShared {
    int smr[NT], sdone[NT];
    float sinit[NT];
};

template <int R>
__device__ inline void smooth_body(int4 d, unsigned char* smraw, SmoothShared& Z, const LevelView& L, const XStore& x,
                                   const float* __restrict__ bvec, const Coef3& W, const uint8_t* __restrict__ fluid,
                                   const Batch& B, const uint8_t* __restrict__ status, uint8_t* __restrict__ status_next,
                                   const SmoothParams& P) {
    using Gm = Geom<R>;
    constexpr int GM = Gm::GMAX, n3 = Gm::n3, nf = Gm::nf, R2 = Gm::R2, sy = R2, sz = R2 * R2;
    SlotImage<float, R> S(smraw, d.y);
    const int G = S.G;
    if (status) pdl_wait();  // the activation flags come from the previous sweep
    stage_meta<R>(S.meta, G, B, d.x, status);
    const int* sb = S.meta + MF_BLOCK * G;
    if (!__syncthreads_or(threadIdx.x < G && sb[threadIdx.x] >= 0)) return;
    pdl_wait();
    for (int t = threadIdx.x; t < G; t += NT) {
        Z.smr[t] = 0;
        Z.sdone[t] = 0;
        Z.sinit[t] = -1.f;
    }
    stage_data<R>(S, SrcX{x}, bvec, W, P.check_fluid ? fluid : nullptr);
    __syncthreads();
    const int my_slot = GM == 1 ? 0 : min((int)threadIdx.x / n3, G - 1);
    // The per-slot residual maximum feeds the early exit and the activation of neighbours.  With no
    // activation output and no exit possible (at most two sweeps and a reduction target below 1:
    // the first sweep only records the initial residual), it is skipped with its two barriers.
    const bool track = status_next || (P.target > 0.f && (P.iters > 2 || (P.iters == 2 && P.target >= 1.f)));
    for (int bi = 0; bi < P.iters; ++bi) {
        float lmax = 0.f;
#pragma unroll
        for (int col = 0; col < 2; ++col) {
            // one slot per CTA (8^3 and 16^3 blocks): each thread visits only cells of this colour;
            // smaller blocks keep one thread per cell so that a slot's threads stay contiguous
            constexpr bool HALF = GM == 1 && R >= 2;
            constexpr int NC = HALF ? n3 / 2 : GM * n3;
            constexpr int RH = R >= 2 ? R / 2 : 1;  // cells of one colour per row (HALF only)
            const int cc = P.reverse ? 1 - col : col;
#pragma unroll
            for (int t0 = 0; t0 < NC; t0 += NT) {
                const int t = t0 + threadIdx.x;
                int sl, i, cx, cy, cz;
                if (HALF) {
                    if (t >= NC) continue;
                    sl = 0;
                    cy = (t / RH) % R;
                    cz = t / (RH * R);
                    cx = 2 * (t % RH) + ((cy + cz + cc) & 1);
                    i = cx + R * (cy + R * cz);
                } else {
                    sl = t / n3;
                    i = t % n3;
                    cx = i % R;
                    cy = (i / R) % R;
                    cz = i / Gm::rr;
                }
                if (sl >= G || sb[sl] < 0 || Z.sdone[sl]) continue;
                if (!HALF && ((cx + cy + cz) & 1) != cc) continue;
                if (P.check_fluid && !S.fluid(sl, i)) continue;
                float* xs = S.xs + sl * Gm::X3;
                const float* bs = S.fs + sl * Gm::FS;
                const float* Ws = bs + n3;
                const float wW = Ws[fidx(0, cx, cy, cz, R)];
                const float wE = Ws[fidx(0, cx + 1, cy, cz, R)];
                const float wS = Ws[nf + fidx(1, cx, cy, cz, R)];
                const float wN = Ws[nf + fidx(1, cx, cy + 1, cz, R)];
                const float wB = Ws[2 * nf + fidx(2, cx, cy, cz, R)];
                const float wT = Ws[2 * nf + fidx(2, cx, cy, cz + 1, R)];
                const float diag = -(wW + wE + wS + wN + wB + wT);
                if (fabsf(diag) < 1e-9f) continue;
                const int q = xi3(cx, cy, cz, R2);
                const float xc = xs[q];
                const float Ax = wW * xs[q - 1] + wE * xs[q + 1] + wS * xs[q - sy] + wN * xs[q + sy] + wB * xs[q - sz] +
                                 wT * xs[q + sz] + diag * xc;
                const float res = bs[i] - Ax;
                xs[q] = xc + P.omega * __fdividef(res, diag);  // a smoother tolerates the 2-ulp quotient
                lmax = fmaxf(lmax, fabsf(res));
            }
            __syncthreads();
        }
        if (!track) continue;
        slot_max(&Z.smr[my_slot], n3, lmax);
        __syncthreads();
        // per-slot early exit (block-uniform); smr keeps the last executed sweep's max
        int more = 0;
        for (int t = threadIdx.x; t < G; t += NT) {
            if (sb[t] < 0 || Z.sdone[t]) continue;
            const float mr = __int_as_float(Z.smr[t]);
            if (bi == 0) Z.sinit[t] = mr;
            if (Z.sinit[t] > 1e-9f && mr < Z.sinit[t] * P.target) Z.sdone[t] = 1;
            else if (bi + 1 < P.iters) {
                Z.smr[t] = 0;
                more = 1;
            }
        }
        if (!__syncthreads_or(more)) break;
    }
    __syncthreads();
    pdl_trigger();
    store_slots<R>(x, sb, S.meta + MF_OFF * G, G, S.xs, Z.sdone);  // sdone reused as per-slot |x| max
    if (!status_next) return;
    for (int t = threadIdx.x; t < G; t += NT) {
        const int b = sb[t];
        if (b < 0 || !(__int_as_float(Z.smr[t]) > P.theta)) continue;
        status_next[b] = 1;
        int cb[3];
        bcoord(L.g, b, cb);
        for (int a = 0; a < 3; ++a)
            for (int sd = -1; sd <= 1; sd += 2) {
                int nc[3] = {cb[0], cb[1], cb[2]};
                nc[a] += sd;
                if (inside(L.g, nc)) status_next[bidx(L.g, nc[0], nc[1], nc[2])] = 1;
            }
    }
}

// smoothActiveBlocks (Smoother.cuh:105-202) for one block colour, batched.  status == nullptr
// means every block is active (no residual-threshold deactivation) and no activation is written.
__global__ void __launch_bounds__(NT, AW_BLOCK_CTAS_PER_SM) k_smooth(LevelView L, XStore x, const float* __restrict__ bvec, Coef3 W,
                                               const uint8_t* __restrict__ fluid, Batch B,
                                               const uint8_t* __restrict__ status, uint8_t* __restrict__ status_next,
                                               SmoothParams P) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ SmoothShared Z;
    const int4 d = B.desc[blockIdx.x];
#define AW_SMOOTH(R) smooth_body<R>(d, smraw, Z, L, x, bvec, W, fluid, B, status, status_next, P)
    AW_SWITCH_RES(d.z, AW_SMOOTH)
#undef AW_SMOOTH
}

// r = b - A x of cell i of slot sl from the staged slot image (0 on air cells when check_fluid)
template <int R, class T>
__device__ __forceinline__ T residual_cell(const SlotImage<T, R>& S, int sl, int i, int check_fluid) {
    using Gm = Geom<R>;
    constexpr int n3 = Gm::n3, nf = Gm::nf, R2 = Gm::R2, sy = R2, sz = R2 * R2;
    T rv = T(0);
    const float* bs = S.fs + sl * Gm::FS;
    if (!check_fluid || S.fluid(sl, i)) {
        const int cx = i % R, cy = (i / R) % R, cz = i / Gm::rr;
        const float* Ws = bs + n3;
        const T wW = Ws[fidx(0, cx, cy, cz, R)];
        const T wE = Ws[fidx(0, cx + 1, cy, cz, R)];
        const T wS = Ws[nf + fidx(1, cx, cy, cz, R)];
        const T wN = Ws[nf + fidx(1, cx, cy + 1, cz, R)];
        const T wB = Ws[2 * nf + fidx(2, cx, cy, cz, R)];
        const T wT = Ws[2 * nf + fidx(2, cx, cy, cz + 1, R)];
        const T diag = -(wW + wE + wS + wN + wB + wT);
        const T* xs = S.xs + sl * Gm::X3;
        const int q = xi3(cx, cy, cz, R2);
        const T Ax = diag * xs[q] + wW * xs[q - 1] + wE * xs[q + 1] + wS * xs[q - sy] + wN * xs[q + sy] +
                     wB * xs[q - sz] + wT * xs[q + sz];
        rv = (T)bs[i] - Ax;
    }
    return rv;
}

// DOTX: the per-CTA partial sums are of x . r instead of r . r (with a zero right-hand side, the
// d . (-A d) of a conjugate-gradient step, taken while d is staged)
template <int R, class Src, bool DOTX = false>
__device__ inline void residual_body(int4 d, unsigned char* smraw, double* dred, const Src& x, const float* __restrict__ bvec,
                                     const Coef3& W, const uint8_t* __restrict__ fluid, const Batch& B, int check_fluid,
                                     float* __restrict__ rout, double* __restrict__ rout64, double* __restrict__ part) {
    using T = typename Src::T;
    using Gm = Geom<R>;
    constexpr int GM = Gm::GMAX, n3 = Gm::n3;
    SlotImage<T, R> S(smraw, d.y);
    const int G = S.G;
    stage_meta<R>(S.meta, G, B, d.x, nullptr);
    pdl_wait();
    stage_data<R>(S, x, bvec, W, check_fluid ? fluid : nullptr);
    __syncthreads();
    pdl_trigger();
    double acc = 0.0;
#pragma unroll
    for (int t0 = 0; t0 < GM * n3; t0 += NT) {
        const int t = t0 + threadIdx.x, sl = t / n3, i = t % n3;
        if (sl >= G) continue;
        const T rv = residual_cell<R>(S, sl, i, check_fluid);
        if (rout) rout[S.off(0, sl) + i] = (float)rv;
        if (rout64) rout64[S.off(0, sl) + i] = (double)rv;
        if (DOTX) acc += (double)S.xs[sl * Gm::X3 + xi3(i % R, (i / R) % R, i / Gm::rr, Gm::R2)] * (double)rv;
        else acc += (double)rv * (double)rv;
    }
    if (part) {
        double tsum = block_sum(acc, dred);
        if (threadIdx.x == 0) part[blockIdx.x] = tsum;
    }
}

// computeExplicitResidual (VCycle.cuh:81-131), batched: r = b - A x on every cell (0 on air cells
// in FV mode); optional per-CTA partial sums of r^2.  Src::T = float for the V-cycle's own
// residual, double for the FP64 residual of the outer defect correction (stored as FP32 into the
// V-cycle right-hand side).
template <class Src>
__global__ void __launch_bounds__(NT, AW_BLOCK_CTAS_PER_SM) k_residual(Src x, const float* __restrict__ bvec, Coef3 W,
                                                 const uint8_t* __restrict__ fluid, Batch B, int check_fluid,
                                                 float* __restrict__ rout, double* __restrict__ rout64,
                                                 double* __restrict__ part) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double dred[32];
    const int4 d = B.desc[blockIdx.x];
#define AW_RESID(R) residual_body<R>(d, smraw, dred, x, bvec, W, fluid, B, check_fluid, rout, rout64, part)
    AW_SWITCH_RES(d.z, AW_RESID)
#undef AW_RESID
}

// qn = -A d in FP64 and the per-CTA partial sums of d . qn (the mixed-precision CG step), in one pass
__global__ void __launch_bounds__(NT, AW_BLOCK_CTAS_PER_SM) k_apply_dot(SrcD x, const float* __restrict__ zero, Coef3 W,
                                                                  const uint8_t* __restrict__ fluid, Batch B,
                                                                  int check_fluid, double* __restrict__ qn,
                                                                  double* __restrict__ part) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double dred[32];
    const int4 d = B.desc[blockIdx.x];
#define AW_APPLY(R) residual_body<R, SrcD, true>(d, smraw, dred, x, zero, W, fluid, B, check_fluid, nullptr, qn, part)
    AW_SWITCH_RES(d.z, AW_APPLY)
#undef AW_APPLY
}

template <int R>
__device__ inline void restrict_body(int4 d, unsigned char* smraw, const float* __restrict__ r, float* __restrict__ bc,
                                     const uint8_t* __restrict__ fluid_c, int check_fluid, const Batch& B) {
    using Gm = Geom<R>;
    constexpr int GM = Gm::GMAX, n3 = Gm::n3, K = 2;
    const int G = d.y;
    int* meta = (int*)smraw;
    stage_meta<R>(meta, G, B, d.x, nullptr);
    pdl_wait();
    pdl_trigger();
    const MetaView S{meta, G};
#pragma unroll
    for (int base = 0; base < GM * n3; base += K * NT) {
        float v[K][8];
        uint8_t fl[K];
        uint32_t dst[K];
        bool ok[K], full[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int t = base + k * NT + threadIdx.x, sl = t / n3, i = t % n3;
            ok[k] = t < GM * n3 && sl < G;
            full[k] = false;
            dst[k] = 0;
            fl[k] = 1;
            if (!ok[k]) continue;
            const int rf = S.m(MF_FINE_RES, sl);
            const uint32_t of = (uint32_t)S.m(MF_FINE_OFF, sl);
            dst[k] = S.off(0, sl) + i;
            if (check_fluid) fl[k] = fluid_c[dst[k]];
            full[k] = rf == 2 * R;
            if (full[k]) {
                const int x = i % R, y = (i / R) % R, z = i / Gm::rr;
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    v[k][c] = r[of + cidx(2 * x + (c & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c >> 2), 2 * R)];
            } else {
                v[k][0] = r[of + i];
            }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!ok[k]) continue;
            float s = v[k][0];
            if (full[k]) {
#pragma unroll
                for (int c = 1; c < 8; ++c) s += v[k][c];
            }
            bc[dst[k]] = fl[k] ? s : 0.f;
        }
    }
}

// restrictResidualsKernel (MultigridTransfer.cuh:9-59), batched over the coarse level's blocks:
// 8-child sum, or a copy for a block that keeps one cell.  Coarse air cells get 0.
__global__ void __launch_bounds__(NT) k_restrict(const float* __restrict__ r, float* __restrict__ bc,
                                                 const uint8_t* __restrict__ fluid_c, int check_fluid, Batch B) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int4 d = B.desc[blockIdx.x];
#define AW_RESTR(R) restrict_body<R>(d, smraw, r, bc, fluid_c, check_fluid, B)
    AW_SWITCH_RES(d.z, AW_RESTR)
#undef AW_RESTR
}

template <int R>
__device__ inline void prolong_body(int4 d, unsigned char* smraw, int* smax, const XStore& xf, const XStore& xc,
                                    const uint8_t* __restrict__ fluid_f, int check_fluid, const Batch& B) {
    using Gm = Geom<R>;
    constexpr int GM = Gm::GMAX, n3 = Gm::n3, K = 2;
    const int G = d.y;
    // FP16 fine storage keeps the updated block in shared memory for the re-encode
    float* xs = (float*)smraw;
    int* meta = (int*)(xs + (xf.f ? 0 : G * Gm::X3));
    stage_meta<R>(meta, G, B, d.x, nullptr);
    pdl_wait();
    pdl_trigger();
    const MetaView S{meta, G};
#pragma unroll
    for (int base = 0; base < GM * n3; base += K * NT) {
        float add[K], cur[K];
        int sl_[K], i_[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int t = base + k * NT + threadIdx.x, sl = t / n3, i = t % n3;
            sl_[k] = -1;
            i_[k] = i;
            add[k] = 0.f;
            cur[k] = 0.f;
            if (t >= GM * n3 || sl >= G) continue;
            sl_[k] = sl;
            const int b = S.m(MF_BLOCK, sl);
            const int rc = S.m(MF_COARSE_RES, sl);
            const uint32_t of = S.off(0, sl), oc = (uint32_t)S.m(MF_COARSE_OFF, sl);
            if (rc && (!check_fluid || fluid_f[of + i])) {
                const uint32_t ci = (R == 2 * rc) ? cidx((i % R) >> 1, ((i / R) % R) >> 1, (i / Gm::rr) >> 1, R / 2)
                                                  : (uint32_t)i;
                add[k] = xc.get(oc + ci, b);
            }
            cur[k] = xf.get(of + i, b);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int sl = sl_[k];
            if (sl < 0) continue;
            const int i = i_[k];
            if (xf.f) xf.f[S.off(0, sl) + i] = cur[k] + add[k];
            else xs[sl * Gm::X3 + xi3(i % R, (i / R) % R, i / Gm::rr, Gm::R2)] = cur[k] + add[k];
        }
    }
    if (xf.f) return;
    __syncthreads();
    store_slots<R>(xf, meta + MF_BLOCK * G, meta + MF_OFF * G, G, xs, smax);
}

// prolongateCorrection (MultigridTransfer.cuh:63-102), batched over the fine level's blocks:
// x_f += x_c[parent] on fluid cells (FP16 fine storage is decoded, updated and re-encoded).
__global__ void __launch_bounds__(NT) k_prolong(XStore xf, XStore xc, const uint8_t* __restrict__ fluid_f,
                                                int check_fluid, Batch B) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ int smax[NT];
    const int4 d = B.desc[blockIdx.x];
#define AW_PROL(R) prolong_body<R>(d, smraw, smax, xf, xc, fluid_f, check_fluid, B)
    AW_SWITCH_RES(d.z, AW_PROL)
#undef AW_PROL
}

// ---- conjugate-gradient outer loop of the mixed-precision solve (FP64 vectors) ----------------
// dot(a, b) over fluid cells (b is FP64, or FP32 when bf is given), per-CTA partial sums
__global__ void k_dot64(const double* __restrict__ a, const double* __restrict__ b, const float* __restrict__ bf,
                        const uint8_t* __restrict__ fluid, size_t n, double* __restrict__ part) {
    pdl_wait();
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (fluid[i]) acc += a[i] * (bf ? (double)bf[i] : b[i]);
    __shared__ double red[32];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) part[blockIdx.x] = t;
    }
}
// z (FP32 V-cycle output) -> search direction d = z + beta d, beta = rho / rho_old (0 when first)
// first_dev (when given) holds the restart flag on the device
__global__ void k_cg_direction(double* __restrict__ d, const float* __restrict__ z, const uint8_t* __restrict__ fluid,
                               const double* __restrict__ sc, int first, const int* first_dev, size_t n) {
    pdl_wait();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (first_dev) first = *first_dev;
    const double beta = first ? 0.0 : sc[0] / sc[1];
    d[i] = fluid[i] ? (double)z[i] + beta * d[i] : 0.0;
}
// qn = -A d (the residual kernel with a zero right-hand side); alpha = rho / (d . A d)
// p += alpha d; r += alpha qn; and the FP32 copy of r for the next V-cycle
// ... and the per-CTA partial sums of |r|^2 over fluid cells (grid-stride, part[blockIdx.x]);
// rho_old = rho for the next iteration's direction (sc[1] is read by no CTA of this kernel)
__global__ void k_cg_update(double* __restrict__ p, double* __restrict__ r, float* __restrict__ rf,
                            const double* __restrict__ d, const double* __restrict__ qn, double* __restrict__ sc,
                            const uint8_t* __restrict__ fluid, size_t n, double* __restrict__ part) {
    pdl_wait();
    const double dq = -sc[2];
    const double alpha = dq != 0.0 ? sc[0] / dq : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) sc[1] = sc[0];
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        p[i] += alpha * d[i];
        const double rv = r[i] + alpha * qn[i];
        r[i] = rv;
        rf[i] = (float)rv;
        if (fluid[i]) acc += rv * rv;
    }
    __shared__ double red[32];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) part[blockIdx.x] = t;
    }
}
// End of one CG iteration inside the device-side loop (one CTA of 256 threads): ||r||^2 into norm2
// from k_cg_update's partial sums (the reduction of k_reduce_sum, so the host loop reads the same
// value), count the iteration, clear the restart flag, and run the loop body again while the
// residual is finite, at or above the tolerance and the iteration limit is not reached.
// st = {iterations, restart, limit}, prm = {||b||, tolerance}.
__global__ void k_cg_check(cudaGraphConditionalHandle h, const double* __restrict__ part, int nparts,
                           double* __restrict__ norm2, const double* __restrict__ prm, int* st) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[i];
    const double t = block_sum(acc, red);
    if (threadIdx.x != 0) return;
    norm2[0] = t;
    const double rel = sqrt(t) / prm[0];
    const int it = st[0] + 1;
    st[0] = it;
    st[1] = 0;
    cudaGraphSetConditional(h, (rel == rel && rel >= prm[1] && it < st[2]) ? 1u : 0u);
}
__global__ void k_fill_zero(float* __restrict__ x, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = 0.f;
}

// ---- conjugate gradients with every vector and scalar in FP32 (AW_PRECISION_FP32_PCG) ----------
// The same V-cycle preconditioner as the mixed form, without its FP64 residual, direction and
// accumulation: the like-for-like baseline of the mixed precision.  Partial sums and scalars are
// FP32 as well.
__device__ inline float block_sum_f(float v, float* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = v;
    __syncthreads();
    float t = 0.f;
    if (w == 0) {
        t = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    return t;  // valid in thread 0
}
__global__ void k_dot32(const float* __restrict__ a, const float* __restrict__ b, const uint8_t* __restrict__ fluid,
                        size_t n, float* __restrict__ part) {
    pdl_wait();
    __shared__ float red[32];
    float acc = 0.f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (fluid[i]) acc += a[i] * b[i];
    const float t = block_sum_f(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}
__global__ void k_reduce_sum32(const float* __restrict__ part, int n, float* out) {
    pdl_wait();
    __shared__ float red[32];
    float acc = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += part[i];
    const float t = block_sum_f(acc, red);
    if (threadIdx.x == 0) *out = t;
}
__global__ void k_cg_direction32(float* __restrict__ d, const float* __restrict__ z, const uint8_t* __restrict__ fluid,
                                 const float* __restrict__ sc, int first, size_t n) {
    pdl_wait();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float beta = first ? 0.f : sc[0] / sc[1];
    d[i] = fluid[i] ? z[i] + beta * d[i] : 0.f;
}
// p += alpha d; r += alpha qn (qn = -A d, alpha = rho / (d . A d)); per-CTA partial sums of |r|^2
__global__ void k_cg_update32(float* __restrict__ p, float* __restrict__ r, const float* __restrict__ d,
                              const float* __restrict__ qn, const float* __restrict__ sc,
                              const uint8_t* __restrict__ fluid, size_t n, float* __restrict__ part) {
    pdl_wait();
    __shared__ float red[32];
    const float dq = -sc[2];
    const float alpha = dq != 0.f ? sc[0] / dq : 0.f;
    float acc = 0.f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        p[i] += alpha * d[i];
        const float rv = r[i] + alpha * qn[i];
        r[i] = rv;
        if (fluid[i]) acc += rv * rv;
    }
    const float t = block_sum_f(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}
__global__ void k_copy_scalar32(float* __restrict__ sc, int dst, int src) {
    pdl_wait();
    sc[dst] = sc[src];
}

__global__ void k_accum64(double* __restrict__ p, const float* __restrict__ e, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] += (double)e[i];
}

__global__ void k_reduce_sum(const double* __restrict__ part, int n, double* out) {
    pdl_wait();
    __shared__ double red[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += part[i];
    double t = block_sum(acc, red);
    if (threadIdx.x == 0) *out = t;
}

// sum of b^2 over fluid cells (or all cells)
__global__ void k_sumsq(const float* __restrict__ v, const uint8_t* __restrict__ fluid, size_t n, int check_fluid,
                        double* part) {
    __shared__ double red[32];
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (!check_fluid || fluid[i]) acc += (double)v[i] * (double)v[i];
    double t = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_zero_scale(float* s, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) s[i] = 0.f;
}

// ---------------------------------- uniform (dense) levels ------------------------------------
struct DenseArgs {
    DenseView d;
    const float* W[3];
    const uint8_t* fluid;
};

__device__ inline float dense_nb(const DenseView& d, const float* x, int i, int j, int k, int a, int s) {
    int q[3] = {i, j, k};
    q[a] += s;
    if (q[a] < 0 || q[a] >= d.D[a]) return 0.f;
    return x[didx(d, q[0], q[1], q[2])];
}

__device__ inline float dense_Ax(const DenseArgs& A, const float* x, int i, int j, int k, float* diag_out) {
    const DenseView& d = A.d;
    float wW = A.W[0][dfidx(d, 0, i, j, k)], wE = A.W[0][dfidx(d, 0, i + 1, j, k)];
    float wS = A.W[1][dfidx(d, 1, i, j, k)], wN = A.W[1][dfidx(d, 1, i, j + 1, k)];
    float wB = A.W[2][dfidx(d, 2, i, j, k)], wT = A.W[2][dfidx(d, 2, i, j, k + 1)];
    float diag = -(wW + wE + wS + wN + wB + wT);
    *diag_out = diag;
    return wW * dense_nb(d, x, i, j, k, 0, -1) + wE * dense_nb(d, x, i, j, k, 0, 1) + wS * dense_nb(d, x, i, j, k, 1, -1) +
           wN * dense_nb(d, x, i, j, k, 1, 1) + wB * dense_nb(d, x, i, j, k, 2, -1) + wT * dense_nb(d, x, i, j, k, 2, 1) +
           diag * x[didx(d, i, j, k)];
}

// Per-cell values of the uniform-level kernels (the caller stores them), shared by the
// one-launch-per-step kernels below and by k_dense_tail, so both forms do the same arithmetic in
// the same order.  Each returns false where the kernel leaves the cell unchanged.
__device__ inline bool dense_smooth_value(const DenseArgs& A, const float* x, const float* __restrict__ b, int t,
                                          int col, float omega, float* out) {
    const DenseView& d = A.d;
    const int i = t % d.D[0], j = (t / d.D[0]) % d.D[1], k = t / (d.D[0] * d.D[1]);
    if (((i + j + k) & 1) != col || !A.fluid[t]) return false;
    float diag;
    const float ax = dense_Ax(A, x, i, j, k, &diag);
    if (fabsf(diag) < 1e-30f) return false;
    *out = x[t] + omega * __fdividef(b[t] - ax, diag);
    return true;
}
__device__ inline float dense_residual_value(const DenseArgs& A, const float* x, const float* __restrict__ b, int t) {
    const DenseView& d = A.d;
    const int i = t % d.D[0], j = (t / d.D[0]) % d.D[1], k = t / (d.D[0] * d.D[1]);
    float diag;
    return A.fluid[t] ? b[t] - dense_Ax(A, x, i, j, k, &diag) : 0.f;
}
// restriction into a dense level from the one-cell-per-block MSBG level (from_msbg) or a dense level
__device__ inline float dense_restrict_value(const DenseView& K, const uint8_t* __restrict__ fluid_c, int from_msbg,
                                             const LevelView& F, const DenseView& Fd, const float* rf, int t) {
    const int i = t % K.D[0], j = (t / K.D[0]) % K.D[1], k = t / (K.D[0] * K.D[1]);
    float s = 0.f;
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                int ci = 2 * i + dx, cj = 2 * j + dy, ck = 2 * k + dz;
                if (from_msbg) {
                    int b = bidx(F.g, ci, cj, ck);
                    if (F.res[b]) s += rf[F.off[0][b]];
                } else {
                    s += rf[didx(Fd, ci, cj, ck)];
                }
            }
    return fluid_c[t] ? s : 0.f;
}
// x_f + x_c[parent] on fluid cells: t is a block of the one-cell MSBG level (to_msbg, *at = its
// cell) or a dense cell (*at = t)
__device__ inline bool dense_prolong_value(const DenseView& K, const float* xc, int to_msbg, const LevelView& F,
                                           const float* xf_msbg, const DenseView& Fd, const float* xf,
                                           const uint8_t* __restrict__ fluid_f, int t, uint32_t* at, float* out) {
    if (to_msbg) {
        if (!F.res[t]) return false;
        const uint32_t ci = F.off[0][t];
        if (!fluid_f[ci]) return false;
        int c[3];
        bcoord(F.g, t, c);
        *at = ci;
        *out = xf_msbg[ci] + xc[didx(K, c[0] >> 1, c[1] >> 1, c[2] >> 1)];
        return true;
    }
    if (!fluid_f[t]) return false;
    const int i = t % Fd.D[0], j = (t / Fd.D[0]) % Fd.D[1], k = t / (Fd.D[0] * Fd.D[1]);
    *at = (uint32_t)t;
    *out = xf[t] + xc[didx(K, i >> 1, j >> 1, k >> 1)];
    return true;
}

__global__ void k_dense_smooth(DenseArgs A, float* x, const float* __restrict__ b, int col, float omega) {
    pdl_wait();
    const DenseView& d = A.d;
    const int n = d.D[0] * d.D[1] * d.D[2];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float v;
    if (t < n && dense_smooth_value(A, x, b, t, col, omega, &v)) x[t] = v;
}

__global__ void k_dense_residual(DenseArgs A, const float* __restrict__ x, const float* __restrict__ b, float* r) {
    pdl_wait();
    const DenseView& d = A.d;
    const int n = d.D[0] * d.D[1] * d.D[2];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) r[t] = dense_residual_value(A, x, b, t);
}

__global__ void k_dense_restrict(DenseView K, const uint8_t* __restrict__ fluid_c, float* __restrict__ bc, int from_msbg,
                                 LevelView F, DenseView Fd, const float* __restrict__ rf) {
    pdl_wait();
    const int n = K.D[0] * K.D[1] * K.D[2];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) bc[t] = dense_restrict_value(K, fluid_c, from_msbg, F, Fd, rf, t);
}

__global__ void k_dense_prolong(DenseView K, const float* __restrict__ xc, int to_msbg, LevelView F, XStore xf_msbg,
                                DenseView Fd, float* __restrict__ xf, const uint8_t* __restrict__ fluid_f) {
    pdl_wait();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = to_msbg ? F.g.nb : Fd.D[0] * Fd.D[1] * Fd.D[2];
    uint32_t at;
    float v;
    if (t < n && dense_prolong_value(K, xc, to_msbg, F, xf_msbg.f, Fd, xf, fluid_f, t, &at, &v))
        (to_msbg ? xf_msbg.f : xf)[at] = v;
}

// ------------------------------- hierarchy setup kernels --------------------------------------
// coarse fluid flags: a coarse cell is fluid iff all of its children are fluid (copy when the
// block keeps one cell)
__global__ void k_coarse_fluid(LevelView F, LevelView K, const uint8_t* __restrict__ ff, uint8_t* __restrict__ fc) {
    const int b = blockIdx.x;
    const int rc = K.res[b], rf = F.res[b];
    if (!rc) return;
    const bool halved = rf == 2 * rc;
    const uint32_t of = F.off[0][b], oc = K.off[0][b];
    const int n3 = rc * rc * rc;
    for (int i = threadIdx.x; i < n3; i += blockDim.x) {
        int x = i % rc, y = (i / rc) % rc, z = i / (rc * rc);
        uint8_t f = 1;
        if (halved) {
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx) f &= ff[of + cidx(2 * x + dx, 2 * y + dy, 2 * z + dz, rf)];
        } else {
            f = ff[of + i];
        }
        fc[oc + i] = f;
    }
}

// coarse 1/rho per face: mean of the 4 fine faces (copy when the block keeps one cell)
// the three axes in one launch: axis = blockIdx.y
struct Face3 {
    float* p[3];
};

__global__ void k_coarse_bbar(LevelView F, LevelView K, Face3 bfs, Face3 bcvs) {
    const int a = blockIdx.y;
    const float* __restrict__ bf = bfs.p[a];
    float* __restrict__ bcv = bcvs.p[a];
    const int b = blockIdx.x;
    const int rc = K.res[b], rf = F.res[b];
    if (!rc) return;
    const bool halved = rf == 2 * rc;
    const int nf = (rc + 1) * rc * rc;
    const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
    for (int i = threadIdx.x; i < nf; i += blockDim.x) {
        int f[3];
        if (a == 0) { f[0] = i % (rc + 1); int rem = i / (rc + 1); f[1] = rem % rc; f[2] = rem / rc; }
        else if (a == 1) { f[0] = i % rc; int rem = i / rc; f[1] = rem % (rc + 1); f[2] = rem / (rc + 1); }
        else { f[0] = i % rc; int rem = i / rc; f[1] = rem % rc; f[2] = rem / rc; }
        float v;
        if (halved) {
            float s = 0.f;
            for (int d1 = 0; d1 < 2; ++d1)
                for (int d2 = 0; d2 < 2; ++d2) {
                    int q[3];
                    q[a] = 2 * f[a];
                    q[t1] = 2 * f[t1] + d1;
                    q[t2] = 2 * f[t2] + d2;
                    s += bf[F.off[1 + a][b] + fidx(a, q[0], q[1], q[2], rf)];
                }
            v = 0.25f * s;
        } else {
            v = bf[F.off[1 + a][b] + i];
        }
        bcv[K.off[1 + a][b] + i] = v;
    }
}

// finite-volume conductance W = geo * bbar: interior h, wall 0, absent neighbour h (Dirichlet),
// same level h, coarser neighbour (2/3) h, finer neighbour (4/3) h  (h = the block's cell size)
__global__ void k_conductance(LevelView L, Face3 bbars, Face3 Ws) {
    const int a = blockIdx.y;
    const float* __restrict__ bbar = bbars.p[a];
    float* __restrict__ W = Ws.p[a];
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    int cb[3];
    bcoord(L.g, b, cb);
    const float H = L.g.bs / (float)r;
    const int nf = (r + 1) * r * r;
    float gl = H, gh = H;
    for (int s = -1; s <= 1; s += 2) {
        int nc[3] = {cb[0], cb[1], cb[2]};
        nc[a] += s;
        float gv;
        if (!inside(L.g, nc)) gv = 0.f;
        else {
            int rn = L.res[bidx(L.g, nc[0], nc[1], nc[2])];
            if (rn == 0 || rn == r) gv = H;
            else if (2 * rn == r) gv = (2.f / 3.f) * H;
            else gv = (4.f / 3.f) * H;
        }
        if (s < 0) gl = gv;
        else gh = gv;
    }
    for (int i = threadIdx.x; i < nf; i += blockDim.x) {
        int fa;
        if (a == 0) fa = i % (r + 1);
        else if (a == 1) fa = (i / r) % (r + 1);
        else fa = i / (r * r);
        float geo = fa == 0 ? gl : (fa == r ? gh : H);
        W[L.off[1 + a][b] + i] = geo * bbar[L.off[1 + a][b] + i];
    }
}

__global__ void k_dense_fluid(DenseView K, int from_msbg, LevelView F, const uint8_t* __restrict__ ff, DenseView Fd,
                              uint8_t* __restrict__ fc) {
    int n = K.D[0] * K.D[1] * K.D[2];
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int i = t % K.D[0], j = (t / K.D[0]) % K.D[1], k = t / (K.D[0] * K.D[1]);
    uint8_t f = 1;
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                int ci = 2 * i + dx, cj = 2 * j + dy, ck = 2 * k + dz;
                uint8_t c;
                if (from_msbg) {
                    int b = bidx(F.g, ci, cj, ck);
                    c = F.res[b] ? ff[F.off[0][b]] : 0;
                } else {
                    c = ff[didx(Fd, ci, cj, ck)];
                }
                f &= c;
            }
    fc[t] = f;
}

// 1/rho on the faces of axis a of a uniform level: the mean of the four faces it covers on the next
// finer level, either the last block-structured level (one cell per block; a face is read from the
// block above it along a, else from the block below, else taken as 1 when neither is active) or the
// previous uniform level.
__global__ void k_dense_bbar(DenseView K, int a, int from_msbg, LevelView F, const float* __restrict__ fb, DenseView Fd,
                             float* __restrict__ bc) {
    const int n = (K.D[0] + (a == 0)) * (K.D[1] + (a == 1)) * (K.D[2] + (a == 2));
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int dx = K.D[0] + (a == 0), dy = K.D[1] + (a == 1);
    const int f[3] = {t % dx, (t / dx) % dy, t / (dx * dy)};
    const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
    float sum = 0.f;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        int q[3];
        q[a] = 2 * f[a];
        q[t1] = 2 * f[t1] + (d & 1);
        q[t2] = 2 * f[t2] + (d >> 1);
        float v = 1.f;
        if (from_msbg) {
            int lo[3] = {q[0], q[1], q[2]};
            lo[a] -= 1;
            const int bh = inside(F.g, q) ? bidx(F.g, q[0], q[1], q[2]) : -1;
            const int bl = inside(F.g, lo) ? bidx(F.g, lo[0], lo[1], lo[2]) : -1;
            if (bh >= 0 && F.res[bh]) v = fb[F.off[1 + a][bh]];           // its low face
            else if (bl >= 0 && F.res[bl]) v = fb[F.off[1 + a][bl] + 1];  // its high face
        } else {
            v = fb[dfidx(Fd, a, q[0], q[1], q[2])];
        }
        sum += v;
    }
    bc[t] = 0.25f * sum;
}

// conductance W = H * bbar on a uniform level, 0 on the domain walls
__global__ void k_dense_conductance(DenseView K, int a, float H, const float* __restrict__ bbar, float* W) {
    int n = (K.D[0] + (a == 0)) * (K.D[1] + (a == 1)) * (K.D[2] + (a == 2));
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int dx = K.D[0] + (a == 0), dy = K.D[1] + (a == 1);
    int f[3] = {t % dx, (t / dx) % dy, t / (dx * dy)};
    W[t] = (f[a] == 0 || f[a] == K.D[a]) ? 0.f : H * bbar[t];
}

// ------------------------------- coarsest FP64 dense solve ------------------------------------
// The coarsest level is a uniform grid (dense level, or the one-cell-per-block MSBG level).
struct Uniform {
    int D[3];
    int msbg;
    LevelView L;       // msbg == 1
    DenseArgs A;       // msbg == 0
    const uint8_t* fluid;
};

__device__ inline int uni_cell(const Uniform& U, int p) {  // cell index of grid position p, or -1
    if (!U.msbg) return p;
    return U.L.res[p] ? (int)U.L.off[0][p] : -1;
}
__device__ inline float uni_W(const Uniform& U, int p, int a, int hi) {
    if (!U.msbg) {
        int c[3] = {p % U.D[0], (p / U.D[0]) % U.D[1], p / (U.D[0] * U.D[1])};
        c[a] += hi;
        return U.A.W[a][dfidx(U.A.d, a, c[0], c[1], c[2])];
    }
    return U.A.W[a][U.L.off[1 + a][p] + hi];
}

// One CTA: enumerate fluid cells, assemble -A, regularise Neumann components, Cholesky, and
// write Minv = -( -A + reg )^-1 so that x = Minv b.  ex_n[0] = n (or -1 when n > EXACT_CAP).
// When the fluid flags match those of the last factorisation (prev) and the coefficients did not
// change (force == 0), the factorisation in place is still exact and the kernel returns at once.
__global__ void __launch_bounds__(512) k_coarse_factor(Uniform U, int* pos_of, int* idx, int* ex_n, double* M,
                                                       double* Minv, uint8_t* prev, int force) {
    __shared__ int cnt, diff;
    {
        const int np0 = U.D[0] * U.D[1] * U.D[2];
        if (threadIdx.x == 0) diff = force;
        __syncthreads();
        for (int p = threadIdx.x; p < np0; p += blockDim.x) {
            const int ci = uni_cell(U, p);
            const uint8_t f = (ci >= 0 && U.fluid[ci]) ? 1 : 0;
            if (f != prev[p]) diff = 1;
        }
        __syncthreads();
        if (!diff) return;
        for (int p = threadIdx.x; p < np0; p += blockDim.x) {
            const int ci = uni_cell(U, p);
            prev[p] = (ci >= 0 && U.fluid[ci]) ? 1 : 0;
        }
    }
    __shared__ int lab[EXACT_CAP];
    __shared__ int dir[EXACT_CAP];
    __shared__ double dsum[EXACT_CAP];
    __shared__ int csz[EXACT_CAP];
    __shared__ int changed;
    __shared__ double piv;
    const int np = U.D[0] * U.D[1] * U.D[2];
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    // deterministic compaction: serial order by position (np <= EXACT_POS_CAP)
    if (threadIdx.x == 0) {
        int c = 0;
        for (int p = 0; p < np; ++p) {
            int ci = uni_cell(U, p);
            if (ci >= 0 && U.fluid[ci]) {
                if (c < EXACT_CAP) idx[c] = p;
                pos_of[p] = c;
                ++c;
            } else {
                pos_of[p] = -1;
            }
        }
        cnt = c;
    }
    __syncthreads();
    const int n = cnt;
    if (n > EXACT_CAP) {
        if (threadIdx.x == 0) ex_n[0] = -1;
        return;
    }
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) M[t] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int p = idx[i];
        int c[3] = {p % U.D[0], (p / U.D[0]) % U.D[1], p / (U.D[0] * U.D[1])};
        double diag = 0.0, off = 0.0;
        for (int a = 0; a < 3; ++a)
            for (int s = 0; s < 2; ++s) {
                double w = uni_W(U, p, a, s);
                diag += w;
                int q[3] = {c[0], c[1], c[2]};
                q[a] += s ? 1 : -1;
                if (q[a] < 0 || q[a] >= U.D[a]) continue;
                int qp = q[0] + U.D[0] * (q[1] + U.D[1] * q[2]);
                int j = pos_of[qp];
                if (j >= 0) {
                    M[(size_t)i * n + j] -= w;
                    off += w;
                }
            }
        M[(size_t)i * n + i] += diag;
        dir[i] = (diag - off) > 1e-12 * diag ? 1 : 0;
        lab[i] = i;
    }
    __syncthreads();
    // connected components by min-label propagation
    for (int it = 0; it < n + 1; ++it) {
        if (threadIdx.x == 0) changed = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            int l = lab[i];
            for (int j = 0; j < n; ++j)
                if (M[(size_t)i * n + j] != 0.0 && j != i && lab[j] < l) l = lab[j];
            if (l < lab[i]) {
                lab[i] = l;
                changed = 1;
            }
        }
        __syncthreads();
        if (!changed) break;
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        dsum[i] = 0.0;
        csz[i] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < n; ++i) {
            int l = lab[i];
            dsum[l] += M[(size_t)i * n + i];
            csz[l] += 1;
            if (dir[i]) dir[l] = 1;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
        int i = t / n, j = t % n;
        int l = lab[i];
        if (lab[j] == l && !dir[l]) M[t] += dsum[l] / ((double)csz[l] * csz[l]);
    }
    __syncthreads();
    // Cholesky (lower, in place)
    for (int j = 0; j < n; ++j) {
        if (threadIdx.x == 0) {
            double s = M[(size_t)j * n + j];
            for (int k = 0; k < j; ++k) s -= M[(size_t)j * n + k] * M[(size_t)j * n + k];
            piv = sqrt(fmax(s, 1e-300));
            M[(size_t)j * n + j] = piv;
        }
        __syncthreads();
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
            double t = M[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) t -= M[(size_t)i * n + k] * M[(size_t)j * n + k];
            M[(size_t)i * n + j] = t / piv;
        }
        __syncthreads();
    }
    // inverse, one column per thread
    for (int col = threadIdx.x; col < n; col += blockDim.x) {
        for (int i = 0; i < n; ++i) {
            double t = (i == col) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) t -= M[(size_t)i * n + k] * Minv[(size_t)k * n + col];
            Minv[(size_t)i * n + col] = t / M[(size_t)i * n + i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double t = Minv[(size_t)i * n + col];
            for (int k = i + 1; k < n; ++k) t -= M[(size_t)k * n + i] * Minv[(size_t)k * n + col];
            Minv[(size_t)i * n + col] = t / M[(size_t)i * n + i];
        }
        for (int i = 0; i < n; ++i) Minv[(size_t)i * n + col] = -Minv[(size_t)i * n + col];
    }
    if (threadIdx.x == 0) ex_n[0] = n;
}

// x = Minv b on the fluid cells of the coarsest level (FP64 accumulation)
// row i of x = Minv b over the n fluid cells of the coarsest level
__device__ inline void coarse_apply_row(const Uniform& U, const int* __restrict__ idx, int n,
                                        const double* __restrict__ Minv, const float* b, float* x, int i) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += Minv[(size_t)i * n + j] * (double)b[uni_cell(U, idx[j])];
    x[uni_cell(U, idx[i])] = (float)s;
}
__global__ void k_coarse_apply(Uniform U, const int* __restrict__ idx, const int* __restrict__ ex_n,
                               const double* __restrict__ Minv, const float* __restrict__ b, float* __restrict__ x) {
    pdl_wait();
    const int n = ex_n[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        coarse_apply_row(U, idx, n, Minv, b, x, i);
}

// The uniform tail of an FV V-cycle in one CTA: the restriction from the level above the tail (the
// last MSBG level, one cell per block, or a larger uniform level) into the first tail level, the
// V-cycle over the tail levels down to the coarsest solve and back, and the prolongation into the
// level above.  Tail levels hold at most TAIL_MAX_CELLS cells, so as separate launches (about 14 on
// a 512/64-cell tail) each step costs a launch's latency rather than its work; here the steps are
// separated by CTA barriers instead.  (A 4096-cell level measured slower in one CTA than as
// launches, so larger uniform levels keep their own launches.)
// Every step applies the per-cell value functions of the separate kernels in the same order, so the
// results are bit-identical to the launch-per-step form.  The CTA reads and writes the levels in
// global memory; __syncthreads orders one step's writes before the next step's reads.  Within a
// step a thread computes the values of up to TAIL_K cells before it stores any of them, so their
// loads are in flight together (a store between them could alias the next cell's loads).
constexpr int TAIL_THREADS = 1024;
constexpr int TAIL_K = 4;             // cells per thread whose loads are issued together
constexpr int TAIL_MAX = 4;           // uniform levels the fused tail handles
constexpr int TAIL_MAX_CELLS = 512;   // largest uniform level it handles
struct TailLevel {
    DenseArgs A;
    float* x;
    float* b;
    float* r;
};
struct DenseTail {
    TailLevel lv[TAIL_MAX];
    int n;                    // uniform levels, lv[n - 1] the coarsest
    int from_msbg;            // the level above is the last MSBG level (F), else a uniform level (Fd)
    LevelView F;
    DenseView Fd;
    const float* rf;          // its residual
    float* xf;                // its x (FP32)
    const uint8_t* fluid_f;   // its fluid flags
    int sweeps, coarsest_iters, exact;
    float omega;
    Uniform U;                // exact coarsest solve
    const int* idx;
    const int* ex_n;
    const double* Minv;
};
__device__ inline int tail_cells(const TailLevel& L) { return L.A.d.D[0] * L.A.d.D[1] * L.A.d.D[2]; }
// One step over n items: value(t, &at, &v) says whether item t writes v at index at; then store.
template <class V, class S>
__device__ __forceinline__ void tail_step(int n, V value, S store) {
    for (int t0 = threadIdx.x; t0 < n; t0 += TAIL_K * blockDim.x) {
        float v[TAIL_K];
        uint32_t at[TAIL_K];
        bool w[TAIL_K];
#pragma unroll
        for (int k = 0; k < TAIL_K; ++k) {
            const int t = t0 + k * (int)blockDim.x;
            w[k] = t < n && value(t, &at[k], &v[k]);
        }
#pragma unroll
        for (int k = 0; k < TAIL_K; ++k)
            if (w[k]) store(at[k], v[k]);
    }
    __syncthreads();
}
__device__ inline void tail_smooth(const TailLevel& L, int iters, int rev, float omega) {
    const int n = tail_cells(L);
    for (int it = 0; it < iters; ++it)
        for (int k = 0; k < 2; ++k) {
            const int col = rev ? 1 - k : k;
            tail_step(
                n,
                [&](int t, uint32_t* at, float* v) {
                    *at = (uint32_t)t;
                    return dense_smooth_value(L.A, L.x, L.b, t, col, omega, v);
                },
                [&](uint32_t at, float v) { L.x[at] = v; });
        }
}
__global__ void __launch_bounds__(TAIL_THREADS) k_dense_tail(DenseTail T) {
    pdl_wait();
    {  // restriction from the level above; the first tail level's x starts at zero
        const TailLevel& C = T.lv[0];
        tail_step(
            tail_cells(C),
            [&](int t, uint32_t* at, float* v) {
                *at = (uint32_t)t;
                *v = dense_restrict_value(C.A.d, C.A.fluid, T.from_msbg, T.F, T.Fd, T.rf, t);
                return true;
            },
            [&](uint32_t at, float v) {
                C.b[at] = v;
                C.x[at] = 0.f;
            });
    }
    for (int m = 0; m + 1 < T.n; ++m) {
        const TailLevel& L = T.lv[m];
        const TailLevel& K = T.lv[m + 1];
        tail_smooth(L, T.sweeps, 0, T.omega);
        tail_step(
            tail_cells(L),
            [&](int t, uint32_t* at, float* v) {
                *at = (uint32_t)t;
                *v = dense_residual_value(L.A, L.x, L.b, t);
                return true;
            },
            [&](uint32_t at, float v) { L.r[at] = v; });
        tail_step(
            tail_cells(K),
            [&](int t, uint32_t* at, float* v) {
                *at = (uint32_t)t;
                *v = dense_restrict_value(K.A.d, K.A.fluid, 0, T.F, L.A.d, L.r, t);
                return true;
            },
            [&](uint32_t at, float v) {
                K.b[at] = v;
                K.x[at] = 0.f;
            });
    }
    const TailLevel& C = T.lv[T.n - 1];
    if (T.exact) {
        const int n = T.ex_n[0];
        for (int i = threadIdx.x; i < n; i += blockDim.x) coarse_apply_row(T.U, T.idx, n, T.Minv, C.b, C.x, i);
        __syncthreads();
    } else {
        tail_smooth(C, T.coarsest_iters, 0, T.omega);
    }
    for (int m = T.n - 2; m >= 0; --m) {
        const TailLevel& L = T.lv[m];
        const TailLevel& K = T.lv[m + 1];
        tail_step(
            tail_cells(L),
            [&](int t, uint32_t* at, float* v) {
                return dense_prolong_value(K.A.d, K.x, 0, T.F, nullptr, L.A.d, L.x, L.A.fluid, t, at, v);
            },
            [&](uint32_t at, float v) { L.x[at] = v; });
        tail_smooth(L, T.sweeps, 1, T.omega);
    }
    const TailLevel& L0 = T.lv[0];
    tail_step(
        T.from_msbg ? T.F.g.nb : T.Fd.D[0] * T.Fd.D[1] * T.Fd.D[2],
        [&](int t, uint32_t* at, float* v) {
            return dense_prolong_value(L0.A.d, L0.x, T.from_msbg, T.F, T.xf, T.Fd, T.xf, T.fluid_f, t, at, v);
        },
        [&](uint32_t at, float v) { T.xf[at] = v; });
}

// ------------------------------------------------------------------------------------------------
// Host orchestration
// ------------------------------------------------------------------------------------------------
static LevelView lview(const aw_solver* S, int m) {
    const MsbgState& G = S->g->st;
    const MGLevel& L = S->lv[m];
    LevelView v;
    v.g = G.geo;
    v.res = L.res.p;
    for (int k = 0; k < 4; ++k) v.off[k] = L.off[k].p;
    return v;
}
static DenseView dview(const MGLevel& L) {
    DenseView d;
    d.D[0] = L.D[0];
    d.D[1] = L.D[1];
    d.D[2] = L.D[2];
    return d;
}
static XStore xstore(aw_solver* S, int m) {
    MGLevel& L = S->lv[m];
    XStore x;
    if (m == 0 && S->x0) {
        x.f = S->x0;
        return x;
    }
    if (L.half) {
        x.h = L.xh.p;
        x.scale = L.xscale.p;
    } else {
        x.f = L.x.p;
    }
    return x;
}
static const float* bptr(aw_solver* S, int m) { return (m == 0 && S->b0) ? S->b0 : S->lv[m].b.p; }
static Coef3 coef(const MGLevel& L) { return Coef3{{L.W[0].p, L.W[1].p, L.W[2].p}}; }
// Slots per CTA.  One-cell blocks take 64 slots (a quarter of the threads), not 256: a level's
// slot image is sized for its largest group, and 256 one-cell slots (70 KB in FP32, 98 KB in FP64)
// held every CTA of the level to 3 (or 2) per SM.  At 64 the image stays under 18 KB (25 KB in FP64)
// and 6 CTAs fit per SM (poisson_256 to 1e-6: 8.05 to 5.90 ms; dam_drop_128 solve 2.08 to 1.86 ms).
// Blocks of 2^3 cells take 16 slots (half the threads) rather than 32: more, shorter CTAs on the
// small levels (dam_drop_128 solve 1.86 to 1.76 ms).
static int slots_per_cta(int r) {
    return r == 1 ? 64 : (r == 2 ? 16 : std::max(1, std::min(256, 256 / (r * r * r))));
}

// Build the CTA batches of one block-structured level from its per-block resolutions.
static aw_status build_batches(MGLevel& L, const Geo& geo) {
    const int nb = (int)L.h_res.size();
    for (int k = 0; k < 3; ++k) {
        std::vector<int> by_res[17];
        for (int b = 0; b < nb; ++b) {
            const int r = L.h_res[b];
            if (!r) continue;
            if (k < 2) {
                int c[3];
                bcoord(geo, b, c);
                if (((c[0] + c[1] + c[2]) & 1) != k) continue;
            }
            by_res[r].push_back(b);
        }
        std::vector<int> blocks;
        std::vector<int4> desc;
        for (int r = 16; r >= 1; --r) {
            const int G = slots_per_cta(r);
            for (size_t i = 0; i < by_res[r].size(); i += G) {
                const int cnt = (int)std::min<size_t>(G, by_res[r].size() - i);
                desc.push_back(make_int4((int)blocks.size(), cnt, r, 0));
                for (int j = 0; j < cnt; ++j) blocks.push_back(by_res[r][i + j]);
            }
            if (!by_res[r].empty()) {
                const int Gm = std::min<int>(G, (int)by_res[r].size());
                const size_t X3 = (size_t)(r + 2) * (r + 2) * (r + 2);
                L.smem_smooth = std::max(L.smem_smooth, slot_image_bytes(Gm, r, sizeof(float)));
                L.smem_x64 = std::max(L.smem_x64, slot_image_bytes(Gm, r, sizeof(double)));
                L.smem_meta = std::max(L.smem_meta, (size_t)Gm * NMETA * 4 + 16);
                L.smem_prolong = std::max(L.smem_prolong, (size_t)Gm * (X3 * 4 + NMETA * 4) + 16);
            }
        }
        L.ndesc[k] = (int)desc.size();
        L.h_blocks[k] = std::move(blocks);
        if (L.ndesc[k]) {
            AW_TRY(L.desc[k].ensure(desc.size()));
            AW_CUDA(cudaMemcpy(L.desc[k].p, desc.data(), desc.size() * sizeof(int4), cudaMemcpyHostToDevice));
        }
    }
    return AW_OK;
}
static Batch batch(const MGLevel& L, int k) { return Batch{L.desc[k].p, L.meta[k].p, (int)L.h_blocks[k].size()}; }

// Slot metadata of one batch of level m, laid out in batch order (field-major): block id, offsets,
// the six face neighbours (cell offset, kind, block) and the block's cells on the adjacent levels.
// One thread per slot, from the level arrays already on the device (no host copy of the offsets).
struct MetaSrc {
    const int* res;
    const uint32_t* off[4];
};
__global__ void k_build_meta(Geo geo, const int* __restrict__ blocks, int n, MetaSrc h, MetaSrc finer, MetaSrc coarser,
                             int* __restrict__ mt) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int b = blocks[j];
    const int r = h.res[b];
    auto F = [&](int f, int v) { mt[(size_t)f * n + j] = v; };
    F(MF_BLOCK, b);
    for (int q = 0; q < 4; ++q) F(MF_OFF + q, (int)h.off[q][b]);
    int c[3];
    bcoord(geo, b, c);
    for (int a = 0; a < 3; ++a)
        for (int sd = 0; sd < 2; ++sd) {
            const int f = MF_NB + 3 * (2 * a + sd);
            int nc[3] = {c[0], c[1], c[2]};
            nc[a] += sd ? 1 : -1;
            int o = 0, kind = NB_NONE, nbk = 0;
            if (inside(geo, nc)) {
                const int q = bidx(geo, nc[0], nc[1], nc[2]);
                const int rn = h.res[q];
                if (rn) {
                    o = (int)h.off[0][q];
                    kind = rn == r ? NB_SAME : (rn < r ? NB_COARSE : NB_FINE);
                    nbk = q;
                }
            }
            F(f, o);
            F(f + 1, kind);
            F(f + 2, nbk);
        }
    F(MF_FINE_OFF, finer.res ? (int)finer.off[0][b] : 0);
    F(MF_FINE_RES, finer.res ? finer.res[b] : 0);
    F(MF_COARSE_OFF, coarser.res ? (int)coarser.off[0][b] : 0);
    F(MF_COARSE_RES, coarser.res ? coarser.res[b] : 0);
}
static MetaSrc meta_src(const MGLevel* L) {
    MetaSrc m{};
    if (!L) return m;
    m.res = L->res.p;
    for (int k = 0; k < 4; ++k) m.off[k] = L->off[k].p;
    return m;
}
// The slot metadata of level m's three batches, built on the device.
static aw_status build_meta(MGLevel& L, const Geo& geo, const MGLevel* finer, const MGLevel* coarser, cudaStream_t s) {
    for (int k = 0; k < 3; ++k) {
        const std::vector<int>& blocks = L.h_blocks[k];
        const size_t n = blocks.size();
        if (!n) continue;
        AW_TRY(L.blk[k].ensure(n));
        AW_CUDA(cudaMemcpyAsync(L.blk[k].p, blocks.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
        AW_TRY(L.meta[k].ensure(NMETA * n));
        k_build_meta<<<nblk(n), 256, 0, s>>>(geo, L.blk[k].p, (int)n, meta_src(&L), meta_src(finer), meta_src(coarser),
                                            L.meta[k].p);
        AW_LAUNCH();
    }
    return AW_OK;
}
static bool fv(const aw_solver* S) { return S->d.operator_mode == AW_OPERATOR_FV; }

static Uniform uniform_of(aw_solver* S, int m) {
    MGLevel& L = S->lv[m];
    Uniform U{};
    if (L.dense) {
        for (int a = 0; a < 3; ++a) U.D[a] = L.D[a];
        U.msbg = 0;
    } else {
        for (int a = 0; a < 3; ++a) U.D[a] = S->g->st.geo.D[a];
        U.msbg = 1;
        U.L = lview(S, m);
    }
    U.A.d = dview(L);
    for (int a = 0; a < 3; ++a) U.A.W[a] = L.W[a].p;
    U.A.fluid = L.fluid.p;
    U.fluid = L.fluid.p;
    return U;
}

// A V-cycle kernel launch, as a programmatic dependent of the kernel before it in the stream (the
// kernels call pdl_wait before reading what it wrote).
template <typename... KArgs, typename... Args>
static aw_status launch_dep(const aw_solver* S, void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem,
                            cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = S->use_pdl ? 1 : 0;
    AW_CUDA(cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...));
    AW_LAUNCH();
    return AW_OK;
}

static aw_status zero_x(aw_solver* S, int m, cudaStream_t s) {
    MGLevel& L = S->lv[m];
    if (L.half) {
        AW_CUDA(cudaMemsetAsync(L.xh.p, 0, L.ncell() * sizeof(__half), s));
        AW_CUDA(cudaMemsetAsync(L.xscale.p, 0, S->g->st.nb * sizeof(float), s));
    } else if (m == 0 && S->x0) {
        AW_CUDA(cudaMemsetAsync(S->x0, 0, L.ncell() * sizeof(float), s));
    } else {
        AW_CUDA(cudaMemsetAsync(L.x.p, 0, L.ncell() * sizeof(float), s));
    }
    return AW_OK;
}

// Red-black block Gauss-Seidel on level m.  The post-smoothing of an FV V-cycle (reverse) runs the
// adjoint order: block colours and cell colours black before red, so that the V-cycle is a
// symmetric preconditioner for CG.  Reference mode keeps the reference's order (VCycle.cuh:251-304).
static aw_status smooth_level(aw_solver* S, int m, int iterations, cudaStream_t s, bool post = false) {
    MGLevel& L = S->lv[m];
    const int cf = fv(S) ? 1 : 0;
    const int rev = post && fv(S) ? 1 : 0;
    if (L.dense) {
        DenseArgs A{dview(L), {L.W[0].p, L.W[1].p, L.W[2].p}, L.fluid.p};
        size_t n = L.ncell();
        for (int it = 0; it < iterations; ++it)
            for (int k = 0; k < 2; ++k) {
                AW_TRY(launch_dep(S, k_dense_smooth, nblk(n), 256, 0, s, A, L.x.p, (const float*)L.b.p, rev ? 1 - k : k,
                                  S->d.omega));
            }
        return AW_OK;
    }
    const int nb = S->g->st.nb;
    // a negative activation threshold keeps every block active: no status arrays
    const bool act = S->d.theta >= 0.f;
    if (act) AW_CUDA(cudaMemsetAsync(L.status[0].p, 1, nb, s));
    SmoothParams P{S->d.omega, S->d.target_reduction, S->d.theta, S->d.block_iterations, cf, rev};
    LevelView V = lview(S, m);
    XStore x = xstore(S, m);
    int cur = 0;
    for (int it = 0; it < iterations; ++it) {
        if (act) AW_CUDA(cudaMemsetAsync(L.status[cur ^ 1].p, 0, nb, s));
        for (int k = 0; k < 2; ++k) {
            const int rb = rev ? 1 - k : k;
            if (!L.ndesc[rb]) continue;
            AW_TRY(launch_dep(S, k_smooth, (unsigned)L.ndesc[rb], 256, L.smem_smooth, s, V, x, bptr(S, m), coef(L),
                              (const uint8_t*)L.fluid.p, batch(L, rb),
                              (const uint8_t*)(act ? L.status[cur].p : nullptr), act ? L.status[cur ^ 1].p : nullptr, P));
        }
        cur ^= 1;
    }
    return AW_OK;
}

static aw_status residual_level(aw_solver* S, int m, double* part, cudaStream_t s) {
    MGLevel& L = S->lv[m];
    const int cf = fv(S) ? 1 : 0;
    if (L.dense) {
        DenseArgs A{dview(L), {L.W[0].p, L.W[1].p, L.W[2].p}, L.fluid.p};
        return launch_dep(S, k_dense_residual, nblk(L.ncell()), 256, 0, s, A, (const float*)L.x.p, (const float*)L.b.p,
                          L.r.p);
    }
    XStore x = xstore(S, m);
    if (L.ndesc[2]) {
        AW_TRY(launch_dep(S, k_residual<SrcX>, (unsigned)L.ndesc[2], 256, L.smem_smooth, s, SrcX{x}, bptr(S, m), coef(L),
                          (const uint8_t*)L.fluid.p, batch(L, 2), cf, L.r.p, (double*)nullptr, part));
    }
    return AW_OK;
}

static aw_status restrict_level(aw_solver* S, int m, cudaStream_t s) {
    MGLevel& F = S->lv[m];
    MGLevel& K = S->lv[m + 1];
    const int cf = fv(S) ? 1 : 0;
    if (K.dense) {
        LevelView Fv = F.dense ? LevelView{} : lview(S, m);
        if (F.dense) Fv.g = S->g->st.geo;
        return launch_dep(S, k_dense_restrict, nblk(K.ncell()), 256, 0, s, dview(K), (const uint8_t*)K.fluid.p, K.b.p,
                          F.dense ? 0 : 1, Fv, dview(F), (const float*)F.r.p);
    }
    if (K.ndesc[2]) {
        AW_TRY(launch_dep(S, k_restrict, (unsigned)K.ndesc[2], 256, K.smem_meta, s, (const float*)F.r.p, K.b.p,
                          (const uint8_t*)K.fluid.p, cf, batch(K, 2)));
    }
    return AW_OK;
}

static aw_status prolong_level(aw_solver* S, int m, cudaStream_t s) {
    MGLevel& F = S->lv[m];
    MGLevel& K = S->lv[m + 1];
    const int cf = fv(S) ? 1 : 0;
    if (K.dense) {
        LevelView Fv = F.dense ? LevelView{} : lview(S, m);
        if (F.dense) Fv.g = S->g->st.geo;
        size_t n = F.dense ? F.ncell() : (size_t)S->g->st.nb;
        XStore xf = F.dense ? XStore{} : xstore(S, m);
        AW_CHECK_ARG(F.dense || xf.f, "FP16 storage on the one-cell MSBG level is not supported");
        return launch_dep(S, k_dense_prolong, nblk(n), 256, 0, s, dview(K), (const float*)K.x.p, F.dense ? 0 : 1, Fv, xf,
                          dview(F), F.x.p, (const uint8_t*)F.fluid.p);
    }
    if (F.ndesc[2]) {
        AW_TRY(launch_dep(S, k_prolong, (unsigned)F.ndesc[2], 256, F.half ? F.smem_prolong : F.smem_meta, s, xstore(S, m),
                          xstore(S, m + 1), (const uint8_t*)F.fluid.p, cf, batch(F, 2)));
    }
    return AW_OK;
}

static aw_status coarsest(aw_solver* S, int m, cudaStream_t s) {
    MGLevel& L = S->lv[m];
    if (fv(S) && S->exact) {
        Uniform U = uniform_of(S, m);
        float* x = L.dense ? L.x.p : (m == 0 && S->x0 ? S->x0 : L.x.p);
        return launch_dep(S, k_coarse_apply, 4, 128, 0, s, U, (const int*)S->ex_idx.p, (const int*)S->ex_n.p,
                          (const double*)S->Minv.p, bptr(S, m), x);
    }
    return smooth_level(S, m, S->d.coarsest_iterations, s);
}

// The uniform levels below level m (the last MSBG level or a uniform one) as one launch
// (k_dense_tail): restriction into them, their V-cycle and the prolongation back into m.
static aw_status dense_tail(aw_solver* S, int m, cudaStream_t s) {
    const int last = (int)S->lv.size() - 1;
    MGLevel& F = S->lv[m];
    DenseTail T{};
    T.n = last - m;
    T.from_msbg = F.dense ? 0 : 1;
    for (int j = 0; j < T.n; ++j) {
        MGLevel& L = S->lv[m + 1 + j];
        T.lv[j].A = DenseArgs{dview(L), {L.W[0].p, L.W[1].p, L.W[2].p}, L.fluid.p};
        T.lv[j].x = L.x.p;
        T.lv[j].b = L.b.p;
        T.lv[j].r = L.r.p;
    }
    if (F.dense) {
        T.Fd = dview(F);
        T.xf = F.x.p;
    } else {
        T.F = lview(S, m);
        T.xf = xstore(S, m).f;
    }
    T.rf = F.r.p;
    T.fluid_f = F.fluid.p;
    T.sweeps = S->d.dense_sweeps;
    T.coarsest_iters = S->d.coarsest_iterations;
    T.exact = S->exact ? 1 : 0;
    T.omega = S->d.omega;
    if (S->exact) {
        T.U = uniform_of(S, last);
        T.idx = S->ex_idx.p;
        T.ex_n = S->ex_n.p;
        T.Minv = S->Minv.p;
    }
    return launch_dep(S, k_dense_tail, 1, TAIL_THREADS, 0, s, T);
}

static aw_status vcycle(aw_solver* S, int m, cudaStream_t s) {
    const int last = (int)S->lv.size() - 1;
    if (m == last) return coarsest(S, m, s);
    MGLevel& L = S->lv[m];
    AW_TRY(smooth_level(S, m, L.dense ? S->d.dense_sweeps : S->d.pre_smooth, s));
    AW_TRY(residual_level(S, m, nullptr, s));
    if (S->tail && m + 1 == S->tail) {
        AW_TRY(dense_tail(S, m, s));
        return smooth_level(S, m, L.dense ? S->d.dense_sweeps : S->d.post_smooth, s, true);
    }
    AW_TRY(restrict_level(S, m, s));
    AW_TRY(zero_x(S, m + 1, s));
    AW_TRY(vcycle(S, m + 1, s));
    AW_TRY(prolong_level(S, m, s));
    AW_TRY(smooth_level(S, m, L.dense ? S->d.dense_sweeps : S->d.post_smooth, s, true));
    return AW_OK;
}

}  // namespace aw

using namespace aw;

// ================================================================================================
// C ABI
// ================================================================================================
extern "C" aw_status aw_solver_default_desc(int32_t mode, aw_solver_desc* d) {
    AW_CHECK_ARG(d && (mode == AW_OPERATOR_FV || mode == AW_OPERATOR_REFERENCE), "bad argument");
    memset(d, 0, sizeof *d);
    d->operator_mode = mode;
    d->precision = AW_PRECISION_FP32;
    d->mg_levels = 0;
    d->pre_smooth = 2;
    d->post_smooth = 2;
    d->coarsest_iterations = 50;
    d->dense_sweeps = 2;
    d->max_cycles = 100;
    d->tolerance = 1e-6;
    if (mode == AW_OPERATOR_REFERENCE) {
        d->block_iterations = 10;     // MAX_BLOCK_ITER
        d->omega = 0.85714f;          // OMEGA
        d->target_reduction = 0.33f;  // TARGET_RESIDUAL_REDUCTION
        d->theta = 1e-4f;             // Smoother.cuh:286
    } else {
        d->block_iterations = 2;
        // Over-relaxed block Gauss-Seidel.  With the symmetric V-cycle preconditioning CG, 1.35
        // reaches 1e-6 on the 4-level poisson_256 layout in 5 iterations (6 at 1.0) and needs 7
        // instead of 9 on the 34.7M-particle dam_drop2_256 step; at 1.5 and above the smoothing
        // degrades and the iteration counts rise again.
        d->omega = 1.35f;
        d->target_reduction = 0.33f;
        d->theta = -1.0f;  // every block stays active (no residual-threshold deactivation)
    }
    return AW_OK;
}

static int ilog2(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

// Coefficients of the block-structured levels from BETA_COEFF_* (stream-ordered): level 0 takes
// them as they are, coarser levels average them (k_coarse_bbar); FV mode multiplies by the face
// geometry (k_conductance), reference mode coarsens with galerkinCoarsen (MSBG.cuh:378-498).
static aw_status build_coefficients(aw_solver* S, cudaStream_t s) {
    MsbgState& G = S->g->st;
    const bool ref = S->d.operator_mode == AW_OPERATOR_REFERENCE;
    const int nb = G.nb;
    for (int m = 0; m < S->nmsbg; ++m) {
        MGLevel& L = S->lv[m];
        LevelView V = lview(S, m);
        Face3 bb{{L.bbar[0].p, L.bbar[1].p, L.bbar[2].p}};
        if (m == 0) {
            for (int a = 0; a < 3; ++a)
                AW_CUDA(cudaMemcpyAsync(L.bbar[a].p, G.ch[AW_BETA_COEFF_X + a], L.nface(a) * sizeof(float),
                                        cudaMemcpyDeviceToDevice, s));
        } else {
            MGLevel& P = S->lv[m - 1];
            Face3 fb{{P.bbar[0].p, P.bbar[1].p, P.bbar[2].p}};
            k_coarse_bbar<<<dim3(nb, 3), 128, 0, s>>>(lview(S, m - 1), V, fb, bb);
            AW_LAUNCH();
        }
        if (!ref) {
            k_conductance<<<dim3(nb, 3), 128, 0, s>>>(V, bb, Face3{{L.W[0].p, L.W[1].p, L.W[2].p}});
            AW_LAUNCH();
            continue;
        }
        for (int a = 0; a < 3; ++a) {
            if (m == 0) {
                AW_CUDA(cudaMemcpyAsync(L.W[a].p, L.bbar[a].p, L.nface(a) * sizeof(float), cudaMemcpyDeviceToDevice,
                                        s));
            } else {
                AW_CUDA(cudaMemsetAsync(L.W[a].p, 0, L.nface(a) * sizeof(float), s));
                k_galerkin_ref<<<nb, 256, 0, s>>>(G.geo, G.level.p, a, m, S->lv[m - 1].W[a].p, L.W[a].p,
                                                  S->lv[m - 1].off[1 + a].p, L.off[1 + a].p);
                AW_LAUNCH();
            }
        }
    }
    // uniform levels below one cell per block (FV mode): 1/rho averaged down face by face, so that
    // their operator follows the density of the finer levels
    for (int m = S->nmsbg; m < (int)S->lv.size(); ++m) {
        MGLevel& L = S->lv[m];
        const MGLevel& P = S->lv[m - 1];
        const bool from_msbg = m == S->nmsbg;
        for (int a = 0; a < 3; ++a) {
            k_dense_bbar<<<nblk(L.nface(a)), 256, 0, s>>>(dview(L), a, from_msbg ? 1 : 0, lview(S, m - 1),
                                                           P.bbar[a].p, dview(P), L.bbar[a].p);
            AW_LAUNCH();
            k_dense_conductance<<<nblk(L.nface(a)), 256, 0, s>>>(dview(L), a, L.H, L.bbar[a].p, L.W[a].p);
            AW_LAUNCH();
        }
    }
    return AW_OK;
}

extern "C" aw_status aw_solver_update_coefficients(aw_solver* S, aw_stream s) {
    AW_CHECK_ARG(S, "null solver");
    S->coef_dirty = true;
    return build_coefficients(S, (cudaStream_t)s);
}

// The multigrid hierarchy of the grid's current layout, built into S.  Every device buffer grows
// only: a re-layout whose levels fit the previous ones reuses their storage, so rebuilding the
// solver after aw_flip_rebuild_levels allocates and frees nothing in the common case.
static void reset_level(MGLevel& L) {
    L.dense = false;
    L.D[0] = L.D[1] = L.D[2] = 0;
    L.H = 0.f;
    L.half = false;
    L.h_res.clear();
    for (int k = 0; k < 4; ++k) L.tot[k] = 0;
    for (int k = 0; k < 3; ++k) {
        L.h_blocks[k].clear();
        L.ndesc[k] = 0;
    }
    L.smem_smooth = L.smem_x64 = L.smem_prolong = L.smem_meta = 0;
    L.maxres = 0;
}

// The stencils assume 2:1 grading between face neighbours.
static aw_status check_grading(const MsbgState& G) {
    const Geo& geo = G.geo;
    for (int b = 0; b < G.nb; ++b) {
        if ((int)G.h_level[b] >= geo.L) continue;
        int c[3];
        bcoord(geo, b, c);
        for (int a = 0; a < 3; ++a) {
            int nc[3] = {c[0], c[1], c[2]};
            nc[a] += 1;
            if (!inside(geo, nc)) continue;
            uint32_t nl = G.h_level[bidx(geo, nc[0], nc[1], nc[2])];
            if ((int)nl < geo.L && std::abs((int)nl - (int)G.h_level[b]) > 1)
                return set_error(AW_ERR_INVALID_ARGUMENT,
                                 "level map is not 2:1 graded (block %d); run aw_msbg_enforce_grading first", b);
        }
    }
    return AW_OK;
}

static aw_status solver_build(aw_solver* S) {
    aw_msbg* g = S->g;
    MsbgState& G = g->st;
    S->exact = false;
    S->coef_dirty = true;
    S->smem_max = S->smem_max64 = 0;
    if (S->cycle) cudaGraphExecDestroy(S->cycle);
    S->cycle = nullptr;
    S->cycle_x0 = S->cycle_b0 = nullptr;
    if (S->cgloop) cudaGraphExecDestroy(S->cgloop);
    S->cgloop = nullptr;
    S->cgloop_p = nullptr;
    S->cycle_kernels = 0;
    S->x0 = nullptr;
    S->b0 = nullptr;
    const bool ref = S->d.operator_mode == AW_OPERATOR_REFERENCE;
    const int nb = G.nb;
    int M = S->d.mg_levels > 0 ? S->d.mg_levels : (ref ? G.geo.L : ilog2(G.geo.R0) + 1);
    if (!ref) M = std::min(M, ilog2(G.geo.R0) + 1);
    cudaStream_t s = 0;
    if (S->lv.size() < (size_t)M) S->lv.resize(M);
    DBuf<uint32_t>& off4 = G.scratch_off4;
    AW_TRY(off4.ensure(4 * (size_t)nb));
    int nlev = M;
    for (int m = 0; m < M; ++m) {
        MGLevel& L = S->lv[m];
        reset_level(L);
        AW_TRY(L.res.ensure(nb));
        AW_TRY(level_offsets(G, m, ref ? 1 : 0, off4.p, L.res.p, L.tot, s));
        for (int k = 0; k < 4; ++k) {
            AW_TRY(L.off[k].ensure(nb));
            AW_CUDA(cudaMemcpy(L.off[k].p, off4.p + (size_t)k * nb, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice));
        }
        L.h_res.resize(nb);
        AW_CUDA(cudaMemcpy(L.h_res.data(), L.res.p, nb * sizeof(int), cudaMemcpyDeviceToHost));
        for (int b = 0; b < nb; ++b) L.maxres = std::max(L.maxres, L.h_res[b]);
        if (L.maxres == 0) {
            nlev = m;
            break;
        }
        AW_TRY(build_batches(L, G.geo));
        AW_TRY(L.status[0].ensure(nb));
        AW_TRY(L.status[1].ensure(nb));
        L.half = (S->d.precision == AW_PRECISION_MIXED) && m >= 1 && m < M - 1 + (ref ? 0 : 1) && L.maxres > 1;
        size_t nc = L.ncell();
        AW_TRY(L.x.ensure(nc));
        AW_TRY(L.b.ensure(nc));
        AW_TRY(L.r.ensure(nc));
        AW_TRY(L.fluid.ensure(nc + 16));  // whole 32-bit words are staged
        AW_CUDA(cudaMemset(L.x.p, 0, nc * sizeof(float)));
        AW_CUDA(cudaMemset(L.b.p, 0, nc * sizeof(float)));
        AW_CUDA(cudaMemset(L.fluid.p, 1, nc + 16));
        if (L.half) {
            AW_TRY(L.xh.ensure(nc));
            AW_TRY(L.xscale.ensure(nb));
            AW_CUDA(cudaMemset(L.xh.p, 0, nc * sizeof(__half)));
            AW_CUDA(cudaMemset(L.xscale.p, 0, nb * sizeof(float)));
        }
        for (int a = 0; a < 3; ++a) {
            AW_TRY(L.W[a].ensure(L.nface(a)));
            AW_TRY(L.bbar[a].ensure(L.nface(a)));
        }
    }
    S->nmsbg = nlev;
    for (int m = 0; m < S->nmsbg; ++m) {
        MGLevel& L = S->lv[m];
        AW_TRY(build_meta(L, G.geo, m > 0 ? &S->lv[m - 1] : nullptr, m + 1 < S->nmsbg ? &S->lv[m + 1] : nullptr, s));
        S->smem_max = std::max({S->smem_max, L.smem_smooth, L.smem_prolong, L.smem_meta});
        S->smem_max64 = std::max(S->smem_max64, L.smem_x64);
    }
    // uniform continuation below one cell per block (FV mode)
    size_t used = (size_t)S->nmsbg;
    if (!ref && S->nmsbg > 0 && S->lv[S->nmsbg - 1].maxres == 1) {
        int Dd[3] = {G.geo.D[0], G.geo.D[1], G.geo.D[2]};
        float H = G.geo.bs;
        while (Dd[0] % 2 == 0 && Dd[1] % 2 == 0 && Dd[2] % 2 == 0 && (long)Dd[0] * Dd[1] * Dd[2] > 64) {
            if (S->lv.size() <= used) S->lv.emplace_back();
            MGLevel& L = S->lv[used++];
            reset_level(L);
            L.dense = true;
            for (int a = 0; a < 3; ++a) L.D[a] = Dd[a] / 2;
            H *= 2.f;
            L.H = H;
            size_t nc = L.ncell();
            AW_TRY(L.x.ensure(nc));
            AW_TRY(L.b.ensure(nc));
            AW_TRY(L.r.ensure(nc));
            AW_TRY(L.fluid.ensure(nc));
            AW_CUDA(cudaMemset(L.x.p, 0, nc * sizeof(float)));
            AW_CUDA(cudaMemset(L.b.p, 0, nc * sizeof(float)));
            for (int a = 0; a < 3; ++a) {
                AW_TRY(L.W[a].ensure(L.nface(a)));
                AW_TRY(L.bbar[a].ensure(L.nface(a)));
            }
            for (int a = 0; a < 3; ++a) Dd[a] /= 2;
        }
        S->lv.resize(used);  // levels beyond the new hierarchy are released
        // the coarsest level is uniform: factorise it densely when small enough
        MGLevel& C = S->lv.back();
        size_t npos = C.dense ? C.ncell() : (size_t)nb;
        if (npos <= (size_t)EXACT_POS_CAP) {
            AW_TRY(S->M.ensure((size_t)EXACT_CAP * EXACT_CAP));
            AW_TRY(S->Minv.ensure((size_t)EXACT_CAP * EXACT_CAP));
            AW_TRY(S->ex_idx.ensure(EXACT_CAP));
            AW_TRY(S->ex_pos.ensure(npos));
            AW_TRY(S->ex_prev.ensure(npos));
            AW_CUDA(cudaMemset(S->ex_prev.p, 0xFF, npos));
            AW_TRY(S->ex_n.ensure(1));
            AW_CUDA(cudaMemset(S->ex_n.p, 0, sizeof(int)));
            S->exact = true;
        }
    }
    S->lv.resize(used);
    // coefficients of every level
    AW_TRY(build_coefficients(S, 0));
    {  // always opted in: static shared memory (k_smooth's per-slot state) counts against the default 48 KB too
        AW_CUDA(cudaFuncSetAttribute(k_smooth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_max));
        AW_CUDA(cudaFuncSetAttribute(k_residual<SrcX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_max));
        AW_CUDA(cudaFuncSetAttribute(k_prolong, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_max));
        AW_CUDA(cudaFuncSetAttribute(k_restrict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_max));
    }
    AW_CUDA(cudaFuncSetAttribute(k_residual<SrcD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_max64));
    AW_CUDA(cudaFuncSetAttribute(k_apply_dot, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_max64));
    if (S->d.precision == AW_PRECISION_MIXED) {
        const size_t nc0 = S->lv[0].ncell();
        AW_TRY(S->cg_r.ensure(nc0));
        AW_TRY(S->cg_d.ensure(nc0));
        AW_TRY(S->cg_q.ensure(nc0));
        AW_TRY(S->cg_sc.ensure(4));
        AW_TRY(S->cg_zero.ensure(nc0));
        AW_CUDA(cudaMemset(S->cg_zero.p, 0, nc0 * sizeof(float)));
        AW_CUDA(cudaMemset(S->cg_d.p, 0, nc0 * sizeof(double)));
    }
    if (S->d.precision == AW_PRECISION_FP32_PCG) {
        const size_t nc0 = S->lv[0].ncell();
        AW_TRY(S->cg32_d.ensure(std::max<size_t>(nc0, 1)));
        AW_TRY(S->cg32_q.ensure(std::max<size_t>(nc0, 1)));
        AW_TRY(S->cg32_sc.ensure(4));
        AW_TRY(S->cg_zero.ensure(std::max<size_t>(nc0, 1)));
        AW_TRY(S->partials32.ensure(4096));
        AW_CUDA(cudaMemset(S->cg_zero.p, 0, std::max<size_t>(nc0, 1) * sizeof(float)));
        AW_CUDA(cudaMemset(S->cg32_d.p, 0, std::max<size_t>(nc0, 1) * sizeof(float)));
    }
    size_t nparts = (size_t)nb + 1024;
    AW_TRY(S->partials.ensure(nparts));
    AW_TRY(S->norm.ensure(2));
    S->use_graph = getenv("AW_NO_GRAPH") == nullptr;
    S->use_pdl = getenv("AW_NO_PDL") == nullptr;
    S->use_devloop = getenv("AW_NO_DEVLOOP") == nullptr;
    // the uniform tail as one launch (FV mode): the uniform levels from the first one of at most
    // TAIL_MAX_CELLS cells down, at most TAIL_MAX of them, below a level that stores x in FP32
    // (AW_NO_DENSE_TAIL keeps one launch per step)
    S->tail = 0;
    if (!ref && S->nmsbg > 0 && getenv("AW_NO_DENSE_TAIL") == nullptr) {
        const int nl = (int)S->lv.size();
        int j = S->nmsbg;
        while (j < nl && S->lv[j].ncell() > (size_t)TAIL_MAX_CELLS) ++j;
        bool ok = j < nl && nl - j <= TAIL_MAX && !S->lv[j - 1].half;
        for (int k = j; ok && k < nl; ++k) ok = S->lv[k].dense && S->lv[k].ncell() <= (size_t)TAIL_MAX_CELLS;
        if (ok) S->tail = j;
    }

    AW_CUDA(cudaDeviceSynchronize());
    return AW_OK;
}

namespace aw {
aw_status solver_relayout(aw_solver* S) {
    AW_CHECK_ARG(S && S->g && S->g->st.allocated, "grid not allocated");
    AW_TRY(check_grading(S->g->st));
    AW_TRY(solver_build(S));
    return aw_solver_setup(S, nullptr, 0);
}
}  // namespace aw

extern "C" aw_status aw_solver_create(aw_msbg* g, const aw_solver_desc* d, aw_solver** out) {
    AW_CHECK_ARG(g && d && out, "null argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    AW_CHECK_ARG(d->operator_mode == AW_OPERATOR_FV || d->operator_mode == AW_OPERATOR_REFERENCE, "bad operator mode");
    AW_CHECK_ARG(d->precision == AW_PRECISION_FP32 || d->precision == AW_PRECISION_MIXED ||
                     d->precision == AW_PRECISION_FP32_PCG,
                 "bad precision");
    AW_CHECK_ARG(d->block_iterations >= 1 && d->pre_smooth >= 0 && d->post_smooth >= 0, "bad smoother settings");
    *out = nullptr;
    MsbgState& G = g->st;
    AW_TRY(check_grading(G));
    std::unique_ptr<aw_solver> S(new aw_solver());
    S->g = g;
    S->d = *d;
    AW_TRY(solver_build(S.get()));
    *out = S.release();
    // default setup: every cell fluid
    return aw_solver_setup(*out, nullptr, 0);
}

extern "C" aw_status aw_solver_destroy(aw_solver* sv) {
    delete sv;
    return AW_OK;
}

extern "C" aw_status aw_solver_setup(aw_solver* S, const uint8_t* d_fluid, aw_stream s_) {
    AW_CHECK_ARG(S, "null solver");
    cudaStream_t s = (cudaStream_t)s_;
    MsbgState& G = S->g->st;
    MGLevel& L0 = S->lv[0];
    if (d_fluid) AW_CUDA(cudaMemcpyAsync(L0.fluid.p, d_fluid, L0.ncell(), cudaMemcpyDeviceToDevice, s));
    else AW_CUDA(cudaMemsetAsync(L0.fluid.p, 1, L0.ncell(), s));
    for (int m = 1; m < (int)S->lv.size(); ++m) {
        MGLevel& L = S->lv[m];
        MGLevel& F = S->lv[m - 1];
        if (!L.dense) {
            k_coarse_fluid<<<G.nb, 128, 0, s>>>(lview(S, m - 1), lview(S, m), F.fluid.p, L.fluid.p);
        } else {
            LevelView Fv = F.dense ? LevelView{} : lview(S, m - 1);
            if (F.dense) Fv.g = G.geo;
            k_dense_fluid<<<nblk(L.ncell()), 256, 0, s>>>(dview(L), F.dense ? 0 : 1, Fv, F.fluid.p, dview(F), L.fluid.p);
        }
        AW_LAUNCH();
    }
    if (S->exact) {
        Uniform U = uniform_of(S, (int)S->lv.size() - 1);
        k_coarse_factor<<<1, 512, 0, s>>>(U, S->ex_pos.p, S->ex_idx.p, S->ex_n.p, S->M.p, S->Minv.p, S->ex_prev.p,
                                          S->coef_dirty ? 1 : 0);
        S->coef_dirty = false;
        AW_LAUNCH();
    }
    return AW_OK;
}

extern "C" aw_status aw_solver_precision(const aw_solver* S, int32_t* precision) {
    AW_CHECK_ARG(S && precision, "null argument");
    *precision = S->d.precision;
    return AW_OK;
}

extern "C" aw_status aw_solver_num_levels(const aw_solver* S, int32_t* n) {
    AW_CHECK_ARG(S && n, "null argument");
    *n = (int32_t)S->lv.size();
    return AW_OK;
}

extern "C" aw_status aw_solver_level_array(aw_solver* S, int32_t m, int32_t which, void** p, uint32_t* count) {
    AW_CHECK_ARG(S && p && m >= 0 && m < (int)S->lv.size(), "bad argument");
    MGLevel& L = S->lv[m];
    uint32_t c = 0;
    void* q = nullptr;
    switch (which) {
        case 0: q = L.half ? (void*)L.xh.p : (void*)L.x.p; c = (uint32_t)L.ncell(); break;
        case 1: q = L.b.p; c = (uint32_t)L.ncell(); break;
        case 2: q = L.r.p; c = (uint32_t)L.ncell(); break;
        case 3: case 4: case 5: q = L.W[which - 3].p; c = (uint32_t)L.nface(which - 3); break;
        case 6: q = L.fluid.p; c = (uint32_t)L.ncell(); break;
        case 7: case 8: case 9: case 10:
            AW_CHECK_ARG(!L.dense, "offsets exist on block-structured levels only");
            q = L.off[which - 7].p;
            c = (uint32_t)S->g->st.nb;
            break;
        case 11:
            AW_CHECK_ARG(!L.dense, "res exists on block-structured levels only");
            q = L.res.p;
            c = (uint32_t)S->g->st.nb;
            break;
        default: return set_error(AW_ERR_INVALID_ARGUMENT, "unknown level array %d", which);
    }
    *p = q;
    if (count) *count = c;
    return AW_OK;
}

extern "C" aw_status aw_smoother_solve_level(aw_solver* S, int32_t m, int32_t iterations, aw_stream s) {
    AW_CHECK_ARG(S && m >= 0 && m < (int)S->lv.size() && iterations >= 0, "bad argument");
    return smooth_level(S, m, iterations, (cudaStream_t)s);
}
extern "C" aw_status aw_mg_residual(aw_solver* S, int32_t m, aw_stream s) {
    AW_CHECK_ARG(S && m >= 0 && m < (int)S->lv.size(), "bad argument");
    return residual_level(S, m, nullptr, (cudaStream_t)s);
}
extern "C" aw_status aw_mg_restrict(aw_solver* S, int32_t m, aw_stream s) {
    AW_CHECK_ARG(S && m >= 0 && m + 1 < (int)S->lv.size(), "bad argument");
    return restrict_level(S, m, (cudaStream_t)s);
}
extern "C" aw_status aw_mg_prolongate(aw_solver* S, int32_t m, aw_stream s) {
    AW_CHECK_ARG(S && m >= 0 && m + 1 < (int)S->lv.size(), "bad argument");
    return prolong_level(S, m, (cudaStream_t)s);
}
// One V-cycle, replayed from a CUDA graph (captured on first use for the current level-0 x/b).
static aw_status run_vcycle(aw_solver* S, cudaStream_t s) {
    if (!S->use_graph) return vcycle(S, 0, s);
    const void* x0 = S->x0 ? (const void*)S->x0 : (const void*)S->lv[0].x.p;
    const void* b0 = S->b0 ? (const void*)S->b0 : (const void*)S->lv[0].b.p;
    if (!S->cycle || S->cycle_x0 != x0 || S->cycle_b0 != b0) {
        if (S->cycle) {
            cudaGraphExecDestroy(S->cycle);
            S->cycle = nullptr;
        }
        if (!S->cap) AW_CUDA(cudaStreamCreateWithFlags(&S->cap, cudaStreamNonBlocking));
        const unsigned long long l0 = g_launches;
        AW_CUDA(cudaStreamBeginCapture(S->cap, cudaStreamCaptureModeThreadLocal));
        aw_status st = vcycle(S, 0, S->cap);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(S->cap, &graph);
        S->cycle_kernels = g_launches - l0;
        g_launches = l0;
        if (st != AW_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) return set_error(AW_ERR_CUDA, "V-cycle capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&S->cycle, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            S->cycle = nullptr;
            return set_error(AW_ERR_CUDA, "V-cycle graph instantiate: %s", cudaGetErrorString(e));
        }
        S->cycle_x0 = x0;
        S->cycle_b0 = b0;
    }
    AW_CUDA(cudaGraphLaunch(S->cycle, s));
    g_launches += S->cycle_kernels;
    return AW_OK;
}

extern "C" aw_status aw_solver_coarsest_solve(aw_solver* S, aw_stream s) {
    AW_CHECK_ARG(S, "null solver");
    return coarsest(S, (int)S->lv.size() - 1, (cudaStream_t)s);
}
extern "C" aw_status aw_vcycle_run(aw_solver* S, aw_stream s) {
    AW_CHECK_ARG(S, "null solver");
    return vcycle(S, 0, (cudaStream_t)s);
}

static aw_status read_norm(aw_solver* S, int nparts, cudaStream_t s, double* out) {
    k_reduce_sum<<<1, 256, 0, s>>>(S->partials.p, nparts, S->norm.p);
    AW_LAUNCH();
    if (!S->h_norm) AW_CUDA(cudaHostAlloc((void**)&S->h_norm, sizeof(double), cudaHostAllocDefault));
    AW_CUDA(cudaMemcpyAsync(S->h_norm, S->norm.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    AW_CUDA(cudaStreamSynchronize(s));
    *out = std::sqrt(*S->h_norm);
    return AW_OK;
}

// Mixed-precision CG iterations on the device until the recursive residual falls below the
// tolerance, turns NaN or the iteration limit is reached: one graph whose while node repeats the
// iteration (V-cycle preconditioner, the two dot products, the direction, A d and the update) and
// a check kernel that sets the loop condition, so no host round trip separates iterations.  The
// kernels and their order are those of the host-driven loop, so the results are identical.  The
// graph is built per pressure array.  Returns false (state unchanged) when the device cannot
// build such a graph; the caller then keeps the host loop.
static aw_status cg_body(aw_solver* S, double* p, unsigned ndot, cudaStream_t s, cudaGraphConditionalHandle h) {
    MGLevel& L0 = S->lv[0];
    const size_t nc = L0.ncell();
    const int cf = fv(S) ? 1 : 0;
    double* sc = S->cg_sc.p;
    k_fill_zero<<<nblk(nc), 256, 0, s>>>(L0.x.p, nc);
    AW_LAUNCH();
    AW_TRY(vcycle(S, 0, s));
    AW_TRY(launch_dep(S, k_dot64, ndot, 256, 0, s, S->cg_r.p, (const double*)nullptr, L0.x.p, L0.fluid.p, nc,
                      S->partials.p));
    AW_TRY(launch_dep(S, k_reduce_sum, 1, 256, 0, s, S->partials.p, (int)ndot, sc + 0));
    AW_TRY(launch_dep(S, k_cg_direction, nblk(nc), 256, 0, s, S->cg_d.p, L0.x.p, L0.fluid.p, sc, 0,
                      (const int*)(S->cgst.p + 1), nc));
    AW_TRY(launch_dep(S, k_apply_dot, (unsigned)L0.ndesc[2], 256, L0.smem_x64, s, SrcD{S->cg_d.p}, S->cg_zero.p,
                      coef(L0), L0.fluid.p, batch(L0, 2), cf, S->cg_q.p, S->partials.p));
    AW_TRY(launch_dep(S, k_reduce_sum, 1, 256, 0, s, S->partials.p, L0.ndesc[2], sc + 2));
    AW_TRY(launch_dep(S, k_cg_update, ndot, 256, 0, s, p, S->cg_r.p, L0.b.p, S->cg_d.p, S->cg_q.p, sc, L0.fluid.p, nc,
                      S->partials.p));
    k_cg_check<<<1, 256, 0, s>>>(h, (const double*)S->partials.p, (int)ndot, S->norm.p, S->cgprm.p, S->cgst.p);
    AW_LAUNCH();
    return AW_OK;
}

static bool cg_devloop_build(aw_solver* S, double* p, unsigned ndot) {
    if (S->cgloop) {
        cudaGraphExecDestroy(S->cgloop);
        S->cgloop = nullptr;
    }
    if (S->cgst.ensure(4) != AW_OK || S->cgprm.ensure(2) != AW_OK) return false;
    if (!S->cap && cudaStreamCreateWithFlags(&S->cap, cudaStreamNonBlocking) != cudaSuccess) return false;
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) return false;
    bool ok = false;
    cudaGraphConditionalHandle h;
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t node;
    if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        if (cudaGraphAddNode(&node, g, nullptr, 0, &cp) == cudaSuccess) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            const unsigned long long l0 = g_launches;
            if (cudaStreamBeginCaptureToGraph(S->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                cudaSuccess) {
                const aw_status st = cg_body(S, p, ndot, S->cap, h);
                cudaGraph_t out = nullptr;
                const cudaError_t e = cudaStreamEndCapture(S->cap, &out);
                S->cgloop_kernels = g_launches - l0;
                g_launches = l0;
                ok = st == AW_OK && e == cudaSuccess && cudaGraphInstantiate(&S->cgloop, g, 0) == cudaSuccess;
            }
        }
    }
    cudaGraphDestroy(g);
    if (!ok) {
        S->cgloop = nullptr;
        cudaGetLastError();
        return false;
    }
    S->cgloop_p = p;
    return true;
}

extern "C" aw_status aw_solve(aw_solver* S, const float* d_b, void* d_p, int32_t* cycles, double* final_rel,
                              aw_stream s_) {
    AW_CHECK_ARG(S && d_b && d_p, "null argument");
    cudaStream_t s = (cudaStream_t)s_;
    MGLevel& L0 = S->lv[0];
    const int cf = fv(S) ? 1 : 0;
    const size_t nc = L0.ncell();
    // ||b||
    int nparts = 256;
    k_sumsq<<<nparts, 256, 0, s>>>(d_b, L0.fluid.p, nc, cf, S->partials.p);
    AW_LAUNCH();
    double bn;
    AW_TRY(read_norm(S, nparts, s, &bn));
    if (!(bn == bn) || std::isinf(bn)) return set_error(AW_ERR_NAN, "right-hand side contains NaN/Inf");
    if (bn == 0.0) bn = 1.0;
    const int nlist = L0.ndesc[2];
    int it = 0;
    double rel = 0;
    aw_status st = AW_OK;
    if (S->d.precision == AW_PRECISION_FP32) {
        S->x0 = (float*)d_p;
        S->b0 = d_b;
        for (;; ++it) {
            st = residual_level(S, 0, S->partials.p, s);
            if (st != AW_OK) break;
            double rn;
            st = read_norm(S, nlist, s, &rn);
            if (st != AW_OK) break;
            rel = rn / bn;
            if (!(rel == rel)) {
                st = set_error(AW_ERR_NAN, "residual became NaN after %d cycles", it);
                break;
            }
            if (rel < S->d.tolerance) break;
            if (it >= S->d.max_cycles) {
                st = set_error(AW_ERR_NOT_CONVERGED, "relative residual %.3e after %d cycles", rel, it);
                break;
            }
            st = run_vcycle(S, s);
            if (st != AW_OK) break;
        }
        S->x0 = nullptr;
        S->b0 = nullptr;
    } else if (S->d.precision == AW_PRECISION_FP32_PCG) {
        // Conjugate gradients preconditioned by the same V-cycle as the mixed form, with the pressure,
        // residual, direction and every scalar in FP32 (the like-for-like FP32 baseline of the mixed
        // precision).  r lives in the level-0 right-hand side array, the V-cycle's input.
        float* p = (float*)d_p;
        float* sc = S->cg32_sc.p;
        int nsm = 148;
        {
            int dev = 0;
            if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        }
        const unsigned ndot = (unsigned)std::min<size_t>((size_t)nsm * 8, S->partials32.n);
        XStore xp, xd;
        xp.f = p;
        xd.f = S->cg32_d.p;
        auto launch_err = [&](const char* what) -> aw_status {
            ++g_launches;
            cudaError_t e = cudaGetLastError();
            return e == cudaSuccess ? AW_OK : set_error(AW_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
        };
        auto read_norm32 = [&](double* out) -> aw_status {
            k_reduce_sum32<<<1, 256, 0, s>>>(S->partials32.p, (int)ndot, sc + 3);
            AW_TRY(launch_err("k_reduce_sum32"));
            if (!S->h_norm) AW_CUDA(cudaHostAlloc((void**)&S->h_norm, sizeof(double), cudaHostAllocDefault));
            AW_CUDA(cudaMemcpyAsync(S->h_norm, sc + 3, sizeof(float), cudaMemcpyDeviceToHost, s));
            AW_CUDA(cudaStreamSynchronize(s));
            float f;
            memcpy(&f, S->h_norm, sizeof f);
            *out = std::sqrt((double)f);
            return AW_OK;
        };
        // r = b - A p into the V-cycle's input; its norm (FP64 partial sums) for the stopping test
        auto true_residual = [&]() -> aw_status {
            k_residual<SrcX><<<L0.ndesc[2], 256, L0.smem_smooth, s>>>(SrcX{xp}, d_b, coef(L0), L0.fluid.p, batch(L0, 2),
                                                                       cf, L0.b.p, nullptr, S->partials.p);
            return launch_err("k_residual");
        };
        st = L0.ndesc[2] ? true_residual() : AW_OK;
        double rn = 0;
        if (st == AW_OK) st = read_norm(S, nlist, s, &rn);
        bool restart = true;
        while (st == AW_OK) {
            rel = rn / bn;
            if (!(rel == rel)) {
                st = set_error(AW_ERR_NAN, "residual became NaN after %d iterations", it);
                break;
            }
            if (rel < S->d.tolerance) {
                if (restart) break;
                st = true_residual();
                if (st == AW_OK) st = read_norm(S, nlist, s, &rn);
                restart = true;
                continue;
            }
            if (it >= S->d.max_cycles) {
                st = set_error(AW_ERR_NOT_CONVERGED, "relative residual %.3e after %d iterations", rel, it);
                break;
            }
            st = zero_x(S, 0, s);
            if (st == AW_OK) st = run_vcycle(S, s);
            if (st != AW_OK) break;
            // the kernels of one iteration as programmatic dependents of one another
            if ((st = launch_dep(S, k_dot32, ndot, 256, 0, s, L0.b.p, L0.x.p, L0.fluid.p, nc, S->partials32.p)) != AW_OK) break;
            if ((st = launch_dep(S, k_reduce_sum32, 1, 256, 0, s, S->partials32.p, (int)ndot, sc + 0)) != AW_OK) break;
            if ((st = launch_dep(S, k_cg_direction32, nblk(nc), 256, 0, s, S->cg32_d.p, L0.x.p, L0.fluid.p, sc,
                                 restart ? 1 : 0, nc)) != AW_OK)
                break;
            if ((st = launch_dep(S, k_residual<SrcX>, (unsigned)L0.ndesc[2], 256, L0.smem_smooth, s, SrcX{xd},
                                 S->cg_zero.p, coef(L0), L0.fluid.p, batch(L0, 2), cf, S->cg32_q.p, (double*)nullptr,
                                 (double*)nullptr)) != AW_OK)
                break;
            if ((st = launch_dep(S, k_dot32, ndot, 256, 0, s, S->cg32_d.p, S->cg32_q.p, L0.fluid.p, nc,
                                 S->partials32.p)) != AW_OK)
                break;
            if ((st = launch_dep(S, k_reduce_sum32, 1, 256, 0, s, S->partials32.p, (int)ndot, sc + 2)) != AW_OK) break;
            if ((st = launch_dep(S, k_cg_update32, ndot, 256, 0, s, p, L0.b.p, S->cg32_d.p, S->cg32_q.p, sc, L0.fluid.p,
                                 nc, S->partials32.p)) != AW_OK)
                break;
            if ((st = launch_dep(S, k_copy_scalar32, 1, 1, 0, s, sc, 1, 0)) != AW_OK) break;
            ++it;
            restart = false;
            st = read_norm32(&rn);
        }
    } else {
        // Mixed precision: conjugate gradients preconditioned by the FP32 V-cycle (FP16-stored coarse
        // corrections), with the residual, the search direction and the pressure accumulation in
        // FP64 and the FP64 coarsest solve inside the V-cycle.  A stand-alone V-cycle iteration
        // stalls or diverges on free-surface domains with four levels; as a preconditioner the same
        // cycle converges on every configuration.  The iterations run in a device-side loop
        // (cg_devloop_build) when the device can build it, else with one host read (||r||) each.
        double* p = (double*)d_p;
        double* sc = S->cg_sc.p;
        // reductions over the level-0 cells: 8 CTAs per SM, grid-stride
        int nsm = 148;
        {
            int dev = 0;
            if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        }
        const unsigned ndot = (unsigned)std::min<size_t>((size_t)nsm * 8, S->partials.n);
        auto launch_err = [&](const char* what) -> aw_status {
            ++g_launches;
            cudaError_t e = cudaGetLastError();
            return e == cudaSuccess ? AW_OK : set_error(AW_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
        };
        auto true_residual = [&]() -> aw_status {
            k_residual<SrcD><<<L0.ndesc[2], 256, L0.smem_x64, s>>>(SrcD{p}, d_b, coef(L0), L0.fluid.p, batch(L0, 2), cf,
                                                                    L0.b.p, S->cg_r.p, S->partials.p);
            return launch_err("k_residual64");
        };
        st = true_residual();
        double rn = 0;
        if (st == AW_OK) st = read_norm(S, nlist, s, &rn);
        bool restart = true;
        while (st == AW_OK) {
            rel = rn / bn;
            if (!(rel == rel)) {
                st = set_error(AW_ERR_NAN, "residual became NaN after %d iterations", it);
                break;
            }
            if (rel < S->d.tolerance) {
                if (restart) break;  // rn is a true residual
                // confirm with the true FP64 residual (the recursive one can drift)
                st = true_residual();
                if (st == AW_OK) st = read_norm(S, nlist, s, &rn);
                restart = true;
                continue;
            }
            if (it >= S->d.max_cycles) {
                st = set_error(AW_ERR_NOT_CONVERGED, "relative residual %.3e after %d iterations", rel, it);
                break;
            }
            if (S->use_graph && S->use_devloop && S->cgloop_p != (const void*)p && !cg_devloop_build(S, p, ndot))
                S->use_devloop = false;  // no such graph on this device: the host loop below
            if (S->use_graph && S->use_devloop) {
                // iterations on the device until the recursive residual converges, turns NaN or the
                // limit is reached; then one read-back of ||r||^2 and the iteration count
                const int st0[4] = {it, restart ? 1 : 0, S->d.max_cycles, 0};
                const double prm[2] = {bn, S->d.tolerance};
                if (!S->h_cg) AW_CUDA(cudaHostAlloc((void**)&S->h_cg, 4 * sizeof(double), cudaHostAllocDefault));
                memcpy(S->h_cg, st0, sizeof st0);
                memcpy(S->h_cg + 2, prm, sizeof prm);
                AW_CUDA(cudaMemcpyAsync(S->cgst.p, S->h_cg, sizeof st0, cudaMemcpyHostToDevice, s));
                AW_CUDA(cudaMemcpyAsync(S->cgprm.p, S->h_cg + 2, sizeof prm, cudaMemcpyHostToDevice, s));
                AW_CUDA(cudaGraphLaunch(S->cgloop, s));
                AW_CUDA(cudaMemcpyAsync(S->h_cg, S->norm.p, sizeof(double), cudaMemcpyDeviceToHost, s));
                AW_CUDA(cudaMemcpyAsync(S->h_cg + 1, S->cgst.p, sizeof(int), cudaMemcpyDeviceToHost, s));
                AW_CUDA(cudaStreamSynchronize(s));
                int it1 = 0;
                memcpy(&it1, S->h_cg + 1, sizeof(int));
                g_launches += S->cgloop_kernels * (unsigned long long)(it1 - it);
                it = it1;
                rn = std::sqrt(S->h_cg[0]);
                restart = false;
                continue;
            }
            // z = V(r): one V-cycle on the FP32 copy of r (in L0.b), from zero
            st = zero_x(S, 0, s);
            if (st == AW_OK) st = run_vcycle(S, s);
            if (st != AW_OK) break;
            // rho = r . z ; d = z + (rho / rho_old) d
            // the kernels of one iteration as programmatic dependents of one another
            if ((st = launch_dep(S, k_dot64, ndot, 256, 0, s, S->cg_r.p, (const double*)nullptr, L0.x.p, L0.fluid.p, nc,
                                 S->partials.p)) != AW_OK)
                break;
            if ((st = launch_dep(S, k_reduce_sum, 1, 256, 0, s, S->partials.p, (int)ndot, sc + 0)) != AW_OK) break;
            if ((st = launch_dep(S, k_cg_direction, nblk(nc), 256, 0, s, S->cg_d.p, L0.x.p, L0.fluid.p, sc,
                                 restart ? 1 : 0, (const int*)nullptr, nc)) != AW_OK)
                break;
            // qn = -A d ; sc[2] = d . qn
            if ((st = launch_dep(S, k_apply_dot, (unsigned)L0.ndesc[2], 256, L0.smem_x64, s, SrcD{S->cg_d.p},
                                 S->cg_zero.p, coef(L0), L0.fluid.p, batch(L0, 2), cf, S->cg_q.p, S->partials.p)) !=
                AW_OK)
                break;
            if ((st = launch_dep(S, k_reduce_sum, 1, 256, 0, s, S->partials.p, L0.ndesc[2], sc + 2)) != AW_OK) break;
            // p += alpha d ; r -= alpha A d ; FP32 copy of r for the next V-cycle ; rho_old = rho
            if ((st = launch_dep(S, k_cg_update, ndot, 256, 0, s, p, S->cg_r.p, L0.b.p, S->cg_d.p, S->cg_q.p, sc,
                                 L0.fluid.p, nc, S->partials.p)) != AW_OK)
                break;
            ++it;
            restart = false;
            st = read_norm(S, ndot, s, &rn);  // ||r|| from k_cg_update's partial sums
        }
    }
    if (cycles) *cycles = it;
    if (final_rel) *final_rel = rel;
    return st;
}
