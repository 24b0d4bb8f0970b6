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
    DBuf<int> blocks[3];
    int ndesc[3] = {0, 0, 0};
    size_t smem_smooth = 0, smem_x = 0, smem_x64 = 0;
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
    // level-0 bindings for the current solve
    float* x0 = nullptr;
    const float* b0 = nullptr;
    // mixed precision
    aw::DBuf<double> p64tmp;
    aw::DBuf<double> partials, norm;
    size_t smem_max = 0;
    // the whole V-cycle as a CUDA graph, captured once per (x0, b0) binding
    cudaStream_t cap = nullptr;
    cudaGraphExec_t cycle = nullptr;
    const void* cycle_x0 = nullptr;
    const void* cycle_b0 = nullptr;
    unsigned long long cycle_kernels = 0;
    bool use_graph = true;
    ~aw_solver() {
        if (cycle) cudaGraphExecDestroy(cycle);
        if (cap) cudaStreamDestroy(cap);
    }
};

namespace aw {

struct SmoothParams {
    float omega, target, theta;
    int iters;
    int check_fluid;
};

__host__ __device__ inline int xi3(int x, int y, int z, int R2) { return (x + 1) + R2 * ((y + 1) + R2 * (z + 1)); }

// Ghost value across face (a, s) of cell c in block b: same level -> mirror cell, coarser
// neighbour -> parent cell, finer neighbour -> mean of the 4 touching cells, outside the domain
// or absent -> 0 (Dirichlet / air).
__device__ inline float ghost_val(const LevelView& L, const XStore& x, int b, const int cb[3], const int c[3], int a, int s) {
    int nc[3] = {cb[0], cb[1], cb[2]};
    nc[a] += s;
    if (!inside(L.g, nc)) return 0.f;
    const int n = bidx(L.g, nc[0], nc[1], nc[2]);
    const int rn = L.res[n], r = L.res[b];
    if (!rn) return 0.f;
    const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
    const int na = s > 0 ? 0 : rn - 1;
    int q[3];
    q[a] = na;
    if (rn == r) {
        q[t1] = c[t1];
        q[t2] = c[t2];
        return x.get(L.off[0][n] + cidx(q[0], q[1], q[2], rn), n);
    }
    if (rn < r) {  // coarser neighbour (2:1 grading: rn == r / 2)
        q[t1] = min(c[t1] >> 1, rn - 1);
        q[t2] = min(c[t2] >> 1, rn - 1);
        return x.get(L.off[0][n] + cidx(q[0], q[1], q[2], rn), n);
    }
    float sum = 0.f;  // finer neighbour (rn == 2 r)
#pragma unroll
    for (int d1 = 0; d1 < 2; ++d1)
#pragma unroll
        for (int d2 = 0; d2 < 2; ++d2) {
            q[t1] = min(2 * c[t1] + d1, rn - 1);
            q[t2] = min(2 * c[t2] + d2, rn - 1);
            sum += x.get(L.off[0][n] + cidx(q[0], q[1], q[2], rn), n);
        }
    return 0.25f * sum;
}

// Stage x (block + 6 halo faces) into xs[(r+2)^3].
__device__ inline void stage_x(const LevelView& L, const XStore& x, int b, const int cb[3], int r, float* xs) {
    const int R2 = r + 2, n3 = r * r * r;
    const uint32_t oc = L.off[0][b];
    for (int i = threadIdx.x; i < n3; i += blockDim.x) {
        int cx = i % r, cy = (i / r) % r, cz = i / (r * r);
        xs[xi3(cx, cy, cz, R2)] = x.get(oc + i, b);
    }
    const int rr = r * r;
    for (int i = threadIdx.x; i < 6 * rr; i += blockDim.x) {
        int face = i / rr, rem = i - face * rr;
        int a = face >> 1, s = (face & 1) ? 1 : -1;
        int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        int c[3];
        c[a] = s > 0 ? r - 1 : 0;
        c[t1] = rem % r;
        c[t2] = rem / r;
        float v = ghost_val(L, x, b, cb, c, a, s);
        int q[3] = {c[0], c[1], c[2]};
        q[a] += s;
        xs[xi3(q[0], q[1], q[2], R2)] = v;
    }
}

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
// contiguously: 1 block of 8^3 or 16^3 cells, 4 of 4^3, 32 of 2^3, 256 of 1^3.  Every slot keeps
// its block and a one-cell halo in shared memory; slots never interact (same colour = no shared
// faces), so each slot's arithmetic, early exit and activation are exactly those of a CTA that
// owns one block.
// ------------------------------------------------------------------------------------------------
struct Batch {
    const int4* desc;  // {first index into blocks, count, res, 0}
    const int* blocks;
};

// Every thread of a batched CTA only ever touches cells of one slot (G * r^3 == 256, or G == 1).
// Reduce a per-thread non-negative value over the threads of each slot: shuffle within aligned
// groups of min(r^3, 32) lanes, then one shared atomicMax per group.
__device__ inline void slot_max(int* dst, int n3, float v) {
    const int grp = n3 < 32 ? n3 : 32;
    int iv = __float_as_int(v);
    for (int o = 1; o < grp; o <<= 1) iv = max(iv, __shfl_xor_sync(0xffffffffu, iv, o));
    if ((threadIdx.x & (grp - 1)) == 0 && iv > 0) atomicMax(dst, iv);
}

__device__ inline float slot_get(const XStore& x, const LevelView& L, int b, uint32_t i) { return x.get(L.off[0][b] + i, b); }

// Stage x of every slot (block interior + halo faces) into xs[slot * X3 + ...].
__device__ inline void stage_slots(const LevelView& L, const XStore& x, const int* sb, int G, int r, float* xs, int stride) {
    const int R2 = r + 2, n3 = r * r * r, rr = r * r;
    for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
        const int sl = t / n3, i = t - sl * n3;
        const int b = sb[sl];
        if (b < 0) continue;
        const int cx = i % r, cy = (i / r) % r, cz = i / rr;
        xs[sl * stride + xi3(cx, cy, cz, R2)] = slot_get(x, L, b, (uint32_t)i);
    }
    for (int t = threadIdx.x; t < G * 6 * rr; t += blockDim.x) {
        const int sl = t / (6 * rr), rem0 = t - sl * 6 * rr;
        const int b = sb[sl];
        if (b < 0) continue;
        const int face = rem0 / rr, rem = rem0 - face * rr;
        const int a = face >> 1, sd = (face & 1) ? 1 : -1;
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        int c[3], cb[3];
        c[a] = sd > 0 ? r - 1 : 0;
        c[t1] = rem % r;
        c[t2] = rem / r;
        bcoord(L.g, b, cb);
        const float v = ghost_val(L, x, b, cb, c, a, sd);
        int q[3] = {c[0], c[1], c[2]};
        q[a] += sd;
        xs[sl * stride + xi3(q[0], q[1], q[2], R2)] = v;
    }
}

// Write every slot's x back: FP32, or FP16 with a fresh per-block scale.
__device__ inline void store_slots(const LevelView& L, const XStore& x, const int* sb, int G, int r, const float* xs,
                                   int stride, int* smax) {
    const int R2 = r + 2, n3 = r * r * r;
    if (x.f) {
        for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
            const int sl = t / n3, i = t - sl * n3;
            const int b = sb[sl];
            if (b < 0) continue;
            const int cx = i % r, cy = (i / r) % r, cz = i / (r * r);
            x.f[L.off[0][b] + i] = xs[sl * stride + xi3(cx, cy, cz, R2)];
        }
        return;
    }
    for (int t = threadIdx.x; t < G; t += blockDim.x) smax[t] = 0;
    __syncthreads();
    {
        float m = 0.f;
        const int sl = (int)threadIdx.x / n3 < G ? (int)threadIdx.x / n3 : 0;
        for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
            const int i = t - (t / n3) * n3;
            if (sb[t / n3] < 0) continue;
            const int cx = i % r, cy = (i / r) % r, cz = i / (r * r);
            m = fmaxf(m, fabsf(xs[(t / n3) * stride + xi3(cx, cy, cz, R2)]));
        }
        slot_max(&smax[G == 1 ? 0 : sl], n3, m);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
        const int sl = t / n3, i = t - sl * n3;
        const int b = sb[sl];
        if (b < 0) continue;
        const float m = __int_as_float(smax[sl]);
        const float inv = m > 0.f ? 32768.f / m : 0.f;
        const int cx = i % r, cy = (i / r) % r, cz = i / (r * r);
        x.h[L.off[0][b] + i] = __float2half_rn(xs[sl * stride + xi3(cx, cy, cz, R2)] * inv);
    }
    for (int t = threadIdx.x; t < G; t += blockDim.x)
        if (sb[t] >= 0) {
            const float m = __int_as_float(smax[t]);
            x.scale[sb[t]] = m > 0.f ? m * (1.f / 32768.f) : 0.f;
        }
}

__host__ __device__ inline int smooth_slot_floats(int r) {
    return (r + 2) * (r + 2) * (r + 2) + r * r * r + 3 * (r + 1) * r * r;
}

// smoothActiveBlocks (Smoother.cuh:105-202) for one block colour, batched.
__global__ void __launch_bounds__(256) k_smooth(LevelView L, XStore x, const float* __restrict__ bvec, Coef3 W,
                                                const uint8_t* __restrict__ fluid, Batch B,
                                                const uint8_t* __restrict__ status, uint8_t* __restrict__ status_next,
                                                SmoothParams P) {
    extern __shared__ float sm[];
    __shared__ int sb[256], smr[256], sdone[256];
    __shared__ float sinit[256];
    const int4 d = B.desc[blockIdx.x];
    const int G = d.y, r = d.z;
    const int R2 = r + 2, n3 = r * r * r, nf = (r + 1) * r * r, X3 = R2 * R2 * R2;
    const int per = smooth_slot_floats(r);
    uint8_t* fsb = (uint8_t*)(sm + G * per);
    for (int t = threadIdx.x; t < G; t += blockDim.x) {
        const int b = B.blocks[d.x + t];
        sb[t] = status[b] ? b : -1;
        smr[t] = 0;
        sdone[t] = 0;
        sinit[t] = -1.f;
    }
    __syncthreads();
    if (!__syncthreads_or(threadIdx.x < G && sb[threadIdx.x] >= 0)) return;
    for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
        const int sl = t / n3, i = t - sl * n3;
        const int b = sb[sl];
        if (b < 0) continue;
        const uint32_t oc = L.off[0][b];
        sm[sl * per + X3 + i] = bvec[oc + i];
        fsb[sl * n3 + i] = fluid[oc + i];
    }
    for (int t = threadIdx.x; t < G * 3 * nf; t += blockDim.x) {
        const int sl = t / (3 * nf), j = t - sl * 3 * nf;
        const int b = sb[sl];
        if (b < 0) continue;
        const int a = j / nf;
        sm[sl * per + X3 + n3 + j] = W.w[a][L.off[1 + a][b] + (j - a * nf)];
    }
    stage_slots(L, x, sb, G, r, sm, per);
    __syncthreads();
    const int sy = R2, sz = R2 * R2;
    const int my_slot = G == 1 ? 0 : min((int)threadIdx.x / n3, G - 1);
    for (int bi = 0; bi < P.iters; ++bi) {
        float lmax = 0.f;
        for (int col = 0; col < 2; ++col) {
            for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
                const int sl = t / n3, i = t - sl * n3;
                if (sb[sl] < 0 || sdone[sl]) continue;
                const int cx = i % r, cy = (i / r) % r, cz = i / (r * r);
                if (((cx + cy + cz) & 1) != col) continue;
                if (P.check_fluid && !fsb[sl * n3 + i]) continue;
                float* xs = sm + sl * per;
                const float* Ws = xs + X3 + n3;
                const float wW = Ws[fidx(0, cx, cy, cz, r)];
                const float wE = Ws[fidx(0, cx + 1, cy, cz, r)];
                const float wS = Ws[nf + fidx(1, cx, cy, cz, r)];
                const float wN = Ws[nf + fidx(1, cx, cy + 1, cz, r)];
                const float wB = Ws[2 * nf + fidx(2, cx, cy, cz, r)];
                const float wT = Ws[2 * nf + fidx(2, cx, cy, cz + 1, r)];
                const float diag = -(wW + wE + wS + wN + wB + wT);
                if (fabsf(diag) < 1e-9f) continue;
                const int q = xi3(cx, cy, cz, R2);
                const float xc = xs[q];
                const float Ax = wW * xs[q - 1] + wE * xs[q + 1] + wS * xs[q - sy] + wN * xs[q + sy] + wB * xs[q - sz] +
                                 wT * xs[q + sz] + diag * xc;
                const float res = xs[X3 + i] - Ax;
                xs[q] = xc + P.omega * (res / diag);
                lmax = fmaxf(lmax, fabsf(res));
            }
            __syncthreads();
        }
        slot_max(&smr[my_slot], n3, lmax);
        __syncthreads();
        // per-slot early exit (block-uniform); smr keeps the last executed sweep's max
        int more = 0;
        for (int t = threadIdx.x; t < G; t += blockDim.x) {
            if (sb[t] < 0 || sdone[t]) continue;
            const float mr = __int_as_float(smr[t]);
            if (bi == 0) sinit[t] = mr;
            if (sinit[t] > 1e-9f && mr < sinit[t] * P.target) sdone[t] = 1;
            else if (bi + 1 < P.iters) {
                smr[t] = 0;
                more = 1;
            }
        }
        if (!__syncthreads_or(more)) break;
    }
    __syncthreads();
    int* smax = sdone;  // reused as per-slot |x| max for FP16 storage
    store_slots(L, x, sb, G, r, sm, per, smax);
    for (int t = threadIdx.x; t < G; t += blockDim.x) {
        const int b = sb[t];
        if (b < 0 || !(__int_as_float(smr[t]) > P.theta)) continue;
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

// computeExplicitResidual (VCycle.cuh:81-131), batched: r = b - A x on every cell (0 on air cells
// in FV mode); optional per-CTA partial sums of r^2.
__global__ void __launch_bounds__(256) k_residual(LevelView L, XStore x, const float* __restrict__ bvec, Coef3 W,
                                                  const uint8_t* __restrict__ fluid, Batch B, int check_fluid,
                                                  float* __restrict__ rout, double* __restrict__ part) {
    extern __shared__ float sm[];
    __shared__ int sb[256];
    __shared__ double dred[32];
    const int4 d = B.desc[blockIdx.x];
    const int G = d.y, r = d.z;
    const int R2 = r + 2, n3 = r * r * r, X3 = R2 * R2 * R2;
    for (int t = threadIdx.x; t < G; t += blockDim.x) sb[t] = B.blocks[d.x + t];
    __syncthreads();
    stage_slots(L, x, sb, G, r, sm, X3);
    __syncthreads();
    const int sy = R2, sz = R2 * R2;
    double acc = 0.0;
    for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
        const int sl = t / n3, i = t - sl * n3;
        const int b = sb[sl];
        const uint32_t oc = L.off[0][b];
        float rv = 0.f;
        if (!check_fluid || fluid[oc + i]) {
            const int cx = i % r, cy = (i / r) % r, cz = i / (r * r);
            const uint32_t ox = L.off[1][b], oy = L.off[2][b], oz = L.off[3][b];
            const float wW = W.w[0][ox + fidx(0, cx, cy, cz, r)];
            const float wE = W.w[0][ox + fidx(0, cx + 1, cy, cz, r)];
            const float wS = W.w[1][oy + fidx(1, cx, cy, cz, r)];
            const float wN = W.w[1][oy + fidx(1, cx, cy + 1, cz, r)];
            const float wB = W.w[2][oz + fidx(2, cx, cy, cz, r)];
            const float wT = W.w[2][oz + fidx(2, cx, cy, cz + 1, r)];
            const float diag = -(wW + wE + wS + wN + wB + wT);
            const float* xs = sm + sl * X3;
            const int q = xi3(cx, cy, cz, R2);
            const float Ax = diag * xs[q] + wW * xs[q - 1] + wE * xs[q + 1] + wS * xs[q - sy] + wN * xs[q + sy] +
                             wB * xs[q - sz] + wT * xs[q + sz];
            rv = bvec[oc + i] - Ax;
        }
        rout[oc + i] = rv;
        acc += (double)rv * (double)rv;
    }
    if (part) {
        double tsum = block_sum(acc, dred);
        if (threadIdx.x == 0) part[blockIdx.x] = tsum;
    }
}

// FP64 residual of the outer defect correction, batched: r = b - A p with p in FP64, stored as
// FP32 into the V-cycle right-hand side, with per-CTA partial sums of r^2.
__global__ void __launch_bounds__(256) k_residual64(LevelView L, const double* __restrict__ p,
                                                    const float* __restrict__ bvec, Coef3 W,
                                                    const uint8_t* __restrict__ fluid, Batch B, int check_fluid,
                                                    float* __restrict__ rout, double* __restrict__ part) {
    extern __shared__ double smd[];
    __shared__ int sb[256];
    __shared__ double dred[32];
    const int4 d = B.desc[blockIdx.x];
    const int G = d.y, r = d.z;
    const int R2 = r + 2, n3 = r * r * r, rr = r * r, X3 = R2 * R2 * R2;
    for (int t = threadIdx.x; t < G; t += blockDim.x) sb[t] = B.blocks[d.x + t];
    __syncthreads();
    for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
        const int sl = t / n3, i = t - sl * n3;
        const int cx = i % r, cy = (i / r) % r, cz = i / rr;
        smd[sl * X3 + xi3(cx, cy, cz, R2)] = p[L.off[0][sb[sl]] + i];
    }
    for (int t = threadIdx.x; t < G * 6 * rr; t += blockDim.x) {
        const int sl = t / (6 * rr), rem0 = t - sl * 6 * rr;
        const int b = sb[sl];
        const int face = rem0 / rr, rem = rem0 - face * rr;
        const int a = face >> 1, sd = (face & 1) ? 1 : -1;
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        int c[3], cb[3];
        c[a] = sd > 0 ? r - 1 : 0;
        c[t1] = rem % r;
        c[t2] = rem / r;
        bcoord(L.g, b, cb);
        int nc[3] = {cb[0], cb[1], cb[2]};
        nc[a] += sd;
        double v = 0.0;
        if (inside(L.g, nc)) {
            const int n = bidx(L.g, nc[0], nc[1], nc[2]);
            const int rn = L.res[n];
            if (rn) {
                int q[3];
                q[a] = sd > 0 ? 0 : rn - 1;
                if (rn == r) {
                    q[t1] = c[t1];
                    q[t2] = c[t2];
                    v = p[L.off[0][n] + cidx(q[0], q[1], q[2], rn)];
                } else if (rn < r) {
                    q[t1] = min(c[t1] >> 1, rn - 1);
                    q[t2] = min(c[t2] >> 1, rn - 1);
                    v = p[L.off[0][n] + cidx(q[0], q[1], q[2], rn)];
                } else {
                    for (int d1 = 0; d1 < 2; ++d1)
                        for (int d2 = 0; d2 < 2; ++d2) {
                            q[t1] = min(2 * c[t1] + d1, rn - 1);
                            q[t2] = min(2 * c[t2] + d2, rn - 1);
                            v += p[L.off[0][n] + cidx(q[0], q[1], q[2], rn)];
                        }
                    v *= 0.25;
                }
            }
        }
        int q[3] = {c[0], c[1], c[2]};
        q[a] += sd;
        smd[sl * X3 + xi3(q[0], q[1], q[2], R2)] = v;
    }
    __syncthreads();
    const int sy = R2, sz = R2 * R2;
    double acc = 0.0;
    for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
        const int sl = t / n3, i = t - sl * n3;
        const int b = sb[sl];
        const uint32_t oc = L.off[0][b];
        double rv = 0.0;
        if (!check_fluid || fluid[oc + i]) {
            const int cx = i % r, cy = (i / r) % r, cz = i / rr;
            const uint32_t ox = L.off[1][b], oy = L.off[2][b], oz = L.off[3][b];
            const double wW = W.w[0][ox + fidx(0, cx, cy, cz, r)];
            const double wE = W.w[0][ox + fidx(0, cx + 1, cy, cz, r)];
            const double wS = W.w[1][oy + fidx(1, cx, cy, cz, r)];
            const double wN = W.w[1][oy + fidx(1, cx, cy + 1, cz, r)];
            const double wB = W.w[2][oz + fidx(2, cx, cy, cz, r)];
            const double wT = W.w[2][oz + fidx(2, cx, cy, cz + 1, r)];
            const double diag = -(wW + wE + wS + wN + wB + wT);
            const double* xs = smd + sl * X3;
            const int q = xi3(cx, cy, cz, R2);
            const double Ax = diag * xs[q] + wW * xs[q - 1] + wE * xs[q + 1] + wS * xs[q - sy] + wN * xs[q + sy] +
                              wB * xs[q - sz] + wT * xs[q + sz];
            rv = (double)bvec[oc + i] - Ax;
        }
        rout[oc + i] = (float)rv;
        acc += rv * rv;
    }
    double tsum = block_sum(acc, dred);
    if (threadIdx.x == 0) part[blockIdx.x] = tsum;
}

__global__ void k_accum64(double* __restrict__ p, const float* __restrict__ e, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] += (double)e[i];
}

__global__ void k_reduce_sum(const double* __restrict__ part, int n, double* out) {
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

// restrictResidualsKernel (MultigridTransfer.cuh:9-59), batched over the coarse level's blocks:
// 8-child sum, or a copy for a block that keeps one cell.  Coarse air cells get 0.
__global__ void __launch_bounds__(256) k_restrict(LevelView F, LevelView K, const float* __restrict__ r,
                                                  float* __restrict__ bc, const uint8_t* __restrict__ fluid_c,
                                                  int check_fluid, Batch B) {
    const int4 d = B.desc[blockIdx.x];
    const int G = d.y, rc = d.z, n3 = rc * rc * rc;
    for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
        const int sl = t / n3, i = t - sl * n3;
        const int b = B.blocks[d.x + sl];
        const int rf = F.res[b];
        const uint32_t of = F.off[0][b], oc = K.off[0][b];
        float s;
        if (rf == 2 * rc) {
            const int x = i % rc, y = (i / rc) % rc, z = i / (rc * rc);
            const int fx = 2 * x, fy = 2 * y, fz = 2 * z;
            s = r[of + cidx(fx, fy, fz, rf)];
            s += r[of + cidx(fx + 1, fy, fz, rf)];
            s += r[of + cidx(fx, fy + 1, fz, rf)];
            s += r[of + cidx(fx + 1, fy + 1, fz, rf)];
            s += r[of + cidx(fx, fy, fz + 1, rf)];
            s += r[of + cidx(fx + 1, fy, fz + 1, rf)];
            s += r[of + cidx(fx, fy + 1, fz + 1, rf)];
            s += r[of + cidx(fx + 1, fy + 1, fz + 1, rf)];
        } else {
            s = r[of + i];
        }
        bc[oc + i] = (!check_fluid || fluid_c[oc + i]) ? s : 0.f;
    }
}

// prolongateCorrection (MultigridTransfer.cuh:63-102), batched over the fine level's blocks:
// x_f += x_c[parent] on fluid cells (FP16 fine storage is decoded, updated and re-encoded).
__global__ void __launch_bounds__(256) k_prolong(LevelView F, LevelView K, XStore xf, XStore xc,
                                                 const uint8_t* __restrict__ fluid_f, int check_fluid, Batch B) {
    extern __shared__ float sm[];
    __shared__ int sb[256], smax[256];
    const int4 d = B.desc[blockIdx.x];
    const int G = d.y, rf = d.z, n3 = rf * rf * rf;
    for (int t = threadIdx.x; t < G; t += blockDim.x) sb[t] = B.blocks[d.x + t];
    __syncthreads();
    const int R2 = rf + 2, X3 = R2 * R2 * R2;
    for (int t = threadIdx.x; t < G * n3; t += blockDim.x) {
        const int sl = t / n3, i = t - sl * n3;
        const int b = sb[sl];
        const int rc = K.res[b];
        const uint32_t of = F.off[0][b], oc = K.off[0][b];
        const int x = i % rf, y = (i / rf) % rf, z = i / (rf * rf);
        float add = 0.f;
        if (rc && (!check_fluid || fluid_f[of + i])) {
            const uint32_t ci = (rf == 2 * rc) ? cidx(x >> 1, y >> 1, z >> 1, rc) : (uint32_t)i;
            add = xc.get(oc + ci, b);
        }
        if (xf.f) xf.f[of + i] += add;
        else sm[sl * X3 + xi3(x, y, z, R2)] = xf.get(of + i, b) + add;
    }
    if (xf.f) return;
    __syncthreads();
    store_slots(F, xf, sb, G, rf, sm, X3, smax);
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

__global__ void k_dense_smooth(DenseArgs A, float* x, const float* __restrict__ b, int col, float omega) {
    const DenseView& d = A.d;
    int n = d.D[0] * d.D[1] * d.D[2];
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int i = t % d.D[0], j = (t / d.D[0]) % d.D[1], k = t / (d.D[0] * d.D[1]);
    if (((i + j + k) & 1) != col || !A.fluid[t]) return;
    float diag;
    float ax = dense_Ax(A, x, i, j, k, &diag);
    if (fabsf(diag) < 1e-30f) return;
    x[t] += omega * (b[t] - ax) / diag;
}

__global__ void k_dense_residual(DenseArgs A, const float* __restrict__ x, const float* __restrict__ b, float* r) {
    const DenseView& d = A.d;
    int n = d.D[0] * d.D[1] * d.D[2];
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int i = t % d.D[0], j = (t / d.D[0]) % d.D[1], k = t / (d.D[0] * d.D[1]);
    float diag;
    r[t] = A.fluid[t] ? b[t] - dense_Ax(A, x, i, j, k, &diag) : 0.f;
}

// restriction into a dense level from the one-cell-per-block MSBG level (first) or a dense level
__global__ void k_dense_restrict(DenseView K, const uint8_t* __restrict__ fluid_c, float* __restrict__ bc, int from_msbg,
                                 LevelView F, DenseView Fd, const float* __restrict__ rf) {
    int n = K.D[0] * K.D[1] * K.D[2];
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int i = t % K.D[0], j = (t / K.D[0]) % K.D[1], k = t / (K.D[0] * K.D[1]);
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
    bc[t] = fluid_c[t] ? s : 0.f;
}

__global__ void k_dense_prolong(DenseView K, const float* __restrict__ xc, int to_msbg, LevelView F, XStore xf_msbg,
                                DenseView Fd, float* __restrict__ xf, const uint8_t* __restrict__ fluid_f) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (to_msbg) {
        if (t >= F.g.nb) return;
        if (!F.res[t]) return;
        uint32_t ci = F.off[0][t];
        if (!fluid_f[ci]) return;
        int c[3];
        bcoord(F.g, t, c);
        xf_msbg.f[ci] += xc[didx(K, c[0] >> 1, c[1] >> 1, c[2] >> 1)];
    } else {
        int n = Fd.D[0] * Fd.D[1] * Fd.D[2];
        if (t >= n) return;
        if (!fluid_f[t]) return;
        int i = t % Fd.D[0], j = (t / Fd.D[0]) % Fd.D[1], k = t / (Fd.D[0] * Fd.D[1]);
        xf[t] += xc[didx(K, i >> 1, j >> 1, k >> 1)];
    }
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
__global__ void k_coarse_bbar(LevelView F, LevelView K, int a, const float* __restrict__ bf, float* __restrict__ bcv) {
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
__global__ void k_conductance(LevelView L, int a, const float* __restrict__ bbar, float* __restrict__ W) {
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

__global__ void k_dense_conductance(DenseView K, int a, float H, float* W) {
    int n = (K.D[0] + (a == 0)) * (K.D[1] + (a == 1)) * (K.D[2] + (a == 2));
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int dx = K.D[0] + (a == 0), dy = K.D[1] + (a == 1);
    int f[3] = {t % dx, (t / dx) % dy, t / (dx * dy)};
    W[t] = (f[a] == 0 || f[a] == K.D[a]) ? 0.f : H;
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
__global__ void __launch_bounds__(512) k_coarse_factor(Uniform U, int* pos_of, int* idx, int* ex_n, double* M,
                                                       double* Minv) {
    __shared__ int cnt;
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
__global__ void k_coarse_apply(Uniform U, const int* __restrict__ idx, const int* __restrict__ ex_n,
                               const double* __restrict__ Minv, const float* __restrict__ b, float* __restrict__ x) {
    const int n = ex_n[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) s += Minv[(size_t)i * n + j] * (double)b[uni_cell(U, idx[j])];
        x[uni_cell(U, idx[i])] = (float)s;
    }
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
static int slots_per_cta(int r) { return std::max(1, std::min(256, 256 / (r * r * r))); }

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
                const size_t Gm = (size_t)std::min<int>(G, (int)by_res[r].size());
                L.smem_smooth = std::max(L.smem_smooth, Gm * (smooth_slot_floats(r) * sizeof(float) + (size_t)r * r * r) + 16);
                L.smem_x = std::max(L.smem_x, Gm * (size_t)(r + 2) * (r + 2) * (r + 2) * sizeof(float));
                L.smem_x64 = std::max(L.smem_x64, Gm * (size_t)(r + 2) * (r + 2) * (r + 2) * sizeof(double));
            }
        }
        L.ndesc[k] = (int)desc.size();
        if (L.ndesc[k]) {
            AW_TRY(L.desc[k].alloc(desc.size()));
            AW_TRY(L.blocks[k].alloc(blocks.size()));
            AW_CUDA(cudaMemcpy(L.desc[k].p, desc.data(), desc.size() * sizeof(int4), cudaMemcpyHostToDevice));
            AW_CUDA(cudaMemcpy(L.blocks[k].p, blocks.data(), blocks.size() * sizeof(int), cudaMemcpyHostToDevice));
        }
    }
    return AW_OK;
}
static Batch batch(const MGLevel& L, int k) { return Batch{L.desc[k].p, L.blocks[k].p}; }
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

static aw_status smooth_level(aw_solver* S, int m, int iterations, cudaStream_t s) {
    MGLevel& L = S->lv[m];
    const int cf = fv(S) ? 1 : 0;
    if (L.dense) {
        DenseArgs A{dview(L), {L.W[0].p, L.W[1].p, L.W[2].p}, L.fluid.p};
        size_t n = L.ncell();
        for (int it = 0; it < iterations; ++it)
            for (int col = 0; col < 2; ++col) {
                k_dense_smooth<<<nblk(n), 256, 0, s>>>(A, L.x.p, L.b.p, col, S->d.omega);
                AW_LAUNCH();
            }
        return AW_OK;
    }
    const int nb = S->g->st.nb;
    AW_CUDA(cudaMemsetAsync(L.status[0].p, 1, nb, s));
    SmoothParams P{S->d.omega, S->d.target_reduction, S->d.theta, S->d.block_iterations, cf};
    LevelView V = lview(S, m);
    XStore x = xstore(S, m);
    int cur = 0;
    for (int it = 0; it < iterations; ++it) {
        AW_CUDA(cudaMemsetAsync(L.status[cur ^ 1].p, 0, nb, s));
        for (int rb = 0; rb < 2; ++rb) {
            if (!L.ndesc[rb]) continue;
            k_smooth<<<L.ndesc[rb], 256, L.smem_smooth, s>>>(V, x, bptr(S, m), coef(L), L.fluid.p, batch(L, rb),
                                                              L.status[cur].p, L.status[cur ^ 1].p, P);
            AW_LAUNCH();
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
        k_dense_residual<<<nblk(L.ncell()), 256, 0, s>>>(A, L.x.p, L.b.p, L.r.p);
        AW_LAUNCH();
        return AW_OK;
    }
    LevelView V = lview(S, m);
    XStore x = xstore(S, m);
    if (L.ndesc[2]) {
        k_residual<<<L.ndesc[2], 256, L.smem_x, s>>>(V, x, bptr(S, m), coef(L), L.fluid.p, batch(L, 2), cf, L.r.p, part);
        AW_LAUNCH();
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
        k_dense_restrict<<<nblk(K.ncell()), 256, 0, s>>>(dview(K), K.fluid.p, K.b.p, F.dense ? 0 : 1, Fv, dview(F), F.r.p);
        AW_LAUNCH();
        return AW_OK;
    }
    if (K.ndesc[2]) {
        k_restrict<<<K.ndesc[2], 256, 0, s>>>(lview(S, m), lview(S, m + 1), F.r.p, K.b.p, K.fluid.p, cf, batch(K, 2));
        AW_LAUNCH();
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
        k_dense_prolong<<<nblk(n), 256, 0, s>>>(dview(K), K.x.p, F.dense ? 0 : 1, Fv, xf, dview(F), F.x.p, F.fluid.p);
        AW_LAUNCH();
        return AW_OK;
    }
    if (F.ndesc[2]) {
        k_prolong<<<F.ndesc[2], 256, F.half ? F.smem_x : 0, s>>>(lview(S, m), lview(S, m + 1), xstore(S, m),
                                                                  xstore(S, m + 1), F.fluid.p, cf, batch(F, 2));
        AW_LAUNCH();
    }
    return AW_OK;
}

static aw_status coarsest(aw_solver* S, int m, cudaStream_t s) {
    MGLevel& L = S->lv[m];
    if (fv(S) && S->exact) {
        Uniform U = uniform_of(S, m);
        float* x = L.dense ? L.x.p : (m == 0 && S->x0 ? S->x0 : L.x.p);
        k_coarse_apply<<<4, 128, 0, s>>>(U, S->ex_idx.p, S->ex_n.p, S->Minv.p, bptr(S, m), x);
        AW_LAUNCH();
        return AW_OK;
    }
    return smooth_level(S, m, S->d.coarsest_iterations, s);
}

static aw_status vcycle(aw_solver* S, int m, cudaStream_t s) {
    const int last = (int)S->lv.size() - 1;
    if (m == last) return coarsest(S, m, s);
    MGLevel& L = S->lv[m];
    AW_TRY(smooth_level(S, m, L.dense ? S->d.dense_sweeps : S->d.pre_smooth, s));
    AW_TRY(residual_level(S, m, nullptr, s));
    AW_TRY(restrict_level(S, m, s));
    AW_TRY(zero_x(S, m + 1, s));
    AW_TRY(vcycle(S, m + 1, s));
    AW_TRY(prolong_level(S, m, s));
    AW_TRY(smooth_level(S, m, L.dense ? S->d.dense_sweeps : S->d.post_smooth, s));
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
        d->omega = 1.0f;
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

extern "C" aw_status aw_solver_create(aw_msbg* g, const aw_solver_desc* d, aw_solver** out) {
    AW_CHECK_ARG(g && d && out, "null argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    AW_CHECK_ARG(d->operator_mode == AW_OPERATOR_FV || d->operator_mode == AW_OPERATOR_REFERENCE, "bad operator mode");
    AW_CHECK_ARG(d->precision == AW_PRECISION_FP32 || d->precision == AW_PRECISION_MIXED, "bad precision");
    AW_CHECK_ARG(d->block_iterations >= 1 && d->pre_smooth >= 0 && d->post_smooth >= 0, "bad smoother settings");
    *out = nullptr;
    MsbgState& G = g->st;
    {  // the stencils assume 2:1 grading between face neighbours
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
    }
    std::unique_ptr<aw_solver> S(new aw_solver());
    S->g = g;
    S->d = *d;
    const bool ref = d->operator_mode == AW_OPERATOR_REFERENCE;
    const int nb = G.nb;
    int M = d->mg_levels > 0 ? d->mg_levels : (ref ? G.geo.L : ilog2(G.geo.R0) + 1);
    if (!ref) M = std::min(M, ilog2(G.geo.R0) + 1);
    cudaStream_t s = 0;
    S->lv.resize(M);
    for (int m = 0; m < M; ++m) {
        MGLevel& L = S->lv[m];
        AW_TRY(L.res.alloc(nb));
        DBuf<uint32_t> off4;
        AW_TRY(off4.alloc(4 * (size_t)nb));
        AW_TRY(level_offsets(G, m, ref ? 1 : 0, off4.p, L.res.p, L.tot, s));
        for (int k = 0; k < 4; ++k) {
            AW_TRY(L.off[k].alloc(nb));
            AW_CUDA(cudaMemcpy(L.off[k].p, off4.p + (size_t)k * nb, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice));
        }
        L.h_res.resize(nb);
        AW_CUDA(cudaMemcpy(L.h_res.data(), L.res.p, nb * sizeof(int), cudaMemcpyDeviceToHost));
        for (int b = 0; b < nb; ++b) L.maxres = std::max(L.maxres, L.h_res[b]);
        if (L.maxres == 0) {
            S->lv.resize(m);
            break;
        }
        AW_TRY(build_batches(L, G.geo));
        AW_TRY(L.status[0].alloc(nb));
        AW_TRY(L.status[1].alloc(nb));
        L.half = (d->precision == AW_PRECISION_MIXED) && m >= 1 && m < M - 1 + (ref ? 0 : 1) && L.maxres > 1;
        size_t nc = L.ncell();
        AW_TRY(L.x.alloc(nc));
        AW_TRY(L.b.alloc(nc));
        AW_TRY(L.r.alloc(nc));
        AW_TRY(L.fluid.alloc(nc));
        AW_CUDA(cudaMemset(L.x.p, 0, nc * sizeof(float)));
        AW_CUDA(cudaMemset(L.b.p, 0, nc * sizeof(float)));
        AW_CUDA(cudaMemset(L.fluid.p, 1, nc));
        if (L.half) {
            AW_TRY(L.xh.alloc(nc));
            AW_TRY(L.xscale.alloc(nb));
            AW_CUDA(cudaMemset(L.xh.p, 0, nc * sizeof(__half)));
            AW_CUDA(cudaMemset(L.xscale.p, 0, nb * sizeof(float)));
        }
        for (int a = 0; a < 3; ++a) {
            AW_TRY(L.W[a].alloc(L.nface(a)));
            AW_TRY(L.bbar[a].alloc(L.nface(a)));
        }
        S->smem_max = std::max({S->smem_max, L.smem_smooth, L.smem_x, L.smem_x64});
    }
    S->nmsbg = (int)S->lv.size();
    // coefficients of the block-structured levels
    for (int m = 0; m < S->nmsbg; ++m) {
        MGLevel& L = S->lv[m];
        LevelView V = lview(S.get(), m);
        for (int a = 0; a < 3; ++a) {
            if (m == 0) {
                AW_CUDA(cudaMemcpy(L.bbar[a].p, G.ch[AW_BETA_COEFF_X + a], L.nface(a) * sizeof(float),
                                   cudaMemcpyDeviceToDevice));
            } else {
                k_coarse_bbar<<<nb, 128>>>(lview(S.get(), m - 1), V, a, S->lv[m - 1].bbar[a].p, L.bbar[a].p);
                AW_LAUNCH();
            }
            if (ref) {
                if (m == 0) {
                    AW_CUDA(cudaMemcpy(L.W[a].p, L.bbar[a].p, L.nface(a) * sizeof(float), cudaMemcpyDeviceToDevice));
                } else {
                    AW_CUDA(cudaMemset(L.W[a].p, 0, L.nface(a) * sizeof(float)));
                    k_galerkin_ref<<<nb, 256>>>(G.geo, G.level.p, a, m, S->lv[m - 1].W[a].p, L.W[a].p,
                                                S->lv[m - 1].off[1 + a].p, L.off[1 + a].p);
                    AW_LAUNCH();
                }
            } else {
                k_conductance<<<nb, 128>>>(V, a, L.bbar[a].p, L.W[a].p);
                AW_LAUNCH();
            }
        }
    }
    // uniform continuation below one cell per block (FV mode)
    if (!ref && S->nmsbg > 0 && S->lv.back().maxres == 1) {
        int Dd[3] = {G.geo.D[0], G.geo.D[1], G.geo.D[2]};
        float H = G.geo.bs;
        while (Dd[0] % 2 == 0 && Dd[1] % 2 == 0 && Dd[2] % 2 == 0 && (long)Dd[0] * Dd[1] * Dd[2] > 64) {
            S->lv.emplace_back();
            MGLevel& L = S->lv.back();
            L.dense = true;
            for (int a = 0; a < 3; ++a) L.D[a] = Dd[a] / 2;
            H *= 2.f;
            L.H = H;
            size_t nc = L.ncell();
            AW_TRY(L.x.alloc(nc));
            AW_TRY(L.b.alloc(nc));
            AW_TRY(L.r.alloc(nc));
            AW_TRY(L.fluid.alloc(nc));
            AW_CUDA(cudaMemset(L.x.p, 0, nc * sizeof(float)));
            AW_CUDA(cudaMemset(L.b.p, 0, nc * sizeof(float)));
            for (int a = 0; a < 3; ++a) {
                AW_TRY(L.W[a].alloc(L.nface(a)));
                k_dense_conductance<<<nblk(L.nface(a)), 256>>>(dview(L), a, H, L.W[a].p);
                AW_LAUNCH();
            }
            for (int a = 0; a < 3; ++a) Dd[a] /= 2;
        }
        // the coarsest level is uniform: factorise it densely when small enough
        MGLevel& C = S->lv.back();
        size_t npos = C.dense ? C.ncell() : (size_t)nb;
        if (npos <= (size_t)EXACT_POS_CAP) {
            AW_TRY(S->M.alloc((size_t)EXACT_CAP * EXACT_CAP));
            AW_TRY(S->Minv.alloc((size_t)EXACT_CAP * EXACT_CAP));
            AW_TRY(S->ex_idx.alloc(EXACT_CAP));
            AW_TRY(S->ex_pos.alloc(npos));
            AW_TRY(S->ex_n.alloc(1));
            AW_CUDA(cudaMemset(S->ex_n.p, 0, sizeof(int)));
            S->exact = true;
        }
    }
    if (S->smem_max > 48 * 1024) {
        AW_CUDA(cudaFuncSetAttribute(k_smooth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_max));
        AW_CUDA(cudaFuncSetAttribute(k_residual, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_max));
        AW_CUDA(cudaFuncSetAttribute(k_prolong, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_max));
        AW_CUDA(cudaFuncSetAttribute(k_residual64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * S->smem_max)));
    }
    size_t nparts = (size_t)nb + 1024;
    AW_TRY(S->partials.alloc(nparts));
    AW_TRY(S->norm.alloc(2));
    S->use_graph = getenv("AW_NO_GRAPH") == nullptr;
    AW_CUDA(cudaDeviceSynchronize());
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
        k_coarse_factor<<<1, 512, 0, s>>>(U, S->ex_pos.p, S->ex_idx.p, S->ex_n.p, S->M.p, S->Minv.p);
        AW_LAUNCH();
    }
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
    double h = 0;
    AW_CUDA(cudaMemcpyAsync(&h, S->norm.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    AW_CUDA(cudaStreamSynchronize(s));
    *out = std::sqrt(h);
    return AW_OK;
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
    } else {
        double* p = (double*)d_p;
        LevelView V = lview(S, 0);
        for (;; ++it) {
            k_residual64<<<L0.ndesc[2], 256, L0.smem_x64, s>>>(V, p, d_b, coef(L0), L0.fluid.p, batch(L0, 2), cf,
                                                                L0.b.p, S->partials.p);
            ++g_launches;
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) {
                st = set_error(AW_ERR_CUDA, "k_residual64: %s", cudaGetErrorString(e));
                break;
            }
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
            st = zero_x(S, 0, s);
            if (st != AW_OK) break;
            st = run_vcycle(S, s);
            if (st != AW_OK) break;
            k_accum64<<<nblk(nc), 256, 0, s>>>(p, L0.x.p, nc);
            ++g_launches;
            e = cudaGetLastError();
            if (e != cudaSuccess) {
                st = set_error(AW_ERR_CUDA, "k_accum64: %s", cudaGetErrorString(e));
                break;
            }
        }
    }
    if (cycles) *cycles = it;
    if (final_rel) *final_rel = rel;
    return st;
}
