// aw_grid.cu — MSBG topology: level map, 2:1 grading, block allocation, offsets, channels.
//
// Reference behaviour followed (paths within the reference project):
//   MSBG.cuh:112-124  computeBlockLayout        MSBG.cuh:139-149  morton3D
//   MSBG.cuh:249-269  initRefinementMap/initBlockInfo
//   MSBG.cuh:316-351  enforceGrading (here iterated to the fixpoint)
//   MSBG.cuh:353-376  countBlockElements       main.cu:270-273   exclusive_scan -> offsets
//   MSBG.cuh:599-659  allocateChannels          MSBG.cuh:679-745  computeCoarse(Face)Offsets
//   MSBG.cuh:400-498  galerkinCoarsen (reference coefficient formula)
#include <cstdarg>
#include <cstring>

#include "aw_internal.cuh"

namespace aw {

static thread_local std::string g_err;
unsigned long long g_launches = 0;

aw_status set_error(aw_status s, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

// ------------------------------------------------------------------------------------------------
// Exclusive scan (three phases: tile scan, carry scan, add).  Tiles of 2048 u32.
// ------------------------------------------------------------------------------------------------
constexpr int SCAN_T = 256, SCAN_V = 8, SCAN_TILE = SCAN_T * SCAN_V;

__device__ inline uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < (SCAN_T / 32) ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < SCAN_T / 32) sh[lane] = s;
    }
    __syncthreads();
    uint32_t pre = (w > 0 ? sh[w - 1] : 0u) + x - v;
    if (total) *total = sh[SCAN_T / 32 - 1];
    __syncthreads();
    return pre;
}

__global__ void k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, size_t n,
                             uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t sh[32];
    size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_V;
    uint32_t v[SCAN_V], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t tot;
    uint32_t pre = block_excl_scan(s, sh, &tot);
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k) {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

__global__ void k_scan_carries(uint32_t* sums, size_t ntiles, uint32_t* total_out) {
    __shared__ uint32_t sh[32];
    uint32_t carry = 0;
    for (size_t base = 0; base < ntiles; base += SCAN_T) {
        size_t i = base + threadIdx.x;
        uint32_t v = i < ntiles ? sums[i] : 0u;
        uint32_t tot;
        uint32_t pre = block_excl_scan(v, sh, &tot);
        if (i < ntiles) sums[i] = pre + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(uint32_t* out, size_t n, const uint32_t* sums) {
    size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_V;
    uint32_t c = sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_V; ++k)
        if (base + k < n) out[base + k] += c;
}

aw_status exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, DBuf<uint32_t>& tmp, cudaStream_t s) {
    size_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (ntiles == 0) ntiles = 1;
    AW_TRY(tmp.ensure(ntiles));
    k_scan_tiles<<<(unsigned)ntiles, SCAN_T, 0, s>>>(in, out, n, tmp.p);
    AW_LAUNCH();
    k_scan_carries<<<1, SCAN_T, 0, s>>>(tmp.p, ntiles, out + n);
    AW_LAUNCH();
    k_scan_add<<<(unsigned)ntiles, SCAN_T, 0, s>>>(out, n, tmp.p);
    AW_LAUNCH();
    return AW_OK;
}

// ------------------------------------------------------------------------------------------------
// Level map kernels
// ------------------------------------------------------------------------------------------------
__host__ __device__ inline uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void k_fill_u32(uint32_t* p, uint32_t v, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_block_info(Geo g, uint32_t* out) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.nb) return;
    int c[3];
    bcoord(g, b, c);
    out[4 * b + 0] = c[0];
    out[4 * b + 1] = c[1];
    out[4 * b + 2] = c[2];
    out[4 * b + 3] = expand_bits(c[0]) | (expand_bits(c[1]) << 1) | (expand_bits(c[2]) << 2);
}

// finest-cell occupancy from particles (one byte per finest cell)
// pos: element (i, a) at pos[i * si + a * sa] (AoS: si = 3, sa = 1; SoA: si = 1, sa = n)
__global__ void k_occupancy(Geo g, const float* __restrict__ pos, int64_t si, int64_t sa, int64_t n, uint8_t* occ) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float h0 = __fdiv_rn(g.bs, (float)g.R0);
    int N[3] = {g.D[0] * g.R0, g.D[1] * g.R0, g.D[2] * g.R0};
    int q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float rel = __fsub_rn(pos[i * si + a * sa], g.dmin[a]);
        int v = (int)floorf(__fdiv_rn(rel, h0));
        q[a] = min(max(v, 0), N[a] - 1);
    }
    occ[(size_t)q[0] + (size_t)N[0] * ((size_t)q[1] + (size_t)N[1] * q[2])] = 1;
}

// per block: does it hold a free-surface cell (occupied, with an unoccupied 6-neighbour)?
__global__ void k_block_surface(Geo g, const uint8_t* __restrict__ occ, uint8_t* bsurf) {
    int b = blockIdx.x;
    int cb[3];
    bcoord(g, b, cb);
    int N[3] = {g.D[0] * g.R0, g.D[1] * g.R0, g.D[2] * g.R0};
    int R = g.R0, n3 = R * R * R;
    __shared__ int hit;
    if (threadIdx.x == 0) hit = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < n3; t += blockDim.x) {
        int c[3] = {cb[0] * R + t % R, cb[1] * R + (t / R) % R, cb[2] * R + t / (R * R)};
        size_t ci = (size_t)c[0] + (size_t)N[0] * ((size_t)c[1] + (size_t)N[1] * c[2]);
        if (!occ[ci]) continue;
        bool surf = false;
        for (int a = 0; a < 3 && !surf; ++a)
            for (int s = -1; s <= 1 && !surf; s += 2) {
                int q[3] = {c[0], c[1], c[2]};
                q[a] += s;
                if (q[a] < 0 || q[a] >= N[a]) continue;
                if (!occ[(size_t)q[0] + (size_t)N[0] * ((size_t)q[1] + (size_t)N[1] * q[2])]) surf = true;
            }
        if (surf) hit = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) bsurf[b] = (uint8_t)hit;
}

struct Thresh {
    int k[8];
};

__global__ void k_levels_from_surface(Geo g, const uint8_t* __restrict__ bsurf, Thresh th, uint32_t* level) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.nb) return;
    int cb[3];
    bcoord(g, b, cb);
    uint32_t lev = (uint32_t)(g.L - 1);
    for (int t = 0; t < g.L - 1; ++t) {
        int K = th.k[t];
        bool hit = false;
        for (int z = max(0, cb[2] - K); z <= min(g.D[2] - 1, cb[2] + K) && !hit; ++z)
            for (int y = max(0, cb[1] - K); y <= min(g.D[1] - 1, cb[1] + K) && !hit; ++y)
                for (int x = max(0, cb[0] - K); x <= min(g.D[0] - 1, cb[0] + K); ++x)
                    if (bsurf[bidx(g, x, y, z)]) {
                        hit = true;
                        break;
                    }
        if (hit) {
            lev = (uint32_t)t;
            break;
        }
    }
    level[b] = lev;
}

// One Jacobi pass of enforceGrading (MSBG.cuh:316-351): level = min(level, nLevel + 1) over
// active 26-neighbours whose level differs by more than one.
__global__ void k_grading(Geo g, const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int* changed) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.nb) return;
    uint32_t l = in[b];
    uint32_t best = l;
    if ((int)l != g.L) {
        int cb[3];
        bcoord(g, b, cb);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!dx && !dy && !dz) continue;
                    int nc[3] = {cb[0] + dx, cb[1] + dy, cb[2] + dz};
                    if (!inside(g, nc)) continue;
                    uint32_t nl = in[bidx(g, nc[0], nc[1], nc[2])];
                    if ((int)nl == g.L) continue;
                    if ((int)l - (int)nl > 1) best = min(best, nl + 1u);
                }
    }
    out[b] = best;
    if (best != l) *changed = 1;
}

// enforceGrading's rule (MSBG.cuh:316-351) to its fixpoint in one CTA, in place, then the number of
// blocks whose level differs from `prev`.  Levels only decrease under the rule, so visiting the
// blocks in any order reaches the same fixpoint as the Jacobi passes of aw_msbg_enforce_grading;
// one launch replaces a host round trip per pass.  out[0] = changed blocks, out[1] = passes
// (-1 when max_passes did not reach the fixpoint).
__global__ void __launch_bounds__(1024) k_grading_fixpoint(Geo g, uint32_t* level, const uint32_t* __restrict__ prev,
                                                           int max_passes, int* out) {
    __shared__ int changed, ndiff;
    int pass = 0;
    for (;;) {
        if (threadIdx.x == 0) changed = 0;
        __syncthreads();
        for (int b = threadIdx.x; b < g.nb; b += blockDim.x) {
            const uint32_t l = level[b];
            if ((int)l == g.L) continue;
            uint32_t best = l;
            int cb[3];
            bcoord(g, b, cb);
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (!dx && !dy && !dz) continue;
                        int nc[3] = {cb[0] + dx, cb[1] + dy, cb[2] + dz};
                        if (!inside(g, nc)) continue;
                        const uint32_t nl = ((volatile const uint32_t*)level)[bidx(g, nc[0], nc[1], nc[2])];
                        if ((int)nl == g.L) continue;
                        if ((int)l - (int)nl > 1) best = min(best, nl + 1u);
                    }
            if (best != l) {
                level[b] = best;
                changed = 1;
            }
        }
        __syncthreads();
        ++pass;
        const int c = changed;
        __syncthreads();
        if (!c || pass > max_passes) break;
    }
    if (threadIdx.x == 0) ndiff = 0;
    __syncthreads();
    int d = 0;
    for (int b = threadIdx.x; b < g.nb; b += blockDim.x) d += level[b] != prev[b];
    if (d) atomicAdd(&ndiff, d);
    __syncthreads();
    if (threadIdx.x == 0) {
        out[0] = ndiff;
        out[1] = changed ? -1 : pass;
    }
}

// The level map of the current particles, graded, compared with the map in use on the device: one
// 8-byte read-back.  *changed = blocks whose level differs.
aw_status relevel_on_device(MsbgState& G, const float* d_pos, int64_t si, int64_t sa, int64_t n,
                            const int32_t* thresholds, int* changed, int* passes, cudaStream_t s) {
    AW_TRY(G.level_prev.ensure((size_t)G.nb));
    AW_CUDA(cudaMemcpyAsync(G.level_prev.p, G.level.p, G.nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    AW_TRY(levels_from_positions(G, d_pos, si, sa, n, thresholds, s));
    AW_TRY(G.flag.ensure(2));
    k_grading_fixpoint<<<1, 1024, 0, s>>>(G.geo, G.level.p, G.level_prev.p, 4 * G.geo.L + 8, G.flag.p);
    AW_LAUNCH();
    int h[2];
    AW_CUDA(cudaMemcpyAsync(h, G.flag.p, sizeof h, cudaMemcpyDeviceToHost, s));
    AW_CUDA(cudaStreamSynchronize(s));
    if (h[1] < 0) return set_error(AW_ERR_STATE, "grading did not reach a fixpoint in %d passes", 4 * G.geo.L + 8);
    *changed = h[0];
    if (passes) *passes = h[1];
    return AW_OK;
}

// countBlockElements (MSBG.cuh:353-376) at MG level m; vanish: res < 1 -> 0 (reference),
// else clamp to 1.  Also writes the per-block res.
__global__ void k_count(Geo g, const uint32_t* __restrict__ level, int m, int vanish, uint32_t* cnt, int* res) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.nb) return;
    uint32_t l = level[b];
    int r = 0;
    if ((int)l < g.L) {
        r = (g.R0 >> l) >> m;
        if (r < 1) r = vanish ? 0 : 1;
    }
    if (res) res[b] = r;
    uint32_t nc = (uint32_t)(r * r * r), nf = r > 0 ? (uint32_t)((r + 1) * r * r) : 0u;
    cnt[b] = nc;
    cnt[g.nb + b] = nf;
    cnt[2 * g.nb + b] = nf;
    cnt[3 * g.nb + b] = nf;
}

// galerkinCoarsen (MSBG.cuh:400-498) — the reference coefficient formula, same float order.
__global__ void k_galerkin_ref(Geo g, const uint32_t* __restrict__ level, int axis, int dest,
                               const float* __restrict__ fine, float* __restrict__ coarse,
                               const uint32_t* __restrict__ foff, const uint32_t* __restrict__ coff) {
    int b = blockIdx.x;
    uint32_t l = level[b];
    if ((int)l >= g.L) return;
    int fr = g.R0 >> (l + dest - 1), cr = g.R0 >> (l + dest);
    if (cr < 1 || fr < 2) return;
    int dimx = cr + (axis == 0), dimy = cr + (axis == 1), dimz = cr + (axis == 2);
    int tot = dimx * dimy * dimz;
    int cb[3];
    bcoord(g, b, cb);
    const float SCF = 1 / (4 * 0.75f), SFC = 2 * SCF;
    for (int i = threadIdx.x; i < tot; i += blockDim.x) {
        int tz = i / (dimx * dimy), rem = i % (dimx * dimy), ty = rem / dimx, tx = rem % dimx;
        int t[3] = {tx, ty, tz};
        float baseS = (float)(1 << l);
        if (t[axis] == 0 || t[axis] == cr) {
            int nc[3] = {cb[0], cb[1], cb[2]};
            nc[axis] += t[axis] == 0 ? -1 : 1;
            uint32_t nl = inside(g, nc) ? level[bidx(g, nc[0], nc[1], nc[2])] : l;
            int diff = (int)l - (int)nl;
            float s = (float)(1 << l);
            if (diff == 1) s *= SCF;
            else if (diff == -1) s *= SFC;
            baseS = s;
        }
        float s = baseS * (float)(1 << dest);
        float sum = 0.f;
        for (int d1 = 0; d1 < 2; ++d1)
            for (int d2 = 0; d2 < 2; ++d2) {
                int q[3] = {2 * tx, 2 * ty, 2 * tz};
                if (axis == 0) { q[1] += d1; q[2] += d2; }
                else if (axis == 1) { q[0] += d1; q[2] += d2; }
                else { q[0] += d1; q[1] += d2; }
                sum += fine[foff[b] + fidx(axis, q[0], q[1], q[2], fr)];
            }
        coarse[coff[b] + fidx(axis, tx, ty, tz, cr)] = s * (sum * 0.25f);
    }
}

__global__ void k_copy_f32(float* dst, const float* src, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}
__global__ void k_fill_f32(float* p, float v, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

static inline unsigned nblk(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Offsets of MG level m (reference semantics when vanish != 0) into d_out[4*nb] and totals.
aw_status level_offsets(MsbgState& G, int m, int vanish, uint32_t* d_off4, int* d_res, uint32_t tot[4], cudaStream_t s) {
    size_t nb = (size_t)G.nb;
    AW_TRY(G.scratch_u32.ensure(4 * (nb + 1)));
    // four scanned rows of nb+1 values (the last one is the row's total), then the four totals
    AW_TRY(G.scratch_scan.ensure(4 * (nb + 1) + 4));
    uint32_t* cnt = G.scratch_u32.p;
    uint32_t* scan = G.scratch_scan.p;
    k_count<<<nblk(nb), 256, 0, s>>>(G.geo, G.level.p, m, vanish, cnt, d_res);
    AW_LAUNCH();
    for (int k = 0; k < 4; ++k) {
        uint32_t* o = scan + k * (nb + 1);
        AW_TRY(exclusive_scan_u32(cnt + k * nb, o, nb, G.scratch_scan_tmp, s));
        AW_CUDA(cudaMemcpyAsync(d_off4 + k * nb, o, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        AW_CUDA(cudaMemcpyAsync(scan + 4 * (nb + 1) + k, o + nb, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    }
    AW_CUDA(cudaMemcpyAsync(tot, scan + 4 * (nb + 1), 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    AW_CUDA(cudaStreamSynchronize(s));
    return AW_OK;
}

}  // namespace aw

using namespace aw;

// ================================================================================================
// C ABI
// ================================================================================================
extern "C" const char* aw_last_error(void) { return g_err.c_str(); }
extern "C" const char* aw_version(void) { return "anitowave-b200 0.1 (sm_100a)"; }
extern "C" uint64_t aw_launch_count(void) { return (uint64_t)g_launches; }

extern "C" uint32_t aw_morton3d(uint32_t x, uint32_t y, uint32_t z) {
    return expand_bits(x) | (expand_bits(y) << 1) | (expand_bits(z) << 2);
}

extern "C" void aw_block_layout(int32_t base_res, int32_t level, uint32_t out[6]) {
    int r = base_res >> level;
    out[0] = (uint32_t)(r * r * r);
    out[1] = (uint32_t)((r + 1) * r * r);
    out[2] = (uint32_t)(r * (r + 1) * r);
    out[3] = (uint32_t)(r * r * (r + 1));
    out[4] = out[0] + out[1] + out[2] + out[3];
    out[5] = (uint32_t)r;
}

extern "C" aw_status aw_msbg_create(const aw_grid_desc* d, aw_msbg** out) {
    AW_CHECK_ARG(d && out, "null argument");
    AW_CHECK_ARG(d->dims[0] > 0 && d->dims[1] > 0 && d->dims[2] > 0, "dims must be positive");
    AW_CHECK_ARG(d->base_res >= 1 && d->base_res <= 16 && (d->base_res & (d->base_res - 1)) == 0,
                 "base_res must be a power of two in [1,16]");
    AW_CHECK_ARG(d->num_levels >= 1 && (d->base_res >> (d->num_levels - 1)) >= 1 && d->num_levels <= 8,
                 "num_levels must satisfy base_res >> (num_levels-1) >= 1");
    AW_CHECK_ARG(d->block_size > 0.f, "block_size must be positive");
    int64_t nb = (int64_t)d->dims[0] * d->dims[1] * d->dims[2];
    AW_CHECK_ARG(nb * (int64_t)d->base_res * d->base_res * d->base_res < (int64_t)1 << 31,
                 "grid too large for 32-bit cell offsets");
    *out = nullptr;
    aw_msbg* g = new aw_msbg();
    MsbgState& G = g->st;
    G.desc = *d;
    G.nb = (int)nb;
    G.geo.D[0] = d->dims[0];
    G.geo.D[1] = d->dims[1];
    G.geo.D[2] = d->dims[2];
    G.geo.bs = d->block_size;
    for (int a = 0; a < 3; ++a) G.geo.dmin[a] = d->domain_min[a];
    G.geo.R0 = d->base_res;
    G.geo.L = d->num_levels;
    G.geo.nb = G.nb;
    aw_status st = G.level.alloc(G.nb);
    if (st == AW_OK) {
        k_fill_u32<<<nblk(G.nb), 256>>>(G.level.p, (uint32_t)(d->num_levels - 1), G.nb);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) st = set_error(AW_ERR_CUDA, "aw_msbg_create: %s", cudaGetErrorString(e));
    }
    if (st != AW_OK) {
        delete g;
        return st;
    }
    *out = g;
    return AW_OK;
}

extern "C" aw_status aw_msbg_destroy(aw_msbg* g) {
    delete g;
    return AW_OK;
}

extern "C" aw_status aw_msbg_desc(const aw_msbg* g, aw_grid_desc* out) {
    AW_CHECK_ARG(g && out, "null argument");
    *out = g->st.desc;
    return AW_OK;
}

extern "C" aw_status aw_msbg_init_refinement_map(aw_msbg* g, uint32_t value, aw_stream s) {
    AW_CHECK_ARG(g, "null grid");
    AW_CHECK_ARG((int)value <= g->st.desc.num_levels, "level value out of range");
    k_fill_u32<<<nblk(g->st.nb), 256, 0, (cudaStream_t)s>>>(g->st.level.p, value, g->st.nb);
    AW_LAUNCH();
    g->st.allocated = false;
    return AW_OK;
}

extern "C" aw_status aw_msbg_refinement_map(aw_msbg* g, uint32_t** d_levels) {
    AW_CHECK_ARG(g && d_levels, "null argument");
    *d_levels = g->st.level.p;
    return AW_OK;
}

extern "C" aw_status aw_msbg_block_info(aw_msbg* g, uint32_t* d_out, aw_stream s) {
    AW_CHECK_ARG(g && d_out, "null argument");
    k_block_info<<<nblk(g->st.nb), 256, 0, (cudaStream_t)s>>>(g->st.geo, d_out);
    AW_LAUNCH();
    return AW_OK;
}

namespace aw {
aw_status levels_from_positions(MsbgState& G, const float* d_pos, int64_t si, int64_t sa, int64_t n,
                                const int32_t* thresholds, cudaStream_t s) {
    Thresh th{};
    for (int t = 0; t < G.geo.L - 1; ++t) {
        AW_CHECK_ARG(thresholds, "thresholds required when num_levels > 1");
        AW_CHECK_ARG(thresholds[t] >= 0 && thresholds[t] % G.geo.R0 == 0, "thresholds must be multiples of base_res");
        th.k[t] = thresholds[t] / G.geo.R0;
    }
    size_t ncell = (size_t)G.nb * G.geo.R0 * G.geo.R0 * G.geo.R0;
    AW_TRY(G.occ.ensure(ncell + G.nb));
    AW_CUDA(cudaMemsetAsync(G.occ.p, 0, ncell + G.nb, s));
    if (n > 0) {
        k_occupancy<<<nblk(n), 256, 0, s>>>(G.geo, d_pos, si, sa, n, G.occ.p);
        AW_LAUNCH();
    }
    k_block_surface<<<G.nb, 256, 0, s>>>(G.geo, G.occ.p, G.occ.p + ncell);
    AW_LAUNCH();
    k_levels_from_surface<<<nblk(G.nb), 256, 0, s>>>(G.geo, G.occ.p + ncell, th, G.level.p);
    AW_LAUNCH();
    G.allocated = false;
    return AW_OK;
}
}  // namespace aw

extern "C" aw_status aw_msbg_levels_from_particles(aw_msbg* g, const float* d_pos, int64_t n,
                                                   const int32_t* thresholds, aw_stream s_) {
    AW_CHECK_ARG(g && (d_pos || n == 0), "null argument");
    return levels_from_positions(g->st, d_pos, 3, 1, n, thresholds, (cudaStream_t)s_);
}

extern "C" aw_status aw_msbg_enforce_grading(aw_msbg* g, int32_t* passes, aw_stream s_) {
    AW_CHECK_ARG(g, "null grid");
    MsbgState& G = g->st;
    cudaStream_t s = (cudaStream_t)s_;
    DBuf<uint32_t> tmp;
    AW_TRY(tmp.alloc(G.nb));
    AW_TRY(G.flag.ensure(1));
    int np = 0;
    for (;;) {
        AW_CUDA(cudaMemsetAsync(G.flag.p, 0, sizeof(int), s));
        k_grading<<<nblk(G.nb), 256, 0, s>>>(G.geo, G.level.p, tmp.p, G.flag.p);
        AW_LAUNCH();
        AW_CUDA(cudaMemcpyAsync(G.level.p, tmp.p, G.nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        int h = 0;
        AW_CUDA(cudaMemcpyAsync(&h, G.flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        AW_CUDA(cudaStreamSynchronize(s));
        ++np;
        if (!h) break;
        if (np > 4 * G.geo.L + 8)
            return set_error(AW_ERR_STATE, "grading did not reach a fixpoint in %d passes", np);
    }
    if (passes) *passes = np;
    G.allocated = false;
    return AW_OK;
}

static const int kCellChannels[] = {AW_PRESSURE, AW_DIVERGENCE, AW_DISTANCE_FIELD, AW_VORTICITY, AW_CELL_TYPE};

extern "C" aw_status aw_msbg_allocate(aw_msbg* g, aw_stream s_) {
    AW_CHECK_ARG(g, "null grid");
    MsbgState& G = g->st;
    cudaStream_t s = (cudaStream_t)s_;
    size_t nb = (size_t)G.nb;
    for (int k = 0; k < 4; ++k) AW_TRY(G.off[k].ensure(nb));
    AW_TRY(G.res.ensure(nb));
    DBuf<uint32_t>& off4 = G.scratch_off4;
    AW_TRY(off4.ensure(4 * nb));
    AW_TRY(level_offsets(G, 0, 1, off4.p, G.res.p, G.tot, s));
    for (int k = 0; k < 4; ++k)
        AW_CUDA(cudaMemcpyAsync(G.off[k].p, off4.p + k * nb, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    // host mirrors (topology is small: one u32 per block)
    G.h_level.resize(nb);
    G.h_res.resize(nb);
    AW_CUDA(cudaMemcpyAsync(G.h_level.data(), G.level.p, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    AW_CUDA(cudaMemcpyAsync(G.h_res.data(), G.res.p, nb * sizeof(int), cudaMemcpyDeviceToHost, s));
    for (int k = 0; k < 4; ++k) {
        G.h_off[k].resize(nb);
        AW_CUDA(cudaMemcpyAsync(G.h_off[k].data(), off4.p + k * nb, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    }
    AW_CUDA(cudaStreamSynchronize(s));
    // one slab for every channel: 5 cell channels, 6 face channels per axis (incl. backup)
    size_t nc = G.tot[0];
    size_t pad = 64;
    size_t total = 0;
    uint32_t cnt[AW_NUM_CHANNELS_EXT] = {};
    for (int c : kCellChannels) cnt[c] = (uint32_t)nc;
    const int face_base[] = {AW_VELOCITY_X, AW_PHASE_FIELD_X, AW_BETA_COEFF_X, AW_MASS_DENSITY_X, AW_MOMENTUM_X,
                             AW_VELOCITY_OLD_X};
    for (int fb : face_base)
        for (int a = 0; a < 3; ++a) cnt[fb + a] = G.tot[1 + a];
    for (int c = 0; c < AW_NUM_CHANNELS_EXT; ++c)
        if (cnt[c]) total += ((cnt[c] + pad - 1) / pad) * pad;
    // grow-only: a re-layout that fits the previous slab reuses it (no free/allocate on the way)
    AW_TRY(G.slab.ensure(total));
    AW_CUDA(cudaMemsetAsync(G.slab.p, 0, total * sizeof(float), s));
    size_t at = 0;
    for (int c = 0; c < AW_NUM_CHANNELS_EXT; ++c) {
        G.ch[c] = cnt[c] ? G.slab.p + at : nullptr;
        G.ch_count[c] = cnt[c];
        if (cnt[c]) at += ((cnt[c] + pad - 1) / pad) * pad;
    }
    // beta = 1 / rho = 1 everywhere by default
    for (int a = 0; a < 3; ++a) {
        k_fill_f32<<<nblk(G.tot[1 + a]), 256, 0, s>>>(G.ch[AW_BETA_COEFF_X + a], 1.f, G.tot[1 + a]);
        AW_LAUNCH();
    }
    AW_CUDA(cudaStreamSynchronize(s));
    G.h_tile_off.clear();  // tiles follow the new resolutions
    G.allocated = true;
    G.pw.src_valid = false;  // a sorted particle order refers to the previous layout
    return AW_OK;
}

extern "C" aw_status aw_msbg_totals(const aw_msbg* g, uint32_t totals[4]) {
    AW_CHECK_ARG(g && totals, "null argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    for (int k = 0; k < 4; ++k) totals[k] = g->st.tot[k];
    return AW_OK;
}

extern "C" aw_status aw_msbg_offsets(aw_msbg* g, int32_t kind, uint32_t** d_offsets) {
    AW_CHECK_ARG(g && d_offsets && kind >= 0 && kind < 4, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    *d_offsets = g->st.off[kind].p;
    return AW_OK;
}

extern "C" aw_status aw_msbg_coarse_offsets(aw_msbg* g, int32_t mg_level, int32_t kind, uint32_t* d_out,
                                            uint32_t* total, aw_stream s_) {
    AW_CHECK_ARG(g && d_out && kind >= 0 && kind < 4 && mg_level >= 0, "bad argument");
    MsbgState& G = g->st;
    cudaStream_t s = (cudaStream_t)s_;
    DBuf<uint32_t> off4;
    AW_TRY(off4.alloc(4 * (size_t)G.nb));
    uint32_t tot[4];
    AW_TRY(level_offsets(G, mg_level, 1, off4.p, nullptr, tot, s));
    AW_CUDA(cudaMemcpyAsync(d_out, off4.p + (size_t)kind * G.nb, G.nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    AW_CUDA(cudaStreamSynchronize(s));
    if (total) *total = tot[kind];
    return AW_OK;
}

extern "C" aw_status aw_msbg_channel(aw_msbg* g, int32_t channel, float** d_ptr, uint32_t* count) {
    AW_CHECK_ARG(g && d_ptr && channel >= 0 && channel < AW_NUM_CHANNELS_EXT, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    *d_ptr = g->st.ch[channel];
    if (count) *count = g->st.ch_count[channel];
    return g->st.ch[channel] ? AW_OK : set_error(AW_ERR_INVALID_ARGUMENT, "channel %d has no storage", channel);
}

extern "C" aw_status aw_msbg_run_galerkin(aw_msbg* g, const float* d_fine[3], float* d_coarse[3], int32_t dest,
                                          aw_stream s_) {
    AW_CHECK_ARG(g && d_fine && d_coarse, "null argument");
    MsbgState& G = g->st;
    // reference: runGalerkin returns for destLevel == 0 or >= MAX_LEVELS (MSBG.cuh:668)
    if (dest <= 0 || dest >= G.geo.L) return AW_OK;
    cudaStream_t s = (cudaStream_t)s_;
    size_t nb = (size_t)G.nb;
    DBuf<uint32_t> fo, co;
    AW_TRY(fo.alloc(4 * nb));
    AW_TRY(co.alloc(4 * nb));
    uint32_t tf[4], tc[4];
    AW_TRY(level_offsets(G, dest - 1, 1, fo.p, nullptr, tf, s));
    AW_TRY(level_offsets(G, dest, 1, co.p, nullptr, tc, s));
    for (int a = 0; a < 3; ++a) {
        k_galerkin_ref<<<G.nb, 256, 0, s>>>(G.geo, G.level.p, a, dest, d_fine[a], d_coarse[a], fo.p + (1 + a) * nb,
                                            co.p + (1 + a) * nb);
        AW_LAUNCH();
    }
    AW_CUDA(cudaStreamSynchronize(s));
    return AW_OK;
}
