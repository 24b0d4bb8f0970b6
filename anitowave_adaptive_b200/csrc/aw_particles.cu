// aw_particles.cu — particle sort, P2G, G2P (FLIP blend), RK3 advection, MAC sampling.
//
// Reference behaviour followed (paths within the reference project), with the defects corrected:
//   P2G.cuh:6-12    kernel weight w = (1 - d^2/R^2)^3, R = cell size  (D1: test inverted there)
//   P2G.cuh:16-135  splat mass and momentum to faces                  (D2: clipped to one block)
//   P2G.cuh:139-171 normalizeVelocity u = P/m if m > 1e-6              (fused here)
//   G2P.cuh:11-80   trilinear MAC interpolation                        (D4/D5: staggering/indexing)
//   G2P.cuh:87-128  FLIP blend v = a (v + du) + (1 - a) u_new
//   G2P.cuh:131-173 Ralston RK3 advection
// New (no reference code): stable particle sort by (block, cell) key.
#include <algorithm>

#include "aw_internal.cuh"

namespace aw {

static inline unsigned nblk(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Strided particle array: element (i, a) at p[i * si + a * sa]  (AoS: si=3, sa=1; SoA: si=1, sa=n)
struct PArr {
    const float* p;
    int64_t si, sa;
    __device__ inline float operator()(int64_t i, int a) const { return p[i * si + a * sa]; }
};
struct PArrW {
    float* p;
    int64_t si, sa;
    __device__ inline float& operator()(int64_t i, int a) const { return p[i * si + a * sa]; }
};

// ghosted face tile of a block of resolution r: per axis (r+1)(r+2)^2 faces; a block's three axes
// padded to 16 bytes
__host__ __device__ inline uint32_t tile_axis(int r) { return (uint32_t)((r + 1) * (r + 2) * (r + 2)); }
__host__ __device__ inline uint32_t tile_block(int r) { return r ? ((3 * tile_axis(r) + 3u) & ~3u) : 0u; }

// sort key: global level-0 cell index (MSBG offsets + cell index), or `invalid` for particles in
// inactive blocks.
__device__ inline uint32_t particle_key(const LevelView& L, const float p[3], uint32_t invalid) {
    int c[3];
    point_block(L.g, p, c);
    int b = bidx(L.g, c[0], c[1], c[2]);
    int r = L.res[b];
    if (!r) return invalid;
    float h = fcell(L.g, r);
    int q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float o = forigin(L.g, a, c[a]);
        int v = (int)floorf(__fdiv_rn(__fsub_rn(p[a], o), h));
        q[a] = min(max(v, 0), r - 1);
    }
    return L.off[0][b] + cidx(q[0], q[1], q[2], r);
}

__global__ void k_keys(LevelView L, PArr pos, int64_t n, uint32_t invalid, uint32_t* keys, uint32_t* count) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float p[3] = {pos(i, 0), pos(i, 1), pos(i, 2)};
    uint32_t k = particle_key(L, p, invalid);
    keys[i] = k;
    // particles arrive mostly in last step's cell order: lanes with the same cell add once
    const unsigned peers = __match_any_sync(__activemask(), k);
    if ((__ffs(peers) - 1) == (int)(threadIdx.x & 31)) atomicAdd(&count[k], (uint32_t)__popc(peers));
}

// ------------------------------------------------------------------------------------------------
// Stable LSD radix sort of (key, index) pairs, digits of up to 11 bits (as few passes as the key
// range allows, the digit width spread evenly over them: 20-bit keys take two 10-bit passes, 22-bit
// keys two 11-bit passes).  Each pass: per-tile digit histograms -> one exclusive scan over (digit,
// tile) -> scatter in which one warp walks its tile in order and ranks equal digits with
// __match_any_sync, so equal keys keep their input order.
// ------------------------------------------------------------------------------------------------
constexpr int RADIX_MAX_BITS = 11, RADIX_MAX_BINS = 1 << RADIX_MAX_BITS;

__global__ void __launch_bounds__(256) k_radix_hist(const uint32_t* __restrict__ keys, int64_t n, int shift, int bins,
                                                    int tile, uint32_t* __restrict__ hist, uint32_t ntiles) {
    __shared__ uint32_t h[RADIX_MAX_BINS];
    for (int i = threadIdx.x; i < bins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    // keys arrive nearly sorted (runs of equal digits, thousands long in crowded cells): a warp whose
    // 32 keys share one digit adds once, so shared-memory atomics do not queue on one address
    const int64_t base = (int64_t)blockIdx.x * tile;
    for (int i = threadIdx.x; i < tile; i += blockDim.x) {
        const int64_t j = base + i;
        const bool valid = j < n;
        const uint32_t dig = valid ? (keys[j] >> shift) & (uint32_t)(bins - 1) : 0xFFFFFFFFu;
        const uint32_t d0 = __shfl_sync(0xffffffffu, dig, 0);
        if (__all_sync(0xffffffffu, dig == d0)) {
            if ((threadIdx.x & 31) == 0 && valid) atomicAdd(&h[dig], 32u);
        } else if (valid) {
            atomicAdd(&h[dig], 1u);
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < bins; d += blockDim.x) hist[(size_t)d * ntiles + blockIdx.x] = h[d];
}

__global__ void __launch_bounds__(256) k_radix_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                       uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int64_t n,
                                                       int shift, int bins, int tile, const uint32_t* __restrict__ offs,
                                                       uint32_t ntiles) {
    extern __shared__ uint32_t cnt[];  // bins per warp
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t t = blockIdx.x * (blockDim.x >> 5) + w;
    uint32_t* c = cnt + w * bins;
    if (t >= ntiles) return;
    for (int d = lane; d < bins; d += 32) c[d] = offs[(size_t)d * ntiles + t];
    __syncwarp();
    const int64_t base = (int64_t)t * tile;
    const unsigned lt = (1u << lane) - 1u;
    for (int ch = 0; ch < tile; ch += 32) {
        const int64_t j = base + ch + lane;
        const bool valid = j < n;
        uint32_t key = 0, val = 0, dig = 0;
        if (valid) {
            key = kin[j];
            val = vin ? vin[j] : (uint32_t)j;
            dig = (key >> shift) & (uint32_t)(bins - 1);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, valid ? dig : (uint32_t)(bins + lane));
        const uint32_t pos = valid ? c[dig] + __popc(peers & lt) : 0u;
        __syncwarp();
        if (valid && (__ffs(peers) - 1) == lane) c[dig] += __popc(peers);
        __syncwarp();
        if (valid) {
            kout[pos] = key;
            vout[pos] = val;
        }
    }
}

static aw_status radix_sort_pairs(uint32_t* keys, uint32_t* keys2, uint32_t* vals, uint32_t* vals2, int64_t n,
                                  uint32_t maxkey, DBuf<uint32_t>& hist, DBuf<uint32_t>& scan_out, DBuf<uint32_t>& tmp,
                                  uint32_t** sorted_vals, cudaStream_t s) {
    int bits = 1;
    while (bits < 32 && (maxkey >> bits)) ++bits;
    const int passes = (bits + RADIX_MAX_BITS - 1) / RADIX_MAX_BITS;
    const int digit = (bits + passes - 1) / passes;
    const int bins = 1 << digit;
    // tiles of 2048 keys, longer for large arrays (down to about 4096 tiles, one wave of warps), so
    // that the (digit, tile) table and its scan stay small
    int tile = 2048;
    while (tile < 16384 && n / (2 * (int64_t)tile) >= 4096) tile *= 2;
    const uint32_t ntiles = (uint32_t)((n + tile - 1) / tile);
    const size_t nh = (size_t)bins * ntiles;
    AW_TRY(hist.ensure(nh));
    AW_TRY(scan_out.ensure(nh + 1));
    uint32_t *kin = keys, *kout = keys2, *vin = nullptr, *vout = vals;
    const int wpb = 8;
    for (int p = 0; p < passes; ++p) {
        const int shift = p * digit;
        k_radix_hist<<<ntiles, 256, 0, s>>>(kin, n, shift, bins, tile, hist.p, ntiles);
        AW_LAUNCH();
        AW_TRY(exclusive_scan_u32(hist.p, scan_out.p, nh, tmp, s));
        const size_t ssm = (size_t)wpb * bins * sizeof(uint32_t);
        if (ssm > 48 * 1024)
            AW_CUDA(cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm));
        k_radix_scatter<<<(ntiles + wpb - 1) / wpb, 32 * wpb, ssm, s>>>(
            kin, vin, kout, vout, n, shift, bins, tile, scan_out.p, ntiles);
        AW_LAUNCH();
        std::swap(kin, kout);
        vin = vout;
        vout = (vout == vals) ? vals2 : vals;
    }
    *sorted_vals = vin;
    return AW_OK;
}

// 64-bit content hash of a particle array: the sum over particles of a mixed hash of (index, x, y, z),
// so that it does not depend on the order the particles are visited in.  mix64 is the splitmix64
// finaliser (S. Vigna).
__device__ inline unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ inline unsigned long long hash3(uint32_t i, float x, float y, float z) {
    const unsigned long long a = ((unsigned long long)__float_as_uint(x) << 32) | __float_as_uint(y);
    const unsigned long long b = ((unsigned long long)__float_as_uint(z) << 32) | i;
    return mix64(mix64(a) ^ b);
}
__device__ inline unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Hash partial sums land in kHashSlots slot pairs (CTA b in slot b mod kHashSlots), so that the
// atomics of many CTAs do not queue on one address; k_hash_fold then sums the slots.
constexpr int kHashSlots = 128;
__device__ inline void hash_block_add(unsigned long long hp, unsigned long long hv, unsigned long long* slots) {
    __shared__ unsigned long long red[2][32];
    hp = warp_sum_u64(hp);
    hv = warp_sum_u64(hv);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) {
        red[0][w] = hp;
        red[1][w] = hv;
    }
    __syncthreads();
    if (w == 0) {
        hp = lane < nw ? red[0][lane] : 0ull;
        hv = lane < nw ? red[1][lane] : 0ull;
        hp = warp_sum_u64(hp);
        hv = warp_sum_u64(hv);
        if (lane == 0) {
            unsigned long long* d = slots + 2 * (blockIdx.x % kHashSlots);
            atomicAdd(d, hp);
            atomicAdd(d + 1, hv);
        }
    }
}
// out[0], out[1] = sums of the slot pairs
__global__ void k_hash_fold(const unsigned long long* __restrict__ slots, unsigned long long* out) {
    unsigned long long hp = 0, hv = 0;
    for (int i = threadIdx.x; i < kHashSlots; i += 32) {
        hp += slots[2 * i];
        hv += slots[2 * i + 1];
    }
    hp = warp_sum_u64(hp);
    hv = warp_sum_u64(hv);
    if (threadIdx.x == 0) {
        out[0] = hp;
        out[1] = hv;
    }
}

// gather pos/vel into SoA sorted order, carry the original ids; with hash, add the content hashes
// of the input positions and velocities into the slot pairs of `hash` (kHashSlots pairs)
__global__ void k_gather(const uint32_t* __restrict__ src, int64_t n, PArr pos, PArr vel, float* __restrict__ soa,
                         const uint32_t* __restrict__ ids_in, uint32_t* __restrict__ ids_out,
                         const uint32_t* __restrict__ keys, uint32_t* __restrict__ keys_sorted,
                         unsigned long long* hash = nullptr) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long hp = 0, hv = 0;
    if (j < n) {
        const uint32_t i = src[j];
        const float x = pos(i, 0), y = pos(i, 1), z = pos(i, 2);
        soa[j] = x;
        soa[n + j] = y;
        soa[2 * n + j] = z;
        if (hash) hp = hash3(i, x, y, z);
        if (vel.p) {
            const float u = vel(i, 0), v = vel(i, 1), w = vel(i, 2);
            soa[3 * n + j] = u;
            soa[4 * n + j] = v;
            soa[5 * n + j] = w;
            if (hash) hv = hash3(i, u, v, w);
        }
        if (ids_out) ids_out[j] = ids_in ? ids_in[i] : i;
        if (keys_sorted) keys_sorted[j] = keys[i];
    }
    if (hash) hash_block_add(hp, hv, hash);  // uniform across the CTA
}

// content hashes of AoS positions and, when given, velocities into the slot pairs (must start at 0)
__global__ void k_hash_aos(const float* __restrict__ pos, const float* __restrict__ vel, int64_t n,
                           unsigned long long* slots) {
    unsigned long long hp = 0, hv = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        hp += hash3((uint32_t)i, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        if (vel) hv += hash3((uint32_t)i, vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
    hash_block_add(hp, hv, slots);
}

// the caller's arrays still hold what the last aw_p2g sorted (positions; velocities too if asked)
__device__ inline bool sort_reusable(const unsigned long long* h, bool need_vel) {
    return h[0] == h[2] && (!need_vel || h[1] == h[3]);
}

aw_status ParticleWork::ensure(int64_t np, uint32_t ncell) {
    AW_TRY(keys.ensure((size_t)np));
    AW_TRY(perm.ensure((size_t)np));
    AW_TRY(perm2.ensure((size_t)np));
    AW_TRY(cell_start.ensure((size_t)ncell + 2));
    AW_TRY(cell_fill.ensure((size_t)ncell + 2));
    AW_TRY(soa.ensure((size_t)np * 6 + kSoaPad));
    AW_TRY(soa2.ensure((size_t)np * 6 + kSoaPad));
    n = np;
    return AW_OK;
}

// Sort (keys -> bucket counts -> scan -> scatter -> per-bucket order) and gather into G.pw.soa.
// After the call: pw.perm[j] = input index of sorted slot j, pw.cell_start[c] = first sorted
// slot of level-0 cell c (c in [0, tot0]; bucket tot0 holds particles of inactive blocks).
aw_status sort_core(MsbgState& G, PArr pos, int64_t n, cudaStream_t s) {
    uint32_t nc = G.tot[0];
    ParticleWork& W = G.pw;
    AW_TRY(W.ensure(n, nc));
    AW_CUDA(cudaMemsetAsync(W.cell_fill.p, 0, ((size_t)nc + 2) * sizeof(uint32_t), s));
    if (n > 0) {
        k_keys<<<nblk(n), 256, 0, s>>>(G.view0(), pos, n, nc, W.keys.p, W.cell_fill.p);
        AW_LAUNCH();
    }
    AW_TRY(exclusive_scan_u32(W.cell_fill.p, W.cell_start.p, (size_t)nc + 1, W.tmp, s));
    W.sorted = W.perm.p;
    W.src_valid = false;  // the recorded order of aw_p2g is replaced
    if (n > 0) {
        // keys are consumed by the sort: keep a copy for aw_sort_particles' key output
        AW_TRY(W.keys2.ensure((size_t)n));
        AW_TRY(W.keys3.ensure((size_t)n));
        AW_CUDA(cudaMemcpyAsync(W.keys3.p, W.keys.p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        AW_TRY(radix_sort_pairs(W.keys3.p, W.keys2.p, W.perm.p, W.perm2.p, n, nc, W.hist, W.hscan, W.tmp, &W.sorted, s));
    }
    return AW_OK;
}

aw_status sort_particles_soa(MsbgState& G, const float* pos_aos, const float* vel_aos, int64_t n, cudaStream_t s,
                             bool record) {
    PArr pos{pos_aos, 3, 1}, vel{vel_aos, 3, 1};
    AW_TRY(sort_core(G, pos, n, s));
    ParticleWork& W = G.pw;
    unsigned long long* hash = nullptr;
    if (record) {
        AW_TRY(W.hash.ensure(4 + 2 * kHashSlots));
        AW_CUDA(cudaMemsetAsync(W.hash.p + 4, 0, 2 * kHashSlots * sizeof(unsigned long long), s));
        hash = W.hash.p + 4;
    }
    if (n > 0) {
        k_gather<<<nblk(n), 256, 0, s>>>(W.sorted, n, pos, vel, W.soa.p, nullptr, nullptr, nullptr, nullptr, hash);
        AW_LAUNCH();
    }
    if (record) {
        k_hash_fold<<<1, 32, 0, s>>>(W.hash.p + 4, W.hash.p);
        AW_LAUNCH();
    }
    if (record) {
        W.src_pos = pos_aos;
        W.src_vel = vel_aos;
        W.src_n = n;
        W.src_valid = true;
    }
    return AW_OK;
}

aw_status sort_core_soa(MsbgState& G, const float* soa_pos, int64_t n, cudaStream_t s) {
    return sort_core(G, PArr{soa_pos, 1, n}, n, s);
}

aw_status gather_soa(MsbgState& G, const float* in_soa, int64_t n, float* out_soa, const uint32_t* ids_in,
                     uint32_t* ids_out, cudaStream_t s) {
    if (n <= 0) return AW_OK;
    PArr pos{in_soa, 1, n}, vel{in_soa + 3 * n, 1, n};
    k_gather<<<nblk(n), 256, 0, s>>>(G.pw.sorted, n, pos, vel, out_soa, ids_in, ids_out, nullptr, nullptr);
    AW_LAUNCH();
    return AW_OK;
}

__global__ void k_cell_count(const uint32_t* __restrict__ cstart, uint32_t nc, float* out) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) out[c] = (float)(cstart[c + 1] - cstart[c]);
}

// ------------------------------------------------------------------------------------------------
// P2G, one pass per particle.  One CTA per block b takes only b's own particles (one contiguous
// range of the cell-sorted array).  Every face within reach of such a particle lies in b's ghosted
// face tile (faces [0,r] along the axis, [-1,r] across it), so the 2x2x2 candidates per axis need
// no index checks: the weight is max(0, 1 - d^2/h^2)^3 and the shared-memory atomics of zero
// weights are predicated off.
//
// The tile accumulates in FP32.  (A fixed-point tile with integer atomics ran faster, but its
// absolute rounding error is amplified by u = P/m on the low-mass faces at the fluid's edge.)
//
// The flush adds every nonzero tile entry into each copy of that physical face held by a block of
// b's resolution (a face on a block boundary has one copy per side).  Faces of neighbours at
// another resolution are at other positions.  Those of a coarser neighbour (half b's resolution)
// lie in a second, coarse tile around b, filled by per-cell register sums like the own tile and
// flushed the same way.  Particles within reach of a finer neighbour add their weights in the
// neighbour's own lattice with global float atomics; those (particle, neighbour) pairs are queued
// per warp and run one pair per lane, so a warp does not pass over every neighbour direction with
// most lanes idle.  A second kernel normalises u = P / m.  The face arrays must start at zero.
// ------------------------------------------------------------------------------------------------
__device__ inline int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

struct FaceAcc {
    float* m[3];
    float* P[3];
    float* Phi[3];  // sum of w * phase (two-phase P2G only)
};

// weights of one particle on the faces of a neighbouring block of resolution rn != r, global atomics.
// N holds that block's origin, 1 / cell size and face offsets (computed once per CTA).
struct CrossNb {
    float o[3];
    float invh;
    uint32_t off[3];
};

template <bool PH>
__device__ __forceinline__ void p2g_cross(const CrossNb& N, int rn, const float X[3], const float V[3], float ph,
                                          const FaceAcc& acc) {
    float q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) q[k] = (X[k] - N.o[k]) * N.invh;
    const float rf = (float)rn;
    if (q[0] <= -1.f || q[1] <= -1.f || q[2] <= -1.f || q[0] >= rf + 1.f || q[1] >= rf + 1.f || q[2] >= rf + 1.f) return;
    // Per component, only the face rows inside the neighbour are visited: for a face neighbour about
    // half of the 2 x 2 x 2 candidates, for edges and corners fewer.
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        const int ia = (int)floorf(q[a]);
        const int j1 = (int)floorf(q[t1] - 0.5f), j2 = (int)floorf(q[t2] - 0.5f);
        const int a0 = max(ia, 0), a1 = min(ia + 1, rn);
        const int b0 = max(j1, 0), b1 = min(j1 + 1, rn - 1);
        const int e0 = max(j2, 0), e1 = min(j2 + 1, rn - 1);
        const uint32_t ob = N.off[a];
#pragma unroll 1
        for (int fa = a0; fa <= a1; ++fa) {
            const float dA = q[a] - (float)fa;
#pragma unroll 1
            for (int f1 = b0; f1 <= b1; ++f1) {
                const float dB = q[t1] - ((float)f1 + 0.5f);
                const float AB = dA * dA + dB * dB;
#pragma unroll 1
                for (int f2 = e0; f2 <= e1; ++f2) {
                    const float dC = q[t2] - ((float)f2 + 0.5f);
                    const float tt = 1.f - (AB + dC * dC);
                    if (tt <= 0.f) continue;
                    const float w = tt * tt * tt;
                    // (fa, f1, f2) along (a, t1, t2) -> the face index of axis a
                    const uint32_t fi = ob + (a == 0 ? (uint32_t)(fa + (rn + 1) * (f1 + rn * f2))
                                                     : (a == 1 ? (uint32_t)(f2 + rn * (fa + (rn + 1) * f1))
                                                               : (uint32_t)(f1 + rn * (f2 + rn * fa))));
                    atomicAdd(&acc.m[a][fi], w);
                    atomicAdd(&acc.P[a][fi], w * V[a]);
                    if (PH && ph != 0.f) atomicAdd(&acc.Phi[a][fi], w * ph);
                }
            }
        }
    }
}

constexpr int P2G_THREADS = 512;  // the most threads a P2G CTA is launched with
constexpr int P2G_XQ = 96;  // per-warp queue of cross-resolution pairs: < 32 waiting + 2 per lane
constexpr int P2G_SLICE = 16;  // particles of one cell per register-accumulation task
constexpr int P2G_MAX_SLICES = 1 << 19;  // 6 * 8^3 * this stays below 2^31
constexpr int P2G_MAX_CELLS = 16 * 16 * 16;  // cells of the largest block (base resolution <= 16)
constexpr int P2G_NEAR_CELLS = 8 * 8 * 8;    // blocks up to this size list their near cells

// one queued (particle, neighbour direction d) pair: the particle's weights on neighbour d's faces
template <bool PH>
__device__ __forceinline__ void p2g_cross_pair(const CrossNb* xn, const int* nres, uint32_t v, int d, uint32_t p0,
                                               const float* __restrict__ soa, int64_t n, const FaceAcc& acc,
                                               const uint32_t* __restrict__ pid, const float* __restrict__ phase) {
    const uint32_t sidx = p0 + v;
    float X[3], V[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        X[k] = soa[(int64_t)k * n + sidx];
        V[k] = soa[(int64_t)(3 + k) * n + sidx];
    }
    const float ph = PH ? phase[pid[sidx]] : 0.f;
    p2g_cross<PH>(xn[d], nres[d], X, V, ph, acc);
}

// Adds every nonzero entry of a ghosted face tile of resolution rr around block cb (faces [0, rr]
// along the axis, [-1, rr] across) into each copy of that face held by a block of resolution rr: a
// face on a plane between two blocks along its axis has one copy per side.  nres / noff: the
// resolution (0 outside the domain or inactive) and face offsets of the 27 blocks around cb,
// direction d = (dx + 1) + 3 (dy + 1) + 9 (dz + 1).
template <bool PH>
__device__ __forceinline__ void p2g_flush_tile(const int* nres, const uint32_t (*noff)[3], int rr, const float* tm,
                                               const float* tp, const float* tq, const FaceAcc& acc) {
    const int R1 = rr + 1, R2 = rr + 2;
    const int TA = (int)tile_axis(rr);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        for (int rem = threadIdx.x; rem < TA; rem += blockDim.x) {
            const float mv = tm[a * TA + rem];
            if (mv == 0.f) continue;
            const float pv = tp[a * TA + rem];
            const float qv2 = PH ? tq[a * TA + rem] : 0.f;
            const int iA = rem % R1;
            const int i1 = (rem / R1) % R2 - 1;
            const int i2 = rem / (R1 * R2) - 1;
            const int s1 = i1 < 0 ? -1 : (i1 >= rr ? 1 : 0), s2 = i2 < 0 ? -1 : (i2 >= rr ? 1 : 0);
            const int l1 = i1 - s1 * rr, l2 = i2 - s2 * rr;
            const int nA = (iA == 0 || iA == rr) ? 2 : 1;
            for (int k = 0; k < nA; ++k) {
                int sA, lA;
                if (iA == 0) { sA = k - 1; lA = k == 0 ? rr : 0; }
                else if (iA == rr) { sA = k; lA = k == 0 ? rr : 0; }
                else { sA = 0; lA = iA; }
                int sd[3];
                sd[a] = sA;
                sd[t1] = s1;
                sd[t2] = s2;
                const int d = (sd[0] + 1) + 3 * (sd[1] + 1) + 9 * (sd[2] + 1);
                if (nres[d] != rr) continue;
                int f[3];
                f[a] = lA;
                f[t1] = l1;
                f[t2] = l2;
                const uint32_t fi = noff[d][a] + fidx(a, f[0], f[1], f[2], rr);
                atomicAdd(&acc.m[a][fi], mv);
                atomicAdd(&acc.P[a][fi], pv);
                if (PH && qv2 != 0.f) atomicAdd(&acc.Phi[a][fi], qv2);
            }
        }
    }
}

template <bool PH>
__global__ void __launch_bounds__(P2G_THREADS, 2) k_p2g_own(LevelView L, const float* __restrict__ soa, int64_t n,
                                                 const uint32_t* __restrict__ cs, FaceAcc acc,
                                                 const uint32_t* __restrict__ pid, const float* __restrict__ phase,
                                                 int smem_floats, uint8_t* __restrict__ occ,
                                                 const int* __restrict__ order) {
    extern __shared__ float sm[];
    __shared__ int nres[27];
    __shared__ uint32_t noff[27][3];
    __shared__ CrossNb xn[27];
    __shared__ int cross, coarse;
    __shared__ uint32_t maxcnt;
    __shared__ int ccount[P2G_MAX_CELLS / 32], cocount[P2G_MAX_CELLS / 32];
    __shared__ uint16_t clist[P2G_MAX_CELLS], colist[P2G_MAX_CELLS];
    __shared__ int nonempty, nnear, ncoarse;
    __shared__ int tctr[2];  // next own / coarse task to hand out
    // near-cell list of the cross-resolution pass (blocks of at most P2G_NEAR_CELLS cells)
    __shared__ uint16_t nl_cell[P2G_NEAR_CELLS];
    __shared__ uint32_t nl_mask[P2G_NEAR_CELLS], nl_pre[P2G_NEAR_CELLS + 1];
    __shared__ uint32_t nmask_tmp[P2G_NEAR_CELLS];
    __shared__ int ncnt_tmp[P2G_NEAR_CELLS];
    __shared__ uint32_t xq_v[(P2G_THREADS / 32) * P2G_XQ];
    __shared__ uint8_t xq_d[(P2G_THREADS / 32) * P2G_XQ];
    const int b = order ? order[blockIdx.x] : (int)blockIdx.x;
    const int r = L.res[b];
    if (!r) {
        if (threadIdx.x == 0) occ[b] = 0;
        return;
    }
    const uint32_t c0 = L.off[0][b];
    const uint32_t p0 = cs[c0], p1 = cs[c0 + (uint32_t)(r * r * r)];
    if (threadIdx.x == 0) occ[b] = p1 > p0 ? 1 : 0;  // read by G2P: blocks around it skip their tiles
    if (p0 == p1) return;
    const Geo& g = L.g;
    // the block's cell starts in the sorted array, after the tiles (smem_floats floats)
    uint32_t* cst = reinterpret_cast<uint32_t*>(sm + smem_floats);
    int cb[3];
    bcoord(g, b, cb);
    const int R1 = r + 1, R2 = r + 2;
    const int TA = (int)tile_axis(r);
    // The coarse tile: the faces of the lattice of half b's resolution around b, with the same
    // ghost rows (faces [0, r/2] along the axis, [-1, r/2] across); its entries outside b hold the
    // deposits into coarser neighbours.
    const int rc = r >> 1;
    const int TAc = rc ? (int)tile_axis(rc) : 0;
    constexpr int NV = PH ? 3 : 2;  // mass, momentum (, phase) per face
    float* am = sm;                   // 3 TA mass
    float* ap = sm + 3 * TA;          // 3 TA momentum
    float* aq = sm + 6 * TA;          // 3 TA phase (PH)
    float* cm = sm + 3 * NV * TA;     // 3 TAc mass of the coarse tile
    float* cp = cm + 3 * TAc;         // 3 TAc momentum
    float* cq = cm + 6 * TAc;         // 3 TAc phase (PH)
    // Blocks of one or two cells per edge hold thousands of particles on a tile of 18 or 48 faces
    // per axis: each warp then deposits into a private copy of the tiles, and the copies are summed
    // before the flush, so that warps do not contend for the same few addresses.
    const int TW = 3 * NV * (TA + TAc);
    const bool priv = r <= 2 && (int)(blockDim.x >> 5) * TW <= smem_floats;
    const int ntile = priv ? (int)(blockDim.x >> 5) * TW : TW;
    float* tw = priv ? sm + (threadIdx.x >> 5) * TW : sm;
    float* amw = tw;
    float* apw = tw + 3 * TA;
    float* aqw = tw + 6 * TA;
    float* cmw = tw + 3 * NV * TA;
    float* cpw = cmw + 3 * TAc;
    float* cqw = cmw + 6 * TAc;
    for (int i = threadIdx.x; i < ntile; i += blockDim.x) sm[i] = 0.f;
    if (threadIdx.x == 0) {
        cross = 0;
        coarse = 0;
        maxcnt = 0;
        tctr[0] = 0;
        tctr[1] = 0;
    }
    __syncthreads();
    if (threadIdx.x < 27) {
        const int d = threadIdx.x;
        const int nc[3] = {cb[0] + d % 3 - 1, cb[1] + (d / 3) % 3 - 1, cb[2] + d / 9 - 1};
        const int nb = inside(g, nc) ? bidx(g, nc[0], nc[1], nc[2]) : -1;
        const int rn = nb >= 0 ? L.res[nb] : 0;
        nres[d] = rn;
#pragma unroll
        for (int k = 0; k < 3; ++k) noff[d][k] = rn ? L.off[1 + k][nb] : 0u;
        if (rn && 2 * rn == r) atomicOr(&coarse, 1 << d);
        if (rn && rn != r && 2 * rn != r) {  // finer (or, in a map that is not 2:1 graded, coarser still)
            atomicOr(&cross, 1 << d);
            xn[d].invh = 1.f / fcell(g, rn);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                xn[d].o[k] = forigin(g, k, nc[k]);
                xn[d].off[k] = L.off[1 + k][nb];
            }
        }
    }
    __syncthreads();
    const int xmask = cross;    // finer neighbours: (particle, neighbour) pairs
    const int cmask = coarse;   // neighbours at half b's resolution: the coarse tile
    const float h = fcell(g, r);
    const float invh = 1.f / h;
    float o[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) o[a] = forigin(g, a, cb[a]);
    // Own particles, cell by cell.  A task is (kind, cell c, slice s): up to `slice` of c's particles
    // (contiguous in the cell-sorted array).  Its thread sums their weights w and w times a value on
    // the 2x3x3 faces of one component a around c in registers, then adds the sums into the tile:
    // one atomic per face and task instead of one per face and particle.  Kinds 0-2 sum mass and
    // momentum of component a = kind; with phases, kinds 3-5 sum w * phase of component kind - 3
    // over the particles whose phase is not 0 (the others add nothing).  Slices hold P2G_SLICE
    // particles unless a crowded cell would push the task count past 6 * 512 * P2G_MAX_SLICES.
    const int nc3 = r * r * r;
    // The block's non-empty cells, in cell order: tasks run over these only, so that lanes do not
    // idle on the air cells of a surface block.
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    // A cell is listed for the coarse tile too when it lies within two of b's cells (one coarse
    // cell, the reach there) of a side towards a coarser neighbour, on every axis that neighbour's
    // direction crosses.
    auto coarse_near = [&](int c) {
        const int cc[3] = {c % r, (c / r) % r, c / (r * r)};
        for (uint32_t mm = (uint32_t)cmask; mm; mm &= mm - 1) {
            const int d = __ffs(mm) - 1;
            const int dd[3] = {d % 3 - 1, (d / 3) % 3 - 1, d / 9 - 1};
            bool nr = true;
#pragma unroll
            for (int k = 0; k < 3; ++k) nr = nr && (dd[k] == 0 || (dd[k] < 0 ? cc[k] <= 1 : cc[k] >= r - 2));
            if (nr) return true;
        }
        return false;
    };
    const int nchunk = (nc3 + 31) / 32;
    for (int ch = wid; ch < nchunk; ch += nwarp) {
        const int c = ch * 32 + lane;
        uint32_t cnt = 0;
        if (c < nc3) {
            const uint32_t a0 = cs[c0 + c], a1 = cs[c0 + c + 1];
            cst[c] = a0;
            if (c == nc3 - 1) cst[nc3] = a1;
            cnt = a1 - a0;
        }
        if (cnt > 0) atomicMax(&maxcnt, cnt);
        const unsigned m = __ballot_sync(0xffffffffu, cnt > 0);
        const unsigned mc = __ballot_sync(0xffffffffu, cnt > 0 && cmask && coarse_near(c));
        if (lane == 0) {
            ccount[ch] = __popc(m);
            cocount[ch] = __popc(mc);
        }
    }
    __syncthreads();
    if (wid == 0) {  // exclusive scans of the per-chunk counts
        int carry = 0, carry2 = 0;
        for (int base = 0; base < nchunk; base += 32) {
            const int ch = base + lane;
            const int v = ch < nchunk ? ccount[ch] : 0;
            const int v2 = ch < nchunk ? cocount[ch] : 0;
            int incl = v, incl2 = v2;
#pragma unroll
            for (int sh = 1; sh < 32; sh <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, sh);
                const int y2 = __shfl_up_sync(0xffffffffu, incl2, sh);
                if (lane >= sh) {
                    incl += y;
                    incl2 += y2;
                }
            }
            if (ch < nchunk) {
                ccount[ch] = carry + incl - v;
                cocount[ch] = carry2 + incl2 - v2;
            }
            carry += __shfl_sync(0xffffffffu, incl, 31);
            carry2 += __shfl_sync(0xffffffffu, incl2, 31);
        }
        if (lane == 0) {
            nonempty = carry;
            ncoarse = carry2;
        }
    }
    __syncthreads();
    for (int ch = wid; ch < nchunk; ch += nwarp) {
        const int c = ch * 32 + lane;
        const bool ne = c < nc3 && cst[c + 1] > cst[c];
        const bool cn = ne && cmask && coarse_near(c);
        const unsigned m = __ballot_sync(0xffffffffu, ne);
        const unsigned mc = __ballot_sync(0xffffffffu, cn);
        if (ne) clist[ccount[ch] + __popc(m & ((1u << lane) - 1u))] = (uint16_t)c;
        if (cn) colist[cocount[ch] + __popc(mc & ((1u << lane) - 1u))] = (uint16_t)c;
    }
    __syncthreads();
    const int ncell = nonempty;
    // Near-cell list of the cross-resolution pass (built here, so that warps that finish their
    // deposit tasks go on to the pass without waiting for the others)
    const int w = wid, nw = nwarp;
    const bool listed = nc3 <= P2G_NEAR_CELLS;
    if (xmask && listed) {
        for (int ch = wid; ch < (ncell + 31) / 32; ch += nwarp) {
            const int k = ch * 32 + lane;
            uint32_t cm = 0;
            int cnt = 0;
            if (k < ncell) {
                const int c = clist[k];
                const int cc[3] = {c % r, (c / r) % r, c / (r * r)};
                for (uint32_t mm = (uint32_t)xmask; mm; mm &= mm - 1) {
                    const int d = __ffs(mm) - 1;
                    const int dd[3] = {d % 3 - 1, (d / 3) % 3 - 1, d / 9 - 1};
                    const float reach = (float)r / (float)nres[d];
                    bool nr = true;
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        nr = nr && (dd[a] == 0 || (dd[a] < 0 ? (float)cc[a] < reach + 0.5f
                                                             : (float)cc[a] > (float)(r - 1) - reach - 0.5f));
                    if (nr) cm |= 1u << d;
                }
                if (cm) cnt = (int)(cst[c + 1] - cst[c]);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, cm != 0);
            if (lane == 0) ccount[ch] = __popc(bal);
            // stash this lane's result in the slot the final list will give it: first the chunk counts
            nmask_tmp[k < P2G_NEAR_CELLS ? k : 0] = k < ncell ? cm : 0u;
            ncnt_tmp[k < P2G_NEAR_CELLS ? k : 0] = cnt;
        }
        __syncthreads();
        if (wid == 0) {  // exclusive scan of the per-chunk counts of near cells
            int carry = 0;
            const int nch = (ncell + 31) / 32;
            for (int base = 0; base < nch; base += 32) {
                const int ch = base + lane;
                const int v = ch < nch ? ccount[ch] : 0;
                int incl = v;
#pragma unroll
                for (int sh = 1; sh < 32; sh <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, sh);
                    if (lane >= sh) incl += y;
                }
                if (ch < nch) ccount[ch] = carry + incl - v;
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) nnear = carry;
        }
        __syncthreads();
        for (int ch = wid; ch < (ncell + 31) / 32; ch += nwarp) {
            const int k = ch * 32 + lane;
            const uint32_t cm = k < ncell ? nmask_tmp[k] : 0u;
            const unsigned bal = __ballot_sync(0xffffffffu, cm != 0);
            if (cm) {
                const int at = ccount[ch] + __popc(bal & ((1u << lane) - 1u));
                nl_cell[at] = clist[k];
                nl_mask[at] = cm;
                nl_pre[at + 1] = ncnt_tmp[k];
            }
        }
        __syncthreads();
        if (wid == 0) {  // inclusive scan of the near cells' particle counts -> nl_pre[0..nnear]
            int carry = 0;
            const int nn = nnear;
            for (int base = 0; base < nn; base += 32) {
                const int k = base + lane;
                const int v = k < nn ? (int)nl_pre[k + 1] : 0;
                int incl = v;
#pragma unroll
                for (int sh = 1; sh < 32; sh <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, sh);
                    if (lane >= sh) incl += y;
                }
                if (k < nn) nl_pre[k + 1] = (uint32_t)(carry + incl);
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) nl_pre[0] = 0;
        }
        __syncthreads();
    }
    const uint32_t mc = maxcnt;
    const int nsl = (int)min((mc + P2G_SLICE - 1) / P2G_SLICE, (uint32_t)P2G_MAX_SLICES);
    const uint32_t slice = nsl ? (mc + nsl - 1) / nsl : 0;
    constexpr int NK = PH ? 6 : 3;
    const int ntask = NK * ncell * nsl;
    // Warps take 32 tasks at a time from a shared counter, so that warps whose tasks hold fewer
    // particles take more of them.
    for (;;) {
        int tb = 0;
        if (lane == 0) tb = atomicAdd(&tctr[0], 32);
        tb = __shfl_sync(0xffffffffu, tb, 0);
        if (tb >= ntask) break;
        const int task = tb + lane;
        if (task >= ntask) continue;
        // neighbouring threads take the kinds of one cell (they read the same particles, so one
        // warp-wide load touches a third as many sectors), then neighbouring cells
        const int kind = task % NK;
        const int rem = task / NK;
        const bool qpass = PH && kind >= 3;
        const int a = qpass ? kind - 3 : kind;
        const int c = clist[rem % ncell], sl = rem / ncell;
        const uint32_t ca = cst[c], ce = cst[c + 1];
        if ((uint32_t)sl * slice >= ce - ca) continue;
        const uint32_t i0 = ca + (uint32_t)sl * slice;
        const uint32_t i1 = ce - i0 > slice ? i0 + slice : ce;
        const int t1 = a == 2 ? 0 : a + 1, t2 = a == 0 ? 2 : a - 1;
        const int cx = c % r, cy = (c / r) % r, cz = c / (r * r);
        const int ka = a == 0 ? cx : (a == 1 ? cy : cz);   // cell index along a
        const int k1 = a == 0 ? cy : (a == 1 ? cz : cx);   // ... along t1
        const int k2 = a == 0 ? cz : (a == 1 ? cx : cy);   // ... along t2
        const float fa0 = (float)ka, f10 = (float)k1 - 0.5f, f20 = (float)k2 - 0.5f;
        const float oa = a == 0 ? o[0] : (a == 1 ? o[1] : o[2]);
        const float o1 = t1 == 0 ? o[0] : (t1 == 1 ? o[1] : o[2]);
        const float o2 = t2 == 0 ? o[0] : (t2 == 1 ? o[1] : o[2]);
        float sw[2][3][3], sv[2][3][3];  // sums of w and of w * (velocity component or phase)
#pragma unroll
        for (int da = 0; da < 2; ++da)
#pragma unroll
            for (int d1 = 0; d1 < 3; ++d1)
#pragma unroll
                for (int d2 = 0; d2 < 3; ++d2) {
                    sw[da][d1][d2] = 0.f;
                    sv[da][d1][d2] = 0.f;
                }
        for (uint32_t i = i0; i < i1; ++i) {
            float val;
            if (qpass) {
                val = phase[pid[i]];
                if (val == 0.f) continue;
            } else {
                val = soa[(int64_t)(3 + a) * n + i];
            }
            const float qa = (soa[(int64_t)a * n + i] - oa) * invh;
            const float q1 = (soa[(int64_t)t1 * n + i] - o1) * invh;
            const float q2 = (soa[(int64_t)t2 * n + i] - o2) * invh;
            // Along a: faces ka and ka + 1.  Across: of the three face rows k - 1, k, k + 1 (centres at
            // k - 0.5, k + 0.5, k + 1.5 in cell units) a particle reaches the centre row k and the side
            // row on its own side of the cell centre; the third is more than one cell away, so its
            // weight is zero and it is skipped.  c is the offset from the centre row, 1 - |c| the
            // distance to the side row.
            const float dA = qa - fa0;
            const float A0 = dA * dA, A1 = (dA - 1.f) * (dA - 1.f);
            const float c1 = q1 - (f10 + 1.f), c2 = q2 - (f20 + 1.f);
            const float s1 = 1.f - fabsf(c1), s2 = 1.f - fabsf(c2);
            const float Bc = c1 * c1, Bs = s1 * s1, Cc = c2 * c2, Cs = s2 * s2;
            const bool lo1 = c1 < 0.f, lo2 = c2 < 0.f;
#pragma unroll
            for (int da = 0; da < 2; ++da) {
                const float A = da ? A1 : A0;
                const float omc = 1.f - (A + Bc), oms = 1.f - (A + Bs);
                float t = fmaxf(omc - Cc, 0.f);
                t = t * t * t;
                sw[da][1][1] += t;
                sv[da][1][1] += t * val;
                t = fmaxf(oms - Cc, 0.f);
                t = t * t * t;
                if (lo1) {
                    sw[da][0][1] += t;
                    sv[da][0][1] += t * val;
                } else {
                    sw[da][2][1] += t;
                    sv[da][2][1] += t * val;
                }
                t = fmaxf(omc - Cs, 0.f);
                t = t * t * t;
                if (lo2) {
                    sw[da][1][0] += t;
                    sv[da][1][0] += t * val;
                } else {
                    sw[da][1][2] += t;
                    sv[da][1][2] += t * val;
                }
                t = fmaxf(oms - Cs, 0.f);
                t = t * t * t;
                const int j1 = lo1 ? 0 : 2, j2 = lo2 ? 0 : 2;
#pragma unroll
                for (int e1 = 0; e1 < 3; e1 += 2)
#pragma unroll
                    for (int e2 = 0; e2 < 3; e2 += 2)
                        if (e1 == j1 && e2 == j2) {
                            sw[da][e1][e2] += t;
                            sv[da][e1][e2] += t * val;
                        }
            }
        }
        // faces fa in {ca, ca+1} along a, f1 in {c1-1, c1, c1+1} and f2 likewise across (tile rows -1..r)
        const int base = a * TA + ka + R1 * (k1 + R2 * k2);
#pragma unroll
        for (int da = 0; da < 2; ++da)
#pragma unroll
            for (int d1 = 0; d1 < 3; ++d1)
#pragma unroll
                for (int d2 = 0; d2 < 3; ++d2) {
                    const float mv = sw[da][d1][d2];
                    if (mv == 0.f) continue;
                    const int e = base + da + d1 * R1 + d2 * R1 * R2;
                    if (qpass) {
                        atomicAdd(&aqw[e], sv[da][d1][d2]);
                    } else {
                        atomicAdd(&amw[e], mv);
                        atomicAdd(&apw[e], sv[da][d1][d2]);
                    }
                }
    }
    // Coarser neighbours.  A coarser neighbour's lattice continues the lattice of half b's
    // resolution anchored at b's origin (every block spans the same length), so its faces within
    // reach of b's particles are entries of the coarse tile outside b.  One of b's cells lies inside
    // half of one coarse cell along every axis, so the faces its particles can reach in that lattice
    // are the same 2 x 2 x 2 for all of them: along a the faces below and above the coarse cell,
    // across it the two face rows on the cell's own side.  A task (kind, listed cell, slice) sums
    // their weights in registers as the own tasks do and adds the sums of the candidates that belong
    // to a coarser neighbour into the coarse tile.
    const int nco = ncoarse;
    const int ntask_c = NK * nco * nsl;
    const float invhc = 0.5f * invh;
    for (;;) {
        int tb = 0;
        if (lane == 0) tb = atomicAdd(&tctr[1], 32);
        tb = __shfl_sync(0xffffffffu, tb, 0);
        if (tb >= ntask_c) break;
        const int task = tb + lane;
        if (task >= ntask_c) continue;
        const int kind = task % NK;
        const int rem = task / NK;
        const bool qpass = PH && kind >= 3;
        const int a = qpass ? kind - 3 : kind;
        const int c = colist[rem % nco], sl = rem / nco;
        const uint32_t ca = cst[c], ce = cst[c + 1];
        if ((uint32_t)sl * slice >= ce - ca) continue;
        const uint32_t i0 = ca + (uint32_t)sl * slice;
        const uint32_t i1 = ce - i0 > slice ? i0 + slice : ce;
        const int t1 = a == 2 ? 0 : a + 1, t2 = a == 0 ? 2 : a - 1;
        const int cx = c % r, cy = (c / r) % r, cz = c / (r * r);
        const int ka = a == 0 ? cx : (a == 1 ? cy : cz);
        const int k1 = a == 0 ? cy : (a == 1 ? cz : cx);
        const int k2 = a == 0 ? cz : (a == 1 ? cx : cy);
        // candidates (ia + da, j1 + d1, j2 + d2): coarse face index along a, coarse cell rows across
        const int ia = ka >> 1, j1 = ((k1 + 1) >> 1) - 1, j2 = ((k2 + 1) >> 1) - 1;
        // the candidates that lie in a coarser neighbour; a face on a plane between two blocks
        // along a belongs to both
        uint32_t live = 0;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int fa = ia + (e >> 2), f1 = j1 + ((e >> 1) & 1), f2 = j2 + (e & 1);
            const int s1 = f1 < 0 ? -1 : (f1 >= rc ? 1 : 0), s2 = f2 < 0 ? -1 : (f2 >= rc ? 1 : 0);
            const int sa0 = fa == 0 ? -1 : 0, sa1 = fa == rc ? 1 : 0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int sa = q ? sa1 : sa0;
                int dxyz[3];
                dxyz[a] = sa;
                dxyz[t1] = s1;
                dxyz[t2] = s2;
                const int d = (dxyz[0] + 1) + 3 * (dxyz[1] + 1) + 9 * (dxyz[2] + 1);
                if ((sa | s1 | s2) != 0 && ((cmask >> d) & 1)) live |= 1u << e;
            }
        }
        if (!live) continue;
        const float oa = a == 0 ? o[0] : (a == 1 ? o[1] : o[2]);
        const float o1 = t1 == 0 ? o[0] : (t1 == 1 ? o[1] : o[2]);
        const float o2 = t2 == 0 ? o[0] : (t2 == 1 ? o[1] : o[2]);
        const float fa0 = (float)ia, f10 = (float)j1 + 0.5f, f20 = (float)j2 + 0.5f;
        float sw[8], sv[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            sw[e] = 0.f;
            sv[e] = 0.f;
        }
        for (uint32_t i = i0; i < i1; ++i) {
            float val;
            if (qpass) {
                val = phase[pid[i]];
                if (val == 0.f) continue;
            } else {
                val = soa[(int64_t)(3 + a) * n + i];
            }
            const float dA = (soa[(int64_t)a * n + i] - oa) * invhc - fa0;
            const float dB = (soa[(int64_t)t1 * n + i] - o1) * invhc - f10;
            const float dC = (soa[(int64_t)t2 * n + i] - o2) * invhc - f20;
            const float A[2] = {dA * dA, (dA - 1.f) * (dA - 1.f)};
            const float B[2] = {dB * dB, (dB - 1.f) * (dB - 1.f)};
            const float C[2] = {dC * dC, (dC - 1.f) * (dC - 1.f)};
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                float t = fmaxf(1.f - ((A[e >> 2] + B[(e >> 1) & 1]) + C[e & 1]), 0.f);
                t = t * t * t;
                sw[e] += t;
                sv[e] += t * val;
            }
        }
        const int Rc1 = rc + 1, Rc2 = rc + 2;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            if (!((live >> e) & 1) || sw[e] == 0.f) continue;
            const int ei = a * TAc + (ia + (e >> 2)) + Rc1 * ((j1 + ((e >> 1) & 1) + 1) + Rc2 * (j2 + (e & 1) + 1));
            if (qpass) {
                atomicAdd(&cqw[ei], sv[e]);
            } else {
                atomicAdd(&cmw[ei], sw[e]);
                atomicAdd(&cpw[ei], sv[e]);
            }
        }
    }
    // Finer neighbours: lanes of a warp take particles a 32nd of the range apart, and the
    // (particle, neighbour) pairs bound for a finer neighbour wait in a per-warp queue and run 32 at
    // a time, one pair per lane, with global atomics, instead of one divergent pass per neighbour
    // direction.  Blocks of up to 8^3 cells visit only the particles of cells near a side that faces
    // such a neighbour, and test only those directions.  The reach is one of the neighbour's cells:
    // half of one of b's cells (its faces across the side sit half a fine cell in; a map that is not
    // 2:1 graded sends a neighbour of a quarter of b's resolution here too, with a reach of four of
    // b's cells).  A cell qualifies for direction d when, on every axis d crosses, its particles can
    // lie within reach of that side; the half-cell margin covers the rounding between a particle's
    // key cell and its position in cell units.  A particle that the exact test drops by rounding has
    // weight (1 - d^2)^3 with d^2 within 1e-7 of 1.
    const int nn = listed ? nnear : 0;
    const uint32_t T = listed ? (xmask ? nl_pre[nn] : 0u) : p1 - p0;
    const uint32_t Ls = (T + 31) / 32;
    uint32_t* qv = xq_v + w * P2G_XQ;
    uint8_t* qd = xq_d + w * P2G_XQ;
    int qn = 0;
    for (uint32_t i = w; xmask && i < Ls; i += nw) {
        const uint32_t f = lane * Ls + i;
        const bool valid = f < T;
        uint32_t v = f, dirs = (uint32_t)xmask;
        if (valid && listed) {  // near cell k holding flat index f: nl_pre[k] <= f < nl_pre[k + 1]
            int lo = 0, hi = nn - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (nl_pre[mid] <= f) lo = mid;
                else hi = mid - 1;
            }
            v = cst[nl_cell[lo]] - p0 + (f - nl_pre[lo]);
            dirs = nl_mask[lo];
        }
        float q[3];
        if (valid) {
            const uint32_t sidx = p0 + v;
#pragma unroll
            for (int k = 0; k < 3; ++k) q[k] = (soa[(int64_t)k * n + sidx] - o[k]) * invh;
        }
        // queued neighbours within reach (half a cell for a finer one)
        uint32_t near = 0;
        if (valid) {
            for (uint32_t mm = dirs; mm; mm &= mm - 1) {
                const int d = __ffs(mm) - 1;
                const int dd[3] = {d % 3 - 1, (d / 3) % 3 - 1, d / 9 - 1};
                const float reach = (float)r / (float)nres[d];
                bool nr = true;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    nr = nr && (dd[k] == 0 || (dd[k] < 0 ? q[k] < reach : q[k] > (float)r - reach));
                if (nr) near |= 1u << d;
            }
        }
        // at most two pairs per lane per round keeps the queue within 31 + 64 entries
        while (__any_sync(0xffffffffu, near)) {
            const uint32_t b1 = near & (0u - near);
            const uint32_t r1 = near & ~b1;
            const uint32_t take = b1 | (r1 & (0u - r1));
            near &= ~take;
            const int cnt = __popc(take);
            int incl = cnt;
#pragma unroll
            for (int sh = 1; sh < 32; sh <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, sh);
                if (lane >= sh) incl += y;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            int slot = qn + incl - cnt;
            for (uint32_t mm = take; mm; mm &= mm - 1, ++slot) {
                qv[slot] = v;
                qd[slot] = (uint8_t)(__ffs(mm) - 1);
            }
            qn += total;
            __syncwarp();
            while (qn >= 32) {
                qn -= 32;
                p2g_cross_pair<PH>(xn, nres, qv[qn + lane], qd[qn + lane], p0, soa, n, acc, pid, phase);
                __syncwarp();
            }
        }
    }
    if (qn > 0 && lane < qn) p2g_cross_pair<PH>(xn, nres, qv[lane], qd[lane], p0, soa, n, acc, pid, phase);
    __syncthreads();
    if (priv) {
        for (int i = threadIdx.x; i < TW; i += blockDim.x) {
            float v = sm[i];
            for (int c = TW; c < ntile; c += TW) v += sm[c + i];
            sm[i] = v;
        }
        __syncthreads();
    }
    // flush: every nonzero entry of the own tile into each copy of its face held by a block of b's
    // resolution, and of the coarse tile into each copy held by a block of half b's resolution
    p2g_flush_tile<PH>(nres, noff, r, am, ap, aq, acc);
    if (cmask) p2g_flush_tile<PH>(nres, noff, rc, cm, cp, cq, acc);
}

constexpr int kOrderMaxBlocks = 8192;  // grids up to this many blocks take their blocks heaviest first
// The blocks in descending order of particle count, by buckets of equal floor(log2(count)) (empty
// and inactive blocks last), for the CTA order of the per-block particle kernels: CTAs start in
// launch order, so the heaviest blocks start first and the last wave holds light ones.  The order
// within a bucket follows the atomics (it has no effect on the results).
__global__ void __launch_bounds__(1024) k_block_order(LevelView L, const uint32_t* __restrict__ cs, int nb,
                                                      int* __restrict__ order) {
    constexpr int NBK = 33;
    __shared__ int hist[NBK], base[NBK];
    auto bucket = [&](int b) {
        const int r = L.res[b];
        if (!r) return 0;
        const uint32_t c0 = L.off[0][b];
        return 32 - __clz((int)(cs[c0 + (uint32_t)(r * r * r)] - cs[c0]));
    };
    if (threadIdx.x < NBK) hist[threadIdx.x] = 0;
    __syncthreads();
    for (int b = threadIdx.x; b < nb; b += blockDim.x) atomicAdd(&hist[bucket(b)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = NBK - 1; k >= 0; --k) {
            base[k] = acc;
            acc += hist[k];
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nb; b += blockDim.x) order[atomicAdd(&base[bucket(b)], 1)] = b;
}

// u = P / m where m > 1e-6, else 0 (normalizeVelocity, P2G.cuh:139-171), over the three axes
__global__ void k_p2g_normalize(const float* __restrict__ m0, const float* __restrict__ P0, float* u0, uint32_t n0,
                                const float* __restrict__ m1, const float* __restrict__ P1, float* u1, uint32_t n1,
                                const float* __restrict__ m2, const float* __restrict__ P2, float* u2, uint32_t n2) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const float *m, *P;
    float* u;
    if (i < n0) { m = m0; P = P0; u = u0; }
    else if ((i -= n0) < n1) { m = m1; P = P1; u = u1; }
    else if ((i -= n1) < n2) { m = m2; P = P2; u = u2; }
    else return;
    const float mv = m[i];
    u[i] = mv > 1e-6f ? P[i] / mv : 0.f;
}

// Two-phase faces: phi = Phi / m where m > 1e-6, else 0; beta = 1 / ((1 - phi) rho0 + phi rho1).
// PHASE_FIELD_* and BETA_COEFF_* (MSBG.cuh:21-29); the reference leaves this accumulation
// commented out (P2G.cuh:94-97).
__global__ void k_p2g_phase(const float* __restrict__ m0, const float* __restrict__ q0, float* phi0, float* beta0,
                            uint32_t n0, const float* __restrict__ m1, const float* __restrict__ q1, float* phi1,
                            float* beta1, uint32_t n1, const float* __restrict__ m2, const float* __restrict__ q2,
                            float* phi2, float* beta2, uint32_t n2, float rho0, float rho1) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const float *m, *q;
    float *phi, *beta;
    if (i < n0) { m = m0; q = q0; phi = phi0; beta = beta0; }
    else if ((i -= n0) < n1) { m = m1; q = q1; phi = phi1; beta = beta1; }
    else if ((i -= n1) < n2) { m = m2; q = q2; phi = phi2; beta = beta2; }
    else return;
    const float mv = m[i];
    const float f = mv > 1e-6f ? fminf(fmaxf(q[i] / mv, 0.f), 1.f) : 0.f;
    phi[i] = f;
    beta[i] = 1.f / ((1.f - f) * rho0 + f * rho1);
}

aw_status p2g_sorted(MsbgState& G, const float* soa, int64_t n, const uint32_t* cstart, float* u[3], float* m[3],
                     float* mom[3], float* cell_count, cudaStream_t s, const PhaseIn* ph) {
    FaceAcc acc;
    for (int a = 0; a < 3; ++a) {
        acc.Phi[a] = nullptr;
        if (ph) {
            AW_TRY(G.p2g_Phi[a].ensure(std::max<uint32_t>(G.tot[1 + a], 1)));
            acc.Phi[a] = G.p2g_Phi[a].p;
            if (G.tot[1 + a]) AW_CUDA(cudaMemsetAsync(acc.Phi[a], 0, G.tot[1 + a] * sizeof(float), s));
        }
        acc.m[a] = m[a];
        if (mom[a]) {
            acc.P[a] = mom[a];
        } else {
            AW_TRY(G.p2g_P[a].ensure(std::max<uint32_t>(G.tot[1 + a], 1)));
            acc.P[a] = G.p2g_P[a].p;
        }
        if (G.tot[1 + a]) {
            AW_CUDA(cudaMemsetAsync(acc.m[a], 0, G.tot[1 + a] * sizeof(float), s));
            AW_CUDA(cudaMemsetAsync(acc.P[a], 0, G.tot[1 + a] * sizeof(float), s));
        }
    }
    int maxres = 0, minres = 1 << 30;
    for (int r : G.h_res)
        if (r) {
            maxres = std::max(maxres, r);
            minres = std::min(minres, r);
        }
    AW_TRY(G.blk_busy.ensure(std::max(G.nb, 1)));
    // Heaviest blocks first, on grids of at most kOrderMaxBlocks blocks: dam_drop_128 (4096 blocks)
    // G2P 0.084 to 0.077 ms and advection 0.149 to 0.137 ms; on dam_drop2_256 (32768 blocks, many
    // more waves) the one-CTA ordering pass cost more than it saved (P2G 2.02 to 2.07 ms, G2P 0.441
    // to 0.457 ms).
    G.blk_order_on = n > 0 && G.nb <= kOrderMaxBlocks;
    if (G.blk_order_on) {
        AW_TRY(G.blk_order.ensure(std::max(G.nb, 1)));
        k_block_order<<<1, 1024, 0, s>>>(G.view0(), cstart, G.nb, G.blk_order.p);
        AW_LAUNCH();
    }
    // (G2P and the advection use it too; any order left from an earlier call is still a permutation of
    // the grid's blocks, so a kernel given one covers every block exactly once)
    const int* order = G.blk_order_on ? G.blk_order.p : nullptr;
    const int NVt = ph ? 9 : 6;
    // the largest tile, or one private tile per warp for blocks of at most two cells per edge
    // 512-thread CTAs: the aw_p2g call takes 0.43 ms on the 3-level dam_drop_128 against 0.48 ms
    // with 256.  A grid with one-cell blocks keeps 256: the tasks of such a block all add into one
    // tile of 18 faces per axis, and more threads on it contend more (the 4-level dam_drop2_256
    // takes 2.96 ms with 512 against 2.85 ms with 256).
    const int nthreads = minres >= 2 ? P2G_THREADS : 256;
    // own tile and coarse tile (half the resolution) of one block
    auto tiles = [&](int r) { return (size_t)NVt * (tile_axis(r) + (r >= 2 ? tile_axis(r / 2) : 0u)); };
    const size_t smem_f = std::max(tiles(maxres), minres <= 2 ? (size_t)(nthreads / 32) * tiles(std::min(maxres, 2)) : 0);
    // then the cell starts of the largest block
    const size_t smem = (smem_f + (((size_t)maxres * maxres * maxres + 1 + 3) & ~(size_t)3)) * sizeof(float);
    if (n > 0) {
        if (ph) {
            // always opted in: the pair queues' static shared memory counts against the default 48 KB too
            AW_CUDA(cudaFuncSetAttribute(k_p2g_own<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_p2g_own<true><<<G.nb, nthreads, smem, s>>>(G.view0(), soa, n, cstart, acc, ph->pid, ph->phase,
                                                           (int)smem_f, G.blk_busy.p, order);
        } else {
            AW_CUDA(cudaFuncSetAttribute(k_p2g_own<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_p2g_own<false><<<G.nb, nthreads, smem, s>>>(G.view0(), soa, n, cstart, acc, nullptr, nullptr,
                                                            (int)smem_f, G.blk_busy.p, order);
        }
        AW_LAUNCH();
    }
    const uint64_t nf = (uint64_t)G.tot[1] + G.tot[2] + G.tot[3];
    if (nf) {
        k_p2g_normalize<<<nblk(nf), 256, 0, s>>>(acc.m[0], acc.P[0], u[0], G.tot[1], acc.m[1], acc.P[1], u[1], G.tot[2],
                                                 acc.m[2], acc.P[2], u[2], G.tot[3]);
        AW_LAUNCH();
        if (ph) {
            k_p2g_phase<<<nblk(nf), 256, 0, s>>>(acc.m[0], acc.Phi[0], ph->phi[0], ph->beta[0], G.tot[1], acc.m[1],
                                                 acc.Phi[1], ph->phi[1], ph->beta[1], G.tot[2], acc.m[2], acc.Phi[2],
                                                 ph->phi[2], ph->beta[2], G.tot[3], ph->rho0, ph->rho1);
            AW_LAUNCH();
        }
    }
    if (cell_count) {
        k_cell_count<<<nblk(G.tot[0]), 256, 0, s>>>(cstart, G.tot[0], cell_count);
        AW_LAUNCH();
    }
    return AW_OK;
}

// ------------------------------------------------------------------------------------------------
// MAC sampling with the block-boundary ghost rule.  Tangential stencil indices outside the block
// read the nearest face of the same axis in the neighbouring block (integer index mapping, so the
// oracle reproduces every choice); outside the domain or in an inactive block the index is
// clamped back into the block.
// ------------------------------------------------------------------------------------------------
// Source face of a (possibly ghost) face index fi of block b: the face itself, the nearest face of the
// same axis in the neighbouring block, or (outside the domain / inactive neighbour) the clamped
// face of b.
__device__ inline uint32_t face_source(const LevelView& L, int a, int b, const int cb[3], int r, const int fi[3]) {
    const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
    const int o1 = fi[t1] < 0 ? -1 : (fi[t1] >= r ? 1 : 0);
    const int o2 = fi[t2] < 0 ? -1 : (fi[t2] >= r ? 1 : 0);
    if (!o1 && !o2) return L.off[1 + a][b] + fidx(a, fi[0], fi[1], fi[2], r);
    int nc[3] = {cb[0], cb[1], cb[2]};
    nc[t1] += o1;
    nc[t2] += o2;
    int rn = 0, n = 0;
    if (inside(L.g, nc)) {
        n = bidx(L.g, nc[0], nc[1], nc[2]);
        rn = L.res[n];
    }
    if (!rn) {
        int q[3] = {fi[0], fi[1], fi[2]};
        q[t1] = min(max(q[t1], 0), r - 1);
        q[t2] = min(max(q[t2], 0), r - 1);
        return L.off[1 + a][b] + fidx(a, q[0], q[1], q[2], r);
    }
    const int sh = __ffs(2 * r) - 1;
    int q[3];
    q[a] = (2 * fi[a] * rn + r) >> sh;
    const int rel1 = 2 * fi[t1] + 1 - o1 * 2 * r;
    const int rel2 = 2 * fi[t2] + 1 - o2 * 2 * r;
    q[t1] = min(max((rel1 * rn) >> sh, 0), rn - 1);
    q[t2] = min(max((rel2 * rn) >> sh, 0), rn - 1);
    return L.off[1 + a][n] + fidx(a, q[0], q[1], q[2], rn);
}

// face_source with the 27-neighbourhood (index (dx+1) + 3 (dy+1) + 9 (dz+1), 13 = the block
// itself) already in shared memory: resolution (0 = outside or inactive) and face offsets per axis
struct NbFaces {
    int r;
    uint32_t off[3];
};
__device__ inline uint32_t face_source_nb(const NbFaces* nbr, int a, int r, const int fi[3]) {
    const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
    const int o1 = fi[t1] < 0 ? -1 : (fi[t1] >= r ? 1 : 0);
    const int o2 = fi[t2] < 0 ? -1 : (fi[t2] >= r ? 1 : 0);
    if (!o1 && !o2) return nbr[13].off[a] + fidx(a, fi[0], fi[1], fi[2], r);
    int dd[3] = {0, 0, 0};
    dd[t1] = o1;
    dd[t2] = o2;
    const NbFaces& N = nbr[(dd[0] + 1) + 3 * (dd[1] + 1) + 9 * (dd[2] + 1)];
    const int rn = N.r;
    if (!rn) {
        int q[3] = {fi[0], fi[1], fi[2]};
        q[t1] = min(max(q[t1], 0), r - 1);
        q[t2] = min(max(q[t2], 0), r - 1);
        return nbr[13].off[a] + fidx(a, q[0], q[1], q[2], r);
    }
    const int sh = __ffs(2 * r) - 1;
    int q[3];
    q[a] = (2 * fi[a] * rn + r) >> sh;
    const int rel1 = 2 * fi[t1] + 1 - o1 * 2 * r;
    const int rel2 = 2 * fi[t2] + 1 - o2 * 2 * r;
    q[t1] = min(max((rel1 * rn) >> sh, 0), rn - 1);
    q[t2] = min(max((rel2 * rn) >> sh, 0), rn - 1);
    return N.off[a] + fidx(a, q[0], q[1], q[2], rn);
}

__device__ inline float face_value(const LevelView& L, const float* __restrict__ u, int a, int b, const int cb[3], int r,
                                   const int fi[3]) {
    return u[face_source(L, a, b, cb, r, fi)];
}

__device__ inline float sample_comp(const LevelView& L, const float* __restrict__ u, int a, const float X[3]) {
    int cb[3];
    point_block(L.g, X, cb);
    const int b = bidx(L.g, cb[0], cb[1], cb[2]);
    const int r = L.res[b];
    if (!r) return 0.f;
    const float h = fcell(L.g, r);
    int i0[3];
    float f[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float o = forigin(L.g, k, cb[k]);
        float s = (X[k] - o) / h;
        int lo = 0;
        if (k != a) {
            s -= 0.5f;
            lo = -1;
        }
        s = fminf(fmaxf(s, (float)lo), (float)r);
        int i = (int)floorf(s);
        i = min(max(i, lo), r - 1);
        i0[k] = i;
        f[k] = s - (float)i;
    }
    float acc = 0.f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                int fi[3] = {i0[0] + dx, i0[1] + dy, i0[2] + dz};
                float w = (dx ? f[0] : 1.f - f[0]) * (dy ? f[1] : 1.f - f[1]) * (dz ? f[2] : 1.f - f[2]);
                acc += w * face_value(L, u, a, b, cb, r, fi);
            }
    return acc;
}

struct Field3 {
    const float* c[3];
};

__global__ void k_g2p(LevelView L, PArr pos, PArrW vel, int64_t n, float alpha, Field3 un, Field3 uo) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float X[3] = {pos(i, 0), pos(i, 1), pos(i, 2)};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float vn = sample_comp(L, un.c[a], a, X);
        float vo = sample_comp(L, uo.c[a], a, X);
        float vp = vel(i, a);
        vel(i, a) = alpha * (vp + (vn - vo)) + (1.f - alpha) * vn;
    }
}

__global__ void k_sample(LevelView L, PArr pts, int64_t n, Field3 u, float* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float X[3] = {pts(i, 0), pts(i, 1), pts(i, 2)};
#pragma unroll
    for (int a = 0; a < 3; ++a) out[3 * i + a] = sample_comp(L, u.c[a], a, X);
}

__global__ void k_advect(LevelView L, PArrW pos, int64_t n, float dt, Field3 u) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Geo& g = L.g;
    const float h0 = g.bs / (float)g.R0;
    float x[3] = {pos(i, 0), pos(i, 1), pos(i, 2)};
    float k1[3], k2[3], k3[3], y[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) k1[a] = sample_comp(L, u.c[a], a, x);
#pragma unroll
    for (int a = 0; a < 3; ++a) y[a] = x[a] + 0.5f * dt * k1[a];
#pragma unroll
    for (int a = 0; a < 3; ++a) k2[a] = sample_comp(L, u.c[a], a, y);
#pragma unroll
    for (int a = 0; a < 3; ++a) y[a] = x[a] + 0.75f * dt * k2[a];
#pragma unroll
    for (int a = 0; a < 3; ++a) k3[a] = sample_comp(L, u.c[a], a, y);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float v = (2.f / 9.f) * k1[a] + (3.f / 9.f) * k2[a] + (4.f / 9.f) * k3[a];
        float lo = g.dmin[a] + 0.01f * h0;
        float hi = g.dmin[a] + (float)g.D[a] * g.bs - 0.01f * h0;
        pos(i, a) = fminf(fmaxf(x[a] + dt * v, lo), hi);
    }
}

// ------------------------------------------------------------------------------------------------
// Ghosted face tiles.  For every block and axis a the tile holds the faces [0,r] along a and
// [-1,r] along both tangential axes (ghost layer filled by face_value's neighbour rule), so a
// trilinear MAC sample anywhere in the block reads 8 tile entries and nothing else.  Layout per
// block: axis-major, entry (iA, i1, i2) at iA + (r+1) ((i1+1) + (r+2) (i2+1)); each block's
// tiles start on a 16-byte boundary so they can be staged with one TMA bulk copy.
// ------------------------------------------------------------------------------------------------

__global__ void k_build_tiles(LevelView L, Field3 u, const uint32_t* __restrict__ toff, float* __restrict__ tiles) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    int cb[3];
    bcoord(L.g, b, cb);
    const int R1 = r + 1, R2 = r + 2;
    const int TA = (int)tile_axis(r);
    float* out = tiles + toff[b];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        const float* ua = u.c[a];
        for (int rem = threadIdx.x; rem < TA; rem += blockDim.x) {
            int fi[3];
            fi[a] = rem % R1;
            fi[t1] = (rem / R1) % R2 - 1;
            fi[t2] = rem / (R1 * R2) - 1;
            out[a * TA + rem] = face_value(L, ua, a, b, cb, r, fi);
        }
    }
}

// Both ghosted tiles of G2P (u_new and u_old) in one pass: every entry's source face is located
// once and read from the two fields.
__global__ void k_build_tiles2(LevelView L, Field3 un, Field3 uo, const uint32_t* __restrict__ toff,
                               float* __restrict__ tn, float* __restrict__ to,
                               const unsigned long long* __restrict__ skip = nullptr) {
    if (skip && sort_reusable(skip, true)) return;  // the drop-in G2P took the sorted path
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    int cb[3];
    bcoord(L.g, b, cb);
    const int R1 = r + 1, R2 = r + 2;
    const int TA = (int)tile_axis(r);
    const uint32_t o = toff[b];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        for (int rem = threadIdx.x; rem < TA; rem += blockDim.x) {
            int fi[3];
            fi[a] = rem % R1;
            fi[t1] = (rem / R1) % R2 - 1;
            fi[t2] = rem / (R1 * R2) - 1;
            const uint32_t src = face_source(L, a, b, cb, r, fi);
            tn[o + a * TA + rem] = un.c[a][src];
            to[o + a * TA + rem] = uo.c[a][src];
        }
    }
}

// Trilinear sample of component a at X from the ghosted tiles (same stencil as sample_comp).
// invh = 1 / (the block's cell size), computed once per block by the caller
__device__ inline float tile_interp(const float* __restrict__ t, int a, int r, const float o[3], float invh,
                                   const float X[3]) {
    const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
    float sA = (X[a] - o[a]) * invh;
    float s1 = (X[t1] - o[t1]) * invh - 0.5f;
    float s2 = (X[t2] - o[t2]) * invh - 0.5f;
    sA = fminf(fmaxf(sA, 0.f), (float)r);
    s1 = fminf(fmaxf(s1, -1.f), (float)r);
    s2 = fminf(fmaxf(s2, -1.f), (float)r);
    const int iA = min(max((int)floorf(sA), 0), r - 1);
    const int i1 = min(max((int)floorf(s1), -1), r - 1);
    const int i2 = min(max((int)floorf(s2), -1), r - 1);
    const float fA = sA - (float)iA, f1 = s1 - (float)i1, f2 = s2 - (float)i2;
    const int R1 = r + 1, R2 = r + 2;
    const float* p = t + a * (int)tile_axis(r) + iA + R1 * ((i1 + 1) + R2 * (i2 + 1));
    const int s_1 = R1, s_2 = R1 * R2;
    const float c00 = p[0] + fA * (p[1] - p[0]);
    const float c10 = p[s_1] + fA * (p[s_1 + 1] - p[s_1]);
    const float c01 = p[s_2] + fA * (p[s_2 + 1] - p[s_2]);
    const float c11 = p[s_1 + s_2] + fA * (p[s_1 + s_2 + 1] - p[s_1 + s_2]);
    const float c0 = c00 + f1 * (c10 - c00);
    const float c1 = c01 + f1 * (c11 - c01);
    return c0 + f2 * (c1 - c0);
}

// The three components of tile_interp at one point, with the per-axis coordinates, floors and
// fractions computed once (the same operations as three calls of tile_interp).
__device__ __forceinline__ void tile_interp3(const float* __restrict__ t, int r, const float o[3], float invh,
                                             const float X[3], float out[3]) {
    const float rf = (float)r;
    int iU[3], iV[3];
    float fU[3], fV[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float u = (X[k] - o[k]) * invh;
        const float su = fminf(fmaxf(u, 0.f), rf);
        const float sv = fminf(fmaxf(u - 0.5f, -1.f), rf);
        iU[k] = min(max((int)floorf(su), 0), r - 1);
        iV[k] = min(max((int)floorf(sv), -1), r - 1);
        fU[k] = su - (float)iU[k];
        fV[k] = sv - (float)iV[k];
    }
    const int R1 = r + 1, R2 = r + 2, TA = (int)tile_axis(r);
    const int s_1 = R1, s_2 = R1 * R2;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        const float fA = fU[a], f1 = fV[t1], f2 = fV[t2];
        const float* p = t + a * TA + iU[a] + R1 * ((iV[t1] + 1) + R2 * (iV[t2] + 1));
        const float c00 = p[0] + fA * (p[1] - p[0]);
        const float c10 = p[s_1] + fA * (p[s_1 + 1] - p[s_1]);
        const float c01 = p[s_2] + fA * (p[s_2 + 1] - p[s_2]);
        const float c11 = p[s_1 + s_2] + fA * (p[s_1 + s_2 + 1] - p[s_1 + s_2]);
        const float c0 = c00 + f1 * (c10 - c00);
        const float c1 = c01 + f1 * (c11 - c01);
        out[a] = c0 + f2 * (c1 - c0);
    }
}

__device__ inline float sample_tiles(const LevelView& L, const uint32_t* __restrict__ toff, const float* __restrict__ tiles,
                                     int a, const float X[3]) {
    int cb[3];
    point_block(L.g, X, cb);
    const int b = bidx(L.g, cb[0], cb[1], cb[2]);
    const int r = L.res[b];
    if (!r) return 0.f;
    const float h = fcell(L.g, r);
    float o[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) o[k] = forigin(L.g, k, cb[k]);
    return tile_interp(tiles + toff[b], a, r, o, 1.f / h, X);
}

// ---- TMA bulk copies (cp.async.bulk, no multicast) and a bounded mbarrier wait ----------------
__device__ inline uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ inline void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ inline void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ inline void tma_bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ inline bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// true when phase `parity` completed; false (and the error flag set) after `polls` polls (2^20 polls,
// about a second, in production)
__device__ inline bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err, int polls = 1 << 20) {
    for (int it = 0; it < polls; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicExch(err, 1);
    return false;
}

// G2P on sorted particles, one CTA per block.
// - The ghosted tile of w = u_new - alpha u_old is built in shared memory from the face arrays (the
//   FLIP blend alpha (v + u_new - u_old) + (1 - alpha) u_new equals alpha v + I(w) because the
//   trilinear interpolation I is linear), and the u_new tile is written to `tn` for the advection
//   that follows.  Every active block writes its u_new tile, with particles or not.
// - The block's particles (a contiguous range of each SoA array) are staged in chunks of G2P_CHUNK
//   by TMA bulk copies (cp.async.bulk, no multicast), two chunks in flight, each behind an mbarrier
//   with a bounded wait.  A copy starts at the 16-byte boundary at or below the chunk's first
//   element and its size is rounded up to 16 bytes, so up to 3 floats past the end of the last array
//   are read: SoA buffers are allocated kSoaPad floats longer.
// - On a wait that runs out, the CTA waits (again bounded) for every copy it issued before it
//   returns, so that no copy lands in shared memory that another CTA may then own.
// arm_only (tests of the timeout path): chunk 0's barrier is armed but its copy is not issued, and
// the waits poll `polls` times.
// Drop-in mode (D.perm set): the particles are the sorted copy that aw_p2g made of the caller's AoS
// arrays; the new velocities go to the caller's array through the sort permutation, no u_new tile is
// written, and the kernel does nothing unless the caller's arrays still hash as they did then.
struct DropIn {
    const uint32_t* perm;            // sorted slot -> caller index (nullptr: FLIP-step SoA state)
    float* aos;                      // caller's AoS array, written through perm
    const unsigned long long* hash;  // {pos, vel} at sort time, {pos, vel} now
};
constexpr int G2P_THREADS = 256;
constexpr int G2P_TB = 4;  // tile entries whose loads a thread issues together
constexpr int G2P_CHUNK = 512;
constexpr int G2P_SLOT = G2P_CHUNK + 8;  // floats per staged array: chunk + alignment head and tail

__device__ inline void g2p_stage_chunk(const float* soa, int64_t n, uint32_t q0, uint32_t q1, float* slot,
                                       uint64_t* bar, bool issue) {
    uint32_t bytes[6];
    const float* src[6];
    uint32_t total = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float* g = soa + (int64_t)k * n + q0;
        const uint32_t head = (uint32_t)(((uintptr_t)g >> 2) & 3u);
        src[k] = g - head;
        bytes[k] = ((q1 - q0 + head) * 4u + 15u) & ~15u;
        total += bytes[k];
    }
    mbar_expect_tx(bar, total);
    if (issue)
#pragma unroll
        for (int k = 0; k < 6; ++k) tma_bulk_load(slot + k * G2P_SLOT, src[k], bytes[k], bar);
}

__global__ void __launch_bounds__(G2P_THREADS) k_g2p_fused(LevelView L, float* __restrict__ soa, int64_t n,
                                                           const uint32_t* __restrict__ cs, float alpha, Field3 un,
                                                           Field3 uo, const uint32_t* __restrict__ toff,
                                                           float* __restrict__ tn, int* err, int polls, int arm_only,
                                                           DropIn D, const uint8_t* __restrict__ occ,
                                                           uint8_t* __restrict__ tile_ok, int untiled,
                                                           const int* __restrict__ order) {
    extern __shared__ __align__(16) float sm[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ NbFaces nbr[27];
    const int b = order ? order[blockIdx.x] : (int)blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    if (D.perm && !sort_reusable(D.hash, true)) return;
    const uint32_t c0 = L.off[0][b];
    const uint32_t p0 = cs[c0], p1 = cs[c0 + (uint32_t)(r * r * r)];
    const uint32_t nchunk = (p1 - p0 + G2P_CHUNK - 1) / G2P_CHUNK;
    if (!tn && !nchunk) return;  // no particles and no u_new tile to write
    const uint32_t tb = tile_block(r);
    float* tw = sm;
    float* stage = sm + tb;  // tb is a multiple of 4 floats
    if (nchunk) {
        if (threadIdx.x == 0) {
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (uint32_t c = 0; c < 2 && c < nchunk; ++c) {
                const uint32_t q0 = p0 + c * G2P_CHUNK, q1 = min(p1, q0 + G2P_CHUNK);
                g2p_stage_chunk(soa, n, q0, q1, stage + c * 6 * G2P_SLOT, &bar[c], !(arm_only && c == 0));
            }
    }
    // ghosted tiles (the copies above are in flight meanwhile).  The 26 neighbours' resolutions
    // and face offsets are read once into shared memory; each thread then locates G2P_TB entries
    // and issues their loads together.
    int cb[3];
    bcoord(L.g, b, cb);
    int busy = 0;
    if (threadIdx.x < 27) {
        const int d = threadIdx.x;
        const int nc[3] = {cb[0] + d % 3 - 1, cb[1] + (d / 3) % 3 - 1, cb[2] + d / 9 - 1};
        const int nb = inside(L.g, nc) ? bidx(L.g, nc[0], nc[1], nc[2]) : -1;
        const int rn = nb >= 0 ? L.res[nb] : 0;
        nbr[d].r = rn;
#pragma unroll
        for (int k = 0; k < 3; ++k) nbr[d].off[k] = rn ? L.off[1 + k][nb] : 0u;
        busy = occ && nb >= 0 && occ[nb];
    }
    // No particle in this block or its 26 neighbours (occ, from this step's P2G): nothing here to
    // interpolate for, and a stage point of the advection reaches this block only from a particle more
    // than a block away; tile_ok[b] = 0 sends such a point to the face arrays instead of the tile.
    // (A block with particles of its own never returns here, so no bulk copy is left in flight.)
    if (!__syncthreads_or(busy) && occ) {
        if (threadIdx.x == 0) tile_ok[b] = 0;
        return;
    }
    if (tile_ok && threadIdx.x == 0) tile_ok[b] = untiled ? 0 : 1;
    {
        const int R1 = r + 1, R2 = r + 2;
        const int TA = (int)tile_axis(r);
        float* tno = tn ? tn + toff[b] : nullptr;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            const float* __restrict__ ua = un.c[a];
            const float* __restrict__ va = uo.c[a];
            for (int base = threadIdx.x; base < TA; base += G2P_TB * blockDim.x) {
                uint32_t src[G2P_TB];
#pragma unroll
                for (int k = 0; k < G2P_TB; ++k) {
                    const int rem = base + k * blockDim.x;
                    src[k] = 0;
                    if (rem < TA) {
                        int fi[3];
                        fi[a] = rem % R1;
                        fi[t1] = (rem / R1) % R2 - 1;
                        fi[t2] = rem / (R1 * R2) - 1;
                        src[k] = face_source_nb(nbr, a, r, fi);
                    }
                }
                float vn[G2P_TB], vo[G2P_TB];
#pragma unroll
                for (int k = 0; k < G2P_TB; ++k) {
                    const bool ok = base + k * (int)blockDim.x < TA;
                    vn[k] = ok ? ua[src[k]] : 0.f;
                    vo[k] = ok ? va[src[k]] : 0.f;
                }
#pragma unroll
                for (int k = 0; k < G2P_TB; ++k) {
                    const int rem = base + k * blockDim.x;
                    if (rem < TA) {
                        if (tno) tno[a * TA + rem] = vn[k];
                        tw[a * TA + rem] = vn[k] - alpha * vo[k];
                    }
                }
            }
        }
    }
    __syncthreads();
    if (!nchunk) return;
    const float invh = 1.f / fcell(L.g, r);
    float o[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) o[a] = forigin(L.g, a, cb[a]);
    for (uint32_t c = 0; c < nchunk; ++c) {
        const int sl = c & 1;
        const bool ok = mbar_wait_bounded(&bar[sl], (c >> 1) & 1u, err, polls);
        if (!__syncthreads_and(ok)) {
            // drain: the copies of chunks c and c + 1 may still be in flight
            if (threadIdx.x == 0)
                for (uint32_t k = c; k < c + 2 && k < nchunk; ++k)
                    if (!(arm_only && k == 0)) mbar_wait_bounded(&bar[k & 1], (k >> 1) & 1u, err, polls);
            __syncthreads();
            return;
        }
        const uint32_t q0 = p0 + c * G2P_CHUNK, q1 = min(p1, q0 + G2P_CHUNK);
        const float* slot = stage + sl * 6 * G2P_SLOT;
        uint32_t head[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) head[k] = (uint32_t)(((uintptr_t)(soa + (int64_t)k * n + q0) >> 2) & 3u);
        for (uint32_t j = threadIdx.x; j < q1 - q0; j += blockDim.x) {
            const float X[3] = {slot[head[0] + j], slot[G2P_SLOT + head[1] + j], slot[2 * G2P_SLOT + head[2] + j]};
            float vout[3];
            tile_interp3(tw, r, o, invh, X, vout);
#pragma unroll
            for (int a = 0; a < 3; ++a) vout[a] += alpha * slot[(3 + a) * G2P_SLOT + head[3 + a] + j];
            if (D.perm) {
                float* dst = D.aos + 3 * (size_t)D.perm[q0 + j];
#pragma unroll
                for (int a = 0; a < 3; ++a) dst[a] = vout[a];
            } else {
#pragma unroll
                for (int a = 0; a < 3; ++a) soa[(int64_t)(3 + a) * n + q0 + j] = vout[a];
            }
        }
        __syncthreads();  // slot sl is free again
        if (threadIdx.x == 0 && c + 2 < nchunk) {
            const uint32_t n0 = p0 + (c + 2) * G2P_CHUNK, n1 = min(p1, n0 + G2P_CHUNK);
            g2p_stage_chunk(soa, n, n0, n1, stage + sl * 6 * G2P_SLOT, &bar[sl], true);
        }
    }
}

// RK3 advection of the sorted particles of one block: the block's u_new tile is staged in shared
// memory by one bulk copy; stage points that leave the block sample the neighbour's tile in global
// memory (same arithmetic as sample_tiles).  The block holding a stage point is located once per
// point, not once per component.
struct PointTile {
    const float* t;  // tile of the block holding the point (nullptr: inactive block, velocity 0)
    int b;           // that block
    int r;
    float o[3];
    float invh;
};
__device__ inline PointTile point_tile(const LevelView& L, const int cb[3], int r, const float o[3], float invh,
                                       const float* __restrict__ tl, const uint32_t* __restrict__ toff,
                                       const float* __restrict__ tg, const float X[3]) {
    PointTile T;
    // A point farther than a margin from every side of block cb lies in cb for point_block as well:
    // its subtraction and division err by a few ulps of the coordinate, far below the margin of
    // 1e-4 block sizes plus 1e-6 of the coordinate's magnitude.  So the exact lookup, with its three
    // divisions, runs only near the sides.
    const float bs = L.g.bs;
    bool inner = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float m = 1e-4f * bs + 1e-6f * (fabsf(o[k]) + bs), d = X[k] - o[k];
        inner = inner && d > m && d < bs - m;
    }
    int pc[3] = {cb[0], cb[1], cb[2]};
    if (!inner) point_block(L.g, X, pc);
    if (pc[0] == cb[0] && pc[1] == cb[1] && pc[2] == cb[2]) {
        T.t = tl;
        T.b = -1;
        T.r = r;
#pragma unroll
        for (int k = 0; k < 3; ++k) T.o[k] = o[k];
        T.invh = invh;
        return T;
    }
    const int b2 = bidx(L.g, pc[0], pc[1], pc[2]);
    T.b = b2;
    T.r = L.res[b2];
    T.t = T.r ? tg + toff[b2] : nullptr;
    T.invh = T.r ? 1.f / fcell(L.g, T.r) : 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) T.o[k] = forigin(L.g, k, pc[k]);
    return T;
}

// The MAC sample of u_new at X from the face arrays, for the rare stage point that lands in a block
// whose tile G2P did not write (no particle within one block of it).  Measured against keeping this
// path out of line (a call, or a separate pass over a list of such particles): inlined, at 80
// registers, the advection runs fastest (0.148 against 0.154-0.161 ms on dam_drop_128).
__device__ __forceinline__ void sample_faces3(const LevelView& L, const Field3& un, const float X[3], float out[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) out[a] = sample_comp(L, un.c[a], a, X);
}

__global__ void __launch_bounds__(256) k_advect_tile(LevelView L, float* __restrict__ soa, int64_t n,
                                                     const uint32_t* __restrict__ cs, float dt,
                                                     const uint32_t* __restrict__ toff, const float* __restrict__ tn_g,
                                                     int* err, DropIn D, const uint8_t* __restrict__ tile_ok, Field3 un,
                                                     const int* __restrict__ order) {
    extern __shared__ __align__(16) float sm[];
    __shared__ __align__(8) uint64_t bar;
    const int b = order ? order[blockIdx.x] : (int)blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    if (D.perm && !sort_reusable(D.hash, false)) return;
    const uint32_t p0 = cs[L.off[0][b]], p1 = cs[L.off[0][b] + (uint32_t)(r * r * r)];
    if (p0 == p1) return;
    const uint32_t tb = tile_block(r);
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar, tb * sizeof(float));
        tma_bulk_load(sm, tn_g + toff[b], tb * sizeof(float), &bar);
    }
    const bool ok = mbar_wait_bounded(&bar, 0, err);
    if (!__syncthreads_and(ok)) {
        // the copy may still be in flight: wait for it (bounded) before the CTA gives up its memory
        if (threadIdx.x == 0) mbar_wait_bounded(&bar, 0, err);
        __syncthreads();
        return;
    }
    const Geo& g = L.g;
    int cb[3];
    bcoord(g, b, cb);
    const float h = fcell(g, r);
    const float invh = 1.f / h;
    float o[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) o[a] = forigin(g, a, cb[a]);
    const float h0 = g.bs / (float)g.R0;
    for (uint32_t i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
        float x[3], k1[3], k2[3], k3[3], y[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) x[a] = soa[(int64_t)a * n + i];
        tile_interp3(sm, r, o, invh, x, k1);
#pragma unroll
        for (int a = 0; a < 3; ++a) y[a] = x[a] + 0.5f * dt * k1[a];
        {
            const PointTile T = point_tile(L, cb, r, o, invh, sm, toff, tn_g, y);
            if (T.t == sm) {  // shared-memory loads when the point stays in the block
                tile_interp3(sm, r, o, invh, y, k2);
            } else if (T.t && tile_ok && !tile_ok[T.b]) {  // no tile written this step: the face arrays
                sample_faces3(L, un, y, k2);
            } else if (T.t) {
                tile_interp3(T.t, T.r, T.o, T.invh, y, k2);
            } else {
                k2[0] = k2[1] = k2[2] = 0.f;
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) y[a] = x[a] + 0.75f * dt * k2[a];
        {
            const PointTile T = point_tile(L, cb, r, o, invh, sm, toff, tn_g, y);
            if (T.t == sm) {  // shared-memory loads when the point stays in the block
                tile_interp3(sm, r, o, invh, y, k3);
            } else if (T.t && tile_ok && !tile_ok[T.b]) {  // no tile written this step: the face arrays
                sample_faces3(L, un, y, k3);
            } else if (T.t) {
                tile_interp3(T.t, T.r, T.o, T.invh, y, k3);
            } else {
                k3[0] = k3[1] = k3[2] = 0.f;
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float v = (2.f / 9.f) * k1[a] + (3.f / 9.f) * k2[a] + (4.f / 9.f) * k3[a];
            const float lo = g.dmin[a] + 0.01f * h0;
            const float hi = g.dmin[a] + (float)g.D[a] * g.bs - 0.01f * h0;
            const float xn = fminf(fmaxf(x[a] + dt * v, lo), hi);
            if (D.perm) D.aos[3 * (size_t)D.perm[i] + a] = xn;
            else soa[(int64_t)a * n + i] = xn;
        }
    }
}

// Drop-in mode, particles of inactive blocks (the last bucket of the sort): G2P samples zero velocity
// there (v = alpha v), RK3 leaves them in place up to the domain clamp.  Caller arrays, through the
// sort permutation; nothing is done unless the arrays still hash as when sorted.
__global__ void k_inactive_aos(Geo g, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ bucket,
                               float* aos, const unsigned long long* __restrict__ hash, int advect, float alpha) {
    if (!sort_reusable(hash, !advect)) return;
    const uint32_t p0 = bucket[0], p1 = bucket[1];
    const float h0 = g.bs / (float)g.R0;
    for (uint32_t j = p0 + blockIdx.x * blockDim.x + threadIdx.x; j < p1; j += gridDim.x * blockDim.x) {
        float* p = aos + 3 * (size_t)perm[j];
        for (int a = 0; a < 3; ++a) {
            if (advect) {
                const float lo = g.dmin[a] + 0.01f * h0;
                const float hi = g.dmin[a] + (float)g.D[a] * g.bs - 0.01f * h0;
                p[a] = fminf(fmaxf(p[a], lo), hi);
            } else {
                p[a] *= alpha;
            }
        }
    }
}

// particles of inactive blocks (the last bucket of the sort) sample zero velocity: v = alpha v
__global__ void k_g2p_inactive(float* soa, int64_t n, const uint32_t* __restrict__ bucket, float alpha) {
    const uint32_t p0 = bucket[0], p1 = bucket[1];
    for (uint32_t i = p0 + blockIdx.x * blockDim.x + threadIdx.x; i < p1; i += gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) soa[(int64_t)(3 + a) * n + i] *= alpha;
}

aw_status ensure_tiles(MsbgState& G) {
    if (G.tile_off.p && G.h_tile_off.size() == (size_t)G.nb) return AW_OK;
    G.h_tile_off.resize(G.nb);
    uint32_t acc = 0;
    for (int b = 0; b < G.nb; ++b) {
        G.h_tile_off[b] = acc;
        acc += tile_block(G.h_res[b]);
    }
    G.tile_tot = acc;
    AW_TRY(G.tile_off.ensure(G.nb));
    AW_CUDA(cudaMemcpy(G.tile_off.p, G.h_tile_off.data(), G.nb * sizeof(uint32_t), cudaMemcpyHostToDevice));
    AW_TRY(G.tiles_new.ensure(std::max<uint32_t>(acc, 4)));
    AW_TRY(G.tiles_old.ensure(std::max<uint32_t>(acc, 4)));
    AW_TRY(G.tile_ok.ensure(std::max(G.nb, 1)));
    AW_TRY(G.err.ensure(4));
    AW_CUDA(cudaMemset(G.err.p, 0, 4 * sizeof(int)));
    return AW_OK;
}

aw_status build_tiles(MsbgState& G, const float* u[3], float* tiles, cudaStream_t s) {
    AW_CHECK_ARG(G.tile_off.p && tiles, "tiles not allocated");
    Field3 f{{u[0], u[1], u[2]}};
    k_build_tiles<<<G.nb, 128, 0, s>>>(G.view0(), f, G.tile_off.p, tiles);
    AW_LAUNCH();
    return AW_OK;
}

// u_new into G.tiles_new and u_old into G.tiles_old, one launch
aw_status build_tiles2(MsbgState& G, const float* un[3], const float* uo[3], cudaStream_t s) {
    AW_CHECK_ARG(G.tile_off.p && G.tiles_new.p && G.tiles_old.p, "tiles not allocated");
    Field3 a{{un[0], un[1], un[2]}}, b{{uo[0], uo[1], uo[2]}};
    k_build_tiles2<<<G.nb, 128, 0, s>>>(G.view0(), a, b, G.tile_off.p, G.tiles_new.p, G.tiles_old.p);
    AW_LAUNCH();
    return AW_OK;
}

aw_status check_device_errors(MsbgState& G, cudaStream_t s) {
    if (!G.err.p) return AW_OK;
    int h[4];
    AW_CUDA(cudaMemcpyAsync(h, G.err.p, sizeof h, cudaMemcpyDeviceToHost, s));
    AW_CUDA(cudaStreamSynchronize(s));
    if (h[1]) {
        // reported once: the flag is cleared so that the next call starts clean
        AW_CUDA(cudaMemsetAsync(G.err.p, 0, 4 * sizeof(int), s));
        AW_CUDA(cudaStreamSynchronize(s));
        return set_error(AW_ERR_STATE, "TMA bulk-copy wait timed out in G2P / advection");
    }
    return AW_OK;
}

aw_status g2p_sorted(MsbgState& G, float* soa, int64_t n, const uint32_t* cs, float alpha, const float* un[3],
                     const float* uo[3], cudaStream_t s) {
    if (n <= 0) return AW_OK;
    AW_TRY(ensure_tiles(G));
    int maxres = 0;
    for (int r : G.h_res) maxres = std::max(maxres, r);
    const size_t smem = ((size_t)tile_block(maxres) + 2 * 6 * G2P_SLOT) * sizeof(float);
    AW_CUDA(cudaFuncSetAttribute(k_g2p_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    Field3 fa{{un[0], un[1], un[2]}}, fb{{uo[0], uo[1], uo[2]}};
    const int arm_only = G.test_copy_timeout ? 1 : 0;
    // AW_TEST_UNTILED (tests of the advection's fallback): every block's u_new tile is reported as not
    // written, so every RK3 stage point outside its own block samples the face arrays
    const int untiled = getenv("AW_TEST_UNTILED") != nullptr ? 1 : 0;
    const int polls = arm_only ? 1 << 10 : 1 << 20;
    G.test_copy_timeout = false;
    k_g2p_fused<<<G.nb, G2P_THREADS, smem, s>>>(G.view0(), soa, n, cs, alpha, fa, fb, G.tile_off.p, G.tiles_new.p,
                                                 G.err.p + 1, polls, arm_only, DropIn{nullptr, nullptr, nullptr}, G.blk_busy.p,
                                                 G.blk_busy.p ? G.tile_ok.p : nullptr, untiled,
                                                 G.blk_order_on ? G.blk_order.p : nullptr);
    AW_LAUNCH();
    k_g2p_inactive<<<16, 256, 0, s>>>(soa, n, cs + G.tot[0], alpha);
    AW_LAUNCH();
    return AW_OK;
}

__global__ void k_advect_tiles(LevelView L, PArrW pos, int64_t n, float dt, const uint32_t* __restrict__ toff,
                               const float* __restrict__ tiles,
                               const unsigned long long* __restrict__ skip = nullptr) {
    if (skip && sort_reusable(skip, false)) return;  // the drop-in advection took the sorted path
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Geo& g = L.g;
    const float h0 = g.bs / (float)g.R0;
    float x[3] = {pos(i, 0), pos(i, 1), pos(i, 2)};
    float k1[3], k2[3], k3[3], y[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) k1[a] = sample_tiles(L, toff, tiles, a, x);
#pragma unroll
    for (int a = 0; a < 3; ++a) y[a] = x[a] + 0.5f * dt * k1[a];
#pragma unroll
    for (int a = 0; a < 3; ++a) k2[a] = sample_tiles(L, toff, tiles, a, y);
#pragma unroll
    for (int a = 0; a < 3; ++a) y[a] = x[a] + 0.75f * dt * k2[a];
#pragma unroll
    for (int a = 0; a < 3; ++a) k3[a] = sample_tiles(L, toff, tiles, a, y);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float v = (2.f / 9.f) * k1[a] + (3.f / 9.f) * k2[a] + (4.f / 9.f) * k3[a];
        float lo = g.dmin[a] + 0.01f * h0;
        float hi = g.dmin[a] + (float)g.D[a] * g.bs - 0.01f * h0;
        pos(i, a) = fminf(fmaxf(x[a] + dt * v, lo), hi);
    }
}

// G2P / sampling on arbitrary (unsorted, AoS) particles through the ghosted tiles
__global__ void k_g2p_tiles(LevelView L, PArr pos, PArrW vel, int64_t n, float alpha, const uint32_t* __restrict__ toff,
                            const float* __restrict__ tn, const float* __restrict__ to,
                            const unsigned long long* __restrict__ skip = nullptr) {
    if (skip && sort_reusable(skip, true)) return;  // the drop-in G2P took the sorted path
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float X[3] = {pos(i, 0), pos(i, 1), pos(i, 2)};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float vn = sample_tiles(L, toff, tn, a, X);
        const float vo = sample_tiles(L, toff, to, a, X);
        const float vp = vel(i, a);
        vel(i, a) = alpha * (vp + (vn - vo)) + (1.f - alpha) * vn;
    }
}

__global__ void k_sample_tiles(LevelView L, PArr pts, int64_t n, const uint32_t* __restrict__ toff,
                               const float* __restrict__ tiles, float* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float X[3] = {pts(i, 0), pts(i, 1), pts(i, 2)};
#pragma unroll
    for (int a = 0; a < 3; ++a) out[3 * i + a] = sample_tiles(L, toff, tiles, a, X);
}

aw_status advect_sorted(MsbgState& G, float* soa, int64_t n, const uint32_t* cs, float dt, const float* un[3],
                        cudaStream_t s) {
    if (n <= 0) return AW_OK;
    int maxres = 0;
    for (int r : G.h_res) maxres = std::max(maxres, r);
    const size_t smem = (size_t)tile_block(maxres) * sizeof(float);
    if (smem > 48 * 1024)
        AW_CUDA(cudaFuncSetAttribute(k_advect_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_advect_tile<<<G.nb, 256, smem, s>>>(G.view0(), soa, n, cs, dt, G.tile_off.p, G.tiles_new.p, G.err.p + 1,
                                          DropIn{nullptr, nullptr, nullptr}, G.blk_busy.p ? G.tile_ok.p : nullptr,
                                          Field3{{un[0], un[1], un[2]}}, G.blk_order_on ? G.blk_order.p : nullptr);
    AW_LAUNCH();
    return AW_OK;
}

aw_status advect_tiles(MsbgState& G, float* pos, int pos_soa, int64_t n, float dt, const float* tiles, cudaStream_t s) {
    if (n <= 0) return AW_OK;
    PArrW P = pos_soa ? PArrW{pos, 1, n} : PArrW{pos, 3, 1};
    k_advect_tiles<<<nblk(n), 256, 0, s>>>(G.view0(), P, n, dt, G.tile_off.p, tiles);
    AW_LAUNCH();
    return AW_OK;
}

aw_status g2p_launch(MsbgState& G, const float* pos, int pos_soa, float* vel, int vel_soa, int64_t n, float alpha,
                     const float* un[3], const float* uo[3], cudaStream_t s) {
    if (n <= 0) return AW_OK;
    PArr P = pos_soa ? PArr{pos, 1, n} : PArr{pos, 3, 1};
    PArrW V = vel_soa ? PArrW{vel, 1, n} : PArrW{vel, 3, 1};
    Field3 a{{un[0], un[1], un[2]}}, b{{uo[0], uo[1], uo[2]}};
    k_g2p<<<nblk(n), 256, 0, s>>>(G.view0(), P, V, n, alpha, a, b);
    AW_LAUNCH();
    return AW_OK;
}

aw_status advect_launch(MsbgState& G, float* pos, int pos_soa, int64_t n, float dt, const float* u[3], cudaStream_t s) {
    if (n <= 0) return AW_OK;
    PArrW P = pos_soa ? PArrW{pos, 1, n} : PArrW{pos, 3, 1};
    Field3 f{{u[0], u[1], u[2]}};
    k_advect<<<nblk(n), 256, 0, s>>>(G.view0(), P, n, dt, f);
    AW_LAUNCH();
    return AW_OK;
}

// Exclusive scan of the per-block tile sizes in one CTA (same order and sums as the host-side
// offsets of the grid's own tiles).
__global__ void __launch_bounds__(1024) k_tile_offsets(const int* __restrict__ res, int nb, uint32_t* __restrict__ toff) {
    __shared__ uint32_t part[1024];
    const int per = (nb + (int)blockDim.x - 1) / (int)blockDim.x;
    const int b0 = (int)threadIdx.x * per, b1 = min(nb, b0 + per);
    uint32_t own = 0;
    for (int b = b0; b < b1; ++b) own += tile_block(res[b]);
    part[threadIdx.x] = own;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        const uint32_t v = (int)threadIdx.x >= o ? part[threadIdx.x - o] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t acc = part[threadIdx.x] - own;
    for (int b = b0; b < b1; ++b) {
        toff[b] = acc;
        acc += tile_block(res[b]);
    }
}

uint64_t tile_total(const std::vector<int>& h_res) {
    uint64_t acc = 0;
    for (int r : h_res) acc += tile_block(r);
    return acc;
}

aw_status g2p_with_tiles(MsbgState& G, float* d_vel, const float* d_pos, int64_t n, float alpha, uint32_t* toff,
                         float* tn, float* to, cudaStream_t s) {
    if (n <= 0) return AW_OK;
    k_tile_offsets<<<1, 1024, 0, s>>>(G.res.p, G.nb, toff);
    AW_LAUNCH();
    Field3 un{{G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]}};
    Field3 uo{{G.ch[AW_VELOCITY_OLD_X], G.ch[AW_VELOCITY_OLD_Y], G.ch[AW_VELOCITY_OLD_Z]}};
    k_build_tiles<<<G.nb, 128, 0, s>>>(G.view0(), un, toff, tn);
    AW_LAUNCH();
    k_build_tiles<<<G.nb, 128, 0, s>>>(G.view0(), uo, toff, to);
    AW_LAUNCH();
    k_g2p_tiles<<<nblk(n), 256, 0, s>>>(G.view0(), PArr{d_pos, 3, 1}, PArrW{d_vel, 3, 1}, n, alpha, toff, tn, to);
    AW_LAUNCH();
    return AW_OK;
}

// Loads the kernels g2p_with_tiles launches on the current device (CUDA loads kernels lazily, at
// their first launch), so that the first launch neither loads code nor takes device memory.
aw_status preload_g2p_with_tiles() {
    cudaFuncAttributes fa;
    AW_CUDA(cudaFuncGetAttributes(&fa, k_tile_offsets));
    AW_CUDA(cudaFuncGetAttributes(&fa, k_build_tiles));
    AW_CUDA(cudaFuncGetAttributes(&fa, k_g2p_tiles));
    return AW_OK;
}

// ================================================================================================
// Adjoint (vector-Jacobian products) of P2G, G2P, RK3 advection and MAC sampling.  No counterpart
// in the reference.  The forward map is differentiated with its discrete decisions held: the cell
// and block of every particle and sample point, each kernel's support, the clamp branches.
// ================================================================================================

// Trilinear tile sample of component a at X (tile_interp) with its adjoint: adds gbar * dI/dX to
// dX and, when tb is given, gbar * weight into the adjoint tile tb (same layout as t).
__device__ inline void tile_interp_vjp(const float* __restrict__ t, float* tb, int a, int r, const float o[3], float h,
                                       const float X[3], float gbar, float dX[3]) {
    const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
    const float rf = (float)r, invh = 1.f / h;
    float sA = (X[a] - o[a]) * invh;
    float s1 = (X[t1] - o[t1]) * invh - 0.5f;
    float s2 = (X[t2] - o[t2]) * invh - 0.5f;
    const float gA = (sA > 0.f && sA < rf) ? invh : 0.f;
    const float g1 = (s1 > -1.f && s1 < rf) ? invh : 0.f;
    const float g2 = (s2 > -1.f && s2 < rf) ? invh : 0.f;
    sA = fminf(fmaxf(sA, 0.f), rf);
    s1 = fminf(fmaxf(s1, -1.f), rf);
    s2 = fminf(fmaxf(s2, -1.f), rf);
    const int iA = min(max((int)floorf(sA), 0), r - 1);
    const int i1 = min(max((int)floorf(s1), -1), r - 1);
    const int i2 = min(max((int)floorf(s2), -1), r - 1);
    const float fA = sA - (float)iA, f1 = s1 - (float)i1, f2 = s2 - (float)i2;
    const int R1 = r + 1, R2 = r + 2;
    const int base = a * (int)tile_axis(r) + iA + R1 * ((i1 + 1) + R2 * (i2 + 1));
    const int s_1 = R1, s_2 = R1 * R2;
    const float* p = t + base;
    const float p000 = p[0], p100 = p[1], p010 = p[s_1], p110 = p[s_1 + 1];
    const float p001 = p[s_2], p101 = p[s_2 + 1], p011 = p[s_1 + s_2], p111 = p[s_1 + s_2 + 1];
    const float dfA = (1.f - f1) * (1.f - f2) * (p100 - p000) + f1 * (1.f - f2) * (p110 - p010) +
                      (1.f - f1) * f2 * (p101 - p001) + f1 * f2 * (p111 - p011);
    const float df1 = (1.f - f2) * ((1.f - fA) * (p010 - p000) + fA * (p110 - p100)) +
                      f2 * ((1.f - fA) * (p011 - p001) + fA * (p111 - p101));
    const float df2 = (1.f - f1) * ((1.f - fA) * (p001 - p000) + fA * (p101 - p100)) +
                      f1 * ((1.f - fA) * (p011 - p010) + fA * (p111 - p110));
    dX[a] += gbar * dfA * gA;
    dX[t1] += gbar * df1 * g1;
    dX[t2] += gbar * df2 * g2;
    if (tb && gbar != 0.f) {
        float* q = tb + base;
        const float wA[2] = {1.f - fA, fA}, w1[2] = {1.f - f1, f1}, w2[2] = {1.f - f2, f2};
#pragma unroll
        for (int k2 = 0; k2 < 2; ++k2)
#pragma unroll
            for (int k1 = 0; k1 < 2; ++k1)
#pragma unroll
                for (int kA = 0; kA < 2; ++kA) atomicAdd(q + kA + k1 * s_1 + k2 * s_2, gbar * wA[kA] * w1[k1] * w2[k2]);
    }
}

// sample_tiles with its adjoint (the block of X is found as in the forward)
__device__ inline void sample_tiles_vjp(const LevelView& L, const uint32_t* __restrict__ toff,
                                        const float* __restrict__ tiles, float* tb, int a, const float X[3], float gbar,
                                        float dX[3]) {
    int cb[3];
    point_block(L.g, X, cb);
    const int b = bidx(L.g, cb[0], cb[1], cb[2]);
    const int r = L.res[b];
    if (!r) return;
    const float h = fcell(L.g, r);
    float o[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) o[k] = forigin(L.g, k, cb[k]);
    tile_interp_vjp(tiles + toff[b], tb ? tb + toff[b] : nullptr, a, r, o, h, X, gbar, dX);
}

// Adjoint of one step's particle update: RK3 advection x' = RK3(x; u6) and the FLIP blend
// v' = alpha v + I(u6, x) - alpha I(uo, x).  xbar/vbar hold the adjoints of x', v' on entry and of
// x, v on exit; the adjoints of the u6 and uo tiles are accumulated into tnb / tob.
__global__ void k_step_particles_vjp(LevelView L, PArr pos, int64_t n, float alpha, float dt,
                                     const uint32_t* __restrict__ toff, const float* __restrict__ tn,
                                     const float* __restrict__ to, float* tnb, float* tob, PArrW xbar, PArrW vbar,
                                     int do_advect, int do_g2p) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Geo& g = L.g;
    const float x[3] = {pos(i, 0), pos(i, 1), pos(i, 2)};
    float gx[3] = {0.f, 0.f, 0.f};
    if (do_advect) {
        const float h0 = g.bs / (float)g.R0;
        float k1[3], k2[3], k3[3], y1[3], y2[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) k1[a] = sample_tiles(L, toff, tn, a, x);
#pragma unroll
        for (int a = 0; a < 3; ++a) y1[a] = x[a] + 0.5f * dt * k1[a];
#pragma unroll
        for (int a = 0; a < 3; ++a) k2[a] = sample_tiles(L, toff, tn, a, y1);
#pragma unroll
        for (int a = 0; a < 3; ++a) y2[a] = x[a] + 0.75f * dt * k2[a];
#pragma unroll
        for (int a = 0; a < 3; ++a) k3[a] = sample_tiles(L, toff, tn, a, y2);
        float k1b[3], k2b[3], k3b[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float v = (2.f / 9.f) * k1[a] + (3.f / 9.f) * k2[a] + (4.f / 9.f) * k3[a];
            const float lo = g.dmin[a] + 0.01f * h0;
            const float hi = g.dmin[a] + (float)g.D[a] * g.bs - 0.01f * h0;
            const float y = x[a] + dt * v;
            const float gb = (y > lo && y < hi) ? xbar(i, a) : 0.f;
            gx[a] = gb;
            k1b[a] = (2.f / 9.f) * dt * gb;
            k2b[a] = (3.f / 9.f) * dt * gb;
            k3b[a] = (4.f / 9.f) * dt * gb;
        }
        float y2b[3] = {0.f, 0.f, 0.f}, y1b[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int a = 0; a < 3; ++a) sample_tiles_vjp(L, toff, tn, tnb, a, y2, k3b[a], y2b);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            gx[a] += y2b[a];
            k2b[a] += 0.75f * dt * y2b[a];
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) sample_tiles_vjp(L, toff, tn, tnb, a, y1, k2b[a], y1b);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            gx[a] += y1b[a];
            k1b[a] += 0.5f * dt * y1b[a];
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) sample_tiles_vjp(L, toff, tn, tnb, a, x, k1b[a], gx);
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) gx[a] = xbar(i, a);
    }
    // FLIP blend
    if (do_g2p)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float gv = vbar(i, a);
            sample_tiles_vjp(L, toff, tn, tnb, a, x, gv, gx);
            sample_tiles_vjp(L, toff, to, tob, a, x, -alpha * gv, gx);
            vbar(i, a) = alpha * gv;
        }
#pragma unroll
    for (int a = 0; a < 3; ++a) xbar(i, a) = gx[a];
}

// Adjoint of y = sample(u, x): adds ybar * weights into the adjoint tile tb and, when xbar is
// given, ybar * dI/dx into xbar.
__global__ void k_sample_vjp(LevelView L, PArr pts, int64_t n, const uint32_t* __restrict__ toff,
                             const float* __restrict__ tiles, PArr ybar, float* tb, PArrW xbar, int with_x) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x[3] = {pts(i, 0), pts(i, 1), pts(i, 2)};
    float gx[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < 3; ++a) sample_tiles_vjp(L, toff, tiles, tb, a, x, ybar(i, a), gx);
    if (with_x)
#pragma unroll
        for (int a = 0; a < 3; ++a) xbar(i, a) += gx[a];
}

// Adjoint tile -> face adjoints: every tile entry adds into the face that supplied it.
__global__ void k_tile_fold(LevelView L, const uint32_t* __restrict__ toff, const float* __restrict__ tb, float* u0,
                            float* u1, float* u2) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    int cb[3];
    bcoord(L.g, b, cb);
    const int R1 = r + 1, R2 = r + 2;
    const int TA = (int)tile_axis(r);
    const float* in = tb + toff[b];
    float* U[3] = {u0, u1, u2};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        for (int rem = threadIdx.x; rem < TA; rem += blockDim.x) {
            const float v = in[a * TA + rem];
            if (v == 0.f) continue;
            int fi[3];
            fi[a] = rem % R1;
            fi[t1] = (rem / R1) % R2 - 1;
            fi[t2] = rem / (R1 * R2) - 1;
            atomicAdd(&U[a][face_source(L, a, b, cb, r, fi)], v);
        }
    }
}

// Adjoint of P2G with the normalisation u = P / m (m > 1e-6): each particle gathers, from every
// face within one cell size (of the face's block) of it, in its own and the 26 neighbouring
// blocks, P_bar = u_bar / m and m_bar = -u_bar u / m, and accumulates
//   vbar_a += w P_bar,   xbar += dw/dx (P_bar v_a + m_bar),   w = (1 - d^2/h^2)^3.
__global__ void k_p2g_vjp(LevelView L, PArr pos, PArr vel, int64_t n, Field3 u, Field3 m, Field3 ub, PArrW xbar,
                          PArrW vbar) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Geo& g = L.g;
    const float X[3] = {pos(i, 0), pos(i, 1), pos(i, 2)};
    const float V[3] = {vel(i, 0), vel(i, 1), vel(i, 2)};
    int pc[3];
    point_block(g, X, pc);
    float xb[3] = {0.f, 0.f, 0.f}, vb[3] = {0.f, 0.f, 0.f};
    for (int d = 0; d < 27; ++d) {
        const int nc[3] = {pc[0] + d % 3 - 1, pc[1] + (d / 3) % 3 - 1, pc[2] + d / 9 - 1};
        if (!inside(g, nc)) continue;
        const int b = bidx(g, nc[0], nc[1], nc[2]);
        const int r = L.res[b];
        if (!r) continue;
        const float h = fcell(g, r);
        const float invh = 1.f / h;
        float q[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) q[k] = (X[k] - forigin(g, k, nc[k])) * invh;
        const float rf = (float)r;
        if (q[0] <= -1.f || q[1] <= -1.f || q[2] <= -1.f || q[0] >= rf + 1.f || q[1] >= rf + 1.f || q[2] >= rf + 1.f)
            continue;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            const int ia = (int)floorf(q[a]);
            const int j1 = (int)floorf(q[t1] - 0.5f), j2 = (int)floorf(q[t2] - 0.5f);
            const uint32_t ob = L.off[1 + a][b];
            for (int da = 0; da < 2; ++da)
                for (int d1 = 0; d1 < 2; ++d1)
                    for (int d2 = 0; d2 < 2; ++d2) {
                        int f[3];
                        f[a] = ia + da;
                        f[t1] = j1 + d1;
                        f[t2] = j2 + d2;
                        if (f[a] < 0 || f[a] > r || f[t1] < 0 || f[t1] >= r || f[t2] < 0 || f[t2] >= r) continue;
                        float dq[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k) dq[k] = q[k] - ((float)f[k] + (k == a ? 0.f : 0.5f));
                        const float d2s = dq[0] * dq[0] + dq[1] * dq[1] + dq[2] * dq[2];
                        if (d2s >= 1.f) continue;
                        const uint32_t fi = ob + fidx(a, f[0], f[1], f[2], r);
                        const float mf = m.c[a][fi];
                        if (!(mf > 1e-6f)) continue;
                        const float gb = ub.c[a][fi];
                        if (gb == 0.f) continue;
                        const float Pbar = gb / mf;
                        const float mbar = -gb * u.c[a][fi] / mf;
                        const float t = 1.f - d2s;
                        vb[a] += t * t * t * Pbar;
                        const float coef = -6.f * t * t * invh * (Pbar * V[a] + mbar);
#pragma unroll
                        for (int k = 0; k < 3; ++k) xb[k] += coef * dq[k];
                    }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        xbar(i, k) += xb[k];
        vbar(i, k) += vb[k];
    }
}

// out[perm[j]] = in[j] for the 6 SoA arrays (adjoint of the gather of the sort)
__global__ void k_unsort6(const uint32_t* __restrict__ perm, int64_t n, const float* __restrict__ in, float* __restrict__ out) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = perm[j];
#pragma unroll
    for (int k = 0; k < 6; ++k) out[(int64_t)k * n + i] = in[(int64_t)k * n + j];
}

aw_status ensure_adjoint_tiles(MsbgState& G) {
    AW_TRY(ensure_tiles(G));
    AW_TRY(G.tiles_bar_new.ensure(std::max<uint32_t>(G.tile_tot, 4)));
    AW_TRY(G.tiles_bar_old.ensure(std::max<uint32_t>(G.tile_tot, 4)));
    return AW_OK;
}

aw_status tile_fold(MsbgState& G, const float* tb, float* ubar[3], cudaStream_t s) {
    k_tile_fold<<<G.nb, 128, 0, s>>>(G.view0(), G.tile_off.p, tb, ubar[0], ubar[1], ubar[2]);
    AW_LAUNCH();
    return AW_OK;
}

aw_status step_particles_vjp(MsbgState& G, const float* pos, int pos_soa, int64_t n, float alpha, float dt,
                             const float* un[3], const float* uo[3], float* xbar, float* vbar, int bar_soa,
                             int do_advect, float* unbar[3], float* uobar[3], cudaStream_t s) {
    if (n <= 0) return AW_OK;
    AW_TRY(ensure_adjoint_tiles(G));
    const int do_g2p = vbar != nullptr;
    if (do_g2p) AW_TRY(build_tiles2(G, un, uo, s));
    else AW_TRY(build_tiles(G, un, G.tiles_new.p, s));
    AW_CUDA(cudaMemsetAsync(G.tiles_bar_new.p, 0, (size_t)G.tile_tot * sizeof(float), s));
    AW_CUDA(cudaMemsetAsync(G.tiles_bar_old.p, 0, (size_t)G.tile_tot * sizeof(float), s));
    PArr P = pos_soa ? PArr{pos, 1, n} : PArr{pos, 3, 1};
    PArrW XB = bar_soa ? PArrW{xbar, 1, n} : PArrW{xbar, 3, 1};
    PArrW VB = bar_soa ? PArrW{vbar, 1, n} : PArrW{vbar, 3, 1};
    k_step_particles_vjp<<<nblk(n), 256, 0, s>>>(G.view0(), P, n, alpha, dt, G.tile_off.p, G.tiles_new.p, G.tiles_old.p,
                                                 G.tiles_bar_new.p, G.tiles_bar_old.p, XB, VB, do_advect, do_g2p);
    AW_LAUNCH();
    AW_TRY(tile_fold(G, G.tiles_bar_new.p, unbar, s));
    if (uobar && do_g2p) AW_TRY(tile_fold(G, G.tiles_bar_old.p, uobar, s));
    return AW_OK;
}

__global__ void k_sample_tiles_w(LevelView L, PArr pts, int64_t n, const uint32_t* __restrict__ toff,
                                 const float* __restrict__ tiles, PArrW out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float X[3] = {pts(i, 0), pts(i, 1), pts(i, 2)};
#pragma unroll
    for (int a = 0; a < 3; ++a) out(i, a) = sample_tiles(L, toff, tiles, a, X);
}

aw_status sample_soa(MsbgState& G, const float* pts_soa, int64_t n, const float* u[3], float* out_soa, cudaStream_t s) {
    if (n <= 0) return AW_OK;
    AW_TRY(ensure_tiles(G));
    AW_TRY(build_tiles(G, u, G.tiles_new.p, s));
    k_sample_tiles_w<<<nblk(n), 256, 0, s>>>(G.view0(), PArr{pts_soa, 1, n}, n, G.tile_off.p, G.tiles_new.p,
                                             PArrW{out_soa, 1, n});
    AW_LAUNCH();
    return AW_OK;
}

aw_status sample_vjp(MsbgState& G, const float* pts, int pts_soa, int64_t n, const float* u[3], const float* ybar,
                     int ybar_soa, float* ubar[3], float* xbar, cudaStream_t s) {
    if (n <= 0) return AW_OK;
    AW_TRY(ensure_adjoint_tiles(G));
    AW_TRY(build_tiles(G, u, G.tiles_new.p, s));
    AW_CUDA(cudaMemsetAsync(G.tiles_bar_new.p, 0, (size_t)G.tile_tot * sizeof(float), s));
    PArr P = pts_soa ? PArr{pts, 1, n} : PArr{pts, 3, 1};
    PArr Y = ybar_soa ? PArr{ybar, 1, n} : PArr{ybar, 3, 1};
    PArrW XB = pts_soa ? PArrW{xbar, 1, n} : PArrW{xbar, 3, 1};
    k_sample_vjp<<<nblk(n), 256, 0, s>>>(G.view0(), P, n, G.tile_off.p, G.tiles_new.p, Y, G.tiles_bar_new.p, XB,
                                         xbar ? 1 : 0);
    AW_LAUNCH();
    return tile_fold(G, G.tiles_bar_new.p, ubar, s);
}

aw_status p2g_vjp(MsbgState& G, const float* pos, const float* vel, int soa, int64_t n, const float* u[3],
                  const float* m[3], const float* ubar[3], float* xbar, float* vbar, cudaStream_t s) {
    if (n <= 0) return AW_OK;
    PArr P = soa ? PArr{pos, 1, n} : PArr{pos, 3, 1};
    PArr V = soa ? PArr{vel, 1, n} : PArr{vel, 3, 1};
    PArrW XB = soa ? PArrW{xbar, 1, n} : PArrW{xbar, 3, 1};
    PArrW VB = soa ? PArrW{vbar, 1, n} : PArrW{vbar, 3, 1};
    Field3 fu{{u[0], u[1], u[2]}}, fm{{m[0], m[1], m[2]}}, fb{{ubar[0], ubar[1], ubar[2]}};
    k_p2g_vjp<<<nblk(n, 128), 128, 0, s>>>(G.view0(), P, V, n, fu, fm, fb, XB, VB);
    AW_LAUNCH();
    return AW_OK;
}

aw_status unsort6(const uint32_t* perm, int64_t n, const float* in, float* out, cudaStream_t s) {
    if (n <= 0) return AW_OK;
    k_unsort6<<<nblk(n), 256, 0, s>>>(perm, n, in, out);
    AW_LAUNCH();
    return AW_OK;
}

}  // namespace aw

using namespace aw;

// ================================================================================================
// C ABI
// ================================================================================================
extern "C" aw_status aw_sort_particles(aw_msbg* g, const float* d_pos, int64_t n, uint32_t* d_keys, uint32_t* d_perm,
                                       aw_stream s_) {
    AW_CHECK_ARG(g && (d_pos || n == 0) && n >= 0 && n < (int64_t)0xFFFFFFFF, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    cudaStream_t s = (cudaStream_t)s_;
    MsbgState& G = g->st;
    PArr pos{d_pos, 3, 1};
    AW_TRY(sort_core(G, pos, n, s));
    if (n > 0 && (d_keys || d_perm)) {
        if (d_perm)
            AW_CUDA(cudaMemcpyAsync(d_perm, G.pw.sorted, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        if (d_keys) {
            k_gather<<<nblk(n), 256, 0, s>>>(G.pw.sorted, n, pos, PArr{nullptr, 3, 1}, G.pw.soa.p, nullptr, nullptr,
                                             G.pw.keys.p, d_keys);
            AW_LAUNCH();
        }
    }
    return AW_OK;
}

extern "C" aw_status aw_p2g(aw_msbg* g, const float* d_pos, const float* d_vel, int64_t n, aw_stream s_) {
    AW_CHECK_ARG(g && ((d_pos && d_vel) || n == 0) && n >= 0 && n < (int64_t)0xFFFFFFFF, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    cudaStream_t s = (cudaStream_t)s_;
    MsbgState& G = g->st;
    AW_TRY(sort_particles_soa(G, d_pos, d_vel, n, s, /*record=*/true));
    float* u[3] = {G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]};
    float* m[3] = {G.ch[AW_MASS_DENSITY_X], G.ch[AW_MASS_DENSITY_Y], G.ch[AW_MASS_DENSITY_Z]};
    float* mo[3] = {G.ch[AW_MOMENTUM_X], G.ch[AW_MOMENTUM_Y], G.ch[AW_MOMENTUM_Z]};
    return p2g_sorted(G, G.pw.soa.p, n, G.pw.cell_start.p, u, m, mo, G.ch[AW_CELL_TYPE], s);
}

extern "C" aw_status aw_p2g_phase(aw_msbg* g, const float* d_pos, const float* d_vel, const float* d_phase, int64_t n,
                                  float rho0, float rho1, aw_stream s_) {
    AW_CHECK_ARG(g && ((d_pos && d_vel && d_phase) || n == 0) && n >= 0 && n < (int64_t)0xFFFFFFFF, "bad argument");
    AW_CHECK_ARG(std::isfinite(rho0) && std::isfinite(rho1) && rho0 > 0.f && rho1 > 0.f, "densities must be positive");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    cudaStream_t s = (cudaStream_t)s_;
    MsbgState& G = g->st;
    AW_TRY(sort_particles_soa(G, d_pos, d_vel, n, s, /*record=*/true));
    float* u[3] = {G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]};
    float* m[3] = {G.ch[AW_MASS_DENSITY_X], G.ch[AW_MASS_DENSITY_Y], G.ch[AW_MASS_DENSITY_Z]};
    float* mo[3] = {G.ch[AW_MOMENTUM_X], G.ch[AW_MOMENTUM_Y], G.ch[AW_MOMENTUM_Z]};
    PhaseIn ph{};
    ph.pid = G.pw.sorted;
    ph.phase = d_phase;
    ph.rho0 = rho0;
    ph.rho1 = rho1;
    for (int a = 0; a < 3; ++a) {
        ph.phi[a] = G.ch[AW_PHASE_FIELD_X + a];
        ph.beta[a] = G.ch[AW_BETA_COEFF_X + a];
    }
    AW_TRY(p2g_sorted(G, G.pw.soa.p, n, G.pw.cell_start.p, u, m, mo, G.ch[AW_CELL_TYPE], s, &ph));
    return beta_sync(G, ph.beta, s);
}

extern "C" aw_status aw_test_arm_copy_timeout(aw_msbg* g) {
    AW_CHECK_ARG(g, "null grid");
    g->st.test_copy_timeout = true;
    return AW_OK;
}

extern "C" aw_status aw_backup_grid_velocity(aw_msbg* g, aw_stream s_) {
    AW_CHECK_ARG(g && g->st.allocated, "grid not allocated");
    MsbgState& G = g->st;
    for (int a = 0; a < 3; ++a)
        AW_CUDA(cudaMemcpyAsync(G.ch[AW_VELOCITY_OLD_X + a], G.ch[AW_VELOCITY_X + a], G.tot[1 + a] * sizeof(float),
                                cudaMemcpyDeviceToDevice, (cudaStream_t)s_));
    return AW_OK;
}

// Drop-in G2P and RK3 on the caller's AoS arrays (G2PManager::performG2P / advect,
// G2P.cuh:198-227).  When the arrays are the ones the last aw_p2g sorted and still hold the same
// contents (64-bit content hashes compared on the device), the block-sorted kernels run on the
// sorted copy aw_p2g made and write the caller's arrays through the sort permutation: G2P builds
// its tile in shared memory and stages the particles by TMA bulk copies.  Otherwise, or for any other
// arrays, the general path samples ghosted tiles in global memory particle by particle.  Both paths
// are launched; the device picks one, so no host synchronisation is needed.
extern "C" aw_status aw_g2p(aw_msbg* g, float* d_vel, const float* d_pos, int64_t n, float alpha, aw_stream s_) {
    AW_CHECK_ARG(g && ((d_pos && d_vel) || n == 0) && n >= 0, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    MsbgState& G = g->st;
    ParticleWork& W = G.pw;
    const float* un[3] = {G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]};
    const float* uo[3] = {G.ch[AW_VELOCITY_OLD_X], G.ch[AW_VELOCITY_OLD_Y], G.ch[AW_VELOCITY_OLD_Z]};
    if (n == 0) return AW_OK;
    cudaStream_t s = (cudaStream_t)s_;
    AW_TRY(ensure_tiles(G));
    const unsigned long long* skip = nullptr;
    if (W.src_valid && W.src_pos == d_pos && W.src_vel == d_vel && W.src_n == n) {
        AW_CUDA(cudaMemsetAsync(W.hash.p + 4, 0, 2 * kHashSlots * sizeof(unsigned long long), s));
        k_hash_aos<<<4 * 148, 256, 0, s>>>(d_pos, d_vel, n, W.hash.p + 4);
        AW_LAUNCH();
        k_hash_fold<<<1, 32, 0, s>>>(W.hash.p + 4, W.hash.p + 2);
        AW_LAUNCH();
        int maxres = 0;
        for (int r : G.h_res) maxres = std::max(maxres, r);
        const size_t smem = ((size_t)tile_block(maxres) + 2 * 6 * G2P_SLOT) * sizeof(float);
        AW_CUDA(cudaFuncSetAttribute(k_g2p_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        Field3 fa{{un[0], un[1], un[2]}}, fb{{uo[0], uo[1], uo[2]}};
        k_g2p_fused<<<G.nb, G2P_THREADS, smem, s>>>(G.view0(), W.soa.p, n, W.cell_start.p, alpha, fa, fb, G.tile_off.p,
                                                     nullptr, G.err.p + 1, 1 << 20, 0, DropIn{W.sorted, d_vel, W.hash.p},
                                                     nullptr, nullptr, 0, G.blk_order_on ? G.blk_order.p : nullptr);
        AW_LAUNCH();
        k_inactive_aos<<<16, 256, 0, s>>>(G.geo, W.sorted, W.cell_start.p + G.tot[0], d_vel, W.hash.p, 0, alpha);
        AW_LAUNCH();
        skip = W.hash.p;
    }
    Field3 a{{un[0], un[1], un[2]}}, b{{uo[0], uo[1], uo[2]}};
    k_build_tiles2<<<G.nb, 128, 0, s>>>(G.view0(), a, b, G.tile_off.p, G.tiles_new.p, G.tiles_old.p, skip);
    AW_LAUNCH();
    k_g2p_tiles<<<nblk(n), 256, 0, s>>>(G.view0(), PArr{d_pos, 3, 1}, PArrW{d_vel, 3, 1}, n, alpha, G.tile_off.p,
                                        G.tiles_new.p, G.tiles_old.p, skip);
    AW_LAUNCH();
    return AW_OK;
}

extern "C" aw_status aw_advect(aw_msbg* g, float* d_pos, int64_t n, float dt, aw_stream s_) {
    AW_CHECK_ARG(g && (d_pos || n == 0) && n >= 0, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    MsbgState& G = g->st;
    ParticleWork& W = G.pw;
    const float* u[3] = {G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]};
    if (n == 0) return AW_OK;
    cudaStream_t s = (cudaStream_t)s_;
    AW_TRY(ensure_tiles(G));
    AW_TRY(build_tiles(G, u, G.tiles_new.p, s));  // both paths sample neighbouring blocks' u_new tiles
    const unsigned long long* skip = nullptr;
    if (W.src_valid && W.src_pos == d_pos && W.src_n == n) {
        AW_CUDA(cudaMemsetAsync(W.hash.p + 4, 0, 2 * kHashSlots * sizeof(unsigned long long), s));
        k_hash_aos<<<4 * 148, 256, 0, s>>>(d_pos, nullptr, n, W.hash.p + 4);
        AW_LAUNCH();
        k_hash_fold<<<1, 32, 0, s>>>(W.hash.p + 4, W.hash.p + 2);
        AW_LAUNCH();
        int maxres = 0;
        for (int r : G.h_res) maxres = std::max(maxres, r);
        const size_t smem = (size_t)tile_block(maxres) * sizeof(float);
        AW_CUDA(cudaFuncSetAttribute(k_advect_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_advect_tile<<<G.nb, 256, smem, s>>>(G.view0(), W.soa.p, n, W.cell_start.p, dt, G.tile_off.p, G.tiles_new.p,
                                              G.err.p + 1, DropIn{W.sorted, d_pos, W.hash.p}, nullptr, Field3{},
                                              G.blk_order_on ? G.blk_order.p : nullptr);
        AW_LAUNCH();
        k_inactive_aos<<<16, 256, 0, s>>>(G.geo, W.sorted, W.cell_start.p + G.tot[0], d_pos, W.hash.p, 1, 0.f);
        AW_LAUNCH();
        skip = W.hash.p;
    }
    k_advect_tiles<<<nblk(n), 256, 0, s>>>(G.view0(), PArrW{d_pos, 3, 1}, n, dt, G.tile_off.p, G.tiles_new.p, skip);
    AW_LAUNCH();
    W.src_valid = false;  // the positions have moved
    return AW_OK;
}

// ------------------------------------------------------------------------------------------------
// Dense resampling for inspection (sampleMSBG, vtx_visualization.cuh:8-62).  Lattice point
// (i, j, k) of an out[0] x out[1] x out[2] lattice over the domain sits at
// domain_min + (i + 0.5) * spacing (spacing = domain extent / out, rounded to float on the host);
// x fastest.  Cell channels take the value of the cell holding the point (0 in inactive blocks);
// the reference's version ignores domain_min.  The velocity takes the MAC trilinear sample.
// ------------------------------------------------------------------------------------------------
struct Lattice {
    int D[3];
    float sp[3];
};

__device__ inline float lattice_coord(const Geo& g, const Lattice& T, int a, int i) {
    return __fadd_rn(g.dmin[a], __fmul_rn(__fadd_rn((float)i, 0.5f), T.sp[a]));
}

__device__ inline void lattice_point(const Geo& g, const Lattice& T, int64_t idx, float X[3]) {
    const int64_t nxy = (int64_t)T.D[0] * T.D[1];
    const int c[3] = {(int)(idx % T.D[0]), (int)((idx / T.D[0]) % T.D[1]), (int)(idx / nxy)};
#pragma unroll
    for (int a = 0; a < 3; ++a) X[a] = lattice_coord(g, T, a, c[a]);
}

// Per-axis lookup of the cell lookup (particle_key's arithmetic split by axis): for lattice
// coordinate i along axis a, the block coordinate and, for every level l, the cell index in a
// block of resolution R0 >> l.  Row tab[a] holds D[a] entries of (1 + L) ints.
__global__ void k_lattice_tables(Geo g, Lattice T, int* tab0, int* tab1, int* tab2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    if (i >= T.D[a]) return;
    int* tab = a == 0 ? tab0 : (a == 1 ? tab1 : tab2);
    const float p = lattice_coord(g, T, a, i);
    const int c = min(max((int)floorf(__fdiv_rn(__fsub_rn(p, g.dmin[a]), g.bs)), 0), g.D[a] - 1);
    const int stride = 1 + g.L;
    tab[i * stride] = c;
    const float o = forigin(g, a, c);
    for (int l = 0; l < g.L; ++l) {
        const int r = g.R0 >> l;
        const float h = fcell(g, r);
        tab[i * stride + 1 + l] = min(max((int)floorf(__fdiv_rn(__fsub_rn(p, o), h)), 0), r - 1);
    }
}

// one CTA row = one lattice x-row (fixed y, z): coalesced writes, per-axis tables for the lookup
__global__ void k_resample_cells(LevelView L, Lattice T, const int* __restrict__ tab0, const int* __restrict__ tab1,
                                 const int* __restrict__ tab2, const float* __restrict__ ch, float* out) {
    const int stride = 1 + L.g.L;
    const int64_t rows = (int64_t)T.D[1] * T.D[2];
    for (int64_t row = blockIdx.x; row < rows; row += gridDim.x) {
        const int y = (int)(row % T.D[1]), z = (int)(row / T.D[1]);
        const int* ty = tab1 + (size_t)y * stride;
        const int* tz = tab2 + (size_t)z * stride;
        float* o = out + row * T.D[0];
        for (int x = threadIdx.x; x < T.D[0]; x += blockDim.x) {
            const int* tx = tab0 + (size_t)x * stride;
            const int b = bidx(L.g, tx[0], ty[0], tz[0]);
            const int r = L.res[b];
            float v = 0.f;
            if (r) {
                const int l = __ffs(L.g.R0) - __ffs(r);  // r = R0 >> l
                v = ch[L.off[0][b] + cidx(tx[1 + l], ty[1 + l], tz[1 + l], r)];
            }
            o[x] = v;
        }
    }
}

__global__ void k_resample_velocity(LevelView L, Lattice T, const uint32_t* __restrict__ toff,
                                    const float* __restrict__ tiles, float* out) {
    const int64_t n = (int64_t)T.D[0] * T.D[1] * T.D[2];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float X[3];
        lattice_point(L.g, T, i, X);
#pragma unroll
        for (int a = 0; a < 3; ++a) out[3 * i + a] = sample_tiles(L, toff, tiles, a, X);
    }
}

static aw_status make_lattice(const MsbgState& G, const int32_t out_dims[3], Lattice& T) {
    for (int a = 0; a < 3; ++a) {
        if (out_dims[a] < 1 || out_dims[a] > (1 << 16))
            return set_error(AW_ERR_INVALID_ARGUMENT, "lattice size %d out of range", out_dims[a]);
        T.D[a] = out_dims[a];
        T.sp[a] = (float)G.geo.D[a] * G.geo.bs / (float)out_dims[a];
    }
    return AW_OK;
}

static unsigned resample_grid(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
}

extern "C" aw_status aw_resample_lattice(aw_msbg* g, const int32_t out_dims[3], float origin[3], float spacing[3]) {
    AW_CHECK_ARG(g && out_dims && origin && spacing, "null argument");
    Lattice T;
    AW_TRY(make_lattice(g->st, out_dims, T));
    for (int a = 0; a < 3; ++a) {
        spacing[a] = T.sp[a];
        origin[a] = g->st.geo.dmin[a] + 0.5f * T.sp[a];
    }
    return AW_OK;
}

extern "C" aw_status aw_resample_cells(aw_msbg* g, int32_t channel, const int32_t out_dims[3], float* d_out,
                                       aw_stream s_) {
    AW_CHECK_ARG(g && out_dims && d_out, "null argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    if (!(channel == AW_PRESSURE || channel == AW_DIVERGENCE || channel == AW_DISTANCE_FIELD ||
          channel == AW_VORTICITY || channel == AW_CELL_TYPE))
        return set_error(AW_ERR_INVALID_ARGUMENT, "channel %d is not a cell channel", channel);
    MsbgState& G = g->st;
    Lattice T;
    AW_TRY(make_lattice(G, out_dims, T));
    cudaStream_t s = (cudaStream_t)s_;
    const int stride = 1 + G.geo.L;
    AW_TRY(G.lattice_tab.ensure((size_t)stride * (T.D[0] + T.D[1] + T.D[2])));
    int* tab[3] = {G.lattice_tab.p, G.lattice_tab.p + (size_t)stride * T.D[0],
                   G.lattice_tab.p + (size_t)stride * (T.D[0] + T.D[1])};
    const int dmax = std::max({T.D[0], T.D[1], T.D[2]});
    k_lattice_tables<<<dim3((dmax + 127) / 128, 3), 128, 0, s>>>(G.geo, T, tab[0], tab[1], tab[2]);
    AW_LAUNCH();
    const int64_t rows = (int64_t)T.D[1] * T.D[2];
    const int threads = T.D[0] >= 256 ? 256 : (T.D[0] >= 128 ? 128 : 64);
    k_resample_cells<<<(unsigned)std::min<int64_t>(rows, 148 * 64), threads, 0, s>>>(G.view0(), T, tab[0], tab[1],
                                                                                   tab[2], G.ch[channel], d_out);
    AW_LAUNCH();
    return AW_OK;
}

extern "C" aw_status aw_resample_velocity(aw_msbg* g, int32_t old, const int32_t out_dims[3], float* d_out,
                                          aw_stream s_) {
    AW_CHECK_ARG(g && out_dims && d_out, "null argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    MsbgState& G = g->st;
    cudaStream_t s = (cudaStream_t)s_;
    Lattice T;
    AW_TRY(make_lattice(G, out_dims, T));
    const int base = old ? AW_VELOCITY_OLD_X : AW_VELOCITY_X;
    const float* u[3] = {G.ch[base], G.ch[base + 1], G.ch[base + 2]};
    AW_TRY(ensure_tiles(G));
    AW_TRY(build_tiles(G, u, G.tiles_old.p, s));
    const int64_t n = (int64_t)T.D[0] * T.D[1] * T.D[2];
    k_resample_velocity<<<resample_grid(n), 256, 0, s>>>(G.view0(), T, G.tile_off.p, G.tiles_old.p, d_out);
    AW_LAUNCH();
    return AW_OK;
}

extern "C" aw_status aw_sample_velocity(aw_msbg* g, const float* d_points, int64_t n, int32_t old, float* d_out,
                                        aw_stream s_) {
    AW_CHECK_ARG(g && ((d_points && d_out) || n == 0) && n >= 0, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    if (n == 0) return AW_OK;
    MsbgState& G = g->st;
    int base = old ? AW_VELOCITY_OLD_X : AW_VELOCITY_X;
    const float* u[3] = {G.ch[base], G.ch[base + 1], G.ch[base + 2]};
    AW_TRY(ensure_tiles(G));
    AW_TRY(build_tiles(G, u, G.tiles_old.p, (cudaStream_t)s_));
    k_sample_tiles<<<nblk(n), 256, 0, (cudaStream_t)s_>>>(G.view0(), PArr{d_points, 3, 1}, n, G.tile_off.p,
                                                          G.tiles_old.p, d_out);
    AW_LAUNCH();
    return AW_OK;
}
