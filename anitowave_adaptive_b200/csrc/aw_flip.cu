// aw_flip.cu — the FLIP step on the MSBG: sort -> P2G -> T-junction sync -> backup -> gravity
// -> walls -> divergence -> multigrid projection -> pressure-gradient update -> G2P -> RK3.
//
// The reference has no time loop, gravity, wall condition, divergence or gradient kernel
// (its headers stop at P2G, the V-cycle and an unused G2P; main.cu:304-317).  The step order
// follows the intent stated at G2P.cuh:177 with the backup taken right after P2G so that
// particles receive gravity and pressure through the FLIP increment.
#include <algorithm>
#include <cmath>
#include <memory>

#include "aw_internal.cuh"

namespace aw {

static inline unsigned nblk(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// T-junction sync: a coarse block's boundary face := mean of the 4 fine faces it covers.
__global__ void k_face_sync(LevelView L, float* u0, float* u1, float* u2) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    int cb[3];
    bcoord(L.g, b, cb);
    float* U[3] = {u0, u1, u2};
#pragma unroll
    for (int dir = 0; dir < 6; ++dir) {
        const int a = dir >> 1, s = (dir & 1) ? 1 : -1;
        int nc[3] = {cb[0], cb[1], cb[2]};
        nc[a] += s;
        if (!inside(L.g, nc)) continue;
        const int n = bidx(L.g, nc[0], nc[1], nc[2]);
        const int rn = L.res[n];
        if (rn != 2 * r) continue;
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        for (int i = threadIdx.x; i < r * r; i += blockDim.x) {
            const int u1 = i % r, u2 = i / r;
            float sum = 0.f;
            for (int d1 = 0; d1 < 2; ++d1)
                for (int d2 = 0; d2 < 2; ++d2) {
                    int q[3];
                    q[a] = s > 0 ? 0 : rn;
                    q[t1] = 2 * u1 + d1;
                    q[t2] = 2 * u2 + d2;
                    sum += U[a][L.off[1 + a][n] + fidx(a, q[0], q[1], q[2], rn)];
                }
            int f[3];
            f[a] = s > 0 ? r : 0;
            f[t1] = u1;
            f[t2] = u2;
            U[a][L.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r)] = 0.25f * sum;
        }
    }
}

__global__ void k_add_const(float* u, size_t n, float v) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) u[i] += v;
}

// solid walls: u.n = 0 on the domain boundary faces
__global__ void k_wall_bc(LevelView L, float* u0, float* u1, float* u2) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    int cb[3];
    bcoord(L.g, b, cb);
    float* U[3] = {u0, u1, u2};
    for (int a = 0; a < 3; ++a) {
        const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        for (int side = 0; side < 2; ++side) {
            if (side == 0 && cb[a] != 0) continue;
            if (side == 1 && cb[a] != L.g.D[a] - 1) continue;
            for (int i = threadIdx.x; i < r * r; i += blockDim.x) {
                int f[3];
                f[a] = side ? r : 0;
                f[t1] = i % r;
                f[t2] = i / r;
                U[a][L.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r)] = 0.f;
            }
        }
    }
}

__global__ void k_fluid_from_count(const uint32_t* __restrict__ cstart, uint32_t nc, uint8_t* fluid, float* count) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    uint32_t k = cstart[c + 1] - cstart[c];
    fluid[c] = k > 0;
    if (count) count[c] = (float)k;
}

__device__ inline void atomic_max_pos(float* addr, float v) {
    atomicMax((int*)addr, __float_as_int(v));  // v >= 0
}

// b = div(u) / dt on fluid cells (face flux sums with the block's own copies); records
// max |div u| (per volume) into *divmax
__global__ void k_divergence(LevelView L, const float* __restrict__ u0, const float* __restrict__ u1,
                             const float* __restrict__ u2, const uint8_t* __restrict__ fluid, float inv_dt, float* bout,
                             float* divmax) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    const float H = L.g.bs / (float)r;
    const uint32_t oc = L.off[0][b], ox = L.off[1][b], oy = L.off[2][b], oz = L.off[3][b];
    float lmax = 0.f;
    for (int i = threadIdx.x; i < r * r * r; i += blockDim.x) {
        const int x = i % r, y = (i / r) % r, z = i / (r * r);
        float d = 0.f;
        if (fluid[oc + i]) {
            d = (u0[ox + fidx(0, x + 1, y, z, r)] - u0[ox + fidx(0, x, y, z, r)]) +
                (u1[oy + fidx(1, x, y + 1, z, r)] - u1[oy + fidx(1, x, y, z, r)]) +
                (u2[oz + fidx(2, x, y, z + 1, r)] - u2[oz + fidx(2, x, y, z, r)]);
            lmax = fmaxf(lmax, fabsf(d) / H);
            d = d * H * H * inv_dt;
        }
        if (bout) bout[oc + i] = d;
    }
    lmax = warp_max(lmax);
    if ((threadIdx.x & 31) == 0 && divmax) atomic_max_pos(divmax, lmax);
}

// pressure of the cell across face (a, s) of cell c, plus whether that cell is fluid; kind 0 =
// outside the domain (wall)
template <class PT>
__device__ inline int ghost_p(const LevelView& L, const PT* __restrict__ p, const uint8_t* __restrict__ fluid, int b,
                              const int cb[3], const int c[3], int a, int s, double* v, bool* fl) {
    int nc[3] = {cb[0], cb[1], cb[2]};
    nc[a] += s;
    *v = 0.0;
    *fl = false;
    if (!inside(L.g, nc)) return 0;
    const int n = bidx(L.g, nc[0], nc[1], nc[2]);
    const int rn = L.res[n], r = L.res[b];
    if (!rn) return 1;
    const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
    int q[3];
    q[a] = s > 0 ? 0 : rn - 1;
    if (rn <= r) {
        const int sh = rn == r ? 0 : 1;
        q[t1] = min(c[t1] >> sh, rn - 1);
        q[t2] = min(c[t2] >> sh, rn - 1);
        uint32_t i = L.off[0][n] + cidx(q[0], q[1], q[2], rn);
        *v = (double)p[i];
        *fl = fluid[i] != 0;
        return 2;
    }
    double sum = 0.0;
    bool any = false;
    for (int d1 = 0; d1 < 2; ++d1)
        for (int d2 = 0; d2 < 2; ++d2) {
            q[t1] = min(2 * c[t1] + d1, rn - 1);
            q[t2] = min(2 * c[t2] + d2, rn - 1);
            uint32_t i = L.off[0][n] + cidx(q[0], q[1], q[2], rn);
            sum += (double)p[i];
            any |= fluid[i] != 0;
        }
    *v = 0.25 * sum;
    *fl = any;
    return 2;
}

// u -= dt (W / area) (p_high - p_low) on faces with a fluid cell on at least one side; wall faces
// are set to zero.
template <class PT>
__global__ void k_gradient(LevelView L, const PT* __restrict__ p, const uint8_t* __restrict__ fluid, const float* W0,
                           const float* W1, const float* W2, float dt, float* u0, float* u1, float* u2) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    int cb[3];
    bcoord(L.g, b, cb);
    const float H = L.g.bs / (float)r;
    const double scale = (double)dt / ((double)H * H);
    const float* Wa[3] = {W0, W1, W2};
    float* U[3] = {u0, u1, u2};
    const int nf = (r + 1) * r * r;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    for (int fi = threadIdx.x; fi < nf; fi += blockDim.x) {
        int f[3];
        if (a == 0) { f[0] = fi % (r + 1); int rem = fi / (r + 1); f[1] = rem % r; f[2] = rem / r; }
        else if (a == 1) { f[0] = fi % r; int rem = fi / r; f[1] = rem % (r + 1); f[2] = rem / (r + 1); }
        else { f[0] = fi % r; int rem = fi / r; f[1] = rem % r; f[2] = rem / r; }
        double pv[2];
        bool fl[2];
        bool wall = false;
        for (int side = 0; side < 2; ++side) {
            int c[3] = {f[0], f[1], f[2]};
            if (side == 0) c[a] -= 1;
            if (c[a] >= 0 && c[a] < r) {
                uint32_t ci = L.off[0][b] + cidx(c[0], c[1], c[2], r);
                pv[side] = (double)p[ci];
                fl[side] = fluid[ci] != 0;
            } else {
                int cin[3] = {f[0], f[1], f[2]};
                cin[a] = side == 0 ? 0 : r - 1;
                int k = ghost_p(L, p, fluid, b, cb, cin, a, side == 0 ? -1 : 1, &pv[side], &fl[side]);
                if (k == 0) wall = true;
            }
        }
        const uint32_t oi = L.off[1 + a][b] + (uint32_t)fi;
        if (wall) {
            U[a][oi] = 0.f;
            continue;
        }
        if (!fl[0] && !fl[1]) continue;
        U[a][oi] = (float)((double)U[a][oi] - scale * (double)Wa[a][oi] * (pv[1] - pv[0]));
    }
}

template <class PT>
__global__ void k_mask_air(PT* p, const uint8_t* fluid, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !fluid[i]) p[i] = (PT)0;
}

// world positions of face centres (axis a) or cell centres (a = 3), one float3 per element
__global__ void k_positions(LevelView L, int a, float* out) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    int cb[3];
    bcoord(L.g, b, cb);
    const float h = L.g.bs / (float)r;
    const int n = a == 3 ? r * r * r : (r + 1) * r * r;
    const uint32_t o = L.off[a == 3 ? 0 : 1 + a][b];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int f[3];
        if (a == 0) { f[0] = i % (r + 1); int rem = i / (r + 1); f[1] = rem % r; f[2] = rem / r; }
        else if (a == 1) { f[0] = i % r; int rem = i / r; f[1] = rem % (r + 1); f[2] = rem / (r + 1); }
        else { f[0] = i % r; int rem = i / r; f[1] = rem % r; f[2] = rem / r; }
        for (int q = 0; q < 3; ++q)
            out[3 * (size_t)(o + i) + q] = L.g.dmin[q] + (float)cb[q] * L.g.bs + h * ((float)f[q] + (q == a ? 0.f : 0.5f));
    }
}

aw_status face_sync(MsbgState& G, float* u[3], cudaStream_t s) {
    k_face_sync<<<G.nb, 64, 0, s>>>(G.view0(), u[0], u[1], u[2]);
    AW_LAUNCH();
    return AW_OK;
}
aw_status wall_bc(MsbgState& G, float* u[3], cudaStream_t s) {
    k_wall_bc<<<G.nb, 64, 0, s>>>(G.view0(), u[0], u[1], u[2]);
    AW_LAUNCH();
    return AW_OK;
}

}  // namespace aw

using namespace aw;

struct aw_flip {
    aw_msbg* g = nullptr;
    aw_flip_desc d{};
    int64_t n = 0;
    DBuf<float> soa[2];
    DBuf<uint32_t> ids[2];
    int cur = 0;
    aw_solver* solver = nullptr;
    DBuf<float> p32, rhs, divmax;
    DBuf<double> p64;
    DBuf<uint8_t> fluid;
    aw_flip_stats stats{};
    cudaEvent_t ev[8] = {};
    ~aw_flip() {
        if (solver) aw_solver_destroy(solver);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
};

extern "C" aw_status aw_flip_create(aw_msbg* g, const aw_flip_desc* d, const float* h_pos, const float* h_vel, int64_t n,
                                    aw_flip** out) {
    AW_CHECK_ARG(g && d && out && ((h_pos && h_vel) || n == 0) && n >= 0 && n < (int64_t)0xFFFFFFFF, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    *out = nullptr;
    std::unique_ptr<aw_flip> F(new aw_flip());
    F->g = g;
    F->d = *d;
    F->n = n;
    MsbgState& G = g->st;
    for (int k = 0; k < 2; ++k) {
        AW_TRY(F->soa[k].alloc((size_t)std::max<int64_t>(n, 1) * 6));
        AW_TRY(F->ids[k].alloc((size_t)std::max<int64_t>(n, 1)));
    }
    // host AoS -> device SoA
    std::vector<float> tmp((size_t)n * 6);
    std::vector<uint32_t> id((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            tmp[(size_t)a * n + i] = h_pos[3 * i + a];
            tmp[(size_t)(3 + a) * n + i] = h_vel[3 * i + a];
        }
        id[i] = (uint32_t)i;
    }
    if (n) {
        AW_CUDA(cudaMemcpy(F->soa[0].p, tmp.data(), tmp.size() * sizeof(float), cudaMemcpyHostToDevice));
        AW_CUDA(cudaMemcpy(F->ids[0].p, id.data(), id.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    }
    aw_solver_desc sd;
    AW_TRY(aw_solver_default_desc(AW_OPERATOR_FV, &sd));
    sd.precision = d->precision;
    sd.tolerance = d->tolerance;
    sd.max_cycles = d->max_cycles;
    AW_TRY(aw_solver_create(g, &sd, &F->solver));
    AW_TRY(F->p32.alloc(G.tot[0]));
    AW_TRY(F->p64.alloc(G.tot[0]));
    AW_TRY(F->rhs.alloc(G.tot[0]));
    AW_TRY(F->fluid.alloc(G.tot[0]));
    AW_TRY(F->divmax.alloc(2));
    for (auto& e : F->ev) AW_CUDA(cudaEventCreate(&e));
    *out = F.release();
    return AW_OK;
}

extern "C" aw_status aw_flip_destroy(aw_flip* f) {
    delete f;
    return AW_OK;
}

extern "C" aw_status aw_flip_solver(aw_flip* f, aw_solver** out) {
    AW_CHECK_ARG(f && out, "null argument");
    *out = f->solver;
    return AW_OK;
}

extern "C" aw_status aw_flip_step(aw_flip* F, aw_stream s_) {
    AW_CHECK_ARG(F, "null simulation");
    cudaStream_t s = (cudaStream_t)s_;
    MsbgState& G = F->g->st;
    const int64_t n = F->n;
    float* U[3] = {G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]};
    float* UO[3] = {G.ch[AW_VELOCITY_OLD_X], G.ch[AW_VELOCITY_OLD_Y], G.ch[AW_VELOCITY_OLD_Z]};
    float* Mm[3] = {G.ch[AW_MASS_DENSITY_X], G.ch[AW_MASS_DENSITY_Y], G.ch[AW_MASS_DENSITY_Z]};
    float* Mo[3] = {G.ch[AW_MOMENTUM_X], G.ch[AW_MOMENTUM_Y], G.ch[AW_MOMENTUM_Z]};
    AW_CUDA(cudaEventRecord(F->ev[0], s));
    // 1. sort by (block, cell)
    AW_TRY(sort_core_soa(G, F->soa[F->cur].p, n, s));
    AW_TRY(gather_soa(G, F->soa[F->cur].p, n, F->soa[F->cur ^ 1].p, F->ids[F->cur].p, F->ids[F->cur ^ 1].p, s));
    F->cur ^= 1;
    float* soa = F->soa[F->cur].p;
    AW_CUDA(cudaEventRecord(F->ev[1], s));
    // 2. P2G (+ normalise) and fluid flags
    float* nomom[3] = {nullptr, nullptr, nullptr};
    (void)Mo;
    AW_TRY(p2g_sorted(G, soa, n, G.pw.cell_start.p, U, Mm, nomom, nullptr, s));
    AW_CUDA(cudaEventRecord(F->ev[2], s));
    k_fluid_from_count<<<nblk(G.tot[0]), 256, 0, s>>>(G.pw.cell_start.p, G.tot[0], F->fluid.p, G.ch[AW_CELL_TYPE]);
    AW_LAUNCH();
    AW_TRY(face_sync(G, U, s));
    // 3. backup, gravity, walls
    for (int a = 0; a < 3; ++a)
        AW_CUDA(cudaMemcpyAsync(UO[a], U[a], G.tot[1 + a] * sizeof(float), cudaMemcpyDeviceToDevice, s));
    for (int a = 0; a < 3; ++a)
        if (F->d.gravity[a] != 0.f) {
            k_add_const<<<nblk(G.tot[1 + a]), 256, 0, s>>>(U[a], G.tot[1 + a], F->d.dt * F->d.gravity[a]);
            AW_LAUNCH();
        }
    AW_TRY(wall_bc(G, U, s));
    // 4. divergence
    AW_CUDA(cudaMemsetAsync(F->divmax.p, 0, 2 * sizeof(float), s));
    k_divergence<<<G.nb, 128, 0, s>>>(G.view0(), U[0], U[1], U[2], F->fluid.p, 1.f / F->d.dt, F->rhs.p, F->divmax.p);
    AW_LAUNCH();
    AW_CUDA(cudaEventRecord(F->ev[3], s));
    // 5. projection
    AW_TRY(aw_solver_setup(F->solver, F->fluid.p, s_));
    void* p;
    if (F->d.precision == AW_PRECISION_MIXED) {
        AW_CUDA(cudaMemsetAsync(F->p64.p, 0, G.tot[0] * sizeof(double), s));
        p = F->p64.p;
    } else {
        AW_CUDA(cudaMemsetAsync(F->p32.p, 0, G.tot[0] * sizeof(float), s));
        p = F->p32.p;
    }
    int32_t cycles = 0;
    double rel = 0;
    aw_status st = aw_solve(F->solver, F->rhs.p, p, &cycles, &rel, s_);
    F->stats.cycles = cycles;
    F->stats.residual = rel;
    if (st != AW_OK) return st;
    AW_CUDA(cudaEventRecord(F->ev[4], s));
    // 6. pressure-gradient update, sync, walls
    void* W[3];
    uint32_t cnt;
    for (int a = 0; a < 3; ++a) AW_TRY(aw_solver_level_array(F->solver, 0, 3 + a, &W[a], &cnt));
    if (F->d.precision == AW_PRECISION_MIXED)
        k_gradient<double><<<G.nb, 128, 0, s>>>(G.view0(), F->p64.p, F->fluid.p, (float*)W[0], (float*)W[1],
                                                (float*)W[2], F->d.dt, U[0], U[1], U[2]);
    else
        k_gradient<float><<<G.nb, 128, 0, s>>>(G.view0(), F->p32.p, F->fluid.p, (float*)W[0], (float*)W[1], (float*)W[2],
                                               F->d.dt, U[0], U[1], U[2]);
    AW_LAUNCH();
    AW_TRY(face_sync(G, U, s));
    AW_TRY(wall_bc(G, U, s));
    k_divergence<<<G.nb, 128, 0, s>>>(G.view0(), U[0], U[1], U[2], F->fluid.p, 1.f / F->d.dt, nullptr, F->divmax.p + 1);
    AW_LAUNCH();
    AW_CUDA(cudaEventRecord(F->ev[5], s));
    // 7. G2P (FLIP blend) on the sorted SoA particles
    const float* un[3] = {U[0], U[1], U[2]};
    const float* uo[3] = {UO[0], UO[1], UO[2]};
    AW_TRY(g2p_sorted(G, soa, n, G.pw.cell_start.p, F->d.alpha, un, uo, s));
    AW_CUDA(cudaEventRecord(F->ev[6], s));
    // 8. RK3 advection through the u_new tiles built for G2P
    AW_TRY(advect_tiles(G, soa, 1, n, F->d.dt, G.tiles_new.p, s));
    AW_CUDA(cudaEventRecord(F->ev[7], s));
    AW_CUDA(cudaEventSynchronize(F->ev[7]));
    AW_TRY(check_device_errors(G, s));
    float dm[2];
    AW_CUDA(cudaMemcpy(dm, F->divmax.p, sizeof dm, cudaMemcpyDeviceToHost));
    F->stats.div_before = dm[0];
    F->stats.div_after = dm[1];
    float t[7];
    for (int k = 0; k < 7; ++k) AW_CUDA(cudaEventElapsedTime(&t[k], F->ev[k], F->ev[k + 1]));
    F->stats.ms_sort = t[0];
    F->stats.ms_p2g = t[1];
    F->stats.ms_other = t[2] + t[4];
    F->stats.ms_solve = t[3];
    F->stats.ms_g2p = t[5];
    F->stats.ms_advect = t[6];
    return AW_OK;
}

extern "C" aw_status aw_flip_stats_get(aw_flip* f, aw_flip_stats* out) {
    AW_CHECK_ARG(f && out, "null argument");
    *out = f->stats;
    return AW_OK;
}

extern "C" aw_status aw_flip_particles(aw_flip* F, float* h_pos, float* h_vel) {
    AW_CHECK_ARG(F, "null simulation");
    const int64_t n = F->n;
    if (!n) return AW_OK;
    std::vector<float> tmp((size_t)n * 6);
    std::vector<uint32_t> id((size_t)n);
    AW_CUDA(cudaDeviceSynchronize());
    AW_CUDA(cudaMemcpy(tmp.data(), F->soa[F->cur].p, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost));
    AW_CUDA(cudaMemcpy(id.data(), F->ids[F->cur].p, id.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    for (int64_t j = 0; j < n; ++j) {
        uint32_t i = id[j];
        for (int a = 0; a < 3; ++a) {
            if (h_pos) h_pos[3 * (size_t)i + a] = tmp[(size_t)a * n + j];
            if (h_vel) h_vel[3 * (size_t)i + a] = tmp[(size_t)(3 + a) * n + j];
        }
    }
    return AW_OK;
}

// ---- FLIP-step building blocks (no counterpart in the reference) -----------------------------
static aw_status channel_triplet(MsbgState& G, int32_t base, float* U[3]) {
    AW_CHECK_ARG(base == AW_VELOCITY_X || base == AW_VELOCITY_OLD_X || base == AW_MOMENTUM_X ||
                     base == AW_MASS_DENSITY_X || base == AW_BETA_COEFF_X || base == AW_PHASE_FIELD_X,
                 "channel must be the x channel of a face-channel triplet");
    for (int a = 0; a < 3; ++a) U[a] = G.ch[base + a];
    return AW_OK;
}

extern "C" aw_status aw_face_positions(aw_msbg* g, int32_t axis, float* d_xyz, aw_stream s) {
    AW_CHECK_ARG(g && d_xyz && axis >= 0 && axis <= 3, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    k_positions<<<g->st.nb, 128, 0, (cudaStream_t)s>>>(g->st.view0(), axis, d_xyz);
    AW_LAUNCH();
    return AW_OK;
}

extern "C" aw_status aw_face_sync(aw_msbg* g, int32_t channel, aw_stream s) {
    AW_CHECK_ARG(g && g->st.allocated, "grid not allocated");
    float* U[3];
    AW_TRY(channel_triplet(g->st, channel, U));
    return face_sync(g->st, U, (cudaStream_t)s);
}

extern "C" aw_status aw_wall_bc(aw_msbg* g, int32_t channel, aw_stream s) {
    AW_CHECK_ARG(g && g->st.allocated, "grid not allocated");
    float* U[3];
    AW_TRY(channel_triplet(g->st, channel, U));
    return wall_bc(g->st, U, (cudaStream_t)s);
}

extern "C" aw_status aw_add_gravity(aw_msbg* g, const float gravity[3], float dt, aw_stream s) {
    AW_CHECK_ARG(g && gravity && g->st.allocated, "bad argument");
    MsbgState& G = g->st;
    for (int a = 0; a < 3; ++a)
        if (gravity[a] != 0.f) {
            k_add_const<<<nblk(G.tot[1 + a]), 256, 0, (cudaStream_t)s>>>(G.ch[AW_VELOCITY_X + a], G.tot[1 + a],
                                                                          dt * gravity[a]);
            AW_LAUNCH();
        }
    return AW_OK;
}

extern "C" aw_status aw_velocity_divergence(aw_msbg* g, const uint8_t* d_fluid, float inv_dt, float* d_out,
                                            float* d_max, aw_stream s) {
    AW_CHECK_ARG(g && d_fluid && g->st.allocated, "bad argument");
    MsbgState& G = g->st;
    k_divergence<<<G.nb, 128, 0, (cudaStream_t)s>>>(G.view0(), G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y],
                                                    G.ch[AW_VELOCITY_Z], d_fluid, inv_dt, d_out, d_max);
    AW_LAUNCH();
    return AW_OK;
}

extern "C" aw_status aw_pressure_gradient(aw_msbg* g, aw_solver* sv, const void* d_p, int32_t p_is_double,
                                          const uint8_t* d_fluid, float dt, aw_stream s_) {
    AW_CHECK_ARG(g && sv && d_p && d_fluid && g->st.allocated, "bad argument");
    MsbgState& G = g->st;
    cudaStream_t s = (cudaStream_t)s_;
    void* W[3];
    uint32_t cnt;
    for (int a = 0; a < 3; ++a) AW_TRY(aw_solver_level_array(sv, 0, 3 + a, &W[a], &cnt));
    if (p_is_double)
        k_gradient<double><<<G.nb, 128, 0, s>>>(G.view0(), (const double*)d_p, d_fluid, (float*)W[0], (float*)W[1],
                                                (float*)W[2], dt, G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y],
                                                G.ch[AW_VELOCITY_Z]);
    else
        k_gradient<float><<<G.nb, 128, 0, s>>>(G.view0(), (const float*)d_p, d_fluid, (float*)W[0], (float*)W[1],
                                               (float*)W[2], dt, G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y],
                                               G.ch[AW_VELOCITY_Z]);
    AW_LAUNCH();
    return AW_OK;
}
