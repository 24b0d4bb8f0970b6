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

// Coefficient sync at T-junctions: the coarse face and the 4 fine faces it covers all take the
// mean of the 4 fine values.  The fine cell's flux uses its own face's coefficient and the coarse
// cell's flux uses the coarse face's, so equal values on both sides keep A symmetric.  Only the
// coarse block writes these faces.
__global__ void k_beta_sync(LevelView L, float* b0, float* b1, float* b2) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    int cb[3];
    bcoord(L.g, b, cb);
    float* B[3] = {b0, b1, b2};
#pragma unroll 1
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
            uint32_t fine[4];
            float sum = 0.f;
            for (int d1 = 0; d1 < 2; ++d1)
                for (int d2 = 0; d2 < 2; ++d2) {
                    int q[3];
                    q[a] = s > 0 ? 0 : rn;
                    q[t1] = 2 * u1 + d1;
                    q[t2] = 2 * u2 + d2;
                    fine[2 * d1 + d2] = L.off[1 + a][n] + fidx(a, q[0], q[1], q[2], rn);
                    sum += B[a][fine[2 * d1 + d2]];
                }
            const float v = 0.25f * sum;
            for (int k = 0; k < 4; ++k) B[a][fine[k]] = v;
            int f[3];
            f[a] = s > 0 ? r : 0;
            f[t1] = u1;
            f[t2] = u2;
            B[a][L.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r)] = v;
        }
    }
}

template <class PT>
__global__ void k_zero_air(PT* p, const uint8_t* __restrict__ fluid, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !fluid[i]) p[i] = PT(0);
}

// the step's pressure into the PRESSURE channel (0 in air cells), for inspection
template <class PT>
__global__ void k_store_pressure(const PT* __restrict__ p, const uint8_t* __restrict__ fluid, size_t n, float* out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = fluid[i] ? (float)p[i] : 0.f;
}

__global__ void k_fill(float* u, size_t n, float v) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) u[i] = v;
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

// max over fluid cells of |div u| per unit volume, the face sums taken in FP64 (for reporting the
// divergence an FP32 velocity field really has, free of the FP32 rounding of the sum itself)
__global__ void k_divergence_max64(LevelView L, const float* __restrict__ u0, const float* __restrict__ u1,
                                   const float* __restrict__ u2, const uint8_t* __restrict__ fluid,
                                   unsigned long long* divmax) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    const double invH = (double)r / (double)L.g.bs;
    const uint32_t oc = L.off[0][b], ox = L.off[1][b], oy = L.off[2][b], oz = L.off[3][b];
    double lmax = 0.0;
    for (int i = threadIdx.x; i < r * r * r; i += blockDim.x) {
        const int x = i % r, y = (i / r) % r, z = i / (r * r);
        if (!fluid || fluid[oc + i]) {
            const double d = ((double)u0[ox + fidx(0, x + 1, y, z, r)] - (double)u0[ox + fidx(0, x, y, z, r)]) +
                             ((double)u1[oy + fidx(1, x, y + 1, z, r)] - (double)u1[oy + fidx(1, x, y, z, r)]) +
                             ((double)u2[oz + fidx(2, x, y, z + 1, r)] - (double)u2[oz + fidx(2, x, y, z, r)]);
            lmax = fmax(lmax, fabs(d) * invH);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    // non-negative doubles order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(divmax, (unsigned long long)__double_as_longlong(lmax));
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

// ---- adjoints of the grid-side linear maps (no counterpart in the reference) -----------------
// k_face_sync^T: a synced coarse face hands a quarter of its adjoint to each of the 4 fine faces
// it was averaged from and keeps none.  Each fine face belongs to one synced coarse face only.
__global__ void k_face_sync_vjp(LevelView L, float* u0, float* u1, float* u2) {
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
            int f[3];
            f[a] = s > 0 ? r : 0;
            f[t1] = u1;
            f[t2] = u2;
            float* cf = &U[a][L.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r)];
            const float g = 0.25f * *cf;
            *cf = 0.f;
            for (int d1 = 0; d1 < 2; ++d1)
                for (int d2 = 0; d2 < 2; ++d2) {
                    int q[3];
                    q[a] = s > 0 ? 0 : rn;
                    q[t1] = 2 * u1 + d1;
                    q[t2] = 2 * u2 + d2;
                    U[a][L.off[1 + a][n] + fidx(a, q[0], q[1], q[2], rn)] += g;
                }
        }
    }
}

// k_divergence^T: ubar_f += (H^2 / dt) (bbar[low cell] - bbar[high cell]) over the fluid cells of the
// face's block (one thread per face, no atomics)
template <class BT>
__global__ void k_divergence_vjp(LevelView L, const BT* __restrict__ bbar, const uint8_t* __restrict__ fluid,
                                 float inv_dt, float* u0, float* u1, float* u2) {
    const int b = blockIdx.x;
    const int r = L.res[b];
    if (!r) return;
    const float H = L.g.bs / (float)r;
    const double sc = (double)H * H * inv_dt;
    float* U[3] = {u0, u1, u2};
    const uint32_t oc = L.off[0][b];
    const int nf = (r + 1) * r * r;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        for (int fi = threadIdx.x; fi < nf; fi += blockDim.x) {
            int f[3];
            if (a == 0) { f[0] = fi % (r + 1); int rem = fi / (r + 1); f[1] = rem % r; f[2] = rem / r; }
            else if (a == 1) { f[0] = fi % r; int rem = fi / r; f[1] = rem % (r + 1); f[2] = rem / (r + 1); }
            else { f[0] = fi % r; int rem = fi / r; f[1] = rem % r; f[2] = rem / r; }
            double acc = 0.0;
            if (f[a] > 0) {  // the face is the high face of the cell below
                int c[3] = {f[0], f[1], f[2]};
                c[a] -= 1;
                const uint32_t ci = oc + cidx(c[0], c[1], c[2], r);
                if (fluid[ci]) acc += (double)bbar[ci];
            }
            if (f[a] < r) {  // and the low face of the cell above
                const uint32_t ci = oc + cidx(f[0], f[1], f[2], r);
                if (fluid[ci]) acc -= (double)bbar[ci];
            }
            if (acc != 0.0) {
                float* p = &U[a][L.off[1 + a][b] + (uint32_t)fi];
                *p = (float)((double)*p + sc * acc);
            }
        }
}

// cells (and their weights) whose pressure forms the value across face (a, s) of cell c (the
// dependence of ghost_p on p); returns the count, 0 for a wall or an absent neighbour
__device__ inline int ghost_cells(const LevelView& L, const uint8_t* __restrict__ fluid, int b, const int cb[3],
                                  const int c[3], int a, int s, uint32_t cells[4], float* w, bool* fl, bool* wall) {
    int nc[3] = {cb[0], cb[1], cb[2]};
    nc[a] += s;
    *fl = false;
    *wall = false;
    if (!inside(L.g, nc)) {
        *wall = true;
        return 0;
    }
    const int n = bidx(L.g, nc[0], nc[1], nc[2]);
    const int rn = L.res[n], r = L.res[b];
    if (!rn) return 0;
    const int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
    int q[3];
    q[a] = s > 0 ? 0 : rn - 1;
    if (rn <= r) {
        const int sh = rn == r ? 0 : 1;
        q[t1] = min(c[t1] >> sh, rn - 1);
        q[t2] = min(c[t2] >> sh, rn - 1);
        cells[0] = L.off[0][n] + cidx(q[0], q[1], q[2], rn);
        *w = 1.f;
        *fl = fluid[cells[0]] != 0;
        return 1;
    }
    int k = 0;
    for (int d1 = 0; d1 < 2; ++d1)
        for (int d2 = 0; d2 < 2; ++d2, ++k) {
            q[t1] = min(2 * c[t1] + d1, rn - 1);
            q[t2] = min(2 * c[t2] + d2, rn - 1);
            cells[k] = L.off[0][n] + cidx(q[0], q[1], q[2], rn);
            *fl = *fl || fluid[cells[k]] != 0;
        }
    *w = 0.25f;
    return 4;
}

// k_gradient^T: ubar on wall faces is cleared; pbar += -dt (W / area) ubar d(p_high - p_low)/dp on
// faces with a fluid cell on either side (float atomics: cells receive from up to 6 faces and from
// neighbouring blocks)
__global__ void k_gradient_vjp(LevelView L, const uint8_t* __restrict__ fluid, const float* W0, const float* W1,
                               const float* W2, float dt, float* u0, float* u1, float* u2, float* pbar) {
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
            uint32_t cells[2][4];
            float cw[2] = {1.f, 1.f};
            int nc[2] = {0, 0};
            bool fl[2] = {false, false};
            bool wall = false;
            for (int side = 0; side < 2; ++side) {
                int c[3] = {f[0], f[1], f[2]};
                if (side == 0) c[a] -= 1;
                if (c[a] >= 0 && c[a] < r) {
                    cells[side][0] = L.off[0][b] + cidx(c[0], c[1], c[2], r);
                    nc[side] = 1;
                    fl[side] = fluid[cells[side][0]] != 0;
                } else {
                    int cin[3] = {f[0], f[1], f[2]};
                    cin[a] = side == 0 ? 0 : r - 1;
                    bool wl;
                    nc[side] = ghost_cells(L, fluid, b, cb, cin, a, side == 0 ? -1 : 1, cells[side], &cw[side],
                                           &fl[side], &wl);
                    wall = wall || wl;
                }
            }
            const uint32_t oi = L.off[1 + a][b] + (uint32_t)fi;
            if (wall) {
                U[a][oi] = 0.f;
                continue;
            }
            if (!fl[0] && !fl[1]) continue;
            const float coef = (float)(-scale * (double)Wa[a][oi] * (double)U[a][oi]);
            if (coef == 0.f) continue;
            for (int k = 0; k < nc[1]; ++k) atomicAdd(&pbar[cells[1][k]], coef * cw[1]);
            for (int k = 0; k < nc[0]; ++k) atomicAdd(&pbar[cells[0][k]], -coef * cw[0]);
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
aw_status beta_sync(MsbgState& G, float* beta[3], cudaStream_t s) {
    k_beta_sync<<<G.nb, 64, 0, s>>>(G.view0(), beta[0], beta[1], beta[2]);
    AW_LAUNCH();
    return AW_OK;
}

aw_status face_sync_vjp(MsbgState& G, float* ubar[3], cudaStream_t s) {
    k_face_sync_vjp<<<G.nb, 64, 0, s>>>(G.view0(), ubar[0], ubar[1], ubar[2]);
    AW_LAUNCH();
    return AW_OK;
}

static aw_status level0_W(aw_solver* sv, float* W[3]) {
    for (int a = 0; a < 3; ++a) {
        void* p;
        uint32_t cnt;
        AW_TRY(aw_solver_level_array(sv, 0, 3 + a, &p, &cnt));
        W[a] = (float*)p;
    }
    return AW_OK;
}

aw_status project_forward(MsbgState& G, aw_solver* sv, const uint8_t* fluid, float dt, int precision, FlipBufs& B,
                          cudaStream_t s) {
    AW_TRY(B.ensure(G));
    float* U[3] = {G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]};
    k_divergence<<<G.nb, 128, 0, s>>>(G.view0(), U[0], U[1], U[2], fluid, 1.f / dt, B.rhs.p, nullptr);
    AW_LAUNCH();
    const bool mixed = precision == AW_PRECISION_MIXED;
    void* p = mixed ? (void*)B.p64.p : (void*)B.p32.p;
    AW_CUDA(cudaMemsetAsync(p, 0, G.tot[0] * (mixed ? sizeof(double) : sizeof(float)), s));
    int32_t cycles;
    double rel;
    AW_TRY(aw_solve(sv, B.rhs.p, p, &cycles, &rel, (aw_stream)s));
    float* W[3];
    AW_TRY(level0_W(sv, W));
    if (mixed)
        k_gradient<double><<<G.nb, 128, 0, s>>>(G.view0(), B.p64.p, fluid, W[0], W[1], W[2], dt, U[0], U[1], U[2]);
    else
        k_gradient<float><<<G.nb, 128, 0, s>>>(G.view0(), B.p32.p, fluid, W[0], W[1], W[2], dt, U[0], U[1], U[2]);
    AW_LAUNCH();
    AW_TRY(face_sync(G, U, s));
    return wall_bc(G, U, s);
}

aw_status project_vjp(MsbgState& G, aw_solver* sv, const uint8_t* fluid, float dt, int precision, float* ubar[3],
                      FlipBufs& B, cudaStream_t s) {
    AW_TRY(B.ensure(G));
    // walls and the T-junction sync, transposed
    AW_TRY(wall_bc(G, ubar, s));
    AW_TRY(face_sync_vjp(G, ubar, s));
    // pressure-gradient update, transposed: pbar (into B.rhs) and the wall faces of ubar
    float* W[3];
    AW_TRY(level0_W(sv, W));
    AW_CUDA(cudaMemsetAsync(B.rhs.p, 0, G.tot[0] * sizeof(float), s));
    k_gradient_vjp<<<G.nb, 128, 0, s>>>(G.view0(), fluid, W[0], W[1], W[2], dt, ubar[0], ubar[1], ubar[2], B.rhs.p);
    AW_LAUNCH();
    k_mask_air<float><<<nblk(G.tot[0]), 256, 0, s>>>(B.rhs.p, fluid, G.tot[0]);
    AW_LAUNCH();
    // the operator is symmetric: bbar = A^-1 pbar is one more solve with the same hierarchy
    const bool mixed = precision == AW_PRECISION_MIXED;
    void* bb = mixed ? (void*)B.p64.p : (void*)B.p32.p;
    AW_CUDA(cudaMemsetAsync(bb, 0, G.tot[0] * (mixed ? sizeof(double) : sizeof(float)), s));
    int32_t cycles;
    double rel;
    AW_TRY(aw_solve(sv, B.rhs.p, bb, &cycles, &rel, (aw_stream)s));
    // divergence, transposed
    if (mixed)
        k_divergence_vjp<double><<<G.nb, 128, 0, s>>>(G.view0(), B.p64.p, fluid, 1.f / dt, ubar[0], ubar[1], ubar[2]);
    else
        k_divergence_vjp<float><<<G.nb, 128, 0, s>>>(G.view0(), B.p32.p, fluid, 1.f / dt, ubar[0], ubar[1], ubar[2]);
    AW_LAUNCH();
    return AW_OK;
}

aw_status FlipBufs::ensure(const MsbgState& G) {
    AW_TRY(p32.ensure(std::max<uint32_t>(G.tot[0], 1)));
    AW_TRY(p64.ensure(std::max<uint32_t>(G.tot[0], 1)));
    AW_TRY(rhs.ensure(std::max<uint32_t>(G.tot[0], 1)));
    AW_TRY(fluid.ensure(std::max<uint32_t>(G.tot[0], 1)));
    AW_TRY(divmax.ensure(2));
    return AW_OK;
}

aw_status StepRecord::ensure(const MsbgState& G, int64_t n) {
    const size_t np = (size_t)std::max<int64_t>(n, 1);
    AW_TRY(perm.ensure(np));
    AW_TRY(soa.ensure(6 * np + kSoaPad));
    for (int a = 0; a < 3; ++a) {
        const size_t nf = std::max<uint32_t>(G.tot[1 + a], 1);
        AW_TRY(u1[a].ensure(nf));
        AW_TRY(m[a].ensure(nf));
        AW_TRY(uo[a].ensure(nf));
        AW_TRY(u6[a].ensure(nf));
    }
    AW_TRY(fluid.ensure(std::max<uint32_t>(G.tot[0], 1)));
    return AW_OK;
}

static aw_status copy_d2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes) AW_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
    return AW_OK;
}

aw_status flip_step_soa(MsbgState& G, aw_solver* solver, const aw_flip_desc& d, FlipBufs& B, const float* soa_in,
                        const uint32_t* ids_in, float* soa_out, uint32_t* ids_out, int64_t n, const uint8_t* fluid_in,
                        StepRecord* rec, cudaEvent_t* ev, aw_flip_stats* st, cudaStream_t s, const FlipPhase* fp,
                        bool warm_start) {
    if (fp && !ids_out) return set_error(AW_ERR_INVALID_ARGUMENT, "two-phase step needs particle ids");
    float* U[3] = {G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]};
    float* UO[3] = {G.ch[AW_VELOCITY_OLD_X], G.ch[AW_VELOCITY_OLD_Y], G.ch[AW_VELOCITY_OLD_Z]};
    float* Mm[3] = {G.ch[AW_MASS_DENSITY_X], G.ch[AW_MASS_DENSITY_Y], G.ch[AW_MASS_DENSITY_Z]};
    const size_t fb[3] = {G.tot[1] * sizeof(float), G.tot[2] * sizeof(float), G.tot[3] * sizeof(float)};
    AW_TRY(B.ensure(G));
    if (rec) AW_TRY(rec->ensure(G, n));
    if (ev) AW_CUDA(cudaEventRecord(ev[0], s));
    // 1. sort by (block, cell)
    AW_TRY(sort_core_soa(G, soa_in, n, s));
    AW_TRY(gather_soa(G, soa_in, n, soa_out, ids_in, ids_out, s));
    if (rec) {
        AW_TRY(copy_d2d(rec->perm.p, G.pw.sorted, (size_t)n * sizeof(uint32_t), s));
        AW_TRY(copy_d2d(rec->soa.p, soa_out, (size_t)n * 6 * sizeof(float), s));
    }
    if (ev) AW_CUDA(cudaEventRecord(ev[1], s));
    // 2. P2G (+ normalise) and fluid flags
    float* nomom[3] = {nullptr, nullptr, nullptr};
    PhaseIn pin{};
    if (fp) {
        pin.pid = ids_out;
        pin.phase = fp->phase;
        pin.rho0 = fp->rho0;
        pin.rho1 = fp->rho1;
        for (int a = 0; a < 3; ++a) {
            pin.phi[a] = G.ch[AW_PHASE_FIELD_X + a];
            pin.beta[a] = G.ch[AW_BETA_COEFF_X + a];
        }
    }
    AW_TRY(p2g_sorted(G, soa_out, n, G.pw.cell_start.p, U, Mm, nomom, nullptr, s, fp ? &pin : nullptr));
    if (ev) AW_CUDA(cudaEventRecord(ev[2], s));
    k_fluid_from_count<<<nblk(G.tot[0]), 256, 0, s>>>(G.pw.cell_start.p, G.tot[0], B.fluid.p, G.ch[AW_CELL_TYPE]);
    AW_LAUNCH();
    if (fluid_in) AW_TRY(copy_d2d(B.fluid.p, fluid_in, G.tot[0], s));
    if (rec) {
        for (int a = 0; a < 3; ++a) {
            AW_TRY(copy_d2d(rec->u1[a].p, U[a], fb[a], s));
            AW_TRY(copy_d2d(rec->m[a].p, Mm[a], fb[a], s));
        }
        AW_TRY(copy_d2d(rec->fluid.p, B.fluid.p, G.tot[0], s));
    }
    AW_TRY(face_sync(G, U, s));
    // 3. backup, gravity, walls
    for (int a = 0; a < 3; ++a) AW_TRY(copy_d2d(UO[a], U[a], fb[a], s));
    for (int a = 0; a < 3; ++a)
        if (d.gravity[a] != 0.f && G.tot[1 + a]) {
            k_add_const<<<nblk(G.tot[1 + a]), 256, 0, s>>>(U[a], G.tot[1 + a], d.dt * d.gravity[a]);
            AW_LAUNCH();
        }
    AW_TRY(wall_bc(G, U, s));
    // 4. divergence
    AW_CUDA(cudaMemsetAsync(B.divmax.p, 0, 2 * sizeof(float), s));
    k_divergence<<<G.nb, 128, 0, s>>>(G.view0(), U[0], U[1], U[2], B.fluid.p, 1.f / d.dt, B.rhs.p, B.divmax.p);
    AW_LAUNCH();
    if (ev) AW_CUDA(cudaEventRecord(ev[3], s));
    // 5. projection (two-phase: coefficients from this step's beta first)
    if (fp) {
        AW_TRY(beta_sync(G, pin.beta, s));
        AW_TRY(aw_solver_update_coefficients(solver, (aw_stream)s));
    }
    AW_TRY(aw_solver_setup(solver, B.fluid.p, (aw_stream)s));
    // initial guess: the previous step's pressure (air cells zeroed: they are Dirichlet p = 0), or 0
    void* p;
    const bool warm = warm_start && B.p_warm && G.tot[0];
    if (d.precision == AW_PRECISION_MIXED) {
        if (warm) k_zero_air<double><<<nblk(G.tot[0]), 256, 0, s>>>(B.p64.p, B.fluid.p, G.tot[0]);
        else AW_CUDA(cudaMemsetAsync(B.p64.p, 0, G.tot[0] * sizeof(double), s));
        p = B.p64.p;
    } else {
        if (warm) k_zero_air<float><<<nblk(G.tot[0]), 256, 0, s>>>(B.p32.p, B.fluid.p, G.tot[0]);
        else AW_CUDA(cudaMemsetAsync(B.p32.p, 0, G.tot[0] * sizeof(float), s));
        p = B.p32.p;
    }
    if (warm) AW_LAUNCH();
    B.p_warm = false;
    int32_t cycles = 0;
    double rel = 0;
    aw_status sst = aw_solve(solver, B.rhs.p, p, &cycles, &rel, (aw_stream)s);
    if (st) {
        st->cycles = cycles;
        st->residual = rel;
    }
    if (sst != AW_OK) return sst;
    B.p_warm = true;
    if (G.tot[0]) {
        if (d.precision == AW_PRECISION_MIXED)
            k_store_pressure<double><<<nblk(G.tot[0]), 256, 0, s>>>(B.p64.p, B.fluid.p, G.tot[0], G.ch[AW_PRESSURE]);
        else
            k_store_pressure<float><<<nblk(G.tot[0]), 256, 0, s>>>(B.p32.p, B.fluid.p, G.tot[0], G.ch[AW_PRESSURE]);
        AW_LAUNCH();
    }
    if (ev) AW_CUDA(cudaEventRecord(ev[4], s));
    // 6. pressure-gradient update, sync, walls
    void* W[3];
    uint32_t cnt;
    for (int a = 0; a < 3; ++a) AW_TRY(aw_solver_level_array(solver, 0, 3 + a, &W[a], &cnt));
    if (d.precision == AW_PRECISION_MIXED)
        k_gradient<double><<<G.nb, 128, 0, s>>>(G.view0(), B.p64.p, B.fluid.p, (float*)W[0], (float*)W[1],
                                                (float*)W[2], d.dt, U[0], U[1], U[2]);
    else
        k_gradient<float><<<G.nb, 128, 0, s>>>(G.view0(), B.p32.p, B.fluid.p, (float*)W[0], (float*)W[1], (float*)W[2],
                                               d.dt, U[0], U[1], U[2]);
    AW_LAUNCH();
    AW_TRY(face_sync(G, U, s));
    AW_TRY(wall_bc(G, U, s));
    k_divergence<<<G.nb, 128, 0, s>>>(G.view0(), U[0], U[1], U[2], B.fluid.p, 1.f / d.dt, nullptr, B.divmax.p + 1);
    AW_LAUNCH();
    if (rec)
        for (int a = 0; a < 3; ++a) {
            AW_TRY(copy_d2d(rec->u6[a].p, U[a], fb[a], s));
            AW_TRY(copy_d2d(rec->uo[a].p, UO[a], fb[a], s));
        }
    if (ev) AW_CUDA(cudaEventRecord(ev[5], s));
    // 7. G2P (FLIP blend) on the sorted SoA particles
    const float* un[3] = {U[0], U[1], U[2]};
    const float* uo[3] = {UO[0], UO[1], UO[2]};
    AW_TRY(g2p_sorted(G, soa_out, n, G.pw.cell_start.p, d.alpha, un, uo, s));
    if (ev) AW_CUDA(cudaEventRecord(ev[6], s));
    // 8. RK3 advection through the u_new tiles built for G2P
    AW_TRY(advect_sorted(G, soa_out, n, G.pw.cell_start.p, d.dt, un, s));
    if (ev) AW_CUDA(cudaEventRecord(ev[7], s));
    if (st) {
        if (ev) AW_CUDA(cudaEventSynchronize(ev[7]));
        AW_TRY(check_device_errors(G, s));
        float dm[2];
        AW_CUDA(cudaMemcpyAsync(dm, B.divmax.p, sizeof dm, cudaMemcpyDeviceToHost, s));
        AW_CUDA(cudaStreamSynchronize(s));
        st->div_before = dm[0];
        st->div_after = dm[1];
        if (ev) {
            float t[7];
            for (int k = 0; k < 7; ++k) AW_CUDA(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]));
            st->ms_sort = t[0];
            st->ms_p2g = t[1];
            st->ms_other = t[2] + t[4];
            st->ms_solve = t[3];
            st->ms_g2p = t[5];
            st->ms_advect = t[6];
        }
    }
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
    aw_solver_desc sd{};
    FlipBufs B;
    DBuf<float> phase;  // two-phase: phase by particle id (empty = one phase)
    float rho0 = 1.f, rho1 = 1.f;
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
        AW_TRY(F->soa[k].alloc((size_t)std::max<int64_t>(n, 1) * 6 + kSoaPad));
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
    F->sd = sd;
    AW_TRY(aw_solver_create(g, &sd, &F->solver));
    AW_TRY(F->B.ensure(G));
    for (auto& e : F->ev) AW_CUDA(cudaEventCreate(&e));
    *out = F.release();
    return AW_OK;
}

extern "C" aw_status aw_flip_set_phase(aw_flip* F, const float* h_phase, float rho0, float rho1) {
    AW_CHECK_ARG(F, "null simulation");
    if (!h_phase) {
        F->phase.free();
        F->rho0 = F->rho1 = 1.f;
        MsbgState& G = F->g->st;
        for (int a = 0; a < 3; ++a)
            if (G.tot[1 + a]) {
                k_fill<<<nblk(G.tot[1 + a]), 256>>>(G.ch[AW_BETA_COEFF_X + a], G.tot[1 + a], 1.f);
                AW_LAUNCH();
            }
        AW_TRY(aw_solver_update_coefficients(F->solver, 0));
        AW_CUDA(cudaStreamSynchronize(0));
        return AW_OK;
    }
    AW_CHECK_ARG(std::isfinite(rho0) && std::isfinite(rho1) && rho0 > 0.f && rho1 > 0.f, "densities must be positive");
    for (int64_t i = 0; i < F->n; ++i)
        AW_CHECK_ARG(h_phase[i] >= 0.f && h_phase[i] <= 1.f, "phase must lie in [0, 1]");
    AW_TRY(F->phase.alloc((size_t)std::max<int64_t>(F->n, 1)));
    if (F->n) AW_CUDA(cudaMemcpy(F->phase.p, h_phase, (size_t)F->n * sizeof(float), cudaMemcpyHostToDevice));
    F->rho0 = rho0;
    F->rho1 = rho1;
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
    const int c = F->cur;
    const FlipPhase fp{F->phase.p, F->rho0, F->rho1};
    aw_status st = flip_step_soa(F->g->st, F->solver, F->d, F->B, F->soa[c].p, F->ids[c].p, F->soa[c ^ 1].p,
                                 F->ids[c ^ 1].p, F->n, nullptr, nullptr, F->ev, &F->stats, s,
                                 F->phase.p ? &fp : nullptr, /*warm_start=*/true);
    F->cur ^= 1;  // the sorted state lives in the other buffer from the gather on
    return st;
}

extern "C" aw_status aw_flip_rebuild_levels(aw_flip* F, const int32_t* h_thresholds, int32_t* changed, aw_stream s_) {
    AW_CHECK_ARG(F, "null simulation");
    cudaStream_t s = (cudaStream_t)s_;
    MsbgState& G = F->g->st;
    if (changed) *changed = 0;
    const float* soa = F->soa[F->cur].p;
    // map, grading and comparison on the device; the host reads one count
    int ndiff = 0;
    AW_TRY(relevel_on_device(G, soa, 1, F->n, F->n, h_thresholds, &ndiff, nullptr, s));
    if (ndiff == 0) {  // same layout: keep the channels and the solver
        G.allocated = true;
        return AW_OK;
    }
    // a new layout: channels, tiles and the solver hierarchy follow it, in the storage they had
    // (grow-only buffers); the particles carry the state
    AW_TRY(aw_msbg_allocate(F->g, s_));
    if (F->solver) AW_TRY(solver_relayout(F->solver));
    else AW_TRY(aw_solver_create(F->g, &F->sd, &F->solver));
    AW_TRY(F->B.ensure(G));
    F->B.p_warm = false;  // cell indices changed
    if (changed) *changed = 1;
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

extern "C" aw_status aw_velocity_divergence_max64(aw_msbg* g, const uint8_t* d_fluid, double* d_max, aw_stream s) {
    AW_CHECK_ARG(g && d_max && g->st.allocated, "bad argument");
    MsbgState& G = g->st;
    AW_CUDA(cudaMemsetAsync(d_max, 0, sizeof(double), (cudaStream_t)s));
    k_divergence_max64<<<G.nb, 128, 0, (cudaStream_t)s>>>(G.view0(), G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y],
                                                          G.ch[AW_VELOCITY_Z], d_fluid, (unsigned long long*)d_max);
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
