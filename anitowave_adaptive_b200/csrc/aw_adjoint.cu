// aw_adjoint.cu — vector-Jacobian products of the FLIP step and a differentiable rollout with
// checkpointing.  No counterpart in the reference (it has no time loop and no gradients).
//
// The map differentiated is the FLIP step of aw_flip_step with its discrete decisions held: the
// cell and block of every particle and sample point, the fluid flags, each P2G kernel's support
// and the clamp branches of sampling and advection.  The adjoints:
//   P2G + normalise   -> a G2P-shaped gather (k_p2g_vjp, one thread per particle)
//   G2P, RK3, sample  -> a P2G-shaped scatter into ghosted adjoint tiles, folded onto the faces
//                        that supplied each tile entry (k_step_particles_vjp, k_tile_fold)
//   projection        -> walls, sync, gradient and divergence transposed around one more solve
//                        with the same multigrid hierarchy (the finite-volume operator is
//                        symmetric, so A^-T = A^-1)
// The rollout keeps the particle state of every `checkpoint_every`-th step on the device; the
// backward pass recomputes each segment from its checkpoint, recording what the step adjoints
// need, and runs the step adjoints in reverse.
#include <algorithm>
#include <cmath>
#include <memory>

#include "aw_internal.cuh"

namespace aw {

static inline unsigned nblk(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

__global__ void k_iota(uint32_t* p, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = (uint32_t)i;
}

// AoS (3 n) -> SoA rows of `out` (first 3 n of a 6 n state)
__global__ void k_aos_to_soa3(const float* __restrict__ in, int64_t n, float* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int a = 0; a < 3; ++a) out[(int64_t)a * n + i] = in[3 * i + a];
}

// SoA positions of the state, written in particle-id order as AoS
__global__ void k_soa_to_aos_by_id(const float* __restrict__ soa, const uint32_t* __restrict__ ids, int64_t n,
                                   float* __restrict__ out) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = ids[j];
#pragma unroll
    for (int a = 0; a < 3; ++a) out[3 * (int64_t)i + a] = soa[(int64_t)a * n + j];
}

// loss = mean_i |x_i - target_{id(i)}|^2 (sum accumulated in FP64); optionally the loss gradient
// xbar = 2 (x - target) / n and vbar = 0 in the state's order
__global__ void k_loss(const float* __restrict__ soa, const uint32_t* __restrict__ ids, int64_t n,
                       const float* __restrict__ target, double* sum, float* bar) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double acc = 0.0;
    if (j < n) {
        const uint32_t i = ids[j];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float d = soa[(int64_t)a * n + j] - target[3 * (int64_t)i + a];
            acc += (double)d * d;
            if (bar) {
                bar[(int64_t)a * n + j] = 2.f * d / (float)n;
                bar[(int64_t)(3 + a) * n + j] = 0.f;
            }
        }
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(sum, acc);
}

__global__ void k_add_into(float* __restrict__ y, const float* __restrict__ x, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
}

// Face adjoint buffers of one grid (three axes).
struct FaceBar {
    DBuf<float> a[3];
    float* p[3] = {nullptr, nullptr, nullptr};
    aw_status ensure(const MsbgState& G) {
        for (int k = 0; k < 3; ++k) {
            AW_TRY(a[k].ensure(std::max<uint32_t>(G.tot[1 + k], 1)));
            p[k] = a[k].p;
        }
        return AW_OK;
    }
    aw_status zero(const MsbgState& G, cudaStream_t s) {
        for (int k = 0; k < 3; ++k)
            if (G.tot[1 + k]) AW_CUDA(cudaMemsetAsync(p[k], 0, G.tot[1 + k] * sizeof(float), s));
        return AW_OK;
    }
};

// Adjoint of one FLIP step.  bar_sorted (6 n SoA: xbar, vbar) holds the adjoint of the step's
// output state (the step's sorted order) and is consumed; bar_in receives the adjoint of the
// step's input state in the input order.
static aw_status flip_step_vjp(MsbgState& G, aw_solver* sv, const aw_flip_desc& d, FlipBufs& B, StepRecord& R,
                               int64_t n, float* bar_sorted, float* bar_in, FaceBar& un, FaceBar& uo, cudaStream_t s) {
    AW_TRY(un.ensure(G));
    AW_TRY(uo.ensure(G));
    AW_TRY(un.zero(G, s));
    AW_TRY(uo.zero(G, s));
    const float* x = R.soa.p;
    const float* v = R.soa.p + 3 * n;
    const float* u6[3] = {R.u6[0].p, R.u6[1].p, R.u6[2].p};
    const float* uold[3] = {R.uo[0].p, R.uo[1].p, R.uo[2].p};
    // RK3 advection and the FLIP blend
    AW_TRY(step_particles_vjp(G, x, 1, n, d.alpha, d.dt, u6, uold, bar_sorted, bar_sorted + 3 * n, 1, 1, un.p, uo.p, s));
    // projection (walls, sync, gradient, solve, divergence)
    AW_TRY(aw_solver_setup(sv, R.fluid.p, (aw_stream)s));
    AW_TRY(project_vjp(G, sv, R.fluid.p, d.dt, d.precision, un.p, B, s));
    // walls before the divergence; gravity is a constant shift; the backup copies u2 into u_old
    AW_TRY(wall_bc(G, un.p, s));
    for (int a = 0; a < 3; ++a)
        if (G.tot[1 + a]) {
            k_add_into<<<nblk(G.tot[1 + a]), 256, 0, s>>>(un.p[a], uo.p[a], G.tot[1 + a]);
            AW_LAUNCH();
        }
    // T-junction sync after P2G
    AW_TRY(face_sync_vjp(G, un.p, s));
    // P2G with its normalisation
    const float* u1[3] = {R.u1[0].p, R.u1[1].p, R.u1[2].p};
    const float* m[3] = {R.m[0].p, R.m[1].p, R.m[2].p};
    const float* ub[3] = {un.p[0], un.p[1], un.p[2]};
    AW_TRY(p2g_vjp(G, x, v, 1, n, u1, m, ub, bar_sorted, bar_sorted + 3 * n, s));
    // the sort's gather, transposed
    return unsort6(R.perm.p, n, bar_sorted, bar_in, s);
}

}  // namespace aw

using namespace aw;

struct aw_rollout {
    aw_msbg* g = nullptr;
    aw_flip_desc d{};
    int64_t n = 0;
    int steps = 0, every = 1;
    aw_solver* solver = nullptr;
    FlipBufs B;
    DBuf<float> state[2];  // 6 n SoA ping-pong
    DBuf<uint32_t> ids[2];
    DBuf<float> pos0;  // initial positions, SoA 3 n
    DBuf<float> u0;    // initial face field of the last forward (three axes concatenated)
    DBuf<float> target;
    std::vector<DBuf<float>> ck_state;
    std::vector<DBuf<uint32_t>> ck_ids;
    std::vector<DBuf<uint8_t>> fluids;  // fluid flags of every forward step
    std::vector<StepRecord> recs;
    DBuf<float> bar[2];
    FaceBar un, uo;
    DBuf<double> loss;
    int final_cur = 0;
    bool have_forward = false, have_flags = false;
    ~aw_rollout() {
        if (solver) aw_solver_destroy(solver);
    }
};

extern "C" aw_status aw_rollout_create(aw_msbg* g, const aw_flip_desc* desc, const float* d_pos0, int64_t n,
                                       int32_t steps, int32_t checkpoint_every, aw_rollout** out) {
    AW_CHECK_ARG(g && desc && out && (d_pos0 || n == 0) && n >= 0 && n < (int64_t)0xFFFFFFFF, "bad argument");
    AW_CHECK_ARG(steps >= 0 && checkpoint_every >= 1, "steps must be >= 0 and checkpoint_every >= 1");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    *out = nullptr;
    std::unique_ptr<aw_rollout> R(new aw_rollout());
    MsbgState& G = g->st;
    R->g = g;
    R->d = *desc;
    R->n = n;
    R->steps = steps;
    R->every = checkpoint_every;
    const size_t np = (size_t)std::max<int64_t>(n, 1);
    for (int k = 0; k < 2; ++k) {
        AW_TRY(R->state[k].alloc(6 * np + kSoaPad));
        AW_TRY(R->ids[k].alloc(np));
        AW_TRY(R->bar[k].alloc(6 * np));
    }
    AW_TRY(R->pos0.alloc(3 * np));
    const size_t nfaces = (size_t)G.tot[1] + G.tot[2] + G.tot[3];
    AW_TRY(R->u0.alloc(std::max<size_t>(nfaces, 1)));
    AW_TRY(R->target.alloc(3 * np));
    const int nck = steps == 0 ? 0 : (steps + checkpoint_every - 1) / checkpoint_every;
    R->ck_state.resize(nck);
    R->ck_ids.resize(nck);
    for (int c = 0; c < nck; ++c) {
        AW_TRY(R->ck_state[c].alloc(6 * np));
        AW_TRY(R->ck_ids[c].alloc(np));
    }
    R->fluids.resize(steps);
    for (int k = 0; k < steps; ++k) AW_TRY(R->fluids[k].alloc(std::max<uint32_t>(G.tot[0], 1)));
    R->recs.resize(std::min(steps, checkpoint_every));
    AW_TRY(R->loss.alloc(1));
    if (n) {
        k_aos_to_soa3<<<nblk(n), 256>>>(d_pos0, n, R->pos0.p);
        AW_LAUNCH();
    }
    aw_solver_desc sd;
    AW_TRY(aw_solver_default_desc(AW_OPERATOR_FV, &sd));
    sd.precision = desc->precision;
    sd.tolerance = desc->tolerance;
    sd.max_cycles = desc->max_cycles;
    AW_TRY(aw_solver_create(g, &sd, &R->solver));
    AW_TRY(R->B.ensure(G));
    AW_CUDA(cudaDeviceSynchronize());
    *out = R.release();
    return AW_OK;
}

extern "C" aw_status aw_rollout_destroy(aw_rollout* r) {
    delete r;
    return AW_OK;
}

static const float* face_ptr(const aw_rollout* R, const float* base, int a) {
    const MsbgState& G = R->g->st;
    size_t o = 0;
    for (int k = 0; k < a; ++k) o += G.tot[1 + k];
    return base + o;
}

extern "C" aw_status aw_rollout_forward(aw_rollout* R, const float* d_u0, const float* d_target, int32_t freeze_fluid,
                                        double* loss, aw_stream s_) {
    AW_CHECK_ARG(R && d_u0 && (d_target || R->n == 0) && loss, "null argument");
    AW_CHECK_ARG(!freeze_fluid || R->have_flags, "freeze_fluid needs an earlier forward without it");
    cudaStream_t s = (cudaStream_t)s_;
    MsbgState& G = R->g->st;
    const int64_t n = R->n;
    const size_t nfaces = (size_t)G.tot[1] + G.tot[2] + G.tot[3];
    if (nfaces) AW_CUDA(cudaMemcpyAsync(R->u0.p, d_u0, nfaces * sizeof(float), cudaMemcpyDeviceToDevice, s));
    if (n) AW_CUDA(cudaMemcpyAsync(R->target.p, d_target, 3 * n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    // initial state: positions, velocities sampled from u0, ids in particle order
    int cur = 0;
    if (n) {
        AW_CUDA(cudaMemcpyAsync(R->state[0].p, R->pos0.p, 3 * n * sizeof(float), cudaMemcpyDeviceToDevice, s));
        const float* u[3] = {face_ptr(R, R->u0.p, 0), face_ptr(R, R->u0.p, 1), face_ptr(R, R->u0.p, 2)};
        AW_TRY(sample_soa(G, R->pos0.p, n, u, R->state[0].p + 3 * n, s));
        k_iota<<<nblk(n), 256, 0, s>>>(R->ids[0].p, n);
        AW_LAUNCH();
    }
    for (int k = 0; k < R->steps; ++k) {
        if (k % R->every == 0) {
            const int c = k / R->every;
            AW_CUDA(cudaMemcpyAsync(R->ck_state[c].p, R->state[cur].p, 6 * n * sizeof(float), cudaMemcpyDeviceToDevice, s));
            AW_CUDA(cudaMemcpyAsync(R->ck_ids[c].p, R->ids[cur].p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        }
        AW_TRY(flip_step_soa(G, R->solver, R->d, R->B, R->state[cur].p, R->ids[cur].p, R->state[cur ^ 1].p,
                             R->ids[cur ^ 1].p, n, freeze_fluid ? R->fluids[k].p : nullptr, nullptr, nullptr, nullptr, s));
        if (!freeze_fluid)
            AW_CUDA(cudaMemcpyAsync(R->fluids[k].p, R->B.fluid.p, G.tot[0], cudaMemcpyDeviceToDevice, s));
        cur ^= 1;
    }
    AW_CUDA(cudaMemsetAsync(R->loss.p, 0, sizeof(double), s));
    if (n) {
        k_loss<<<nblk(n), 256, 0, s>>>(R->state[cur].p, R->ids[cur].p, n, R->target.p, R->loss.p, nullptr);
        AW_LAUNCH();
    }
    double h = 0;
    AW_CUDA(cudaMemcpyAsync(&h, R->loss.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    AW_CUDA(cudaStreamSynchronize(s));
    AW_TRY(check_device_errors(G, s));
    *loss = n ? h / (double)n : 0.0;
    R->final_cur = cur;
    R->have_forward = true;
    if (!freeze_fluid) R->have_flags = true;
    return AW_OK;
}

extern "C" aw_status aw_rollout_final_positions(aw_rollout* R, float* d_pos, aw_stream s_) {
    AW_CHECK_ARG(R && (d_pos || R->n == 0), "null argument");
    AW_CHECK_ARG(R->have_forward, "no forward run yet");
    if (!R->n) return AW_OK;
    const int c = R->final_cur;
    k_soa_to_aos_by_id<<<nblk(R->n), 256, 0, (cudaStream_t)s_>>>(R->state[c].p, R->ids[c].p, R->n, d_pos);
    AW_LAUNCH();
    return AW_OK;
}

extern "C" aw_status aw_vjp_rollout(aw_rollout* R, float* d_u0_bar, aw_stream s_) {
    AW_CHECK_ARG(R && d_u0_bar, "null argument");
    AW_CHECK_ARG(R->have_forward, "aw_vjp_rollout needs aw_rollout_forward first");
    cudaStream_t s = (cudaStream_t)s_;
    MsbgState& G = R->g->st;
    const int64_t n = R->n;
    const size_t nfaces = (size_t)G.tot[1] + G.tot[2] + G.tot[3];
    if (nfaces) AW_CUDA(cudaMemsetAsync(d_u0_bar, 0, nfaces * sizeof(float), s));
    if (!n) return AW_OK;
    // loss gradient in the final state's order
    AW_CUDA(cudaMemsetAsync(R->loss.p, 0, sizeof(double), s));
    const int fc = R->final_cur;
    k_loss<<<nblk(n), 256, 0, s>>>(R->state[fc].p, R->ids[fc].p, n, R->target.p, R->loss.p, R->bar[0].p);
    AW_LAUNCH();
    int cb = 0;
    const int nseg = R->steps == 0 ? 0 : (R->steps + R->every - 1) / R->every;
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int k0 = seg * R->every, k1 = std::min(R->steps, k0 + R->every);
        // recompute the segment from its checkpoint with the forward's fluid flags, recording
        int cur = 0;
        AW_CUDA(cudaMemcpyAsync(R->state[0].p, R->ck_state[seg].p, 6 * n * sizeof(float), cudaMemcpyDeviceToDevice, s));
        AW_CUDA(cudaMemcpyAsync(R->ids[0].p, R->ck_ids[seg].p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        for (int k = k0; k < k1; ++k) {
            AW_TRY(flip_step_soa(G, R->solver, R->d, R->B, R->state[cur].p, R->ids[cur].p, R->state[cur ^ 1].p,
                                 R->ids[cur ^ 1].p, n, R->fluids[k].p, &R->recs[k - k0], nullptr, nullptr, s));
            cur ^= 1;
        }
        for (int k = k1 - 1; k >= k0; --k) {
            AW_TRY(flip_step_vjp(G, R->solver, R->d, R->B, R->recs[k - k0], n, R->bar[cb].p, R->bar[cb ^ 1].p, R->un,
                                 R->uo, s));
            cb ^= 1;
        }
    }
    // v0 = sample(u0, x0): u0_bar = I^T v0_bar (the initial state is in particle order)
    float* ub[3] = {d_u0_bar, d_u0_bar + G.tot[1], d_u0_bar + G.tot[1] + G.tot[2]};
    const float* u[3] = {face_ptr(R, R->u0.p, 0), face_ptr(R, R->u0.p, 1), face_ptr(R, R->u0.p, 2)};
    AW_TRY(sample_vjp(G, R->pos0.p, 1, n, u, R->bar[cb].p + 3 * n, 1, ub, nullptr, s));
    AW_CUDA(cudaStreamSynchronize(s));
    AW_TRY(check_device_errors(G, s));
    // the recompute overwrote the state buffers: the forward's final state is gone
    R->have_forward = false;
    return AW_OK;
}

// ---- VJPs of the single C-ABI calls -----------------------------------------------------------
extern "C" aw_status aw_vjp_p2g(aw_msbg* g, const float* d_pos, const float* d_vel, int64_t n, const float* const d_u_bar[3],
                                float* d_pos_bar, float* d_vel_bar, aw_stream s_) {
    AW_CHECK_ARG(g && n >= 0 && n < (int64_t)0xFFFFFFFF && (n == 0 || (d_pos && d_vel && d_u_bar && d_pos_bar && d_vel_bar)),
                 "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    if (!n) return AW_OK;
    cudaStream_t s = (cudaStream_t)s_;
    MsbgState& G = g->st;
    float* u[3];
    float* m[3];
    for (int a = 0; a < 3; ++a) {
        AW_TRY(G.adj_u[a].ensure(std::max<uint32_t>(G.tot[1 + a], 1)));
        AW_TRY(G.adj_m[a].ensure(std::max<uint32_t>(G.tot[1 + a], 1)));
        u[a] = G.adj_u[a].p;
        m[a] = G.adj_m[a].p;
    }
    // the forward mass and velocity of these particles (the grid's channels stay untouched)
    AW_TRY(sort_particles_soa(G, d_pos, d_vel, n, s));
    float* nomom[3] = {nullptr, nullptr, nullptr};
    AW_TRY(p2g_sorted(G, G.pw.soa.p, n, G.pw.cell_start.p, u, m, nomom, nullptr, s));
    const float* cu[3] = {u[0], u[1], u[2]};
    const float* cm[3] = {m[0], m[1], m[2]};
    const float* ub[3] = {d_u_bar[0], d_u_bar[1], d_u_bar[2]};
    return p2g_vjp(G, d_pos, d_vel, 0, n, cu, cm, ub, d_pos_bar, d_vel_bar, s);
}

extern "C" aw_status aw_vjp_g2p(aw_msbg* g, const float* d_pos, int64_t n, float alpha, float* d_vel_bar,
                                float* d_pos_bar, float* const d_un_bar[3], float* const d_uo_bar[3], aw_stream s_) {
    AW_CHECK_ARG(g && n >= 0 && (n == 0 || (d_pos && d_vel_bar && d_pos_bar && d_un_bar && d_uo_bar)), "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    if (!n) return AW_OK;
    MsbgState& G = g->st;
    const float* un[3] = {G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]};
    const float* uo[3] = {G.ch[AW_VELOCITY_OLD_X], G.ch[AW_VELOCITY_OLD_Y], G.ch[AW_VELOCITY_OLD_Z]};
    float* unb[3] = {d_un_bar[0], d_un_bar[1], d_un_bar[2]};
    float* uob[3] = {d_uo_bar[0], d_uo_bar[1], d_uo_bar[2]};
    return step_particles_vjp(G, d_pos, 0, n, alpha, 0.f, un, uo, d_pos_bar, d_vel_bar, 0, 0, unb, uob,
                              (cudaStream_t)s_);
}

extern "C" aw_status aw_vjp_advect(aw_msbg* g, const float* d_pos, int64_t n, float dt, float* d_pos_bar,
                                   float* const d_u_bar[3], aw_stream s_) {
    AW_CHECK_ARG(g && n >= 0 && (n == 0 || (d_pos && d_pos_bar && d_u_bar)), "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    if (!n) return AW_OK;
    MsbgState& G = g->st;
    const float* u[3] = {G.ch[AW_VELOCITY_X], G.ch[AW_VELOCITY_Y], G.ch[AW_VELOCITY_Z]};
    float* ub[3] = {d_u_bar[0], d_u_bar[1], d_u_bar[2]};
    return step_particles_vjp(G, d_pos, 0, n, 0.f, dt, u, u, d_pos_bar, nullptr, 0, 1, ub, nullptr, (cudaStream_t)s_);
}

extern "C" aw_status aw_vjp_sample(aw_msbg* g, const float* d_points, int64_t n, int32_t old, const float* d_out_bar,
                                   float* const d_u_bar[3], float* d_points_bar, aw_stream s_) {
    AW_CHECK_ARG(g && n >= 0 && (n == 0 || (d_points && d_out_bar && d_u_bar)), "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    if (!n) return AW_OK;
    MsbgState& G = g->st;
    const int base = old ? AW_VELOCITY_OLD_X : AW_VELOCITY_X;
    const float* u[3] = {G.ch[base], G.ch[base + 1], G.ch[base + 2]};
    float* ub[3] = {d_u_bar[0], d_u_bar[1], d_u_bar[2]};
    return sample_vjp(G, d_points, 0, n, u, d_out_bar, 0, ub, d_points_bar, (cudaStream_t)s_);
}

extern "C" aw_status aw_project(aw_msbg* g, aw_solver* sv, const uint8_t* d_fluid, float dt, aw_stream s_) {
    AW_CHECK_ARG(g && sv && d_fluid && dt > 0.f, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    int32_t prec;
    AW_TRY(aw_solver_precision(sv, &prec));
    AW_TRY(aw_solver_setup(sv, d_fluid, s_));
    return project_forward(g->st, sv, d_fluid, dt, prec, g->st.proj, (cudaStream_t)s_);
}

extern "C" aw_status aw_vjp_project(aw_msbg* g, aw_solver* sv, const uint8_t* d_fluid, float dt, float* const d_u_bar[3],
                                    aw_stream s_) {
    AW_CHECK_ARG(g && sv && d_fluid && d_u_bar && dt > 0.f, "bad argument");
    AW_CHECK_ARG(g->st.allocated, "grid not allocated");
    int32_t prec;
    AW_TRY(aw_solver_precision(sv, &prec));
    AW_TRY(aw_solver_setup(sv, d_fluid, s_));
    float* ub[3] = {d_u_bar[0], d_u_bar[1], d_u_bar[2]};
    return project_vjp(g->st, sv, d_fluid, dt, prec, ub, g->st.proj, (cudaStream_t)s_);
}
