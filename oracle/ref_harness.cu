// ref_harness.cu — C-ABI harness around the reference's OWN CUDA kernels and managers.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/build_ref.py directly against the reference
// headers where they lie (include path = <reference root>/include); nothing of the reference is
// copied.  The output goes to oracle/_ref/libawref.so, is used by tests/golden/make_ref_golden.py
// on a GPU box to produce the committed fixtures, and by oracle/ref_timing.py for timings.
//
// The reference compiles its constants in: BLOCK_BASE_RES 16, MAX_LEVELS 3 (MSBG.cuh:4-5).
// Calls are restricted to the inputs on which the reference is memory-safe and well defined:
// single-level (or level-uniform) maps with every block active (the reference-exact tier).  The smoother
// is driven with one thread per CTA: smoothActiveBlocks' early exit is evaluated by thread 0
// only (Smoother.cuh:183-185), so a 1-thread CTA is the launch shape in which that exit is
// block-uniform and the kernel is free of the divergent barrier.
// the reference headers rely on the includes that precede them in main.cu:1-4
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <vector>
#include <algorithm>
#include <thrust/device_ptr.h>
#include <thrust/scan.h>

#include <MSBG.cuh>
#include <P2G.cuh>
#include <VCycle.cuh>
#include <G2P.cuh>

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {

struct Grid {
    MSBGManager* mg = nullptr;
    std::vector<uint32_t> h_level;
    ~Grid() { delete mg; }
};

// Setup sequence of main.cu:98-278 with a given refinement map (no markActiveBlocks).
Grid* make_grid(const int dims[3], const uint32_t* levels, bool channels) {
    Grid* G = new Grid();
    G->mg = new MSBGManager(make_int3(dims[0], dims[1], dims[2]), 1.0f, make_float3(0, 0, 0));
    MSBG& g = G->mg->grid;
    G->h_level.assign(levels, levels + g.numBlocks);
    cudaMemcpy(g.d_refinementMap, levels, g.numBlocks * sizeof(uint32_t), cudaMemcpyHostToDevice);
    uint32_t *c, *fx, *fy, *fz;
    cudaMalloc(&c, g.numBlocks * sizeof(uint32_t));
    cudaMalloc(&fx, g.numBlocks * sizeof(uint32_t));
    cudaMalloc(&fy, g.numBlocks * sizeof(uint32_t));
    cudaMalloc(&fz, g.numBlocks * sizeof(uint32_t));
    int nb = (g.numBlocks + 255) / 256;
    countBlockElements<<<nb, 256>>>(g.d_refinementMap, c, fx, fy, fz, g.numBlocks);
    cudaDeviceSynchronize();
    std::vector<uint32_t> hc(g.numBlocks), hx(g.numBlocks), hy(g.numBlocks), hz(g.numBlocks);
    cudaMemcpy(hc.data(), c, g.numBlocks * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hx.data(), fx, g.numBlocks * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hy.data(), fy, g.numBlocks * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hz.data(), fz, g.numBlocks * 4, cudaMemcpyDeviceToHost);
    g.totalCells = g.totalFacesX = g.totalFacesY = g.totalFacesZ = 0;
    for (uint32_t i = 0; i < g.numBlocks; ++i) {
        g.totalCells += hc[i];
        g.totalFacesX += hx[i];
        g.totalFacesY += hy[i];
        g.totalFacesZ += hz[i];
    }
    thrust::exclusive_scan(thrust::device_ptr<uint32_t>(c), thrust::device_ptr<uint32_t>(c) + g.numBlocks,
                           thrust::device_ptr<uint32_t>(g.d_cellOffsets));
    thrust::exclusive_scan(thrust::device_ptr<uint32_t>(fx), thrust::device_ptr<uint32_t>(fx) + g.numBlocks,
                           thrust::device_ptr<uint32_t>(g.d_faceXOffsets));
    thrust::exclusive_scan(thrust::device_ptr<uint32_t>(fy), thrust::device_ptr<uint32_t>(fy) + g.numBlocks,
                           thrust::device_ptr<uint32_t>(g.d_faceYOffsets));
    thrust::exclusive_scan(thrust::device_ptr<uint32_t>(fz), thrust::device_ptr<uint32_t>(fz) + g.numBlocks,
                           thrust::device_ptr<uint32_t>(g.d_faceZOffsets));
    cudaDeviceSynchronize();
    cudaFree(c);
    cudaFree(fx);
    cudaFree(fy);
    cudaFree(fz);
    if (channels) G->mg->allocateChannels();
    return G;
}

std::vector<float*> channel_table(const float* const* dev_table) {
    std::vector<float*> h(NUM_CHANNELS);
    cudaMemcpy(h.data(), dev_table, NUM_CHANNELS * sizeof(float*), cudaMemcpyDeviceToHost);
    return h;
}

float* upload(const float* h, size_t n) {
    float* d = nullptr;
    cudaMalloc(&d, std::max<size_t>(n, 1) * sizeof(float));
    if (n) cudaMemcpy(d, h, n * sizeof(float), cudaMemcpyHostToDevice);
    return d;
}
void download(float* h, const float* d, size_t n) {
    if (n) cudaMemcpy(h, d, n * sizeof(float), cudaMemcpyDeviceToHost);
}

// AdaptiveSmoother::solveLevel (Smoother.cuh:249-291) with one thread per CTA.
void solve_level_1t(AdaptiveSmoother& sm, MSBGManager& mg, int mgLevel, float* x, float* b, float* bx, float* by,
                    float* bz, uint32_t* c_off, uint32_t* fx_off, uint32_t* fy_off, uint32_t* fz_off, int iterations) {
    int curr = 0, next = 1;
    cudaMemset(sm.d_activeCount[curr], 0, sizeof(uint32_t));
    cudaMemset(sm.d_blockStatus[curr], 0, sm.numBlocks * sizeof(uint32_t));
    int blocks = (sm.numBlocks + 255) / 256;
    initActiveBlocks<<<blocks, 256>>>(mg.grid, sm.d_activeList[curr], sm.d_activeCount[curr], sm.d_blockStatus[curr],
                                      MAX_LEVELS - 1, mgLevel);
    cudaDeviceSynchronize();
    for (int iter = 0; iter < iterations; iter++) {
        uint32_t h_count = 0;
        cudaMemcpy(&h_count, sm.d_activeCount[curr], sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (h_count == 0) break;
        thrust::device_ptr<uint32_t> ptr(sm.d_activeList[curr]);
        MortonCompare comp(mg.grid.d_blockInfo);
        thrust::sort(thrust::device, ptr, ptr + h_count, comp);
        cudaMemset(sm.d_activeCount[next], 0, sizeof(uint32_t));
        cudaMemset(sm.d_blockStatus[next], 0, sm.numBlocks * sizeof(uint32_t));
        for (int rb = 0; rb < 2; rb++) {
            smoothActiveBlocks<<<h_count, 1>>>(mg.grid, x, b, bx, by, bz, c_off, fx_off, fy_off, fz_off,
                                               sm.d_activeList[curr], h_count, sm.d_activeList[next],
                                               sm.d_activeCount[next], sm.d_blockStatus[next], rb, 1e-4f, mgLevel);
        }
        cudaDeviceSynchronize();
        std::swap(curr, next);
    }
}

// VCycleSolver::runCycle (VCycle.cuh:251-304) with the 1-thread smoother driver.
void run_cycle_1t(VCycleSolver& S, MSBGManager& mg, int level) {
    if (level == S.maxLevels - 1) {
        solve_level_1t(S.smoother, mg, level, S.levels_x[level], S.levels_b[level], S.levels_beta_x[level],
                       S.levels_beta_y[level], S.levels_beta_z[level], S.levels_c_off[level], S.levels_fx_off[level],
                       S.levels_fy_off[level], S.levels_fz_off[level], 50);
        return;
    }
    solve_level_1t(S.smoother, mg, level, S.levels_x[level], S.levels_b[level], S.levels_beta_x[level],
                   S.levels_beta_y[level], S.levels_beta_z[level], S.levels_c_off[level], S.levels_fx_off[level],
                   S.levels_fy_off[level], S.levels_fz_off[level], 2);
    float* r;
    cudaMalloc(&r, std::max<uint32_t>(S.levels_total_cells[level], 1) * sizeof(float));
    computeExplicitResidual<<<mg.grid.numBlocks, 256>>>(
        mg.grid, S.levels_c_off[level], S.levels_fx_off[level], S.levels_beta_x[level], S.levels_fy_off[level],
        S.levels_beta_y[level], S.levels_fz_off[level], S.levels_beta_z[level], S.levels_x[level], S.levels_b[level], r,
        level);
    S.transfer.restrictResiduals(mg, r, S.levels_b[level + 1], S.levels_c_off[level], S.levels_c_off[level + 1], level);
    cudaFree(r);
    uint32_t cs = S.levels_total_cells[level + 1];
    if (cs > 0) zeroVector<<<(cs + 255) / 256, 256>>>(S.levels_x[level + 1], cs);
    run_cycle_1t(S, mg, level + 1);
    S.transfer.prolongateAndCorrect(mg, S.levels_x[level], S.levels_x[level + 1], S.levels_c_off[level],
                                    S.levels_c_off[level + 1], level);
    solve_level_1t(S.smoother, mg, level, S.levels_x[level], S.levels_b[level], S.levels_beta_x[level],
                   S.levels_beta_y[level], S.levels_beta_z[level], S.levels_c_off[level], S.levels_fx_off[level],
                   S.levels_fy_off[level], S.levels_fz_off[level], 2);
}

}  // namespace

REF_API int ref_constants(int out[2]) {
    out[0] = BLOCK_BASE_RES;
    out[1] = MAX_LEVELS;
    return 0;
}

REF_API int ref_device_ok(void) {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}

REF_API void ref_layout(int level, uint32_t out[6]) {
    BlockLayout l = computeBlockLayout((uint8_t)level);
    out[0] = l.numCells;
    out[1] = l.numFacesX;
    out[2] = l.numFacesY;
    out[3] = l.numFacesZ;
    out[4] = l.totalSize;
    out[5] = (uint32_t)l.res;
}

REF_API uint32_t ref_morton(uint32_t x, uint32_t y, uint32_t z) { return morton3D(x, y, z); }

// initBlockInfo (MSBG.cuh:256-269) via the MSBGManager constructor; out: 5 u32 per block
REF_API int ref_block_info(const int dims[3], uint32_t* out) {
    uint32_t nb = (uint32_t)dims[0] * dims[1] * dims[2];
    std::vector<uint32_t> lv(nb, 0);
    Grid* G = make_grid(dims, lv.data(), false);
    std::vector<BlockInfo> h(nb);
    cudaMemcpy(h.data(), G->mg->grid.d_blockInfo, nb * sizeof(BlockInfo), cudaMemcpyDeviceToHost);
    for (uint32_t b = 0; b < nb; ++b) {
        out[5 * b + 0] = (uint32_t)h[b].coord.x;
        out[5 * b + 1] = (uint32_t)h[b].coord.y;
        out[5 * b + 2] = (uint32_t)h[b].coord.z;
        out[5 * b + 3] = h[b].level;
        out[5 * b + 4] = h[b].morton;
    }
    delete G;
    return (int)cudaGetLastError();
}

// enforceGrading (MSBG.cuh:316-351) repeated until the map stops changing (max 64 passes)
REF_API int ref_grading(const int dims[3], uint32_t* levels, int* passes) {
    uint32_t nb = (uint32_t)dims[0] * dims[1] * dims[2];
    uint32_t* d;
    cudaMalloc(&d, nb * sizeof(uint32_t));
    cudaMemcpy(d, levels, nb * 4, cudaMemcpyHostToDevice);
    int3 D = make_int3(dims[0], dims[1], dims[2]);
    dim3 t(4, 4, 4), g((dims[0] + 3) / 4, (dims[1] + 3) / 4, (dims[2] + 3) / 4);
    std::vector<uint32_t> prev(levels, levels + nb), cur(nb);
    int p = 0;
    for (; p < 64; ++p) {
        enforceGrading<<<g, t>>>(d, D);
        cudaDeviceSynchronize();
        cudaMemcpy(cur.data(), d, nb * 4, cudaMemcpyDeviceToHost);
        if (cur == prev) break;
        prev = cur;
    }
    std::memcpy(levels, cur.data(), nb * 4);
    if (passes) *passes = p + 1;
    cudaFree(d);
    return (int)cudaGetLastError();
}

// countBlockElements + exclusive_scan (main.cu:224-273): out = 4*nb offsets, totals[4]
REF_API int ref_offsets(const int dims[3], const uint32_t* levels, uint32_t* out, uint32_t* totals) {
    Grid* G = make_grid(dims, levels, false);
    MSBG& g = G->mg->grid;
    uint32_t nb = g.numBlocks;
    cudaMemcpy(out, g.d_cellOffsets, nb * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(out + nb, g.d_faceXOffsets, nb * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(out + 2 * nb, g.d_faceYOffsets, nb * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(out + 3 * nb, g.d_faceZOffsets, nb * 4, cudaMemcpyDeviceToHost);
    totals[0] = g.totalCells;
    totals[1] = g.totalFacesX;
    totals[2] = g.totalFacesY;
    totals[3] = g.totalFacesZ;
    delete G;
    return (int)cudaGetLastError();
}

// computeCoarseOffsets / computeCoarseFaceOffsets (MSBG.cuh:679-745)
REF_API int ref_coarse_offsets(const int dims[3], const uint32_t* levels, int mgLevel, int kind, uint32_t* out,
                               uint32_t* total) {
    Grid* G = make_grid(dims, levels, false);
    uint32_t nb = G->mg->grid.numBlocks;
    uint32_t* d;
    cudaMalloc(&d, nb * 4);
    uint32_t t = 0;
    if (kind == 0) computeCoarseOffsets(*G->mg, mgLevel, d, t);
    else computeCoarseFaceOffsets(*G->mg, mgLevel, kind - 1, d, t);
    cudaMemcpy(out, d, nb * 4, cudaMemcpyDeviceToHost);
    *total = t;
    cudaFree(d);
    delete G;
    return (int)cudaGetLastError();
}

// MSBGManager::runGalerkin (MSBG.cuh:661-676) between the reference's coarse offsets
REF_API int ref_galerkin(const int dims[3], const uint32_t* levels, int dest, const float* const* fine,
                         float* const* coarse) {
    Grid* G = make_grid(dims, levels, false);
    uint32_t nb = G->mg->grid.numBlocks;
    uint32_t *fo[3], *co[3], tf[3], tc[3];
    float *df[3], *dc[3];
    for (int a = 0; a < 3; ++a) {
        cudaMalloc(&fo[a], nb * 4);
        cudaMalloc(&co[a], nb * 4);
        computeCoarseFaceOffsets(*G->mg, dest - 1, a, fo[a], tf[a]);
        computeCoarseFaceOffsets(*G->mg, dest, a, co[a], tc[a]);
        df[a] = upload(fine[a], tf[a]);
        cudaMalloc(&dc[a], std::max<uint32_t>(tc[a], 1) * 4);
        cudaMemset(dc[a], 0, std::max<uint32_t>(tc[a], 1) * 4);
    }
    G->mg->runGalerkin(df[0], df[1], df[2], fo[0], fo[1], fo[2], dc[0], dc[1], dc[2], co[0], co[1], co[2], dest);
    for (int a = 0; a < 3; ++a) {
        download(coarse[a], dc[a], tc[a]);
        cudaFree(df[a]);
        cudaFree(dc[a]);
        cudaFree(fo[a]);
        cudaFree(co[a]);
    }
    delete G;
    return (int)cudaGetLastError();
}

// MG-level kernels on the reference hierarchy built by VCycleSolver::init (VCycle.cuh:177-249).
// op: 0 = computeExplicitResidual, 1 = restrictResiduals (r of `level` -> b of level+1),
//     2 = prolongateAndCorrect (x of level+1 -> x of level), 3 = solveLevel(iterations),
//     4 = runCycle from `level` (1-thread smoother).
// io arrays (host, FP32): x[level], b[level], beta x/y/z[level] are uploaded (beta only when
// `set_beta`), then the op runs, then x, b, r of `level` and x, b of level+1 are downloaded.
REF_API int ref_mg_op(const int dims[3], const uint32_t* levels, const float* const* fine_beta, int level, int op,
                      int iterations, float* x, float* b, float* r, float* x1, float* b1, const float* xin1) {
    Grid* G = make_grid(dims, levels, true);
    MSBGManager& mg = *G->mg;
    std::vector<float*> fx = channel_table(mg.grid.d_faceXData), fy = channel_table(mg.grid.d_faceYData),
                        fz = channel_table(mg.grid.d_faceZData);
    cudaMemcpy(fx[BETA_COEFF_X], fine_beta[0], mg.grid.totalFacesX * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(fy[BETA_COEFF_Y], fine_beta[1], mg.grid.totalFacesY * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(fz[BETA_COEFF_Z], fine_beta[2], mg.grid.totalFacesZ * 4, cudaMemcpyHostToDevice);
    VCycleSolver S(MAX_LEVELS, mg.grid.numBlocks);
    S.init(mg);
    uint32_t n0 = S.levels_total_cells[level];
    uint32_t n1 = level + 1 < MAX_LEVELS ? S.levels_total_cells[level + 1] : 0;
    cudaMemcpy(S.levels_x[level], x, n0 * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(S.levels_b[level], b, n0 * 4, cudaMemcpyHostToDevice);
    if (n1 && xin1) cudaMemcpy(S.levels_x[level + 1], xin1, n1 * 4, cudaMemcpyHostToDevice);
    float* dr = nullptr;
    cudaMalloc(&dr, std::max<uint32_t>(n0, 1) * 4);
    cudaMemset(dr, 0, std::max<uint32_t>(n0, 1) * 4);
    if (op == 0 || op == 1) {
        computeExplicitResidual<<<mg.grid.numBlocks, 256>>>(
            mg.grid, S.levels_c_off[level], S.levels_fx_off[level], S.levels_beta_x[level], S.levels_fy_off[level],
            S.levels_beta_y[level], S.levels_fz_off[level], S.levels_beta_z[level], S.levels_x[level],
            S.levels_b[level], dr, level);
        cudaDeviceSynchronize();
        if (op == 1) S.transfer.restrictResiduals(mg, dr, S.levels_b[level + 1], S.levels_c_off[level],
                                                  S.levels_c_off[level + 1], level);
    } else if (op == 2) {
        S.transfer.prolongateAndCorrect(mg, S.levels_x[level], S.levels_x[level + 1], S.levels_c_off[level],
                                        S.levels_c_off[level + 1], level);
    } else if (op == 3) {
        solve_level_1t(S.smoother, mg, level, S.levels_x[level], S.levels_b[level], S.levels_beta_x[level],
                       S.levels_beta_y[level], S.levels_beta_z[level], S.levels_c_off[level], S.levels_fx_off[level],
                       S.levels_fy_off[level], S.levels_fz_off[level], iterations);
    } else if (op == 4) {
        run_cycle_1t(S, mg, level);
    }
    cudaDeviceSynchronize();
    download(x, S.levels_x[level], n0);
    download(b, S.levels_b[level], n0);
    if (r) download(r, dr, n0);
    if (n1 && x1) download(x1, S.levels_x[level + 1], n1);
    if (n1 && b1) download(b1, S.levels_b[level + 1], n1);
    cudaFree(dr);
    int err = (int)cudaGetLastError();
    delete G;
    return err;
}

// coarse coefficient arrays of VCycleSolver::init at `level` (beta x/y/z) for a given fine beta
REF_API int ref_level_beta(const int dims[3], const uint32_t* levels, const float* const* fine_beta, int level,
                           float* const* out) {
    Grid* G = make_grid(dims, levels, true);
    MSBGManager& mg = *G->mg;
    std::vector<float*> fx = channel_table(mg.grid.d_faceXData), fy = channel_table(mg.grid.d_faceYData),
                        fz = channel_table(mg.grid.d_faceZData);
    cudaMemcpy(fx[BETA_COEFF_X], fine_beta[0], mg.grid.totalFacesX * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(fy[BETA_COEFF_Y], fine_beta[1], mg.grid.totalFacesY * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(fz[BETA_COEFF_Z], fine_beta[2], mg.grid.totalFacesZ * 4, cudaMemcpyHostToDevice);
    VCycleSolver S(MAX_LEVELS, mg.grid.numBlocks);
    S.init(mg);
    uint32_t t[3];
    uint32_t* tmp;
    cudaMalloc(&tmp, mg.grid.numBlocks * 4);
    for (int a = 0; a < 3; ++a) computeCoarseFaceOffsets(mg, level, a, tmp, t[a]);
    cudaFree(tmp);
    download(out[0], S.levels_beta_x[level], t[0]);
    download(out[1], S.levels_beta_y[level], t[1]);
    download(out[2], S.levels_beta_z[level], t[2]);
    delete G;
    return (int)cudaGetLastError();
}

// normalizeVelocity (P2G.cuh:139-171) on given momentum / mass face arrays -> velocity
REF_API int ref_normalize(const int dims[3], const uint32_t* levels, const float* const* mom, const float* const* mass,
                          float* const* vel) {
    Grid* G = make_grid(dims, levels, true);
    MSBGManager& mg = *G->mg;
    std::vector<float*> t[3] = {channel_table(mg.grid.d_faceXData), channel_table(mg.grid.d_faceYData),
                                channel_table(mg.grid.d_faceZData)};
    uint32_t tot[3] = {mg.grid.totalFacesX, mg.grid.totalFacesY, mg.grid.totalFacesZ};
    const int MOM[3] = {MOMENTUM_X, MOMENTUM_Y, MOMENTUM_Z}, MAS[3] = {MASS_DENSITY_X, MASS_DENSITY_Y, MASS_DENSITY_Z},
              VEL[3] = {VELOCITY_X, VELOCITY_Y, VELOCITY_Z};
    for (int a = 0; a < 3; ++a) {
        cudaMemcpy(t[a][MOM[a]], mom[a], tot[a] * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(t[a][MAS[a]], mass[a], tot[a] * 4, cudaMemcpyHostToDevice);
    }
    for (int a = 0; a < 3; ++a)
        normalizeVelocity<<<mg.grid.numBlocks, 256>>>(mg.grid, (DataChannel)MOM[a], (DataChannel)MAS[a],
                                                       (DataChannel)VEL[a], a);
    cudaDeviceSynchronize();
    for (int a = 0; a < 3; ++a) download(vel[a], t[a][VEL[a]], tot[a]);
    delete G;
    return (int)cudaGetLastError();
}

// ---- Transfer kernels launched directly (no G2PManager / P2GTransfer calls) --------------------
// The managers' host paths are avoided on purpose: G2PManager::performG2P copies a pointer table
// into a host stack array and leaks a device allocation per call (G2P.cuh:198-211).  Here the
// backup fields and the device pointer table of g2pUpdateKernel are built by the harness.
namespace {

struct TransferGrid {
    Grid* G = nullptr;
    std::vector<float*> fx, fy, fz;
    float* backup[3] = {nullptr, nullptr, nullptr};
    float** d_backup = nullptr;
    uint32_t tot[3] = {0, 0, 0};
    ~TransferGrid() {
        for (float* p : backup)
            if (p) cudaFree(p);
        if (d_backup) cudaFree(d_backup);
        delete G;
    }
};

// single-level map (every block at `level`), channels allocated, VELOCITY_* = un, backup = uo
TransferGrid* make_transfer_grid(const int dims[3], uint32_t level, const float* const* un, const float* const* uo) {
    TransferGrid* T = new TransferGrid();
    uint32_t nb = (uint32_t)dims[0] * dims[1] * dims[2];
    std::vector<uint32_t> lv(nb, level);
    T->G = make_grid(dims, lv.data(), true);
    MSBG& g = T->G->mg->grid;
    T->fx = channel_table(g.d_faceXData);
    T->fy = channel_table(g.d_faceYData);
    T->fz = channel_table(g.d_faceZData);
    T->tot[0] = g.totalFacesX;
    T->tot[1] = g.totalFacesY;
    T->tot[2] = g.totalFacesZ;
    float* vel[3] = {T->fx[VELOCITY_X], T->fy[VELOCITY_Y], T->fz[VELOCITY_Z]};
    for (int a = 0; a < 3; ++a) {
        if (un) cudaMemcpy(vel[a], un[a], T->tot[a] * sizeof(float), cudaMemcpyHostToDevice);
        else cudaMemset(vel[a], 0, T->tot[a] * sizeof(float));
        cudaMalloc(&T->backup[a], std::max<uint32_t>(T->tot[a], 1) * sizeof(float));
        if (uo) cudaMemcpy(T->backup[a], uo[a], T->tot[a] * sizeof(float), cudaMemcpyHostToDevice);
        else cudaMemcpy(T->backup[a], vel[a], T->tot[a] * sizeof(float), cudaMemcpyDeviceToDevice);
    }
    cudaMalloc(&T->d_backup, 3 * sizeof(float*));
    cudaMemcpy(T->d_backup, T->backup, 3 * sizeof(float*), cudaMemcpyHostToDevice);
    return T;
}

float3 domain_size(const MSBG& g) {
    return make_float3(g.indexDims.x * g.blockSize, g.indexDims.y * g.blockSize, g.indexDims.z * g.blockSize);
}

}  // namespace

// g2pUpdateKernel (G2P.cuh:87-128) on a single-level map: VELOCITY_* = un, backup fields = uo;
// vel (n float3, in/out), pos (n float3)
REF_API int ref_g2p_blend(const int dims[3], uint32_t level, const float* const* un, const float* const* uo,
                          const float* pos, float* vel, uint32_t n, float alpha) {
    TransferGrid* T = make_transfer_grid(dims, level, un, uo);
    float3 *dp = nullptr, *dv = nullptr;
    cudaMalloc(&dp, std::max<uint32_t>(n, 1) * sizeof(float3));
    cudaMalloc(&dv, std::max<uint32_t>(n, 1) * sizeof(float3));
    cudaMemcpy(dp, pos, n * sizeof(float3), cudaMemcpyHostToDevice);
    cudaMemcpy(dv, vel, n * sizeof(float3), cudaMemcpyHostToDevice);
    if (n) g2pUpdateKernel<<<(n + 255) / 256, 256>>>(T->G->mg->grid, dv, dp, n, T->d_backup, alpha);
    cudaDeviceSynchronize();
    cudaMemcpy(vel, dv, n * sizeof(float3), cudaMemcpyDeviceToHost);
    cudaFree(dp);
    cudaFree(dv);
    int err = (int)cudaGetLastError();
    delete T;
    return err;
}

// advectParticlesKernel (G2P.cuh:131-173) on a single-level map with VELOCITY_* = u; pos in/out
REF_API int ref_advect(const int dims[3], uint32_t level, const float* const* u, float* pos, uint32_t n, float dt) {
    TransferGrid* T = make_transfer_grid(dims, level, u, nullptr);
    float3* dp = nullptr;
    cudaMalloc(&dp, std::max<uint32_t>(n, 1) * sizeof(float3));
    cudaMemcpy(dp, pos, n * sizeof(float3), cudaMemcpyHostToDevice);
    if (n) advectParticlesKernel<<<(n + 255) / 256, 256>>>(T->G->mg->grid, dp, n, dt, domain_size(T->G->mg->grid));
    cudaDeviceSynchronize();
    cudaMemcpy(pos, dp, n * sizeof(float3), cudaMemcpyDeviceToHost);
    cudaFree(dp);
    int err = (int)cudaGetLastError();
    delete T;
    return err;
}

// Timing of the reference's own kernels (CUDA events, ms per call) on a single-level map with every
// block active, launched directly in the launch shapes of the reference's managers:
//   ms_out[0] p2g + the three normalizeVelocity launches     (P2GTransfer::run, P2G.cuh:175-195)
//   ms_out[1] three D2D backup copies + g2pUpdateKernel      (G2PManager, G2P.cuh:192-211)
//   ms_out[2] advectParticlesKernel                          (G2PManager::advect, G2P.cuh:216-227)
//   ms_out[3] one V-cycle from level 0 with 1-thread smoother CTAs (runCycle, VCycle.cuh:251-304)
// Progress goes to stderr after each stage.  The velocity fields are zero and the coefficients one.
REF_API int ref_time_kernels(const int dims[3], uint32_t level, const float* pos, const float* vel, uint32_t n,
                             int reps, float* ms_out) {
    TransferGrid* T = make_transfer_grid(dims, level, nullptr, nullptr);
    MSBGManager& mg = *T->G->mg;
    MSBG& g = mg.grid;
    float3 *dp = nullptr, *dv = nullptr, *dp2 = nullptr;
    cudaMalloc(&dp, std::max<uint32_t>(n, 1) * sizeof(float3));
    cudaMalloc(&dv, std::max<uint32_t>(n, 1) * sizeof(float3));
    cudaMalloc(&dp2, std::max<uint32_t>(n, 1) * sizeof(float3));
    cudaMemcpy(dp, pos, n * sizeof(float3), cudaMemcpyHostToDevice);
    cudaMemcpy(dv, vel, n * sizeof(float3), cudaMemcpyHostToDevice);
    cudaMemcpy(dp2, dp, n * sizeof(float3), cudaMemcpyDeviceToDevice);
    std::vector<float*> cc = channel_table(g.d_cellData);
    const int face_ch[] = {BETA_COEFF_X, MASS_DENSITY_X, MOMENTUM_X, PHASE_FIELD_X};
    std::vector<float> ones(std::max({T->tot[0], T->tot[1], T->tot[2], 1u}), 1.f);
    for (int c : face_ch) {
        cudaMemset(T->fx[c], 0, T->tot[0] * 4);
        cudaMemset(T->fy[c + 1], 0, T->tot[1] * 4);
        cudaMemset(T->fz[c + 2], 0, T->tot[2] * 4);
    }
    cudaMemcpy(T->fx[BETA_COEFF_X], ones.data(), T->tot[0] * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(T->fy[BETA_COEFF_Y], ones.data(), T->tot[1] * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(T->fz[BETA_COEFF_Z], ones.data(), T->tot[2] * 4, cudaMemcpyHostToDevice);
    cudaMemset(cc[PRESSURE], 0, g.totalCells * 4);
    cudaMemset(cc[DIVERGENCE], 0, g.totalCells * 4);
    cudaDeviceSynchronize();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const unsigned pb = (n + 255) / 256;
    auto run_p2g = [&]() {
        if (n) p2g<<<pb, 256>>>(g, dp, dv, n, 1.0f, 0.0f);
        normalizeVelocity<<<g.numBlocks, 256>>>(g, MOMENTUM_X, MASS_DENSITY_X, VELOCITY_X, AXIS_X);
        normalizeVelocity<<<g.numBlocks, 256>>>(g, MOMENTUM_Y, MASS_DENSITY_Y, VELOCITY_Y, AXIS_Y);
        normalizeVelocity<<<g.numBlocks, 256>>>(g, MOMENTUM_Z, MASS_DENSITY_Z, VELOCITY_Z, AXIS_Z);
    };
    float* vch[3] = {T->fx[VELOCITY_X], T->fy[VELOCITY_Y], T->fz[VELOCITY_Z]};
    auto run_g2p = [&]() {
        for (int a = 0; a < 3; ++a)
            cudaMemcpyAsync(T->backup[a], vch[a], T->tot[a] * sizeof(float), cudaMemcpyDeviceToDevice);
        if (n) g2pUpdateKernel<<<pb, 256>>>(g, dv, dp, n, T->d_backup, 0.95f);
    };
    auto run_advect = [&]() {
        if (n) advectParticlesKernel<<<pb, 256>>>(g, dp2, n, 1.0f / 240, domain_size(g));
    };
    auto timed = [&](auto&& fn, int r) {
        fn();
        cudaDeviceSynchronize();
        cudaEventRecord(e0);
        for (int i = 0; i < r; ++i) fn();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        return t / r;
    };
    ms_out[0] = timed(run_p2g, reps);
    fprintf(stderr, "ref_time_kernels: p2g %.4f ms (%s)\n", ms_out[0], cudaGetErrorString(cudaGetLastError()));
    ms_out[1] = timed(run_g2p, reps);
    fprintf(stderr, "ref_time_kernels: g2p %.4f ms (%s)\n", ms_out[1], cudaGetErrorString(cudaGetLastError()));
    ms_out[2] = timed(run_advect, reps);
    fprintf(stderr, "ref_time_kernels: advect %.4f ms (%s)\n", ms_out[2], cudaGetErrorString(cudaGetLastError()));
    {
        VCycleSolver S(MAX_LEVELS, g.numBlocks);
        S.init(mg);
        ms_out[3] = timed([&]() { run_cycle_1t(S, mg, 0); }, 1);
        fprintf(stderr, "ref_time_kernels: vcycle (1-thread smoother CTAs) %.4f ms (%s)\n", ms_out[3],
                cudaGetErrorString(cudaGetLastError()));
    }
    cudaFree(dp);
    cudaFree(dv);
    cudaFree(dp2);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int err = (int)cudaGetLastError();
    delete T;
    return err;
}
