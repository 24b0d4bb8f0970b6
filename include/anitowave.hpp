/*
 * anitowave.hpp — C++ host classes with the reference's names, over the C ABI of anitowave.h.
 *
 * Code written against fonzy1243/AnitoWave_Adaptive's managers keeps its call sites:
 *
 *   reference (header-only CUDA C++)                      here
 *   MSBGManager(dims, blockSize, domainMin)   MSBG.cuh:506 MSBGManager(dims, blockSize, domainMin, baseRes, levels)
 *   MSBGManager::allocateChannels()            MSBG.cuh:599 allocateChannels()  (counts + scan + one slab)
 *   MSBGManager::runGalerkin(...)              MSBG.cuh:661 runGalerkin(fine, coarse, destLevel)
 *   computeCoarseOffsets / computeCoarseFaceOffsets  MSBG.cuh:679,707  same names
 *   P2GTransfer::run(mg, d_pos, d_vel, n)      P2G.cuh:175  same signature (+ optional stream)
 *   G2PManager::{init, cleanup, backupGridVelocity, performG2P, advect}  G2P.cuh:179-227  same
 *   AdaptiveSmoother::solveLevel(mg, level, ..., iterations)  Smoother.cuh:249  (level arrays
 *                                              are the solver's own: solveLevel(mg, level, iterations))
 *   MultigridTransfer::{restrictResiduals, prolongateAndCorrect}  MultigridTransfer.cuh:107,129
 *   VCycleSolver(levels, nBlocks)::{init(mg), runCycle(mg, 0)}  VCycle.cuh:161,177,251
 *
 * Differences a caller sees: errors throw anitowave::Error (the reference ignored them); every
 * call takes an optional stream and does not synchronise unless anitowave.h says it does; the
 * velocity backup lives in the grid (VELOCITY_OLD_*) instead of G2PManager-owned buffers; the
 * constants BLOCK_BASE_RES and MAX_LEVELS are constructor arguments.  Define
 * ANITOWAVE_GLOBAL_NAMES before including to also get the names in the global namespace.
 */
#ifndef ANITOWAVE_HPP
#define ANITOWAVE_HPP

#include <cstdint>
#include <stdexcept>
#include <string>

#include "anitowave.h"

namespace anitowave {

class Error : public std::runtime_error {
public:
    Error(aw_status s, const char* msg) : std::runtime_error(std::string(msg ? msg : "")), status(s) {}
    aw_status status;
};

inline void check(aw_status s) {
    if (s != AW_OK) throw Error(s, aw_last_error());
}

class MSBGManager {
public:
    MSBGManager(const int dims[3], float blockSize, const float domainMin[3], int baseRes = 16, int numLevels = 3) {
        aw_grid_desc d;
        for (int a = 0; a < 3; ++a) {
            d.dims[a] = dims[a];
            d.domain_min[a] = domainMin[a];
        }
        d.block_size = blockSize;
        d.base_res = baseRes;
        d.num_levels = numLevels;
        check(aw_msbg_create(&d, &g_));
    }
    ~MSBGManager() {
        if (g_) aw_msbg_destroy(g_);
    }
    MSBGManager(const MSBGManager&) = delete;
    MSBGManager& operator=(const MSBGManager&) = delete;

    aw_msbg* handle() const { return g_; }
    uint32_t numBlocks() const {
        aw_grid_desc d;
        check(aw_msbg_desc(g_, &d));
        return (uint32_t)d.dims[0] * d.dims[1] * d.dims[2];
    }

    // initRefinementMap (MSBG.cuh:249-254)
    void initRefinementMap(uint32_t value, aw_stream s = nullptr) { check(aw_msbg_init_refinement_map(g_, value, s)); }
    // d_refinementMap (MSBG.cuh:80)
    uint32_t* refinementMap() const {
        uint32_t* p = nullptr;
        check(aw_msbg_refinement_map(g_, &p));
        return p;
    }
    // level map from particles (replaces markActiveBlocks, MSBG.cuh:271-314)
    void levelsFromParticles(const float* d_pos, int64_t n, const int32_t* thresholds, aw_stream s = nullptr) {
        check(aw_msbg_levels_from_particles(g_, d_pos, n, thresholds, s));
    }
    // enforceGrading (MSBG.cuh:316-351) to its fixpoint; returns the passes it took
    int enforceGrading(aw_stream s = nullptr) {
        int32_t passes = 0;
        check(aw_msbg_enforce_grading(g_, &passes, s));
        return passes;
    }
    // countBlockElements + exclusive scan + allocateChannels (MSBG.cuh:353-376, 599-659)
    void allocateChannels(aw_stream s = nullptr) { check(aw_msbg_allocate(g_, s)); }
    // runGalerkin (MSBG.cuh:661-676)
    void runGalerkin(const float* fine[3], float* coarse[3], int destLevel, aw_stream s = nullptr) {
        check(aw_msbg_run_galerkin(g_, fine, coarse, destLevel, s));
    }
    // d_cellData / d_face*Data channel pointers (MSBG.cuh:92-95)
    float* channel(int ch, uint32_t* count = nullptr) const {
        float* p = nullptr;
        uint32_t n = 0;
        check(aw_msbg_channel(g_, ch, &p, &n));
        if (count) *count = n;
        return p;
    }
    // totalCells, totalFacesX/Y/Z (MSBG.cuh:98-101)
    void totals(uint32_t out[4]) const { check(aw_msbg_totals(g_, out)); }
    // d_cellOffsets / d_face*Offsets (MSBG.cuh:86-89): kind 0 cells, 1..3 faces
    uint32_t* offsets(int kind) const {
        uint32_t* p = nullptr;
        check(aw_msbg_offsets(g_, kind, &p));
        return p;
    }

private:
    aw_msbg* g_ = nullptr;
};

// computeCoarseOffsets (MSBG.cuh:679-705)
inline void computeCoarseOffsets(MSBGManager& mg, int mgLevel, uint32_t* d_offsets_out, uint32_t& totalSize_out,
                                 aw_stream s = nullptr) {
    check(aw_msbg_coarse_offsets(mg.handle(), mgLevel, 0, d_offsets_out, &totalSize_out, s));
}
// computeCoarseFaceOffsets (MSBG.cuh:707-745), axis 0..2
inline void computeCoarseFaceOffsets(MSBGManager& mg, int mgLevel, int axis, uint32_t* d_offsets_out,
                                     uint32_t& totalSize_out, aw_stream s = nullptr) {
    check(aw_msbg_coarse_offsets(mg.handle(), mgLevel, 1 + axis, d_offsets_out, &totalSize_out, s));
}

// P2GTransfer (P2G.cuh:173-195)
class P2GTransfer {
public:
    void run(MSBGManager& mg, const float* d_pos, const float* d_vel, uint32_t numParticles, aw_stream s = nullptr) {
        check(aw_p2g(mg.handle(), d_pos, d_vel, numParticles, s));
    }
    // run() plus the phase field and beta = 1/rho (PHASE_FIELD_*, BETA_COEFF_*; MSBG.cuh:21-29)
    void runPhase(MSBGManager& mg, const float* d_pos, const float* d_vel, const float* d_phase, uint32_t numParticles,
                  float rho0, float rho1, aw_stream s = nullptr) {
        check(aw_p2g_phase(mg.handle(), d_pos, d_vel, d_phase, numParticles, rho0, rho1, s));
    }
};

// G2PManager (G2P.cuh:175-228)
class G2PManager {
public:
    void init(MSBGManager&) {}  // the backup channels VELOCITY_OLD_* belong to the grid
    void cleanup() {}
    void backupGridVelocity(MSBGManager& mg, aw_stream s = nullptr) { check(aw_backup_grid_velocity(mg.handle(), s)); }
    void performG2P(MSBGManager& mg, float* p_vel, const float* p_pos, uint32_t n, float alpha = 0.97f,
                    aw_stream s = nullptr) {
        check(aw_g2p(mg.handle(), p_vel, p_pos, n, alpha, s));
    }
    void advect(MSBGManager& mg, float* p_pos, uint32_t n, float dt, aw_stream s = nullptr) {
        check(aw_advect(mg.handle(), p_pos, n, dt, s));
    }
};

class VCycleSolver;

// AdaptiveSmoother (Smoother.cuh:227-292) on the level arrays of its VCycleSolver
class AdaptiveSmoother {
public:
    void solveLevel(MSBGManager&, int mgLevel, int iterations, aw_stream s = nullptr) {
        check(aw_smoother_solve_level(sv_, mgLevel, iterations, s));
    }

private:
    friend class VCycleSolver;
    aw_solver* sv_ = nullptr;
};

// MultigridTransfer (MultigridTransfer.cuh:104-150) on the level arrays of its VCycleSolver
class MultigridTransfer {
public:
    // residual of level mgLevel restricted into the right-hand side of mgLevel + 1
    void restrictResiduals(MSBGManager&, int mgLevel, aw_stream s = nullptr) {
        check(aw_mg_residual(sv_, mgLevel, s));
        check(aw_mg_restrict(sv_, mgLevel, s));
    }
    // x[mgLevel] += P x[mgLevel + 1]
    void prolongateAndCorrect(MSBGManager&, int mgLevel, aw_stream s = nullptr) {
        check(aw_mg_prolongate(sv_, mgLevel, s));
    }

private:
    friend class VCycleSolver;
    aw_solver* sv_ = nullptr;
};

// VCycleSolver (VCycle.cuh:140-305).  levels = 0 picks the default depth; desc = nullptr picks the
// reference operator and smoother constants (AW_OPERATOR_REFERENCE).
class VCycleSolver {
public:
    VCycleSolver(int levels, uint32_t /*numBlocks*/, const aw_solver_desc* desc = nullptr) {
        if (desc) d_ = *desc;
        else check(aw_solver_default_desc(AW_OPERATOR_REFERENCE, &d_));
        if (levels > 0) d_.mg_levels = levels;
    }
    ~VCycleSolver() {
        if (sv_) aw_solver_destroy(sv_);
    }
    VCycleSolver(const VCycleSolver&) = delete;
    VCycleSolver& operator=(const VCycleSolver&) = delete;

    // init (VCycle.cuh:177-249): offsets, level arrays and coefficients of every level
    void init(MSBGManager& mg) {
        if (sv_) aw_solver_destroy(sv_);
        sv_ = nullptr;
        check(aw_solver_create(mg.handle(), &d_, &sv_));
        smoother.sv_ = sv_;
        transfer.sv_ = sv_;
    }
    // runCycle(mg, 0) (VCycle.cuh:251-304): one V-cycle on the level-0 arrays x (PRESSURE-like) and b
    void runCycle(MSBGManager&, int level, aw_stream s = nullptr) {
        if (level != 0) throw Error(AW_ERR_UNSUPPORTED, "runCycle runs the whole cycle from level 0");
        check(aw_vcycle_run(sv_, s));
    }
    // coefficients of every level again from the grid's current BETA_COEFF_* (after runPhase)
    void updateCoefficients(aw_stream s = nullptr) { check(aw_solver_update_coefficients(sv_, s)); }
    // level array of the hierarchy: which 0 = x, 1 = b, 2 = r (floats)
    float* levelArray(int level, int which, uint32_t* count = nullptr) const {
        void* p = nullptr;
        uint32_t n = 0;
        check(aw_solver_level_array(sv_, level, which, &p, &n));
        if (count) *count = n;
        return (float*)p;
    }
    aw_solver* handle() const { return sv_; }

    AdaptiveSmoother smoother;
    MultigridTransfer transfer;

private:
    aw_solver_desc d_{};
    aw_solver* sv_ = nullptr;
};

}  // namespace anitowave

#ifdef ANITOWAVE_GLOBAL_NAMES
using anitowave::AdaptiveSmoother;
using anitowave::computeCoarseFaceOffsets;
using anitowave::computeCoarseOffsets;
using anitowave::G2PManager;
using anitowave::MSBGManager;
using anitowave::MultigridTransfer;
using anitowave::P2GTransfer;
using anitowave::VCycleSolver;
#endif

#endif /* ANITOWAVE_HPP */
