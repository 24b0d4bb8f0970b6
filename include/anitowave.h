/*
 * anitowave.h — C ABI of the B200 (sm_100a) FLIP-on-MSBG library.
 *
 * Drop-in boundary for the hot path of fonzy1243/AnitoWave_Adaptive: MSBG block allocation and
 * level map, P2G, G2P, Smoother, MultigridTransfer and VCycle.  Every entry point below names
 * the reference interface it replaces (path:line within the reference project).
 *
 * Conventions
 *   - Plain C types only.  `aw_stream` is a cudaStream_t (NULL = legacy default stream).
 *   - Every call returns aw_status; aw_last_error() gives a thread-local message.
 *   - No call synchronises the device unless its comment says so ("syncs").
 *   - Device pointers are marked d_*; host pointers h_*.  Caller buffers are borrowed.
 *   - The library owns all grid, solver and simulation memory behind opaque handles.
 *   - Particle positions/velocities cross the boundary as float3 AoS (x,y,z per particle),
 *     as in the reference (P2G.cuh:18-19, G2P.cuh:89-90).
 */
#ifndef ANITOWAVE_H
#define ANITOWAVE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct CUstream_st* aw_stream;

typedef enum aw_status {
    AW_OK = 0,
    AW_ERR_INVALID_ARGUMENT = 1,
    AW_ERR_CUDA = 2,
    AW_ERR_OUT_OF_MEMORY = 3,
    AW_ERR_NOT_CONVERGED = 4,
    AW_ERR_NAN = 5,
    AW_ERR_STATE = 6,
    AW_ERR_UNSUPPORTED = 7,
    AW_ERR_IO = 8  /* a file could not be written */
} aw_status;

/* Data channels, numbered as the reference's DataChannel enum (MSBG.cuh:12-50).
 * Face channels (velocity, phase, beta, mass, momentum) live in the per-axis face tables,
 * cell channels (pressure, divergence, distance, vorticity, cell type) in the cell table. */
enum {
    AW_VELOCITY_X = 0, AW_VELOCITY_Y = 1, AW_VELOCITY_Z = 2,
    AW_PRESSURE = 3,
    AW_PHASE_FIELD_X = 4, AW_PHASE_FIELD_Y = 5, AW_PHASE_FIELD_Z = 6,
    AW_BETA_COEFF_X = 7, AW_BETA_COEFF_Y = 8, AW_BETA_COEFF_Z = 9,
    AW_MASS_DENSITY_X = 10, AW_MASS_DENSITY_Y = 11, AW_MASS_DENSITY_Z = 12,
    AW_MOMENTUM_X = 13, AW_MOMENTUM_Y = 14, AW_MOMENTUM_Z = 15,
    AW_DIVERGENCE = 16, AW_DISTANCE_FIELD = 17, AW_VORTICITY = 18, AW_CELL_TYPE = 19,
    AW_NUM_CHANNELS = 20,
    /* channels with no counterpart in the reference's enum */
    AW_VELOCITY_OLD_X = 20, AW_VELOCITY_OLD_Y = 21, AW_VELOCITY_OLD_Z = 22, /* G2P.cuh:174 backup */
    AW_NUM_CHANNELS_EXT = 23
};

/* Grid descriptor: MSBGManager(dims, blockSize, domainMin) (MSBG.cuh:506) plus the two
 * compile-time constants BLOCK_BASE_RES and MAX_LEVELS (MSBG.cuh:4-5) made runtime values. */
typedef struct aw_grid_desc {
    int32_t dims[3];       /* blocks per axis */
    float block_size;      /* world edge length of a block */
    float domain_min[3];   /* world position of block (0,0,0)'s low corner */
    int32_t base_res;      /* cells per block edge at level 0 (power of two, 1..16) */
    int32_t num_levels;    /* number of levels; level value num_levels marks an inactive block */
} aw_grid_desc;

typedef struct aw_msbg aw_msbg;
typedef struct aw_solver aw_solver;
typedef struct aw_flip aw_flip;

const char* aw_last_error(void);
const char* aw_version(void);
/* number of kernels this library has launched in this process (all threads) */
uint64_t aw_launch_count(void);

/* ---- layout helpers ------------------------------------------------------------------------ */
/* morton3D (MSBG.cuh:147-149) */
uint32_t aw_morton3d(uint32_t x, uint32_t y, uint32_t z);
/* computeBlockLayout (MSBG.cuh:112-124): out = {numCells, numFacesX, numFacesY, numFacesZ,
 * totalSize, res} */
void aw_block_layout(int32_t base_res, int32_t level, uint32_t out[6]);

/* ---- MSBG grid ------------------------------------------------------------------------------ */
/* MSBGManager::MSBGManager (MSBG.cuh:506-542).  Allocates topology; every block starts at
 * level num_levels-1 (the coarsest), like the demo's initRefinementMap (main.cu:159). */
aw_status aw_msbg_create(const aw_grid_desc* desc, aw_msbg** out);
/* MSBGManager::~MSBGManager / cleanup (MSBG.cuh:544-597) */
aw_status aw_msbg_destroy(aw_msbg* g);
aw_status aw_msbg_desc(const aw_msbg* g, aw_grid_desc* out);
/* initRefinementMap (MSBG.cuh:249-254) */
aw_status aw_msbg_init_refinement_map(aw_msbg* g, uint32_t value, aw_stream s);
/* device pointer to the refinement map (u32 per block, x-fastest linear order, MSBG.cuh:161).
 * After writing it, call aw_msbg_enforce_grading and aw_msbg_allocate again. */
aw_status aw_msbg_refinement_map(aw_msbg* g, uint32_t** d_levels);
/* initBlockInfo (MSBG.cuh:256-269): d_coord_morton = 4 u32 per block {x, y, z, morton} */
aw_status aw_msbg_block_info(aw_msbg* g, uint32_t* d_coord_morton, aw_stream s);
/* Level map from particles — replaces markActiveBlocks (MSBG.cuh:271-314).  A block's level is
 * the first k with a free-surface cell within thresholds[k] finest cells (Chebyshev distance;
 * thresholds are multiples of base_res), else num_levels-1.  d_pos: float3 AoS. */
aw_status aw_msbg_levels_from_particles(aw_msbg* g, const float* d_pos, int64_t n, const int32_t* h_thresholds,
                                        aw_stream s);
/* enforceGrading (MSBG.cuh:316-351, driven by main.cu:192-196) iterated to its fixpoint.
 * syncs (reads a changed flag per pass). */
aw_status aw_msbg_enforce_grading(aw_msbg* g, int32_t* passes, aw_stream s);
/* countBlockElements (MSBG.cuh:353-376) + exclusive scan (main.cu:270-273) + allocateChannels
 * (MSBG.cuh:599-659).  syncs (totals are needed on the host to size the channels). */
aw_status aw_msbg_allocate(aw_msbg* g, aw_stream s);
/* totals {cells, facesX, facesY, facesZ} (MSBG::totalCells..totalFacesZ, MSBG.cuh:98-101) */
aw_status aw_msbg_totals(const aw_msbg* g, uint32_t totals[4]);
/* per-block offsets at MG level 0: kind 0 = cells, 1..3 = faces x/y/z (MSBG.cuh:86-89) */
aw_status aw_msbg_offsets(aw_msbg* g, int32_t kind, uint32_t** d_offsets);
/* computeCoarseOffsets (kind 0) / computeCoarseFaceOffsets (kind 1..3) (MSBG.cuh:679-745):
 * per-block offsets at MG level mg_level, res = (base_res >> level) >> mg_level, blocks whose
 * res drops below one own nothing.  d_out: u32[num blocks]. */
aw_status aw_msbg_coarse_offsets(aw_msbg* g, int32_t mg_level, int32_t kind, uint32_t* d_out, uint32_t* total,
                                 aw_stream s);
/* device pointer of a channel (MSBG::d_cellData / d_face*Data, MSBG.cuh:92-95) */
aw_status aw_msbg_channel(aw_msbg* g, int32_t channel, float** d_ptr, uint32_t* count);
/* galerkinCoarsen x3 (MSBGManager::runGalerkin, MSBG.cuh:400-498,661-676), reference formula:
 * coarse = 2^native * 2^dest * sigma * mean(4 fine).  Offsets are the reference's coarse
 * offsets at dest-1 and dest. */
aw_status aw_msbg_run_galerkin(aw_msbg* g, const float* d_fine[3], float* d_coarse[3], int32_t dest_level,
                               aw_stream s);

/* ---- particle <-> grid transfers ------------------------------------------------------------ */
/* P2GTransfer::run (P2G.cuh:173-195) with the weight test and cross-block splat corrected:
 * every face gathers w = (1 - d^2/h^2)^3 (d < h, h = the face's cell size) from all particles,
 * writes MASS_DENSITY_*, MOMENTUM_* and VELOCITY_* = momentum/mass (0 where mass <= 1e-6), and
 * the particle count per cell into CELL_TYPE (as float).  Sorts the particles internally. */
aw_status aw_p2g(aw_msbg* g, const float* d_pos, const float* d_vel, int64_t n, aw_stream s);
/* aw_p2g for two phases: particle i also carries a phase d_phase[i] in [0,1].  Adds PHASE_FIELD_* =
 * sum w phase / sum w (0 where mass <= 1e-6) and BETA_COEFF_* = 1 / ((1 - phi) rho0 + phi rho1),
 * the face coefficients beta = 1/rho of the Poisson equation, with beta made equal on the coarse
 * face and the 4 fine faces of each T-junction (their mean).  The reference allocates these
 * channels (MSBG.cuh:21-29) and leaves their accumulation commented out (P2G.cuh:94-97). */
aw_status aw_p2g_phase(aw_msbg* g, const float* d_pos, const float* d_vel, const float* d_phase, int64_t n, float rho0,
                       float rho1, aw_stream s);
/* G2PManager::backupGridVelocity (G2P.cuh:192-196): VELOCITY_OLD_* = VELOCITY_* */
aw_status aw_backup_grid_velocity(aw_msbg* g, aw_stream s);
/* G2PManager::performG2P (G2P.cuh:198-211): v = alpha (v + u_new - u_old) + (1 - alpha) u_new,
 * trilinear MAC samples with the staggering corrected. */
aw_status aw_g2p(aw_msbg* g, float* d_vel, const float* d_pos, int64_t n, float alpha, aw_stream s);
/* No counterpart in the reference.  aw_g2p with the same arguments and results, for callers that
 * cannot let a library allocate device memory (an allocator that owns the whole GPU, a fixed device
 * budget, code where cudaMalloc's implicit device synchronisation is not allowed): its tile scratch
 * is a fixed static device array (16.25 MiB, held by every device that loads it until exit).
 * Limits: at most 65,536 blocks and 2,097,152 tile floats per velocity field (sum over active
 * blocks of 3 (r+1) (r+2)^2, rounded up to a multiple of 4); larger grids return
 * AW_ERR_INVALID_ARGUMENT.  The first call on a device looks up the array (with that device
 * current) and should come before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race. */
aw_status aw_g2p_noalloc(aw_msbg* g, float* d_vel, const float* d_pos, int64_t n, float alpha, aw_stream s);

/* Test hook, no counterpart in the reference.  The next G2P launch of a FLIP step on this grid arms
 * its first particle-copy barrier without issuing the copy and polls it only 1,024 times, so that
 * the bounded wait runs out without any fault: the CTAs drain their other copies and return, the
 * step returns AW_ERR_STATE, and the following step runs normally. */
aw_status aw_test_arm_copy_timeout(aw_msbg* g);
/* G2PManager::advect (G2P.cuh:216-227): Ralston RK3 through VELOCITY_*, clamped to the domain
 * interior (margin 0.01 finest cells). */
aw_status aw_advect(aw_msbg* g, float* d_pos, int64_t n, float dt, aw_stream s);
/* trilinear MAC sample of VELOCITY_* (or VELOCITY_OLD_* when old != 0) at n points */
aw_status aw_sample_velocity(aw_msbg* g, const float* d_points, int64_t n, int32_t old, float* d_out, aw_stream s);
/* stable sort of particles by (block, cell) key; d_perm[i] = original index of sorted slot i.
 * d_keys gets the sorted keys (global cell index; 0xFFFFFFFF for inactive blocks). */
aw_status aw_sort_particles(aw_msbg* g, const float* d_pos, int64_t n, uint32_t* d_keys, uint32_t* d_perm,
                            aw_stream s);

/* ---- FLIP-step building blocks (no counterpart in the reference: D14) ---------------------- */
/* world positions of face centres (axis 0..2) or cell centres (axis 3), float3 per element */
aw_status aw_face_positions(aw_msbg* g, int32_t axis, float* d_xyz, aw_stream s);
/* level-interface sync of a face-channel triplet (channel = its x channel): a coarse block's
 * boundary face := mean of the 4 fine faces it covers */
aw_status aw_face_sync(aw_msbg* g, int32_t channel, aw_stream s);
/* solid walls: zero the domain-boundary faces of a face-channel triplet */
aw_status aw_wall_bc(aw_msbg* g, int32_t channel, aw_stream s);
/* VELOCITY_* += dt * gravity */
aw_status aw_add_gravity(aw_msbg* g, const float gravity[3], float dt, aw_stream s);
/* d_out = net face flux / dt per fluid cell (the projection right-hand side); optional d_max
 * (device float, must start at 0) receives max |div u| per unit volume */
aw_status aw_velocity_divergence(aw_msbg* g, const uint8_t* d_fluid, float inv_dt, float* d_out, float* d_max,
                                 aw_stream s);
/* *d_max (device double) = max over fluid cells (every cell when d_fluid is NULL) of |div u| per unit
 * volume, the face sums of VELOCITY_* taken in FP64.  No counterpart in the reference: it reports
 * the divergence an FP32 field really has, free of the rounding of an FP32 sum. */
aw_status aw_velocity_divergence_max64(aw_msbg* g, const uint8_t* d_fluid, double* d_max, aw_stream s);

/* ---- pressure solver -------------------------------------------------------------------------- */
enum { AW_OPERATOR_FV = 0, AW_OPERATOR_REFERENCE = 1 };
/* AW_PRECISION_FP32: V-cycle iteration on an FP32 pressure (runCycle repeated, VCycle.cuh:251-304).
 * AW_PRECISION_MIXED: conjugate gradients preconditioned by the V-cycle, FP32 arithmetic inside the
 *   cycle with FP16-stored coarse corrections (per-block scale), FP64 residual, direction, pressure
 *   accumulation and coarsest solve; the pressure is FP64.
 * AW_PRECISION_FP32_PCG: the same preconditioned conjugate gradients with every vector and scalar in
 *   FP32 and FP32 storage on every level; the pressure is FP32.  No counterpart in the reference: the
 *   like-for-like FP32 baseline of the mixed form. */
enum { AW_PRECISION_FP32 = 0, AW_PRECISION_MIXED = 1, AW_PRECISION_FP32_PCG = 2 };

typedef struct aw_solver_desc {
    int32_t operator_mode;       /* AW_OPERATOR_FV (finite-volume, symmetric) or _REFERENCE */
    int32_t precision;           /* AW_PRECISION_FP32, _MIXED or _FP32_PCG */
    int32_t mg_levels;           /* block-structured MG levels (0 = default) */
    int32_t pre_smooth;          /* runCycle pre-smoothing iterations (VCycle.cuh:262) */
    int32_t post_smooth;         /* runCycle post-smoothing iterations (VCycle.cuh:303) */
    int32_t coarsest_iterations; /* smoother iterations at the coarsest level (VCycle.cuh:255) */
    int32_t block_iterations;    /* MAX_BLOCK_ITER (Smoother.cuh:10) */
    int32_t dense_sweeps;        /* red-black sweeps on the uniform coarse levels (FV) */
    float omega;                 /* OMEGA (Smoother.cuh:9) */
    float target_reduction;      /* TARGET_RESIDUAL_REDUCTION (Smoother.cuh:11); 0 disables */
    float theta;                 /* activation threshold (Smoother.cuh:286) */
    int32_t max_cycles;
    double tolerance;            /* relative residual ||b - A p|| / ||b|| */
} aw_solver_desc;

aw_status aw_solver_default_desc(int32_t operator_mode, aw_solver_desc* out);
/* VCycleSolver(levels, nBlocks) + init (VCycle.cuh:161,177-249): builds offsets, level arrays
 * and coefficients of every MG level.  Reference mode takes BETA_COEFF_* as the fine
 * coefficients and coarsens them with galerkinCoarsen; FV mode derives conductances from the
 * geometry and BETA_COEFF_* (1/rho).  syncs. */
aw_status aw_solver_create(aw_msbg* g, const aw_solver_desc* desc, aw_solver** out);
aw_status aw_solver_destroy(aw_solver* sv);
/* Per-step setup: fluid flags of level 0 (d_fluid: u8 per cell, NULL = every cell fluid),
 * coarse flags, and the FP64 factorisation of the coarsest level. */
aw_status aw_solver_setup(aw_solver* sv, const uint8_t* d_fluid, aw_stream s);
/* Rebuild every block-structured level's coefficients from the grid's current BETA_COEFF_*
 * (after aw_p2g_phase; before aw_solver_setup, whose coarsest factorisation uses them).
 * Stream-ordered; no counterpart in the reference, whose coefficients are fixed at init. */
aw_status aw_solver_update_coefficients(aw_solver* sv, aw_stream s);
aw_status aw_solver_num_levels(const aw_solver* sv, int32_t* n);
/* precision of the solver (AW_PRECISION_FP32, _MIXED or _FP32_PCG) */
aw_status aw_solver_precision(const aw_solver* sv, int32_t* precision);
/* level arrays: which 0 = x, 1 = b, 2 = r (float), 3..5 = coefficients x/y/z (float),
 * 6 = fluid (u8), 7 = cell offsets, 8..10 = face offsets (u32; MSBG levels only) */
aw_status aw_solver_level_array(aw_solver* sv, int32_t level, int32_t which, void** d_ptr, uint32_t* count);
/* AdaptiveSmoother::solveLevel (Smoother.cuh:249-291) on MG level `level` */
aw_status aw_smoother_solve_level(aw_solver* sv, int32_t level, int32_t iterations, aw_stream s);
/* computeExplicitResidual (VCycle.cuh:81-131): r = b - A x on MG level `level` */
aw_status aw_mg_residual(aw_solver* sv, int32_t level, aw_stream s);
/* MultigridTransfer::restrictResiduals (MultigridTransfer.cuh:107-127): b[level+1] = R r[level] */
aw_status aw_mg_restrict(aw_solver* sv, int32_t level, aw_stream s);
/* MultigridTransfer::prolongateAndCorrect (MultigridTransfer.cuh:129-149): x[level] += P x[level+1] */
aw_status aw_mg_prolongate(aw_solver* sv, int32_t level, aw_stream s);
/* coarsest-level solve (VCycle.cuh:252-256): FP64 dense solve of the uniform coarsest level in FV
 * mode, coarsest_iterations smoother iterations in reference mode */
aw_status aw_solver_coarsest_solve(aw_solver* sv, aw_stream s);
/* VCycleSolver::runCycle(mg, 0) (VCycle.cuh:251-304) on the level-0 arrays x, b */
aw_status aw_vcycle_run(aw_solver* sv, aw_stream s);
/* Solve A p = b on level 0 to desc.tolerance.  FP32 precision: p is float*, V-cycles in place.
 * Mixed precision: p is double*, outer defect correction with the FP64 residual, FP64
 * accumulation and FP64 coarsest solve; V-cycle in FP32 with FP16 coarse corrections.
 * syncs (one residual norm read per cycle).  Returns AW_ERR_NOT_CONVERGED if max_cycles ran out. */
aw_status aw_solve(aw_solver* sv, const float* d_b, void* d_p, int32_t* cycles, double* final_rel, aw_stream s);
/* pressure-gradient update of VELOCITY_*: u -= dt (W/area) (p_high - p_low) on faces with a fluid
 * cell on either side (level-0 conductances W of the solver); wall faces are zeroed.
 * d_p is float (p_is_double = 0) or double. */
aw_status aw_pressure_gradient(aw_msbg* g, aw_solver* sv, const void* d_p, int32_t p_is_double,
                               const uint8_t* d_fluid, float dt, aw_stream s);

/* ---- FLIP simulation ------------------------------------------------------------------------- */
typedef struct aw_flip_desc {
    float dt;
    float alpha;          /* FLIP/PIC blend */
    float gravity[3];
    int32_t precision;    /* pressure solve precision */
    double tolerance;
    int32_t max_cycles;
} aw_flip_desc;

typedef struct aw_flip_stats {
    int32_t cycles;          /* V-cycles of the last projection */
    double residual;         /* final relative residual */
    double div_before;       /* max |div u| * dt before projection (fluid cells) */
    double div_after;        /* max |div u| * dt after projection */
    float ms_sort, ms_p2g, ms_solve, ms_g2p, ms_advect, ms_other;
} aw_flip_stats;

/* One FLIP time step per call on library-owned SoA particle state. */
aw_status aw_flip_create(aw_msbg* g, const aw_flip_desc* desc, const float* h_pos, const float* h_vel, int64_t n,
                         aw_flip** out);
aw_status aw_flip_destroy(aw_flip* f);
/* One step.  The pressure solve starts from the previous step's pressure (air cells zeroed) once a
 * step on the current layout has converged, from zero otherwise. */
aw_status aw_flip_step(aw_flip* f, aw_stream s);
aw_status aw_flip_stats_get(aw_flip* f, aw_flip_stats* out);
/* copy particle state to host in the original particle order (AoS) */
aw_status aw_flip_particles(aw_flip* f, float* h_pos, float* h_vel);
aw_status aw_flip_solver(aw_flip* f, aw_solver** out);
/* Between steps: rebuild the level map from the simulation's current particle positions (the rule
 * of aw_msbg_levels_from_particles with these thresholds, graded to the same fixpoint as
 * aw_msbg_enforce_grading).  The map, its grading and the comparison with the map in use run on the
 * device; the host reads back one count.  When the map is unchanged nothing else happens.  When it
 * changed, the grid is laid out again (aw_msbg_allocate) and the solver hierarchy rebuilt; channel
 * pointers and solver handles obtained before are then stale.  No grid state needs remapping: P2G
 * regenerates it from the particles every step.  *changed (optional) = 1 when the layout changed.
 * syncs.  No counterpart in the reference (markActiveBlocks + grading + allocateChannels were a
 * one-time setup there, main.cu:154-278). */
aw_status aw_flip_rebuild_levels(aw_flip* f, const int32_t* h_thresholds, int32_t* changed, aw_stream s);
/* Two-phase simulation: h_phase[i] in [0,1] is the phase of particle i (original order) and rho0,
 * rho1 > 0 the densities of phase 0 and 1.  Every later step runs aw_p2g_phase's deposit, rebuilds
 * the solver's coefficients from BETA_COEFF_* and projects with beta = 1/rho.  The particle
 * velocity transfer keeps unit particle mass.  h_phase = NULL returns to one phase (beta = 1).
 * The differentiable rollout does not take a phase.  syncs. */
aw_status aw_flip_set_phase(aw_flip* f, const float* h_phase, float rho0, float rho1);

/* ---- inspection: dense resampling and binary VTK (vtx_visualization.cuh:8-218) ----------------
 * The lattice has out_dims[0] x out_dims[1] x out_dims[2] points over the domain, x fastest;
 * point (i, j, k) sits at domain_min + (i + 0.5) * spacing with spacing = domain extent / out_dims
 * (float).  aw_resample_lattice reports origin (point 0) and spacing for the VTK header. */
aw_status aw_resample_lattice(aw_msbg* g, const int32_t out_dims[3], float origin[3], float spacing[3]);
/* sampleMSBG (vtx_visualization.cuh:8-62): a cell channel (PRESSURE, DIVERGENCE, DISTANCE_FIELD,
 * VORTICITY or CELL_TYPE) at every lattice point: the value of the level-0 cell holding it, 0 in
 * inactive blocks.  d_out: one float per point.  Corrected: domain_min is honoured.  The FLIP step
 * leaves its pressure in PRESSURE (0 in air cells). */
aw_status aw_resample_cells(aw_msbg* g, int32_t channel, const int32_t out_dims[3], float* d_out, aw_stream s);
/* The MAC velocity (VELOCITY_*, or VELOCITY_OLD_* when old) at every lattice point, with
 * aw_sample_velocity's trilinear rule; d_out: float3 per point.  No counterpart in the reference. */
aw_status aw_resample_velocity(aw_msbg* g, int32_t old, const int32_t out_dims[3], float* d_out, aw_stream s);
/* exportUniformPressure_VTK (vtx_visualization.cuh:64-127) in legacy VTK BINARY encoding (big
 * endian): STRUCTURED_POINTS with ncomp 1 (SCALARS) or 3 (VECTORS) floats per point, x fastest.
 * Host data.  AW_ERR_IO if the file cannot be written. */
aw_status aw_vtk_write_structured_points(const char* path, const int32_t dims[3], const float origin[3],
                                         const float spacing[3], const char* name, int32_t ncomp, const float* h_data);
/* exportMultigrid_VTK (vtx_visualization.cuh:129-195), binary: one hexahedron per block with its
 * level as CELL_DATA refineLevel (-1 for inactive blocks).  syncs. */
aw_status aw_vtk_write_blocks(aw_msbg* g, const char* path);
/* exportParticles_VTK (vtx_visualization.cuh:197-218), binary POLYDATA: n float3 host positions as
 * vertices, with one optional float per particle (h_scalar, may be NULL) named `name`. */
aw_status aw_vtk_write_particles(const char* path, const float* h_pos, int64_t n, const char* name,
                                 const float* h_scalar);

/* ---- projection and adjoints (no counterpart in the reference) ------------------------------
 * The vector-Jacobian products differentiate the forward calls with their discrete decisions
 * held fixed: the block and cell of every particle and sample point, the fluid flags, the P2G
 * kernel supports and the clamp branches of sampling and advection.  Face-array adjoints
 * (d_*_bar[3]) have the layout of the VELOCITY_* channels; particle adjoints are float3 AoS.
 * "+=" marks outputs that are accumulated into, "in/out" adjoints that are replaced. */
typedef struct aw_rollout aw_rollout;

/* the projection of the FLIP step on VELOCITY_*: divergence, solve (aw_solver_setup with d_fluid
 * first, done here), pressure-gradient update, T-junction sync, walls.  syncs (aw_solve). */
aw_status aw_project(aw_msbg* g, aw_solver* sv, const uint8_t* d_fluid, float dt, aw_stream s);
/* VJP of aw_project: d_u_bar (in/out) from the adjoint of the projected velocity to the adjoint of
 * its input.  One more solve with the same operator (the finite-volume operator is symmetric).
 * syncs. */
aw_status aw_vjp_project(aw_msbg* g, aw_solver* sv, const uint8_t* d_fluid, float dt, float* const d_u_bar[3],
                         aw_stream s);
/* VJP of aw_p2g's VELOCITY_* output (P2G with u = P/m): given d_u_bar, d_pos_bar and d_vel_bar +=.
 * Recomputes the forward mass and velocity of these particles internally (the grid's channels are
 * not touched).  A G2P-shaped gather: one thread per particle. */
aw_status aw_vjp_p2g(aw_msbg* g, const float* d_pos, const float* d_vel, int64_t n, const float* const d_u_bar[3],
                     float* d_pos_bar, float* d_vel_bar, aw_stream s);
/* VJP of aw_g2p with the current VELOCITY_* / VELOCITY_OLD_* as u_new / u_old: d_vel_bar in/out,
 * d_pos_bar +=, d_un_bar and d_uo_bar +=.  A P2G-shaped scatter through ghosted adjoint tiles. */
aw_status aw_vjp_g2p(aw_msbg* g, const float* d_pos, int64_t n, float alpha, float* d_vel_bar, float* d_pos_bar,
                     float* const d_un_bar[3], float* const d_uo_bar[3], aw_stream s);
/* VJP of aw_advect through VELOCITY_*: d_pos = positions before advection, d_pos_bar in/out,
 * d_u_bar +=. */
aw_status aw_vjp_advect(aw_msbg* g, const float* d_pos, int64_t n, float dt, float* d_pos_bar, float* const d_u_bar[3],
                        aw_stream s);
/* VJP of aw_sample_velocity: d_u_bar += I^T d_out_bar; d_points_bar (optional) += (dI/dx)^T d_out_bar */
aw_status aw_vjp_sample(aw_msbg* g, const float* d_points, int64_t n, int32_t old, const float* d_out_bar,
                        float* const d_u_bar[3], float* d_points_bar, aw_stream s);

/* Differentiable rollout: particles start at d_pos0 (AoS, copied) with velocities sampled from a
 * MAC face field u0, take `steps` FLIP steps of desc, and the loss is the mean over particles of
 * |x_final - target|^2.  The particle state of every checkpoint_every-th step is kept on the
 * device; aw_vjp_rollout recomputes each segment from its checkpoint and runs the step adjoints
 * backwards through it. */
aw_status aw_rollout_create(aw_msbg* g, const aw_flip_desc* desc, const float* d_pos0, int64_t n, int32_t steps,
                            int32_t checkpoint_every, aw_rollout** out);
aw_status aw_rollout_destroy(aw_rollout* r);
/* d_u0: the three face arrays of u0 concatenated (x, y, z; sizes from aw_msbg_totals); d_target:
 * AoS per particle (copied).  freeze_fluid != 0 reuses the fluid flags of the last forward run
 * without it, so that finite differences see the same discrete decisions as the adjoint.
 * syncs; writes *loss. */
aw_status aw_rollout_forward(aw_rollout* r, const float* d_u0, const float* d_target, int32_t freeze_fluid,
                             double* loss, aw_stream s);
/* final positions of the last forward run, AoS in particle order */
aw_status aw_rollout_final_positions(aw_rollout* r, float* d_pos, aw_stream s);
/* d loss / d u0 (layout of d_u0) for the last forward run.  The recompute reuses the state
 * buffers, so run aw_rollout_forward again before another aw_vjp_rollout.  syncs. */
aw_status aw_vjp_rollout(aw_rollout* r, float* d_u0_bar, aw_stream s);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* ANITOWAVE_H */
