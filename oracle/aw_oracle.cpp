// aw_oracle.cpp — FP64 OpenMP CPU restatement of the AnitoWave_Adaptive FLIP-on-MSBG path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle used by tests/, by __graft_entry__.smoke()
// and by the cpu_baseline / --impl reference legs of bench.py.  Nothing in the product library
// (anitowave_adaptive_b200/) links, loads or calls it.
//
// Precision contract: every value (weights, velocities, pressures, residuals) is computed in
// FP64.  Every *discrete decision* (block of a particle, cell of a particle, sort key, fluid
// flag) is computed with the same IEEE-754 single-precision operations the GPU performs, so that
// maps, keys and sort orders are bit-exact between the two.  Build with -ffp-contract=off.
//
// Reference files followed (paths relative to the reference project root):
//   MSBG.cuh:112-124   computeBlockLayout           -> layout_count()
//   MSBG.cuh:139-149   expandBits / morton3D          -> oc_morton3d()
//   MSBG.cuh:151-191   index helpers                  -> cidx()/fidx()/block helpers
//   MSBG.cuh:316-351   enforceGrading                 -> oc_enforce_grading() (iterated to fixpoint)
//   MSBG.cuh:353-376   countBlockElements + main.cu:270-273 exclusive_scan -> offsets()
//   MSBG.cuh:378-498   getScalingFactor/galerkinCoarsen -> oc_galerkin_ref()
//   MSBG.cuh:679-745   computeCoarseOffsets/FaceOffsets -> offsets(mg, vanish=true)
//   P2G.cuh:6-12,16-135 kernel weight and splat       -> p2g() (gather form, D1/D2 corrected)
//   P2G.cuh:139-171    normalizeVelocity               -> p2g() (u = P/m if m > 1e-6)
//   MSBG.cuh:21-29, P2G.cuh:94-97 phase field, beta = 1/rho -> oc_p2g_phase(), oc_beta_sync()
//   G2P.cuh:11-80      interpolateComponent            -> sample() (D4/D5 corrected staggering)
//   G2P.cuh:87-128     g2pUpdateKernel (FLIP blend)    -> g2p()
//   G2P.cuh:131-173    advectParticlesKernel (RK3)     -> advect()
//   Smoother.cuh:105-223 smoothActiveBlocks/solveLevel -> smooth_level()
//   MultigridTransfer.cuh:9-102 restrict / prolongate  -> restrict_level()/prolong_level()
//   VCycle.cuh:81-131  computeExplicitResidual         -> residual()
//   VCycle.cuh:251-304 runCycle                        -> vcycle()
//
// Corrections of reference defects (each is a deliberate deviation, listed once here):
//   D1  P2G weight test inverted (P2G.cuh:9): here w = (1-d^2/R^2)^3 for d < R, else 0.
//   D2  P2G clipped to the particle's block (P2G.cuh:67-76): here every face within R of the
//       particle receives weight, in any block (gather form: each face sums all particles in its
//       support, R = the face's own cell size).
//   D3  accumulators never cleared (P2G.cuh:175-187): here every face value is recomputed.
//   D4/D5 G2P staggering and face indexing (G2P.cuh:37-39, 58-65): here the tangential
//       coordinates are shifted by half a cell and faces use the face index maps.
//   D8  T-junction ghost lookups swapped (Smoother.cuh:72-91, VCycle.cuh:57-75): here a fine
//       cell reads its coarse parent; a coarse cell reads the mean of the 4 touching fine cells.
//   D9  divergent early-exit (Smoother.cuh:183-185): here the exit test is block-uniform.
//   D10 inactive blocks indexing c_blockLayouts[MAX_LEVELS]: here inactive blocks own nothing.
//   D12 grading ran a fixed 3 passes (main.cu:192-196): here it iterates to the fixpoint.
//   D13 fine operator had no h-scaling: here the finite-volume operator ("FV mode") uses face
//       conductances area/distance, symmetric at level interfaces.
//   D14 FLIP-step pieces absent from the reference (sort, gravity, walls, divergence, gradient,
//       defect correction) are specified here.
//
// Parity status: layouts, Morton codes, offsets, grading, Galerkin coefficients, restriction,
// prolongation, residual and the smoother in "reference mode" are pinned against fixtures
// produced by the reference's own CUDA build (tests/golden).  The FV-mode operator, P2G, G2P,
// the projection and the adjoint have no counterpart in the reference; they are pinned by
// analytic cases (manufactured Poisson solution, hydrostatic column, constant-field transfers,
// finite differences).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OC_API extern "C" __attribute__((visibility("default")))

namespace {

// ----------------------------------------------------------------------------------------------
// Geometry and index helpers (MSBG.cuh:112-191)
// ----------------------------------------------------------------------------------------------
struct Geo {
    int D[3];
    float bs;
    float dmin[3];
    int R0;
    int L;
    int nb() const { return D[0] * D[1] * D[2]; }
};

inline int bidx(const Geo& g, int x, int y, int z) { return x + g.D[0] * (y + g.D[1] * z); }
inline void bcoord(const Geo& g, int b, int c[3]) {
    c[0] = b % g.D[0];
    c[1] = (b / g.D[0]) % g.D[1];
    c[2] = b / (g.D[0] * g.D[1]);
}
inline bool inside(const Geo& g, const int c[3]) {
    return c[0] >= 0 && c[1] >= 0 && c[2] >= 0 && c[0] < g.D[0] && c[1] < g.D[1] && c[2] < g.D[2];
}
inline uint32_t cidx(int x, int y, int z, int r) { return (uint32_t)(x + r * (y + r * z)); }
// face index of axis a at integer coords (x,y,z): MSBG.cuh:169-179
inline uint32_t fidx(int a, int x, int y, int z, int r) {
    if (a == 0) return (uint32_t)(x + (r + 1) * (y + r * z));
    if (a == 1) return (uint32_t)(x + r * (y + (r + 1) * z));
    return (uint32_t)(x + r * (y + r * z));
}
inline uint32_t nfaces(int a, int r) { (void)a; return (uint32_t)((r + 1) * r * r); }

// float origin of a block, computed with the single-precision operations the GPU uses
inline float forigin(const Geo& g, int a, int c) { return g.dmin[a] + (float)c * g.bs; }
inline float fcell(const Geo& g, int r) { return g.bs / (float)r; }

// The block a point belongs to (worldToBlockCoord, MSBG.cuh:151-159), clamped into the domain.
inline void point_block(const Geo& g, const float p[3], int c[3]) {
    for (int a = 0; a < 3; ++a) {
        float rel = p[a] - g.dmin[a];
        int v = (int)std::floor(rel / g.bs);
        c[a] = std::min(std::max(v, 0), g.D[a] - 1);
    }
}

uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// ----------------------------------------------------------------------------------------------
// One multigrid level.  MSBG levels hold per-block resolutions; dense levels are uniform grids.
// ----------------------------------------------------------------------------------------------
struct Lvl {
    bool dense = false;
    int D[3] = {0, 0, 0};  // dense dims
    double H = 0;          // dense cell size
    std::vector<int> res;  // MSBG: cells per block edge (0 = no storage)
    std::vector<uint32_t> off[4];
    uint32_t tot[4] = {0, 0, 0, 0};
    std::vector<double> W[3];  // conductances (FV) or coefficients (reference mode)
    std::vector<double> bbar[3];
    std::vector<uint8_t> fluid;
    std::vector<double> x, b, r;
    std::vector<double> Minv;  // dense inverse for the coarsest level
    int nexact = 0;
    std::vector<int> exact_cells;
};

struct Params {
    int mode = 0;  // 0 = FV, 1 = reference operator
    int pre = 2, post = 2, coarsest_iters = 50, block_iters = 2, dense_sweeps = 2;
    double omega = 1.0;
    double target = 0.33;
    double theta = -1.0;
    int max_exact = 1024;
    double lambda = 1.0;  // prolongation scale
    int coarse_all = 1;   // FV: a coarse cell is fluid iff all its children are fluid
};

struct Ctx {
    Geo g;
    std::vector<uint32_t> level;
    Params P;
    std::vector<Lvl> lv;  // solver hierarchy (built on demand)
    bool built = false;
};

inline int lg2(int v) { int l = 0; while ((1 << l) < v) ++l; return l; }

// Offsets for a block-structured level: res per block -> counts -> exclusive scan (linear order)
void make_offsets(Lvl& L, int nb) {
    for (int k = 0; k < 4; ++k) L.off[k].assign(nb, 0);
    uint32_t acc[4] = {0, 0, 0, 0};
    for (int b = 0; b < nb; ++b) {
        int r = L.res[b];
        uint32_t cnt[4];
        cnt[0] = (uint32_t)(r * r * r);
        cnt[1] = cnt[2] = cnt[3] = r > 0 ? (uint32_t)((r + 1) * r * r) : 0u;
        for (int k = 0; k < 4; ++k) {
            L.off[k][b] = acc[k];
            acc[k] += cnt[k];
        }
    }
    for (int k = 0; k < 4; ++k) L.tot[k] = acc[k];
}

// res of block b at MG level m.  vanish=true is the reference semantics (computeCoarseOffsets,
// MSBG.cuh:689-694, with D10 fixed); vanish=false clamps at one cell (FV hierarchy).
int res_at(const Ctx& C, int b, int m, bool vanish) {
    uint32_t l = C.level[b];
    if ((int)l >= C.g.L) return 0;
    int r = C.g.R0 >> l;
    int rm = r >> m;
    if (rm < 1) rm = vanish ? 0 : 1;
    return rm;
}

// ----------------------------------------------------------------------------------------------
// Ghost values across a block boundary (getPressureLevel / getVectorLevel with D8 corrected)
// kind: 0 = wall (outside the domain), 1 = absent neighbour (air, value 0), 2 = value
// ----------------------------------------------------------------------------------------------
struct Ghost {
    int kind;
    double v;
    bool fluid;
};

Ghost ghost(const Geo& g, const Lvl& L, const double* x, int b, const int cb[3], const int c[3], int a,
            int s) {
    int nc[3] = {cb[0], cb[1], cb[2]};
    nc[a] += s;
    if (!inside(g, nc)) return {0, 0.0, false};
    int n = bidx(g, nc[0], nc[1], nc[2]);
    int r = L.res[b], rn = L.res[n];
    if (rn == 0) return {1, 0.0, false};
    int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
    int na = (s > 0) ? 0 : rn - 1;
    if (rn == r) {
        int q[3];
        q[a] = na; q[t1] = c[t1]; q[t2] = c[t2];
        uint32_t i = L.off[0][n] + cidx(q[0], q[1], q[2], rn);
        return {2, x ? x[i] : 0.0, L.fluid.empty() ? true : (bool)L.fluid[i]};
    }
    if (2 * rn == r) {  // neighbour coarser: parent cell
        int q[3];
        q[a] = na; q[t1] = c[t1] / 2; q[t2] = c[t2] / 2;
        uint32_t i = L.off[0][n] + cidx(q[0], q[1], q[2], rn);
        return {2, x ? x[i] : 0.0, L.fluid.empty() ? true : (bool)L.fluid[i]};
    }
    // neighbour finer: mean of the 4 touching fine cells
    double sum = 0.0;
    bool anyf = false;
    for (int d1 = 0; d1 < 2; ++d1)
        for (int d2 = 0; d2 < 2; ++d2) {
            int q[3];
            q[a] = na; q[t1] = 2 * c[t1] + d1; q[t2] = 2 * c[t2] + d2;
            uint32_t i = L.off[0][n] + cidx(q[0], q[1], q[2], rn);
            if (x) sum += x[i];
            if (L.fluid.empty() || L.fluid[i]) anyf = true;
        }
    return {2, 0.25 * sum, anyf};
}

// value of the neighbour cell across (a, s) from cell c of block b
inline double nbr(const Geo& g, const Lvl& L, const double* x, int b, const int cb[3], const int c[3], int a,
                  int s) {
    int r = L.res[b];
    int q[3] = {c[0], c[1], c[2]};
    q[a] += s;
    if (q[a] >= 0 && q[a] < r) return x[L.off[0][b] + cidx(q[0], q[1], q[2], r)];
    Ghost gh = ghost(g, L, x, b, cb, c, a, s);
    return gh.v;
}

inline double face_W(const Lvl& L, int b, int a, const int c[3], int s) {
    int r = L.res[b];
    int f[3] = {c[0], c[1], c[2]};
    if (s > 0) f[a] += 1;
    return L.W[a][L.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r)];
}

// (A x)_i = sum_f W_f (g_f - x_i) at cell c of block b, plus its diagonal -sum W_f
inline double apply_cell(const Geo& g, const Lvl& L, const double* x, int b, const int cb[3], const int c[3],
                         double* diag_out) {
    double s = 0.0, d = 0.0;
    double xi = x[L.off[0][b] + cidx(c[0], c[1], c[2], L.res[b])];
    for (int a = 0; a < 3; ++a)
        for (int sd = -1; sd <= 1; sd += 2) {
            double w = face_W(L, b, a, c, sd);
            double v = nbr(g, L, x, b, cb, c, a, sd);
            s += w * v;
            d -= w;
        }
    if (diag_out) *diag_out = d;
    return s + d * xi;
}

// ---------------------------- dense (uniform) levels -------------------------------------------
inline uint32_t didx(const Lvl& L, int i, int j, int k) { return (uint32_t)(i + L.D[0] * (j + L.D[1] * k)); }
inline uint32_t dfidx(const Lvl& L, int a, int i, int j, int k) {
    if (a == 0) return (uint32_t)(i + (L.D[0] + 1) * (j + L.D[1] * k));
    if (a == 1) return (uint32_t)(i + L.D[0] * (j + (L.D[1] + 1) * k));
    return (uint32_t)(i + L.D[0] * (j + L.D[1] * k));
}
inline double dense_apply(const Lvl& L, const double* x, int i, int j, int k, double* diag_out) {
    int c[3] = {i, j, k};
    double s = 0.0, d = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int sd = -1; sd <= 1; sd += 2) {
            int f[3] = {i, j, k};
            if (sd > 0) f[a] += 1;
            double w = L.W[a][dfidx(L, a, f[0], f[1], f[2])];
            int q[3] = {c[0], c[1], c[2]};
            q[a] += sd;
            double v = 0.0;
            if (q[a] >= 0 && q[a] < L.D[a]) v = x[didx(L, q[0], q[1], q[2])];
            s += w * v;
            d -= w;
        }
    if (diag_out) *diag_out = d;
    return s + d * x[didx(L, i, j, k)];
}

// ----------------------------------------------------------------------------------------------
// Hierarchy construction
// ----------------------------------------------------------------------------------------------
void fv_conductance(const Ctx& C, Lvl& L) {
    const Geo& g = C.g;
    int nb = g.nb();
    for (int a = 0; a < 3; ++a) L.W[a].assign(L.tot[1 + a], 0.0);
    for (int b = 0; b < nb; ++b) {
        int r = L.res[b];
        if (!r) continue;
        int cb[3];
        bcoord(g, b, cb);
        double H = (double)g.bs / r;
        for (int a = 0; a < 3; ++a) {
            int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            for (int fa = 0; fa <= r; ++fa)
                for (int u = 0; u < r; ++u)
                    for (int v = 0; v < r; ++v) {
                        int f[3];
                        f[a] = fa; f[t1] = u; f[t2] = v;
                        uint32_t i = L.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r);
                        double geo;
                        if (fa > 0 && fa < r) {
                            geo = H;
                        } else {
                            int nc[3] = {cb[0], cb[1], cb[2]};
                            nc[a] += (fa == 0) ? -1 : 1;
                            if (!inside(g, nc)) {
                                geo = 0.0;
                            } else {
                                int rn = L.res[bidx(g, nc[0], nc[1], nc[2])];
                                if (rn == 0 || rn == r) geo = H;
                                else if (2 * rn == r) geo = (2.0 / 3.0) * H;
                                else geo = (4.0 / 3.0) * H;
                            }
                        }
                        L.W[a][i] = geo * L.bbar[a][i];
                    }
        }
    }
}

void dense_conductance(Lvl& L) {
    for (int a = 0; a < 3; ++a) {
        int n = (L.D[0] + (a == 0)) * (L.D[1] + (a == 1)) * (L.D[2] + (a == 2));
        L.W[a].assign(n, 0.0);
        for (int k = 0; k < L.D[2] + (a == 2); ++k)
            for (int j = 0; j < L.D[1] + (a == 1); ++j)
                for (int i = 0; i < L.D[0] + (a == 0); ++i) {
                    int f[3] = {i, j, k};
                    uint32_t fi = dfidx(L, a, i, j, k);
                    if (f[a] == 0 || f[a] == L.D[a]) L.W[a][fi] = 0.0;
                    else L.W[a][fi] = L.H * L.bbar[a][fi];
                }
    }
}

// Symmetric dense inverse for the coarsest level (Cholesky of -A, with one rank-1 term per
// Neumann component, i.e. a connected set of fluid cells that touches no Dirichlet face).
void build_exact(Lvl& L, const Geo& g) {
    // enumerate fluid cells
    std::vector<int> ids;
    size_t ncell = L.dense ? (size_t)L.D[0] * L.D[1] * L.D[2] : L.tot[0];
    for (size_t i = 0; i < ncell; ++i)
        if (L.fluid[i]) ids.push_back((int)i);
    int n = (int)ids.size();
    L.nexact = n;
    L.exact_cells = ids;
    L.Minv.assign((size_t)n * n, 0.0);
    if (n == 0) return;
    std::vector<int> pos(ncell, -1);
    for (int i = 0; i < n; ++i) pos[ids[i]] = i;
    // assemble -A (positive semi-definite)
    std::vector<double> M((size_t)n * n, 0.0);
    std::vector<double> e(ncell, 0.0);
    std::vector<char> dirichlet(n, 0);
    for (int col = 0; col < n; ++col) {
        std::fill(e.begin(), e.end(), 0.0);
        e[ids[col]] = 1.0;
        for (int row = 0; row < n; ++row) {
            int ci = ids[row];
            double d, ax;
            if (L.dense) {
                int i = ci % L.D[0], j = (ci / L.D[0]) % L.D[1], k = ci / (L.D[0] * L.D[1]);
                ax = dense_apply(L, e.data(), i, j, k, &d);
            } else {
                // locate block of cell ci (res-1 blocks: one cell per block, or general)
                int b = (int)(std::upper_bound(L.off[0].begin(), L.off[0].end(), (uint32_t)ci) - L.off[0].begin()) - 1;
                while (b > 0 && L.res[b] == 0) --b;
                int r = L.res[b];
                int loc = ci - (int)L.off[0][b];
                int c[3] = {loc % r, (loc / r) % r, loc / (r * r)};
                int cb[3];
                bcoord(g, b, cb);
                ax = apply_cell(g, L, e.data(), b, cb, c, &d);
            }
            M[(size_t)row * n + col] = -ax;
        }
    }
    // Dirichlet-touching rows: -A row sum > 0
    for (int i = 0; i < n; ++i) {
        double s = 0;
        for (int j = 0; j < n; ++j) s += M[(size_t)i * n + j];
        if (s > 1e-12 * std::fabs(M[(size_t)i * n + i])) dirichlet[i] = 1;
    }
    // connected components
    std::vector<int> comp(n, -1);
    int ncomp = 0;
    for (int s0 = 0; s0 < n; ++s0) {
        if (comp[s0] >= 0) continue;
        std::vector<int> st = {s0};
        comp[s0] = ncomp;
        while (!st.empty()) {
            int u = st.back();
            st.pop_back();
            for (int v = 0; v < n; ++v)
                if (comp[v] < 0 && M[(size_t)u * n + v] != 0.0) {
                    comp[v] = ncomp;
                    st.push_back(v);
                }
        }
        ++ncomp;
    }
    for (int c = 0; c < ncomp; ++c) {
        bool dir = false;
        int cnt = 0;
        double dsum = 0;
        for (int i = 0; i < n; ++i)
            if (comp[i] == c) {
                cnt++;
                dsum += M[(size_t)i * n + i];
                if (dirichlet[i]) dir = true;
            }
        if (dir) continue;
        double sc = dsum / cnt / cnt;  // rank-1 regulariser scaled to the diagonal
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                if (comp[i] == c && comp[j] == c) M[(size_t)i * n + j] += sc;
    }
    // Cholesky and explicit inverse of (-A + reg); Minv = -(...)^-1 so that x = Minv * b solves A x = b
    std::vector<double> Lc = M;
    for (int j = 0; j < n; ++j) {
        double s = Lc[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) s -= Lc[(size_t)j * n + k] * Lc[(size_t)j * n + k];
        s = std::sqrt(std::max(s, 1e-300));
        Lc[(size_t)j * n + j] = s;
        for (int i = j + 1; i < n; ++i) {
            double t = Lc[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) t -= Lc[(size_t)i * n + k] * Lc[(size_t)j * n + k];
            Lc[(size_t)i * n + j] = t / s;
        }
    }
    for (int col = 0; col < n; ++col) {
        std::vector<double> y(n, 0.0);
        for (int i = 0; i < n; ++i) {
            double t = (i == col) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) t -= Lc[(size_t)i * n + k] * y[k];
            y[i] = t / Lc[(size_t)i * n + i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double t = y[i];
            for (int k = i + 1; k < n; ++k) t -= Lc[(size_t)k * n + i] * y[k];
            y[i] = t / Lc[(size_t)i * n + i];
        }
        for (int i = 0; i < n; ++i) L.Minv[(size_t)i * n + col] = -y[i];
    }
}

void build_hierarchy(Ctx& C, const double* bbar0[3], const uint8_t* fluid0, const double* W0ref[3],
                     int mg_levels) {
    const Geo& g = C.g;
    int nb = g.nb();
    C.lv.clear();
    bool ref = C.P.mode == 1;
    int M = mg_levels > 0 ? mg_levels : (ref ? g.L : lg2(g.R0) + 1);
    for (int m = 0; m < M; ++m) {
        Lvl L;
        L.res.resize(nb);
        for (int b = 0; b < nb; ++b) L.res[b] = res_at(C, b, m, ref);
        make_offsets(L, nb);
        L.fluid.assign(L.tot[0], 1);
        for (int a = 0; a < 3; ++a) L.bbar[a].assign(L.tot[1 + a], 1.0);
        if (m == 0) {
            if (fluid0) std::copy(fluid0, fluid0 + L.tot[0], L.fluid.begin());
            for (int a = 0; a < 3; ++a)
                if (bbar0[a]) std::copy(bbar0[a], bbar0[a] + L.tot[1 + a], L.bbar[a].begin());
        } else {
            Lvl& F = C.lv[m - 1];
            for (int b = 0; b < nb; ++b) {
                int r = L.res[b], rf = F.res[b];
                if (!r) continue;
                bool halved = (rf == 2 * r);
                for (int z = 0; z < r; ++z)
                    for (int y = 0; y < r; ++y)
                        for (int x = 0; x < r; ++x) {
                            uint8_t fl = C.P.coarse_all ? 1 : 0;
                            if (halved) {
                                for (int dz = 0; dz < 2; ++dz)
                                    for (int dy = 0; dy < 2; ++dy)
                                        for (int dx = 0; dx < 2; ++dx) {
                                            uint8_t cf = F.fluid[F.off[0][b] + cidx(2 * x + dx, 2 * y + dy, 2 * z + dz, rf)];
                                            fl = C.P.coarse_all ? (fl & cf) : (fl | cf);
                                        }
                            } else {
                                fl = F.fluid[F.off[0][b] + cidx(x, y, z, rf)];
                            }
                            L.fluid[L.off[0][b] + cidx(x, y, z, r)] = fl;
                        }
                for (int a = 0; a < 3; ++a) {
                    int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
                    for (int fa = 0; fa <= r; ++fa)
                        for (int u = 0; u < r; ++u)
                            for (int v = 0; v < r; ++v) {
                                int f[3];
                                f[a] = fa; f[t1] = u; f[t2] = v;
                                double val;
                                if (halved) {
                                    double s = 0;
                                    for (int d1 = 0; d1 < 2; ++d1)
                                        for (int d2 = 0; d2 < 2; ++d2) {
                                            int q[3];
                                            q[a] = 2 * fa; q[t1] = 2 * u + d1; q[t2] = 2 * v + d2;
                                            s += F.bbar[a][F.off[1 + a][b] + fidx(a, q[0], q[1], q[2], rf)];
                                        }
                                    val = 0.25 * s;
                                } else {
                                    val = F.bbar[a][F.off[1 + a][b] + fidx(a, f[0], f[1], f[2], rf)];
                                }
                                L.bbar[a][L.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r)] = val;
                            }
                }
            }
        }
        if (ref) {
            for (int a = 0; a < 3; ++a) L.W[a].assign(L.tot[1 + a], 0.0);
            if (m == 0) {
                for (int a = 0; a < 3; ++a)
                    for (uint32_t i = 0; i < L.tot[1 + a]; ++i) L.W[a][i] = W0ref[a] ? W0ref[a][i] : 1.0;
            }
        } else {
            fv_conductance(C, L);
        }
        L.x.assign(L.tot[0], 0.0);
        L.b.assign(L.tot[0], 0.0);
        L.r.assign(L.tot[0], 0.0);
        C.lv.push_back(std::move(L));
        if (ref && m > 0) {
            // Galerkin coarse coefficients, reference formula (MSBG.cuh:400-498), in FP64
            Lvl& Lc = C.lv[m];
            Lvl& F = C.lv[m - 1];
            for (int b = 0; b < nb; ++b) {
                uint32_t l = C.level[b];
                if ((int)l >= g.L) continue;
                int fr = g.R0 >> (l + m - 1), cr = g.R0 >> (l + m);
                if (cr < 1 || fr < 2) continue;
                int cb[3];
                bcoord(g, b, cb);
                for (int a = 0; a < 3; ++a) {
                    int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
                    for (int fa = 0; fa <= cr; ++fa)
                        for (int u = 0; u < cr; ++u)
                            for (int v = 0; v < cr; ++v) {
                                int t[3];
                                t[a] = fa; t[t1] = u; t[t2] = v;
                                double s = (double)(1 << l);
                                if (fa == 0 || fa == cr) {
                                    int nc[3] = {cb[0], cb[1], cb[2]};
                                    nc[a] += fa == 0 ? -1 : 1;
                                    int nl = inside(g, nc) ? (int)C.level[bidx(g, nc[0], nc[1], nc[2])] : (int)l;
                                    int diff = (int)l - nl;
                                    if (diff == 1) s *= 1.0 / 3.0;
                                    else if (diff == -1) s *= 2.0 / 3.0;
                                }
                                s *= (double)(1 << m);
                                double sum = 0;
                                for (int d1 = 0; d1 < 2; ++d1)
                                    for (int d2 = 0; d2 < 2; ++d2) {
                                        int q[3] = {2 * t[0], 2 * t[1], 2 * t[2]};
                                        // reference loop order: axis X -> (y += d1, z += d2) etc.
                                        int a1 = (a == 0) ? 1 : 0, a2 = (a == 2) ? 1 : 2;
                                        q[a1] += d1;
                                        q[a2] += d2;
                                        sum += F.W[a][F.off[1 + a][b] + fidx(a, q[0], q[1], q[2], fr)];
                                    }
                                Lc.W[a][Lc.off[1 + a][b] + fidx(a, t[0], t[1], t[2], cr)] = s * (sum * 0.25);
                            }
                }
            }
        }
    }
    if (!ref) {
        // dense continuation: all blocks are one cell at the last MSBG level
        int Dd[3] = {g.D[0], g.D[1], g.D[2]};
        double H = g.bs;
        Lvl* prev = &C.lv.back();
        bool first = true;
        while (Dd[0] % 2 == 0 && Dd[1] % 2 == 0 && Dd[2] % 2 == 0 && (long)Dd[0] * Dd[1] * Dd[2] > 64) {
            Lvl L;
            L.dense = true;
            for (int a = 0; a < 3; ++a) L.D[a] = Dd[a] / 2;
            L.H = 2 * H;
            size_t nc = (size_t)L.D[0] * L.D[1] * L.D[2];
            L.fluid.assign(nc, 0);
            for (int a = 0; a < 3; ++a) {
                int n = (L.D[0] + (a == 0)) * (L.D[1] + (a == 1)) * (L.D[2] + (a == 2));
                L.bbar[a].assign(n, 1.0);
            }
            for (int k = 0; k < L.D[2]; ++k)
                for (int j = 0; j < L.D[1]; ++j)
                    for (int i = 0; i < L.D[0]; ++i) {
                        uint8_t fl = C.P.coarse_all ? 1 : 0;
                        for (int dz = 0; dz < 2; ++dz)
                            for (int dy = 0; dy < 2; ++dy)
                                for (int dx = 0; dx < 2; ++dx) {
                                    int ci = 2 * i + dx, cj = 2 * j + dy, ck = 2 * k + dz;
                                    uint8_t cf = 0;
                                    if (first) {
                                        int b = bidx(g, ci, cj, ck);
                                        if (prev->res[b]) cf = prev->fluid[prev->off[0][b]];
                                    } else {
                                        cf = prev->fluid[didx(*prev, ci, cj, ck)];
                                    }
                                    fl = C.P.coarse_all ? (fl & cf) : (fl | cf);
                                }
                        L.fluid[didx(L, i, j, k)] = fl;
                    }
            dense_conductance(L);
            L.x.assign(nc, 0.0);
            L.b.assign(nc, 0.0);
            L.r.assign(nc, 0.0);
            C.lv.push_back(std::move(L));
            prev = &C.lv.back();
            first = false;
            for (int a = 0; a < 3; ++a) Dd[a] /= 2;
            H *= 2;
        }
        Lvl& last = C.lv.back();
        size_t nlast = last.dense ? (size_t)last.D[0] * last.D[1] * last.D[2] : last.tot[0];
        size_t nf = 0;
        for (size_t i = 0; i < nlast; ++i) nf += last.fluid[i];
        if ((int)nf <= C.P.max_exact) build_exact(last, g);
    }
    C.built = true;
}

// ----------------------------------------------------------------------------------------------
// Smoother (Smoother.cuh:105-202, 249-291) — block red-black on block parity, block-local
// red-black Gauss-Seidel sweeps with early exit, adaptive activation with threshold theta.
// post (FV mode): the adjoint order, block and cell colours black before red, which makes the
// V-cycle a symmetric preconditioner; reference mode keeps one order (VCycle.cuh:251-304).
// ----------------------------------------------------------------------------------------------
void smooth_level(Ctx& C, int m, int iterations, bool post = false) {
    const Geo& g = C.g;
    Lvl& L = C.lv[m];
    int nb = g.nb();
    const double w = C.P.omega;
    const int rev = post && C.P.mode == 0 ? 1 : 0;
    if (L.dense) {
        for (int it = 0; it < iterations; ++it)
            for (int k2 = 0; k2 < 2; ++k2) {
                const int col = rev ? 1 - k2 : k2;
#pragma omp parallel for collapse(2) schedule(static)
                for (int k = 0; k < L.D[2]; ++k)
                    for (int j = 0; j < L.D[1]; ++j)
                        for (int i = (j + k + col) & 1; i < L.D[0]; i += 2) {
                            uint32_t ci = didx(L, i, j, k);
                            if (!L.fluid[ci]) continue;
                            double d;
                            double ax = dense_apply(L, L.x.data(), i, j, k, &d);
                            if (std::fabs(d) < 1e-300) continue;
                            L.x[ci] += w * (L.b[ci] - ax) / d;
                        }
            }
        return;
    }
    std::vector<uint8_t> active(nb, 0), next(nb, 0);
    for (int b = 0; b < nb; ++b) active[b] = L.res[b] > 0;
    const bool ref = C.P.mode == 1;
    for (int it = 0; it < iterations; ++it) {
        bool any = false;
        for (int b = 0; b < nb; ++b) any |= active[b] != 0;
        if (!any) break;
        std::fill(next.begin(), next.end(), 0);
        for (int k2 = 0; k2 < 2; ++k2) {
            const int rb = rev ? 1 - k2 : k2;
            std::vector<double> maxres(nb, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
            for (int b = 0; b < nb; ++b) {
                if (!active[b]) continue;
                int cb[3];
                bcoord(g, b, cb);
                if ((cb[0] + cb[1] + cb[2]) % 2 != rb) continue;
                int r = L.res[b];
                if (r < 1) continue;
                double init = -1.0, mr = 0.0;
                for (int bi = 0; bi < C.P.block_iters; ++bi) {
                    mr = 0.0;
                    for (int k3 = 0; k3 < 2; ++k3)
                        for (int z = 0; z < r; ++z)
                            for (int y = 0; y < r; ++y)
                                for (int x = 0; x < r; ++x) {
                                    if ((x + y + z) % 2 != (rev ? 1 - k3 : k3)) continue;
                                    uint32_t ci = L.off[0][b] + cidx(x, y, z, r);
                                    if (!ref && !L.fluid[ci]) continue;
                                    int c[3] = {x, y, z};
                                    double d;
                                    double ax = apply_cell(g, L, L.x.data(), b, cb, c, &d);
                                    if (std::fabs(d) < 1e-9) continue;
                                    double res = L.b[ci] - ax;
                                    L.x[ci] += w * (res / d);
                                    mr = std::max(mr, std::fabs(res));
                                }
                    if (bi == 0) init = mr;
                    if (init > 1e-9 && mr < init * C.P.target) break;
                }
                maxres[b] = mr;
            }
            for (int b = 0; b < nb; ++b) {
                if (!active[b]) continue;
                int cb[3];
                bcoord(g, b, cb);
                if ((cb[0] + cb[1] + cb[2]) % 2 != rb || L.res[b] < 1) continue;
                if (maxres[b] > C.P.theta) {
                    next[b] = 1;
                    for (int a = 0; a < 3; ++a)
                        for (int s = -1; s <= 1; s += 2) {
                            int nc[3] = {cb[0], cb[1], cb[2]};
                            nc[a] += s;
                            if (inside(g, nc)) next[bidx(g, nc[0], nc[1], nc[2])] = 1;
                        }
                }
            }
        }
        for (int b = 0; b < nb; ++b) active[b] = next[b] && L.res[b] > 0;
    }
}

void residual_level(Ctx& C, int m, const double* x, const double* bvec, double* r) {
    const Geo& g = C.g;
    Lvl& L = C.lv[m];
    const bool ref = C.P.mode == 1;
    if (L.dense) {
#pragma omp parallel for collapse(2)
        for (int k = 0; k < L.D[2]; ++k)
            for (int j = 0; j < L.D[1]; ++j)
                for (int i = 0; i < L.D[0]; ++i) {
                    uint32_t ci = didx(L, i, j, k);
                    r[ci] = L.fluid[ci] ? bvec[ci] - dense_apply(L, x, i, j, k, nullptr) : 0.0;
                }
        return;
    }
    int nb = g.nb();
#pragma omp parallel for schedule(dynamic, 4)
    for (int b = 0; b < nb; ++b) {
        int r0 = L.res[b];
        if (!r0) continue;
        int cb[3];
        bcoord(g, b, cb);
        for (int z = 0; z < r0; ++z)
            for (int y = 0; y < r0; ++y)
                for (int xx = 0; xx < r0; ++xx) {
                    uint32_t ci = L.off[0][b] + cidx(xx, y, z, r0);
                    if (!ref && !L.fluid[ci]) { r[ci] = 0.0; continue; }
                    int c[3] = {xx, y, z};
                    r[ci] = bvec[ci] - apply_cell(g, L, x, b, cb, c, nullptr);
                }
    }
}

// restriction m -> m+1 (MultigridTransfer.cuh:9-59): 8-child sum; copy for clamped one-cell blocks
void restrict_level(Ctx& C, int m) {
    const Geo& g = C.g;
    Lvl& F = C.lv[m];
    Lvl& K = C.lv[m + 1];
    std::fill(K.b.begin(), K.b.end(), 0.0);
    if (K.dense) {
        for (int k = 0; k < K.D[2]; ++k)
            for (int j = 0; j < K.D[1]; ++j)
                for (int i = 0; i < K.D[0]; ++i) {
                    double s = 0;
                    for (int dz = 0; dz < 2; ++dz)
                        for (int dy = 0; dy < 2; ++dy)
                            for (int dx = 0; dx < 2; ++dx) {
                                int ci = 2 * i + dx, cj = 2 * j + dy, ck = 2 * k + dz;
                                if (F.dense) s += F.r[didx(F, ci, cj, ck)];
                                else {
                                    int b = bidx(g, ci, cj, ck);
                                    if (F.res[b]) s += F.r[F.off[0][b]];
                                }
                            }
                    K.b[didx(K, i, j, k)] = K.fluid[didx(K, i, j, k)] ? s : 0.0;
                }
        return;
    }
    int nb = g.nb();
    for (int b = 0; b < nb; ++b) {
        int r = K.res[b], rf = F.res[b];
        if (!r) continue;
        bool halved = rf == 2 * r;
        for (int z = 0; z < r; ++z)
            for (int y = 0; y < r; ++y)
                for (int x = 0; x < r; ++x) {
                    double s = 0;
                    if (halved) {
                        for (int dz = 0; dz < 2; ++dz)
                            for (int dy = 0; dy < 2; ++dy)
                                for (int dx = 0; dx < 2; ++dx)
                                    s += F.r[F.off[0][b] + cidx(2 * x + dx, 2 * y + dy, 2 * z + dz, rf)];
                    } else {
                        s = F.r[F.off[0][b] + cidx(x, y, z, rf)];
                    }
                    uint32_t ci = K.off[0][b] + cidx(x, y, z, r);
                    K.b[ci] = (C.P.mode == 1 || K.fluid[ci]) ? s : 0.0;
                }
    }
}

// prolongation m+1 -> m (MultigridTransfer.cuh:63-102): injection add into fluid cells
void prolong_level(Ctx& C, int m) {
    const Geo& g = C.g;
    Lvl& F = C.lv[m];
    Lvl& K = C.lv[m + 1];
    const bool ref = C.P.mode == 1;
    if (K.dense) {
        if (F.dense) {
            for (int k = 0; k < F.D[2]; ++k)
                for (int j = 0; j < F.D[1]; ++j)
                    for (int i = 0; i < F.D[0]; ++i) {
                        uint32_t ci = didx(F, i, j, k);
                        if (F.fluid[ci]) F.x[ci] += C.P.lambda * K.x[didx(K, i / 2, j / 2, k / 2)];
                    }
        } else {
            for (int b = 0; b < g.nb(); ++b) {
                if (!F.res[b]) continue;
                int cb[3];
                bcoord(g, b, cb);
                uint32_t ci = F.off[0][b];
                if (F.fluid[ci]) F.x[ci] += C.P.lambda * K.x[didx(K, cb[0] / 2, cb[1] / 2, cb[2] / 2)];
            }
        }
        return;
    }
    for (int b = 0; b < g.nb(); ++b) {
        int r = K.res[b], rf = F.res[b];
        if (!r) continue;
        bool halved = rf == 2 * r;
        for (int z = 0; z < rf; ++z)
            for (int y = 0; y < rf; ++y)
                for (int x = 0; x < rf; ++x) {
                    uint32_t ci = F.off[0][b] + cidx(x, y, z, rf);
                    if (!ref && !F.fluid[ci]) continue;
                    double v = halved ? K.x[K.off[0][b] + cidx(x / 2, y / 2, z / 2, r)] : K.x[K.off[0][b] + cidx(x, y, z, r)];
                    F.x[ci] += C.P.lambda * v;
                }
    }
}

void coarsest_solve(Ctx& C, int m) {
    Lvl& L = C.lv[m];
    if (C.P.mode == 1 || L.Minv.empty()) {
        smooth_level(C, m, C.P.coarsest_iters);
        return;
    }
    int n = L.nexact;
    std::vector<double> bb(n);
    for (int i = 0; i < n; ++i) bb[i] = L.b[L.exact_cells[i]];
    for (int i = 0; i < n; ++i) {
        double s = 0;
        for (int j = 0; j < n; ++j) s += L.Minv[(size_t)i * n + j] * bb[j];
        L.x[L.exact_cells[i]] = s;
    }
}

void vcycle(Ctx& C, int m) {
    int last = (int)C.lv.size() - 1;
    if (m == last) {
        coarsest_solve(C, m);
        return;
    }
    Lvl& L = C.lv[m];
    if (L.dense) smooth_level(C, m, C.P.dense_sweeps);
    else smooth_level(C, m, C.P.pre);
    residual_level(C, m, L.x.data(), L.b.data(), L.r.data());
    restrict_level(C, m);
    std::fill(C.lv[m + 1].x.begin(), C.lv[m + 1].x.end(), 0.0);
    vcycle(C, m + 1);
    prolong_level(C, m);
    if (L.dense) smooth_level(C, m, C.P.dense_sweeps, true);
    else smooth_level(C, m, C.P.post, true);
}

double norm2(const std::vector<double>& v) {
    double s = 0;
    for (double x : v) s += x * x;
    return std::sqrt(s);
}

// ----------------------------------------------------------------------------------------------
// Particles: keys, stable sort, P2G, G2P, RK3
// ----------------------------------------------------------------------------------------------
struct PartGrid {
    const Geo* g;
    const std::vector<uint32_t>* level;
    std::vector<int> res;  // per block native res (0 inactive)
    std::vector<uint32_t> off[4];
    uint32_t tot[4];
};

PartGrid make_pgrid(const Ctx& C) {
    PartGrid P;
    P.g = &C.g;
    P.level = &C.level;
    int nb = C.g.nb();
    P.res.resize(nb);
    for (int b = 0; b < nb; ++b) P.res[b] = res_at(C, b, 0, true);
    Lvl tmp;
    tmp.res = P.res;
    make_offsets(tmp, nb);
    for (int k = 0; k < 4; ++k) {
        P.off[k] = tmp.off[k];
        P.tot[k] = tmp.tot[k];
    }
    return P;
}

// sort key of a particle: global cell index (block offset + cell index) or 0xFFFFFFFF
uint32_t particle_key(const PartGrid& P, const float p[3]) {
    const Geo& g = *P.g;
    int c[3];
    point_block(g, p, c);
    int b = bidx(g, c[0], c[1], c[2]);
    int r = P.res[b];
    if (!r) return 0xFFFFFFFFu;
    float h = fcell(g, r);
    int q[3];
    for (int a = 0; a < 3; ++a) {
        float o = forigin(g, a, c[a]);
        float loc = p[a] - o;
        int v = (int)std::floor(loc / h);
        q[a] = std::min(std::max(v, 0), r - 1);
    }
    return P.off[0][b] + cidx(q[0], q[1], q[2], r);
}

inline double kernel_w(double d2, double R2) {
    if (d2 >= R2) return 0.0;
    double t = 1.0 - d2 / R2;
    return t * t * t;
}

// Ghost face value for G2P.  Tangential stencil indices outside the block read the nearest face
// of the same axis in the neighbouring block, mapped with integer arithmetic (positions in
// half-cells): normal index round-half-up(fi * rn / r), tangential floor((2 fi + 1 - 2 o r) rn /
// (2 r)).  Outside the domain or in an inactive block the index is clamped into the block.
double face_value_at(const Ctx& C, const PartGrid& PG, const double* u, int a, int b, const int cb[3], int r,
                     int fi[3]) {
    const Geo& g = C.g;
    int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
    int o1 = fi[t1] < 0 ? -1 : (fi[t1] >= r ? 1 : 0);
    int o2 = fi[t2] < 0 ? -1 : (fi[t2] >= r ? 1 : 0);
    if (!o1 && !o2) return u[PG.off[1 + a][b] + fidx(a, fi[0], fi[1], fi[2], r)];
    int nc[3] = {cb[0], cb[1], cb[2]};
    nc[t1] += o1;
    nc[t2] += o2;
    int rn = 0, n = 0;
    if (inside(g, nc)) {
        n = bidx(g, nc[0], nc[1], nc[2]);
        rn = PG.res[n];
    }
    if (!rn) {
        int q[3] = {fi[0], fi[1], fi[2]};
        q[t1] = std::min(std::max(q[t1], 0), r - 1);
        q[t2] = std::min(std::max(q[t2], 0), r - 1);
        return u[PG.off[1 + a][b] + fidx(a, q[0], q[1], q[2], r)];
    }
    int q[3];
    q[a] = (2 * fi[a] * rn + r) / (2 * r);
    int rel1 = 2 * fi[t1] + 1 - o1 * 2 * r;
    int rel2 = 2 * fi[t2] + 1 - o2 * 2 * r;
    q[t1] = std::min(std::max((rel1 * rn) / (2 * r), 0), rn - 1);
    q[t2] = std::min(std::max((rel2 * rn) / (2 * r), 0), rn - 1);
    return u[PG.off[1 + a][n] + fidx(a, q[0], q[1], q[2], rn)];
}

// Trilinear MAC sample of component a at world point X (interpolateComponent, G2P.cuh:11-72,
// with D4/D5 corrected).
double sample(const Ctx& C, const PartGrid& PG, const double* u, int a, const double X[3]) {
    const Geo& g = C.g;
    float Xf[3] = {(float)X[0], (float)X[1], (float)X[2]};
    int cb[3];
    point_block(g, Xf, cb);
    int b = bidx(g, cb[0], cb[1], cb[2]);
    int r = PG.res[b];
    if (!r) return 0.0;
    double h = (double)fcell(g, r);
    int i0[3];
    double f[3];
    for (int k = 0; k < 3; ++k) {
        double o = (double)forigin(g, k, cb[k]);
        double s = (X[k] - o) / h;
        int lo, hi;
        if (k == a) { lo = 0; hi = r; }
        else { s -= 0.5; lo = -1; hi = r; }
        s = std::min(std::max(s, (double)lo), (double)hi);
        int i = (int)std::floor(s);
        i = std::min(std::max(i, lo), hi - 1);
        i0[k] = i;
        f[k] = s - i;
    }
    double acc = 0.0;
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                int fi[3] = {i0[0] + dx, i0[1] + dy, i0[2] + dz};
                double wv = (dx ? f[0] : 1 - f[0]) * (dy ? f[1] : 1 - f[1]) * (dz ? f[2] : 1 - f[2]);
                acc += wv * face_value_at(C, PG, u, a, b, cb, r, fi);
            }
    return acc;
}

}  // namespace

// ================================================================================================
// C ABI
// ================================================================================================
OC_API uint32_t oc_morton3d(uint32_t x, uint32_t y, uint32_t z) {
    return expand_bits(x) | (expand_bits(y) << 1) | (expand_bits(z) << 2);
}

OC_API void oc_block_layout(int R0, int level, uint32_t out[6]) {
    int r = R0 >> level;
    out[0] = (uint32_t)(r * r * r);
    out[1] = (uint32_t)((r + 1) * r * r);
    out[2] = (uint32_t)(r * (r + 1) * r);
    out[3] = (uint32_t)(r * r * (r + 1));
    out[4] = out[0] + out[1] + out[2] + out[3];
    out[5] = (uint32_t)r;
}

OC_API int oc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
OC_API void oc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// Level map from particle occupancy: finest-cell occupancy -> free-surface cells -> block
// Chebyshev distance thresholds (in cells, multiples of R0).  Inactive value = L never produced.
OC_API int oc_levels_from_particles(const int D[3], float bs, const float dmin[3], int R0, int L,
                                    const float* pos, int64_t n, const int* thresholds, uint32_t* levels) {
    Geo g{{D[0], D[1], D[2]}, bs, {dmin[0], dmin[1], dmin[2]}, R0, L};
    int N[3] = {D[0] * R0, D[1] * R0, D[2] * R0};
    size_t nc = (size_t)N[0] * N[1] * N[2];
    std::vector<uint8_t> occ(nc, 0);
    float h0 = bs / (float)R0;
    for (int64_t i = 0; i < n; ++i) {
        int q[3];
        for (int a = 0; a < 3; ++a) {
            float rel = pos[3 * i + a] - dmin[a];
            int v = (int)std::floor(rel / h0);
            q[a] = std::min(std::max(v, 0), N[a] - 1);
        }
        occ[(size_t)q[0] + (size_t)N[0] * ((size_t)q[1] + (size_t)N[1] * q[2])] = 1;
    }
    int nb = g.nb();
    std::vector<uint8_t> bsurf(nb, 0);
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j)
            for (int i = 0; i < N[0]; ++i) {
                size_t ci = (size_t)i + (size_t)N[0] * ((size_t)j + (size_t)N[1] * k);
                if (!occ[ci]) continue;
                bool surf = false;
                int c[3] = {i, j, k};
                for (int a = 0; a < 3 && !surf; ++a)
                    for (int s = -1; s <= 1 && !surf; s += 2) {
                        int q[3] = {c[0], c[1], c[2]};
                        q[a] += s;
                        if (q[a] < 0 || q[a] >= N[a]) continue;
                        if (!occ[(size_t)q[0] + (size_t)N[0] * ((size_t)q[1] + (size_t)N[1] * q[2])]) surf = true;
                    }
                if (surf) bsurf[bidx(g, i / R0, j / R0, k / R0)] = 1;
            }
    for (int b = 0; b < nb; ++b) {
        int cb[3];
        bcoord(g, b, cb);
        uint32_t lev = (uint32_t)(L - 1);
        for (int t = 0; t < L - 1; ++t) {
            int K = thresholds[t] / R0;
            bool hit = false;
            for (int z = std::max(0, cb[2] - K); z <= std::min(D[2] - 1, cb[2] + K) && !hit; ++z)
                for (int y = std::max(0, cb[1] - K); y <= std::min(D[1] - 1, cb[1] + K) && !hit; ++y)
                    for (int x = std::max(0, cb[0] - K); x <= std::min(D[0] - 1, cb[0] + K); ++x)
                        if (bsurf[bidx(g, x, y, z)]) { hit = true; break; }
            if (hit) { lev = (uint32_t)t; break; }
        }
        levels[b] = lev;
    }
    return 0;
}

// 2:1 grading to the fixpoint (enforceGrading, MSBG.cuh:316-351, iterated).  Jacobi passes.
OC_API int oc_enforce_grading(const int D[3], int L, uint32_t* levels, int* passes_out) {
    Geo g{{D[0], D[1], D[2]}, 1.f, {0, 0, 0}, 1, L};
    int nb = g.nb();
    std::vector<uint32_t> nxt(levels, levels + nb);
    int passes = 0;
    while (true) {
        bool changed = false;
        for (int b = 0; b < nb; ++b) {
            uint32_t l = levels[b];
            if ((int)l == L) continue;
            int cb[3];
            bcoord(g, b, cb);
            uint32_t best = l;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (!dx && !dy && !dz) continue;
                        int nc[3] = {cb[0] + dx, cb[1] + dy, cb[2] + dz};
                        if (!inside(g, nc)) continue;
                        uint32_t nl = levels[bidx(g, nc[0], nc[1], nc[2])];
                        if ((int)nl == L) continue;
                        if ((int)l - (int)nl > 1) best = std::min(best, nl + 1u);
                    }
            nxt[b] = best;
            if (best != l) changed = true;
        }
        ++passes;
        std::copy(nxt.begin(), nxt.end(), levels);
        if (!changed) break;
    }
    if (passes_out) *passes_out = passes;
    return 0;
}

OC_API void* oc_create(const int D[3], float bs, const float dmin[3], int R0, int L, const uint32_t* levels) {
    Ctx* C = new Ctx();
    C->g = Geo{{D[0], D[1], D[2]}, bs, {dmin[0], dmin[1], dmin[2]}, R0, L};
    C->level.assign(levels, levels + C->g.nb());
    return C;
}
OC_API void oc_destroy(void* h) { delete (Ctx*)h; }

OC_API void oc_set_params(void* h, int mode, int pre, int post, int coarsest_iters, int block_iters,
                          int dense_sweeps, double omega, double target, double theta, double lambda) {
    Ctx* C = (Ctx*)h;
    C->P.mode = mode;
    C->P.pre = pre;
    C->P.post = post;
    C->P.coarsest_iters = coarsest_iters;
    C->P.block_iters = block_iters;
    C->P.dense_sweeps = dense_sweeps;
    C->P.omega = omega;
    C->P.target = target;
    C->P.theta = theta;
    C->P.lambda = lambda;
    C->built = false;
}

// FV hierarchy rule for coarse fluid flags: 1 = a coarse cell is fluid iff all its children are,
// 0 = iff any child is.
OC_API void oc_set_coarse_all(void* h, int all) {
    Ctx* C = (Ctx*)h;
    C->P.coarse_all = all;
    C->built = false;
}

// Offsets at MG level m (vanish = reference semantics).  out: 4*nb (cell, fx, fy, fz); tot: 4
OC_API void oc_offsets(void* h, int m, int vanish, uint32_t* out, uint32_t* tot) {
    Ctx* C = (Ctx*)h;
    int nb = C->g.nb();
    Lvl L;
    L.res.resize(nb);
    for (int b = 0; b < nb; ++b) L.res[b] = res_at(*C, b, m, vanish != 0);
    make_offsets(L, nb);
    for (int k = 0; k < 4; ++k) {
        std::copy(L.off[k].begin(), L.off[k].end(), out + (size_t)k * nb);
        tot[k] = L.tot[k];
    }
}

// Galerkin coarse coefficient (reference formula, single precision as the reference computes it)
OC_API void oc_galerkin_ref(void* h, int dest, const float* fine[3], float* coarse[3]) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    int nb = g.nb();
    Lvl F, K;
    F.res.resize(nb);
    K.res.resize(nb);
    for (int b = 0; b < nb; ++b) {
        F.res[b] = res_at(*C, b, dest - 1, true);
        K.res[b] = res_at(*C, b, dest, true);
    }
    make_offsets(F, nb);
    make_offsets(K, nb);
    const float SCF = 1 / (4 * 0.75f);
    const float SFC = 2 * SCF;
    for (int b = 0; b < nb; ++b) {
        uint32_t l = C->level[b];
        if ((int)l >= g.L) continue;
        int fr = g.R0 >> (l + dest - 1), cr = g.R0 >> (l + dest);
        if (cr < 1 || fr < 2) continue;
        int cb[3];
        bcoord(g, b, cb);
        for (int a = 0; a < 3; ++a) {
            int dim[3] = {cr + (a == 0), cr + (a == 1), cr + (a == 2)};
            for (int tz = 0; tz < dim[2]; ++tz)
                for (int ty = 0; ty < dim[1]; ++ty)
                    for (int tx = 0; tx < dim[0]; ++tx) {
                        int t[3] = {tx, ty, tz};
                        float baseS = (float)(1 << l);
                        if (t[a] == 0 || t[a] == cr) {
                            int nc[3] = {cb[0], cb[1], cb[2]};
                            nc[a] += t[a] == 0 ? -1 : 1;
                            uint32_t nl = inside(g, nc) ? C->level[bidx(g, nc[0], nc[1], nc[2])] : l;
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
                                if (a == 0) { q[1] += d1; q[2] += d2; }
                                else if (a == 1) { q[0] += d1; q[2] += d2; }
                                else { q[0] += d1; q[1] += d2; }
                                sum += fine[a][F.off[1 + a][b] + fidx(a, q[0], q[1], q[2], fr)];
                            }
                        coarse[a][K.off[1 + a][b] + fidx(a, tx, ty, tz, cr)] = s * (sum * 0.25f);
                    }
        }
    }
}

// Build the solver hierarchy.  bbar/W0 may be null.  fluid0 may be null (all fluid).
OC_API int oc_build(void* h, const double* bx, const double* by, const double* bz, const uint8_t* fluid0,
                    int mg_levels) {
    Ctx* C = (Ctx*)h;
    const double* bb[3] = {bx, by, bz};
    const double* nul[3] = {nullptr, nullptr, nullptr};
    if (C->P.mode == 1) build_hierarchy(*C, nul, fluid0, bb, mg_levels);
    else build_hierarchy(*C, bb, fluid0, nul, mg_levels);
    return (int)C->lv.size();
}

OC_API int oc_num_levels(void* h) { return (int)((Ctx*)h)->lv.size(); }

// Level info: [dense, D0, D1, D2, ncell, nfx, nfy, nfz]
OC_API void oc_level_info(void* h, int m, int64_t* out) {
    Lvl& L = ((Ctx*)h)->lv[m];
    out[0] = L.dense;
    out[1] = L.D[0];
    out[2] = L.D[1];
    out[3] = L.D[2];
    if (L.dense) {
        out[4] = (int64_t)L.D[0] * L.D[1] * L.D[2];
        for (int a = 0; a < 3; ++a) out[5 + a] = (int64_t)L.W[a].size();
    } else {
        for (int k = 0; k < 4; ++k) out[4 + k] = L.tot[k];
    }
}

// Access level arrays: which 0=x 1=b 2=r 3=Wx 4=Wy 5=Wz 6=fluid(as double)
OC_API void oc_get(void* h, int m, int which, double* out) {
    Lvl& L = ((Ctx*)h)->lv[m];
    if (which == 0) std::copy(L.x.begin(), L.x.end(), out);
    else if (which == 1) std::copy(L.b.begin(), L.b.end(), out);
    else if (which == 2) std::copy(L.r.begin(), L.r.end(), out);
    else if (which >= 3 && which <= 5) std::copy(L.W[which - 3].begin(), L.W[which - 3].end(), out);
    else if (which == 6)
        for (size_t i = 0; i < L.fluid.size(); ++i) out[i] = L.fluid[i];
}
OC_API void oc_set(void* h, int m, int which, const double* in) {
    Lvl& L = ((Ctx*)h)->lv[m];
    if (which == 0) std::copy(in, in + L.x.size(), L.x.begin());
    else if (which == 1) std::copy(in, in + L.b.size(), L.b.begin());
    else if (which >= 3 && which <= 5) std::copy(in, in + L.W[which - 3].size(), L.W[which - 3].begin());
}

OC_API void oc_smooth(void* h, int m, int iterations) { smooth_level(*(Ctx*)h, m, iterations); }
OC_API void oc_residual(void* h, int m) {
    Ctx* C = (Ctx*)h;
    Lvl& L = C->lv[m];
    residual_level(*C, m, L.x.data(), L.b.data(), L.r.data());
}
OC_API void oc_restrict(void* h, int m) { restrict_level(*(Ctx*)h, m); }
OC_API void oc_prolong(void* h, int m) { prolong_level(*(Ctx*)h, m); }
OC_API void oc_vcycle(void* h) { vcycle(*(Ctx*)h, 0); }
OC_API void oc_coarsest(void* h) {
    Ctx* C = (Ctx*)h;
    coarsest_solve(*C, (int)C->lv.size() - 1);
}

// Defect-correction solve of A p = b on level 0 to relative residual tol (FP64 throughout).
// p (in/out), b (in).  history (optional, max_cycles+1 entries) gets ||r||/||b|| per cycle.
OC_API int oc_solve(void* h, double* p, const double* b, double tol, int max_cycles, double* history) {
    Ctx* C = (Ctx*)h;
    Lvl& L = C->lv[0];
    size_t n = L.tot[0];
    std::vector<double> r(n), pv(p, p + n);
    double bn = 0;
    for (size_t i = 0; i < n; ++i) bn += (L.fluid[i] || C->P.mode == 1) ? b[i] * b[i] : 0.0;
    bn = std::sqrt(bn);
    if (bn == 0) bn = 1;
    int it = 0;
    for (;; ++it) {
        residual_level(*C, 0, pv.data(), b, r.data());
        double rel = norm2(r) / bn;
        if (history) history[it] = rel;
        if (rel < tol || it >= max_cycles) break;
        std::copy(r.begin(), r.end(), L.b.begin());
        std::fill(L.x.begin(), L.x.end(), 0.0);
        vcycle(*C, 0);
        for (size_t i = 0; i < n; ++i) pv[i] += L.x[i];
    }
    std::copy(pv.begin(), pv.end(), p);
    return it;
}

OC_API void oc_apply(void* h, int m, const double* x, double* y) {
    Ctx* C = (Ctx*)h;
    Lvl& L = C->lv[m];
    std::vector<double> z(L.x.size(), 0.0);
    residual_level(*C, m, x, z.data(), y);
    for (size_t i = 0; i < L.x.size(); ++i) y[i] = -y[i];
}

// ---------------------------------- particles ------------------------------------------------
OC_API void oc_particle_keys(void* h, const float* pos, int64_t n, uint32_t* keys, int64_t* perm) {
    Ctx* C = (Ctx*)h;
    PartGrid PG = make_pgrid(*C);
    std::vector<uint32_t> k(n);
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) k[i] = particle_key(PG, pos + 3 * i);
    std::vector<int64_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return k[a] < k[b]; });
    if (keys) std::copy(k.begin(), k.end(), keys);
    if (perm) std::copy(idx.begin(), idx.end(), perm);
}

// P2G (gather form) on sorted or unsorted particles.  u/m per axis (level-0 face layout).
// cell_count: particles per level-0 cell.
namespace {
template <class PT>
void p2g_impl(Ctx* C, const PT* pos, const PT* vel, int64_t n, double* ux, double* uy, double* uz, double* mx,
              double* my, double* mz, uint32_t* cell_count, const float* phase = nullptr, double* const* phi = nullptr) {
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
    std::vector<uint32_t> k(n);
    for (int64_t i = 0; i < n; ++i) {
        const float pf[3] = {(float)pos[3 * i], (float)pos[3 * i + 1], (float)pos[3 * i + 2]};
        k[i] = particle_key(PG, pf);
    }
    std::vector<int64_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return k[a] < k[b]; });
    std::vector<int64_t> start(PG.tot[0] + 1, 0);
    for (int64_t i = 0; i < n; ++i)
        if (k[i] != 0xFFFFFFFFu) start[k[i] + 1]++;
    for (size_t c = 0; c < PG.tot[0]; ++c) start[c + 1] += start[c];
    if (cell_count)
        for (size_t c = 0; c < PG.tot[0]; ++c) cell_count[c] = (uint32_t)(start[c + 1] - start[c]);
    double* U[3] = {ux, uy, uz};
    double* Mm[3] = {mx, my, mz};
    int nb = g.nb();
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nb; ++b) {
        int r = PG.res[b];
        if (!r) continue;
        int cb[3];
        bcoord(g, b, cb);
        double h_ = (double)fcell(g, r);
        double R2 = h_ * h_;
        double org[3];
        for (int a = 0; a < 3; ++a) org[a] = (double)forigin(g, a, cb[a]);
        for (int a = 0; a < 3; ++a) {
            int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            for (int fa = 0; fa <= r; ++fa)
                for (int u1 = 0; u1 < r; ++u1)
                    for (int u2 = 0; u2 < r; ++u2) {
                        int f[3];
                        f[a] = fa; f[t1] = u1; f[t2] = u2;
                        double xf[3];
                        for (int q = 0; q < 3; ++q) xf[q] = org[q] + h_ * (f[q] + (q == a ? 0.0 : 0.5));
                        double msum = 0, psum = 0, qsum = 0;
                        // blocks intersecting the support box
                        int blo[3], bhi[3];
                        for (int q = 0; q < 3; ++q) {
                            blo[q] = std::max(0, (int)std::floor((xf[q] - h_ - g.dmin[q]) / g.bs));
                            bhi[q] = std::min(g.D[q] - 1, (int)std::floor((xf[q] + h_ - g.dmin[q]) / g.bs));
                        }
                        for (int nz = blo[2]; nz <= bhi[2]; ++nz)
                            for (int ny = blo[1]; ny <= bhi[1]; ++ny)
                                for (int nx = blo[0]; nx <= bhi[0]; ++nx) {
                                    int nbk = bidx(g, nx, ny, nz);
                                    int rn = PG.res[nbk];
                                    if (!rn) continue;
                                    int ncb[3] = {nx, ny, nz};
                                    double hn = (double)fcell(g, rn);
                                    int clo[3], chi[3];
                                    for (int q = 0; q < 3; ++q) {
                                        double o = (double)forigin(g, q, ncb[q]);
                                        clo[q] = std::max(0, (int)std::floor((xf[q] - h_ - o) / hn));
                                        chi[q] = std::min(rn - 1, (int)std::floor((xf[q] + h_ - o) / hn));
                                    }
                                    for (int cz = clo[2]; cz <= chi[2]; ++cz)
                                        for (int cy = clo[1]; cy <= chi[1]; ++cy)
                                            for (int cx = clo[0]; cx <= chi[0]; ++cx) {
                                                uint32_t key = PG.off[0][nbk] + cidx(cx, cy, cz, rn);
                                                for (int64_t s = start[key]; s < start[key + 1]; ++s) {
                                                    int64_t p = idx[s];
                                                    double d2 = 0;
                                                    for (int q = 0; q < 3; ++q) {
                                                        double dd = (double)pos[3 * p + q] - xf[q];
                                                        d2 += dd * dd;
                                                    }
                                                    double w = kernel_w(d2, R2);
                                                    msum += w;
                                                    psum += w * (double)vel[3 * p + a];
                                                    if (phase) qsum += w * (double)phase[p];
                                                }
                                            }
                                }
                        uint32_t fi = PG.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r);
                        Mm[a][fi] = msum;
                        U[a][fi] = msum > 1e-6 ? psum / msum : 0.0;
                        if (phase) phi[a][fi] = msum > 1e-6 ? std::min(1.0, std::max(0.0, qsum / msum)) : 0.0;
                    }
        }
    }
}

}  // namespace

OC_API void oc_p2g(void* h, const float* pos, const float* vel, int64_t n, double* ux, double* uy, double* uz,
                   double* mx, double* my, double* mz, uint32_t* cell_count) {
    p2g_impl((Ctx*)h, pos, vel, n, ux, uy, uz, mx, my, mz, cell_count);
}
// Two-phase P2G: also the face phase phi = sum w phase / sum w (0 where the mass is <= 1e-6),
// the channel PHASE_FIELD_* (MSBG.cuh:21-29) whose accumulation P2G.cuh:94-97 leaves commented out.
OC_API void oc_p2g_phase(void* h, const float* pos, const float* vel, const float* phase, int64_t n, double* ux,
                         double* uy, double* uz, double* mx, double* my, double* mz, double* px, double* py,
                         double* pz, uint32_t* cell_count) {
    double* phi[3] = {px, py, pz};
    p2g_impl((Ctx*)h, pos, vel, n, ux, uy, uz, mx, my, mz, cell_count, phase, phi);
}

// Face coefficients at T-junctions: the coarse face and the 4 fine faces it covers all take the
// mean of the 4 fine values (equal coefficients on both sides keep the FV operator symmetric).
OC_API void oc_beta_sync(void* h, double* bx, double* by, double* bz) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
    double* B[3] = {bx, by, bz};
    for (int b = 0; b < g.nb(); ++b) {
        int r = PG.res[b];
        if (!r) continue;
        int cb[3];
        bcoord(g, b, cb);
        for (int a = 0; a < 3; ++a) {
            int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            for (int s = -1; s <= 1; s += 2) {
                int nc[3] = {cb[0], cb[1], cb[2]};
                nc[a] += s;
                if (!inside(g, nc)) continue;
                int n = bidx(g, nc[0], nc[1], nc[2]);
                int rn = PG.res[n];
                if (rn != 2 * r) continue;
                for (int u1 = 0; u1 < r; ++u1)
                    for (int u2 = 0; u2 < r; ++u2) {
                        uint32_t fine[4];
                        double sum = 0;
                        for (int k = 0; k < 4; ++k) {
                            int q[3];
                            q[a] = s > 0 ? 0 : rn;
                            q[t1] = 2 * u1 + k / 2;
                            q[t2] = 2 * u2 + k % 2;
                            fine[k] = PG.off[1 + a][n] + fidx(a, q[0], q[1], q[2], rn);
                            sum += B[a][fine[k]];
                        }
                        for (int k = 0; k < 4; ++k) B[a][fine[k]] = 0.25 * sum;
                        int f[3];
                        f[a] = s > 0 ? r : 0;
                        f[t1] = u1;
                        f[t2] = u2;
                        B[a][PG.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r)] = 0.25 * sum;
                    }
            }
        }
    }
}

// P2G on FP64 particle state (the differentiable rollout); cells of particles from float(pos)
OC_API void oc_p2g64(void* h, const double* pos, const double* vel, int64_t n, double* ux, double* uy, double* uz,
                     double* mx, double* my, double* mz, uint32_t* cell_count) {
    p2g_impl((Ctx*)h, pos, vel, n, ux, uy, uz, mx, my, mz, cell_count);
}

// T-junction sync: a coarse block's boundary face := mean of the 4 fine faces it covers.
OC_API void oc_face_sync(void* h, double* ux, double* uy, double* uz) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
    double* U[3] = {ux, uy, uz};
    int nb = g.nb();
    for (int b = 0; b < nb; ++b) {
        int r = PG.res[b];
        if (!r) continue;
        int cb[3];
        bcoord(g, b, cb);
        for (int a = 0; a < 3; ++a) {
            int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            for (int s = -1; s <= 1; s += 2) {
                int nc[3] = {cb[0], cb[1], cb[2]};
                nc[a] += s;
                if (!inside(g, nc)) continue;
                int n = bidx(g, nc[0], nc[1], nc[2]);
                int rn = PG.res[n];
                if (rn != 2 * r) continue;
                for (int u1 = 0; u1 < r; ++u1)
                    for (int u2 = 0; u2 < r; ++u2) {
                        double sum = 0;
                        for (int d1 = 0; d1 < 2; ++d1)
                            for (int d2 = 0; d2 < 2; ++d2) {
                                int q[3];
                                q[a] = s > 0 ? 0 : rn;
                                q[t1] = 2 * u1 + d1;
                                q[t2] = 2 * u2 + d2;
                                sum += U[a][PG.off[1 + a][n] + fidx(a, q[0], q[1], q[2], rn)];
                            }
                        int f[3];
                        f[a] = s > 0 ? r : 0;
                        f[t1] = u1;
                        f[t2] = u2;
                        U[a][PG.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r)] = 0.25 * sum;
                    }
            }
        }
    }
}

// Zero faces on the domain boundary (solid walls, u.n = 0).
OC_API void oc_wall_bc(void* h, double* ux, double* uy, double* uz) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
    double* U[3] = {ux, uy, uz};
    for (int b = 0; b < g.nb(); ++b) {
        int r = PG.res[b];
        if (!r) continue;
        int cb[3];
        bcoord(g, b, cb);
        for (int a = 0; a < 3; ++a) {
            int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            for (int side = 0; side < 2; ++side) {
                if (side == 0 && cb[a] != 0) continue;
                if (side == 1 && cb[a] != g.D[a] - 1) continue;
                for (int u1 = 0; u1 < r; ++u1)
                    for (int u2 = 0; u2 < r; ++u2) {
                        int f[3];
                        f[a] = side ? r : 0;
                        f[t1] = u1;
                        f[t2] = u2;
                        U[a][PG.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r)] = 0.0;
                    }
            }
        }
    }
}

// rhs b = div(u)/dt on fluid cells (level 0 layout); fluid from cell_count > 0
OC_API void oc_divergence(void* h, const double* ux, const double* uy, const double* uz, const uint8_t* fluid,
                          double inv_dt, double* bout) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
    const double* U[3] = {ux, uy, uz};
    for (int b = 0; b < g.nb(); ++b) {
        int r = PG.res[b];
        if (!r) continue;
        double H = (double)g.bs / r;
        for (int z = 0; z < r; ++z)
            for (int y = 0; y < r; ++y)
                for (int x = 0; x < r; ++x) {
                    uint32_t ci = PG.off[0][b] + cidx(x, y, z, r);
                    if (!fluid[ci]) { bout[ci] = 0.0; continue; }
                    int c[3] = {x, y, z};
                    double d = 0;
                    for (int a = 0; a < 3; ++a) {
                        int hi[3] = {c[0], c[1], c[2]};
                        hi[a] += 1;
                        d += U[a][PG.off[1 + a][b] + fidx(a, hi[0], hi[1], hi[2], r)] -
                             U[a][PG.off[1 + a][b] + fidx(a, c[0], c[1], c[2], r)];
                    }
                    bout[ci] = d * H * H * inv_dt;
                }
    }
}

// Pressure-gradient update on level 0 face copies: u -= dt * (W/area) * (p_high - p_low) on
// faces with a fluid cell on at least one side.  Uses the level-0 hierarchy (oc_build first).
OC_API void oc_gradient_update(void* h, const double* p, double dt, double* ux, double* uy, double* uz) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    Lvl& L = C->lv[0];
    double* U[3] = {ux, uy, uz};
    for (int b = 0; b < g.nb(); ++b) {
        int r = L.res[b];
        if (!r) continue;
        int cb[3];
        bcoord(g, b, cb);
        double H = (double)g.bs / r;
        double area = H * H;
        for (int a = 0; a < 3; ++a) {
            int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            for (int fa = 0; fa <= r; ++fa)
                for (int u1 = 0; u1 < r; ++u1)
                    for (int u2 = 0; u2 < r; ++u2) {
                        int f[3];
                        f[a] = fa; f[t1] = u1; f[t2] = u2;
                        uint32_t fi = L.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r);
                        double W = L.W[a][fi];
                        // low and high cells
                        double pv[2];
                        bool fl[2];
                        bool wall = false;
                        for (int side = 0; side < 2; ++side) {
                            int c[3] = {f[0], f[1], f[2]};
                            if (side == 0) c[a] -= 1;
                            if (c[a] >= 0 && c[a] < r) {
                                uint32_t ci = L.off[0][b] + cidx(c[0], c[1], c[2], r);
                                pv[side] = p[ci];
                                fl[side] = L.fluid[ci];
                            } else {
                                int cin[3] = {f[0], f[1], f[2]};
                                if (side == 0) cin[a] = 0; else cin[a] = r - 1;
                                Ghost gh = ghost(g, L, p, b, cb, cin, a, side == 0 ? -1 : 1);
                                if (gh.kind == 0) wall = true;
                                pv[side] = gh.v;
                                fl[side] = gh.fluid;
                            }
                        }
                        if (wall) { U[a][fi] = 0.0; continue; }
                        if (!fl[0] && !fl[1]) continue;
                        U[a][fi] -= dt * (W / area) * (pv[1] - pv[0]);
                    }
        }
    }
}

// G2P FLIP blend (g2pUpdateKernel, G2P.cuh:87-128) for every particle.
OC_API void oc_g2p(void* h, const float* pos, int64_t n, const double* un[3], const double* uo[3], double alpha,
                   const float* vin, double* vout) {
    Ctx* C = (Ctx*)h;
    PartGrid PG = make_pgrid(*C);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double X[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        for (int a = 0; a < 3; ++a) {
            double vn = sample(*C, PG, un[a], a, X);
            double vo = sample(*C, PG, uo[a], a, X);
            double vp = vin[3 * i + a];
            vout[3 * i + a] = alpha * (vp + (vn - vo)) + (1.0 - alpha) * vn;
        }
    }
}

// Sample velocity (3 components) at positions.
OC_API void oc_sample(void* h, const double* X, int64_t n, const double* u[3], double* out) {
    Ctx* C = (Ctx*)h;
    PartGrid PG = make_pgrid(*C);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) out[3 * i + a] = sample(*C, PG, u[a], a, X + 3 * i);
}

// Ralston RK3 advection (advectParticlesKernel, G2P.cuh:131-173), clamp to the domain interior
// with a margin of 0.01 finest cells.
OC_API void oc_advect(void* h, const double* u[3], double dt, const double* xin, int64_t n, double* xout) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
    double h0 = (double)g.bs / g.R0;
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = g.dmin[a] + 0.01 * h0;
        hi[a] = g.dmin[a] + (double)g.D[a] * g.bs - 0.01 * h0;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double x[3] = {xin[3 * i], xin[3 * i + 1], xin[3 * i + 2]};
        double k1[3], k2[3], k3[3], x2[3], x3[3];
        for (int a = 0; a < 3; ++a) k1[a] = sample(*C, PG, u[a], a, x);
        for (int a = 0; a < 3; ++a) x2[a] = x[a] + 0.5 * dt * k1[a];
        for (int a = 0; a < 3; ++a) k2[a] = sample(*C, PG, u[a], a, x2);
        for (int a = 0; a < 3; ++a) x3[a] = x[a] + 0.75 * dt * k2[a];
        for (int a = 0; a < 3; ++a) k3[a] = sample(*C, PG, u[a], a, x3);
        for (int a = 0; a < 3; ++a) {
            double v = (2.0 / 9.0) * k1[a] + (3.0 / 9.0) * k2[a] + (4.0 / 9.0) * k3[a];
            double y = x[a] + dt * v;
            xout[3 * i + a] = std::min(std::max(y, lo[a]), hi[a]);
        }
    }
}

// ================================================================================================
// Adjoint of the FLIP step (vector-Jacobian products), FP64.
//
// The forward map differentiated is the step above with its discrete decisions held fixed: the
// cell of every particle, the fluid flags, each kernel's support, the clamp branches of the
// trilinear sample and of the advection.  Every VJP accumulates (+=) into its output adjoints.
// The projection's adjoint reuses the forward solve: the FV operator is symmetric, so
// b_bar = A^{-1} p_bar is one more solve with the same hierarchy.
// ================================================================================================
namespace {

// index (into the axis-a face array) of the face that supplies ghost face fi of block b — the
// rule of face_value_at
uint32_t face_src(const Ctx& C, const PartGrid& PG, int a, int b, const int cb[3], int r, const int fi[3]) {
    const Geo& g = C.g;
    int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
    int o1 = fi[t1] < 0 ? -1 : (fi[t1] >= r ? 1 : 0);
    int o2 = fi[t2] < 0 ? -1 : (fi[t2] >= r ? 1 : 0);
    if (!o1 && !o2) return PG.off[1 + a][b] + fidx(a, fi[0], fi[1], fi[2], r);
    int nc[3] = {cb[0], cb[1], cb[2]};
    nc[t1] += o1;
    nc[t2] += o2;
    int rn = 0, n = 0;
    if (inside(g, nc)) {
        n = bidx(g, nc[0], nc[1], nc[2]);
        rn = PG.res[n];
    }
    if (!rn) {
        int q[3] = {fi[0], fi[1], fi[2]};
        q[t1] = std::min(std::max(q[t1], 0), r - 1);
        q[t2] = std::min(std::max(q[t2], 0), r - 1);
        return PG.off[1 + a][b] + fidx(a, q[0], q[1], q[2], r);
    }
    int q[3];
    q[a] = (2 * fi[a] * rn + r) / (2 * r);
    int rel1 = 2 * fi[t1] + 1 - o1 * 2 * r;
    int rel2 = 2 * fi[t2] + 1 - o2 * 2 * r;
    q[t1] = std::min(std::max((rel1 * rn) / (2 * r), 0), rn - 1);
    q[t2] = std::min(std::max((rel2 * rn) / (2 * r), 0), rn - 1);
    return PG.off[1 + a][n] + fidx(a, q[0], q[1], q[2], rn);
}

// Trilinear MAC sample of component a at X as a stencil: 8 source faces, their weights and the
// derivative of each weight with respect to X (zero along a clamped axis).
struct Stencil {
    int n = 0;
    uint32_t idx[8];
    double w[8];
    double dw[8][3];
};

Stencil sample_stencil(const Ctx& C, const PartGrid& PG, int a, const double X[3]) {
    Stencil S;
    const Geo& g = C.g;
    float Xf[3] = {(float)X[0], (float)X[1], (float)X[2]};
    int cb[3];
    point_block(g, Xf, cb);
    int b = bidx(g, cb[0], cb[1], cb[2]);
    int r = PG.res[b];
    if (!r) return S;
    double h = (double)fcell(g, r);
    int i0[3];
    double f[3], df[3];
    for (int k = 0; k < 3; ++k) {
        double o = (double)forigin(g, k, cb[k]);
        double s = (X[k] - o) / h;
        int lo = 0, hi = r;
        if (k != a) { s -= 0.5; lo = -1; }
        df[k] = (s > lo && s < hi) ? 1.0 / h : 0.0;
        s = std::min(std::max(s, (double)lo), (double)hi);
        int i = (int)std::floor(s);
        i = std::min(std::max(i, lo), hi - 1);
        i0[k] = i;
        f[k] = s - i;
    }
    S.n = 8;
    int k = 0;
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx, ++k) {
                int fi[3] = {i0[0] + dx, i0[1] + dy, i0[2] + dz};
                double wx = dx ? f[0] : 1 - f[0], wy = dy ? f[1] : 1 - f[1], wz = dz ? f[2] : 1 - f[2];
                double sx = dx ? 1.0 : -1.0, sy = dy ? 1.0 : -1.0, sz = dz ? 1.0 : -1.0;
                S.idx[k] = face_src(C, PG, a, b, cb, r, fi);
                S.w[k] = wx * wy * wz;
                S.dw[k][0] = sx * wy * wz * df[0];
                S.dw[k][1] = wx * sy * wz * df[1];
                S.dw[k][2] = wx * wy * sz * df[2];
            }
    return S;
}

inline void atomic_add(double* p, double v) {
#pragma omp atomic
    *p += v;
}

// y = I(u, X) for one component: ubar[idx] += w * ybar; Xbar += ybar * sum_k dw_k u[idx_k]
void sample_vjp(const Ctx& C, const PartGrid& PG, const double* u, int a, const double X[3], double ybar,
                double* ubar, double* Xbar) {
    Stencil S = sample_stencil(C, PG, a, X);
    for (int k = 0; k < S.n; ++k) {
        if (ubar) atomic_add(&ubar[S.idx[k]], S.w[k] * ybar);
        if (Xbar)
            for (int j = 0; j < 3; ++j) Xbar[j] += ybar * S.dw[k][j] * u[S.idx[k]];
    }
}

double sample_val(const Ctx& C, const PartGrid& PG, const double* u, int a, const double X[3]) {
    Stencil S = sample_stencil(C, PG, a, X);
    double acc = 0;
    for (int k = 0; k < S.n; ++k) acc += S.w[k] * u[S.idx[k]];
    return acc;
}

}  // namespace

// Sample (3 components) at FP64 points through the stencil form (equals oc_sample).
OC_API void oc_sample_stencil(void* h, const double* X, int64_t n, const double* u[3], double* out) {
    Ctx* C = (Ctx*)h;
    PartGrid PG = make_pgrid(*C);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) out[3 * i + a] = sample_val(*C, PG, u[a], a, X + 3 * i);
}

// VJP of y = sample(u, X): ubar += I^T ybar; Xbar += (dI/dX)^T ybar (Xbar may be null)
OC_API void oc_sample_vjp(void* h, const double* X, int64_t n, const double* u[3], const double* ybar, double* ubar[3],
                          double* Xbar) {
    Ctx* C = (Ctx*)h;
    PartGrid PG = make_pgrid(*C);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a)
            sample_vjp(*C, PG, u[a], a, X + 3 * i, ybar[3 * i + a], ubar[a], Xbar ? Xbar + 3 * i : nullptr);
}

// G2P on FP64 state: v' = alpha (v + I(un) - I(uo)) + (1 - alpha) I(un)
OC_API void oc_g2p64(void* h, const double* X, int64_t n, const double* un[3], const double* uo[3], double alpha,
                     const double* vin, double* vout) {
    Ctx* C = (Ctx*)h;
    PartGrid PG = make_pgrid(*C);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            double vn = sample_val(*C, PG, un[a], a, X + 3 * i);
            double vo = sample_val(*C, PG, uo[a], a, X + 3 * i);
            vout[3 * i + a] = alpha * (vin[3 * i + a] + (vn - vo)) + (1.0 - alpha) * vn;
        }
}

// VJP of oc_g2p64.  vbar: adjoint of v' on input, adjoint of v on output.  Xbar, unbar, uobar +=.
OC_API void oc_g2p_vjp(void* h, const double* X, int64_t n, const double* un[3], const double* uo[3], double alpha,
                       double* vbar, double* Xbar, double* unbar[3], double* uobar[3]) {
    Ctx* C = (Ctx*)h;
    PartGrid PG = make_pgrid(*C);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            const double g = vbar[3 * i + a];
            sample_vjp(*C, PG, un[a], a, X + 3 * i, g, unbar[a], Xbar + 3 * i);
            sample_vjp(*C, PG, uo[a], a, X + 3 * i, -alpha * g, uobar[a], Xbar + 3 * i);
            vbar[3 * i + a] = alpha * g;
        }
}

// VJP of oc_advect (Ralston RK3 + clamp).  xbar: adjoint of x' on input, of x on output.
OC_API void oc_advect_vjp(void* h, const double* u[3], double dt, const double* xin, int64_t n, double* xbar,
                          double* ubar[3]) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
    double h0 = (double)g.bs / g.R0;
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = g.dmin[a] + 0.01 * h0;
        hi[a] = g.dmin[a] + (double)g.D[a] * g.bs - 0.01 * h0;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double* x = xin + 3 * i;
        double k1[3], k2[3], k3[3], y1[3], y2[3];
        for (int a = 0; a < 3; ++a) k1[a] = sample_val(*C, PG, u[a], a, x);
        for (int a = 0; a < 3; ++a) y1[a] = x[a] + 0.5 * dt * k1[a];
        for (int a = 0; a < 3; ++a) k2[a] = sample_val(*C, PG, u[a], a, y1);
        for (int a = 0; a < 3; ++a) y2[a] = x[a] + 0.75 * dt * k2[a];
        for (int a = 0; a < 3; ++a) k3[a] = sample_val(*C, PG, u[a], a, y2);
        double gx[3], k1b[3], k2b[3], k3b[3], y1b[3] = {0, 0, 0}, y2b[3] = {0, 0, 0};
        for (int a = 0; a < 3; ++a) {
            double v = (2.0 / 9.0) * k1[a] + (3.0 / 9.0) * k2[a] + (4.0 / 9.0) * k3[a];
            double y = x[a] + dt * v;
            double gb = (y > lo[a] && y < hi[a]) ? xbar[3 * i + a] : 0.0;
            gx[a] = gb;
            k1b[a] = (2.0 / 9.0) * dt * gb;
            k2b[a] = (3.0 / 9.0) * dt * gb;
            k3b[a] = (4.0 / 9.0) * dt * gb;
        }
        for (int a = 0; a < 3; ++a) sample_vjp(*C, PG, u[a], a, y2, k3b[a], ubar[a], y2b);
        for (int a = 0; a < 3; ++a) {
            gx[a] += y2b[a];
            k2b[a] += 0.75 * dt * y2b[a];
        }
        for (int a = 0; a < 3; ++a) sample_vjp(*C, PG, u[a], a, y1, k2b[a], ubar[a], y1b);
        for (int a = 0; a < 3; ++a) {
            gx[a] += y1b[a];
            k1b[a] += 0.5 * dt * y1b[a];
        }
        for (int a = 0; a < 3; ++a) sample_vjp(*C, PG, u[a], a, x, k1b[a], ubar[a], gx);
        for (int a = 0; a < 3; ++a) xbar[3 * i + a] = gx[a];
    }
}

// VJP of oc_p2g64 through the normalisation u = P/m (m > 1e-6): given ubar per face and the
// forward u, m, accumulate pos_bar and vel_bar per particle.  Every particle gathers from the
// faces within one cell size (of the face's block) of it, in its own and the 26 neighbouring
// blocks.
OC_API void oc_p2g_vjp(void* h, const double* pos, const double* vel, int64_t n, const double* u[3],
                       const double* m[3], const double* ubar[3], double* pos_bar, double* vel_bar) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        const double* X = pos + 3 * i;
        float Xf[3] = {(float)X[0], (float)X[1], (float)X[2]};
        int pc[3];
        point_block(g, Xf, pc);
        double xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0};
        for (int d = 0; d < 27; ++d) {
            int nc[3] = {pc[0] + d % 3 - 1, pc[1] + (d / 3) % 3 - 1, pc[2] + d / 9 - 1};
            if (!inside(g, nc)) continue;
            int b = bidx(g, nc[0], nc[1], nc[2]);
            int r = PG.res[b];
            if (!r) continue;
            double hh = (double)fcell(g, r);
            double q[3];
            for (int k = 0; k < 3; ++k) q[k] = (X[k] - (double)forigin(g, k, nc[k])) / hh;
            bool out = false;
            for (int k = 0; k < 3; ++k) out |= q[k] <= -1.0 || q[k] >= r + 1.0;
            if (out) continue;
            for (int a = 0; a < 3; ++a) {
                int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
                int ia = (int)std::floor(q[a]);
                int j1 = (int)std::floor(q[t1] - 0.5), j2 = (int)std::floor(q[t2] - 0.5);
                for (int da = 0; da < 2; ++da)
                    for (int d1 = 0; d1 < 2; ++d1)
                        for (int d2 = 0; d2 < 2; ++d2) {
                            int f[3];
                            f[a] = ia + da;
                            f[t1] = j1 + d1;
                            f[t2] = j2 + d2;
                            if (f[a] < 0 || f[a] > r || f[t1] < 0 || f[t1] >= r || f[t2] < 0 || f[t2] >= r) continue;
                            double Q[3];
                            for (int k = 0; k < 3; ++k) Q[k] = f[k] + (k == a ? 0.0 : 0.5);
                            double dq[3] = {q[0] - Q[0], q[1] - Q[1], q[2] - Q[2]};
                            double d2s = dq[0] * dq[0] + dq[1] * dq[1] + dq[2] * dq[2];
                            if (d2s >= 1.0) continue;
                            uint32_t fi = PG.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r);
                            double mf = m[a][fi];
                            if (!(mf > 1e-6)) continue;
                            double Pbar = ubar[a][fi] / mf;
                            double mbar = -ubar[a][fi] * u[a][fi] / mf;
                            double t = 1.0 - d2s;
                            double w = t * t * t;
                            double coef = -6.0 * t * t / hh * (Pbar * vel[3 * i + a] + mbar);
                            vb[a] += w * Pbar;
                            for (int k = 0; k < 3; ++k) xb[k] += coef * dq[k];
                        }
            }
        }
        for (int k = 0; k < 3; ++k) {
            pos_bar[3 * i + k] += xb[k];
            vel_bar[3 * i + k] += vb[k];
        }
    }
}

// VJP of oc_face_sync: fine faces receive a quarter of each synced coarse face's adjoint, which
// is then cleared.  In place on ubar.
OC_API void oc_face_sync_vjp(void* h, double* ux, double* uy, double* uz) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
    double* U[3] = {ux, uy, uz};
    for (int b = 0; b < g.nb(); ++b) {
        int r = PG.res[b];
        if (!r) continue;
        int cb[3];
        bcoord(g, b, cb);
        for (int a = 0; a < 3; ++a) {
            int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            for (int s = -1; s <= 1; s += 2) {
                int nc[3] = {cb[0], cb[1], cb[2]};
                nc[a] += s;
                if (!inside(g, nc)) continue;
                int n = bidx(g, nc[0], nc[1], nc[2]);
                int rn = PG.res[n];
                if (rn != 2 * r) continue;
                for (int u1 = 0; u1 < r; ++u1)
                    for (int u2 = 0; u2 < r; ++u2) {
                        int f[3];
                        f[a] = s > 0 ? r : 0;
                        f[t1] = u1;
                        f[t2] = u2;
                        uint32_t ci = PG.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r);
                        double gbar = U[a][ci];
                        U[a][ci] = 0.0;
                        for (int d1 = 0; d1 < 2; ++d1)
                            for (int d2 = 0; d2 < 2; ++d2) {
                                int q[3];
                                q[a] = s > 0 ? 0 : rn;
                                q[t1] = 2 * u1 + d1;
                                q[t2] = 2 * u2 + d2;
                                U[a][PG.off[1 + a][n] + fidx(a, q[0], q[1], q[2], rn)] += 0.25 * gbar;
                            }
                    }
            }
        }
    }
}

// VJP of oc_divergence: ubar += D^T bbar (fluid cells only)
OC_API void oc_divergence_vjp(void* h, const double* bbar, const uint8_t* fluid, double inv_dt, double* ux, double* uy,
                              double* uz) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    PartGrid PG = make_pgrid(*C);
    double* U[3] = {ux, uy, uz};
    for (int b = 0; b < g.nb(); ++b) {
        int r = PG.res[b];
        if (!r) continue;
        double H = (double)g.bs / r;
        for (int z = 0; z < r; ++z)
            for (int y = 0; y < r; ++y)
                for (int x = 0; x < r; ++x) {
                    uint32_t ci = PG.off[0][b] + cidx(x, y, z, r);
                    if (!fluid[ci]) continue;
                    double s = bbar[ci] * H * H * inv_dt;
                    int c[3] = {x, y, z};
                    for (int a = 0; a < 3; ++a) {
                        int hi[3] = {c[0], c[1], c[2]};
                        hi[a] += 1;
                        U[a][PG.off[1 + a][b] + fidx(a, hi[0], hi[1], hi[2], r)] += s;
                        U[a][PG.off[1 + a][b] + fidx(a, c[0], c[1], c[2], r)] -= s;
                    }
                }
    }
}

// VJP of oc_gradient_update: ubar (in place) := ubar with wall faces cleared; pbar += -dt (W/area)
// (d(p_high - p_low)/dp)^T ubar on faces with a fluid cell on either side.
OC_API void oc_gradient_vjp(void* h, double dt, double* ux, double* uy, double* uz, double* pbar) {
    Ctx* C = (Ctx*)h;
    const Geo& g = C->g;
    Lvl& L = C->lv[0];
    double* U[3] = {ux, uy, uz};
    for (int b = 0; b < g.nb(); ++b) {
        int r = L.res[b];
        if (!r) continue;
        int cb[3];
        bcoord(g, b, cb);
        double H = (double)g.bs / r;
        double area = H * H;
        for (int a = 0; a < 3; ++a) {
            int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
            for (int fa = 0; fa <= r; ++fa)
                for (int u1 = 0; u1 < r; ++u1)
                    for (int u2 = 0; u2 < r; ++u2) {
                        int f[3];
                        f[a] = fa; f[t1] = u1; f[t2] = u2;
                        uint32_t fi = L.off[1 + a][b] + fidx(a, f[0], f[1], f[2], r);
                        // cells (and weights) of the low and high pressure values
                        uint32_t cells[2][4];
                        double cw[2][4];
                        int nc_[2] = {0, 0};
                        bool fl[2] = {false, false};
                        bool wall = false;
                        for (int side = 0; side < 2; ++side) {
                            int c[3] = {f[0], f[1], f[2]};
                            if (side == 0) c[a] -= 1;
                            if (c[a] >= 0 && c[a] < r) {
                                uint32_t ci = L.off[0][b] + cidx(c[0], c[1], c[2], r);
                                cells[side][0] = ci;
                                cw[side][0] = 1.0;
                                nc_[side] = 1;
                                fl[side] = L.fluid[ci];
                                continue;
                            }
                            int cin[3] = {f[0], f[1], f[2]};
                            cin[a] = side == 0 ? 0 : r - 1;
                            int s = side == 0 ? -1 : 1;
                            int nb3[3] = {cb[0], cb[1], cb[2]};
                            nb3[a] += s;
                            if (!inside(g, nb3)) { wall = true; continue; }
                            int n = bidx(g, nb3[0], nb3[1], nb3[2]);
                            int rn = L.res[n];
                            if (!rn) continue;
                            int na = s > 0 ? 0 : rn - 1;
                            if (rn == r || 2 * rn == r) {
                                int sh = rn == r ? 0 : 1;
                                int q[3];
                                q[a] = na; q[t1] = cin[t1] >> sh; q[t2] = cin[t2] >> sh;
                                uint32_t ci = L.off[0][n] + cidx(q[0], q[1], q[2], rn);
                                cells[side][0] = ci;
                                cw[side][0] = 1.0;
                                nc_[side] = 1;
                                fl[side] = L.fluid[ci];
                            } else {
                                int k = 0;
                                for (int d1 = 0; d1 < 2; ++d1)
                                    for (int d2 = 0; d2 < 2; ++d2, ++k) {
                                        int q[3];
                                        q[a] = na; q[t1] = 2 * cin[t1] + d1; q[t2] = 2 * cin[t2] + d2;
                                        uint32_t ci = L.off[0][n] + cidx(q[0], q[1], q[2], rn);
                                        cells[side][k] = ci;
                                        cw[side][k] = 0.25;
                                        fl[side] = fl[side] || L.fluid[ci];
                                    }
                                nc_[side] = 4;
                            }
                        }
                        if (wall) { U[a][fi] = 0.0; continue; }
                        if (!fl[0] && !fl[1]) continue;
                        double coef = -dt * (L.W[a][fi] / area) * U[a][fi];
                        for (int k = 0; k < nc_[1]; ++k) pbar[cells[1][k]] += coef * cw[1][k];
                        for (int k = 0; k < nc_[0]; ++k) pbar[cells[0][k]] -= coef * cw[0][k];
                    }
        }
    }
}
