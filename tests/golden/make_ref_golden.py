"""Generate golden fixtures from the reference's OWN CUDA build (oracle/_ref/libawref.so).

Runs on a machine with a GPU (the reference is CUDA-only and has no CPU code).  Inputs are seeded
and restricted to the cases on which the reference is well defined and memory-safe: every block
active, and single-level maps wherever a kernel reads across block boundaries (reference
constants: 16^3 base blocks, 3 levels).  Writes tests/golden/ref_*.npz (or the directory given as
the first argument).  The fixtures pin the oracle (tests/test_golden.py, CPU) and the library's
reference-operator mode (tests/test_golden_gpu.py).

    python tests/golden/make_ref_golden.py [outdir] [--only=transfer]
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libawref.so")

u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C")


def load():
    L = C.CDLL(LIB)
    L.ref_constants.argtypes = [i32p]
    L.ref_device_ok.restype = C.c_int
    L.ref_layout.argtypes = [C.c_int, u32p]
    L.ref_morton.restype = C.c_uint32
    L.ref_morton.argtypes = [C.c_uint32] * 3
    L.ref_block_info.argtypes = [i32p, u32p]
    L.ref_grading.argtypes = [i32p, u32p, i32p]
    L.ref_offsets.argtypes = [i32p, u32p, u32p, u32p]
    L.ref_coarse_offsets.argtypes = [i32p, u32p, C.c_int, C.c_int, u32p, u32p]
    PP = C.POINTER(C.c_void_p)
    L.ref_galerkin.argtypes = [i32p, u32p, C.c_int, PP, PP]
    L.ref_mg_op.argtypes = [i32p, u32p, PP, C.c_int, C.c_int, C.c_int, f32p, f32p, C.c_void_p, C.c_void_p,
                            C.c_void_p, C.c_void_p]
    L.ref_level_beta.argtypes = [i32p, u32p, PP, C.c_int, PP]
    L.ref_normalize.argtypes = [i32p, u32p, PP, PP, PP]
    L.ref_g2p_blend.argtypes = [i32p, C.c_uint32, PP, PP, f32p, f32p, C.c_uint32, C.c_float]
    L.ref_advect.argtypes = [i32p, C.c_uint32, PP, f32p, C.c_uint32, C.c_float]
    return L


def ptrs(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def coarse_offsets(L, dims, lv, m):
    nb = int(np.prod(dims))
    out = np.zeros((4, nb), np.uint32)
    tot = np.zeros(4, np.uint32)
    for k in range(4):
        o = np.zeros(nb, np.uint32)
        t = np.zeros(1, np.uint32)
        assert L.ref_coarse_offsets(np.array(dims, np.int32), lv, m, k, o, t) == 0
        out[k], tot[k] = o, t[0]
    return out, tot


def transfer_fixtures(L, outdir):
    """g2pUpdateKernel (G2P.cuh:87-128) and advectParticlesKernel (G2P.cuh:131-173) on inputs where
    the reference is in bounds and its MAC staggering defects do not matter: single-level maps with
    every block active, a velocity field uniform per axis, and particles at least two cells from the
    domain walls (the reference samples 0 across the wall).  This pins the FLIP blend algebra and the
    RK3 stages given identical sampled velocities.  Reference grid: block size 1, origin 0."""
    rng = np.random.default_rng(2025)
    out = {}
    for case, (dims, level) in enumerate((((2, 2, 2), 0), ((3, 2, 2), 1))):
        d = np.array(dims, np.int32)
        nb = int(np.prod(dims))
        lv = np.full(nb, level, np.uint32)
        _, t = coarse_offsets(L, dims, lv, 0)
        h = 1.0 / (16 >> level)
        n = 4096
        lo = np.array([2 * h] * 3)
        hi = np.array(dims, np.float64) - 2 * h
        pos = (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)
        vel = rng.standard_normal((n, 3)).astype(np.float32)
        cn = rng.standard_normal(3).astype(np.float32)
        co = rng.standard_normal(3).astype(np.float32)
        un = [np.full(int(t[1 + a]), cn[a], np.float32) for a in range(3)]
        uo = [np.full(int(t[1 + a]), co[a], np.float32) for a in range(3)]
        alpha, dt = np.float32(0.95), np.float32(1.0 / 240)
        v_out = vel.copy()
        assert L.ref_g2p_blend(d, level, ptrs(un), ptrs(uo), pos.reshape(-1), v_out.reshape(-1), n, alpha) == 0
        x_out = pos.copy()
        assert L.ref_advect(d, level, ptrs(un), x_out.reshape(-1), n, dt) == 0
        k = f"c{case}_"
        out.update({k + "dims": d, k + "level": np.uint32(level), k + "pos": pos, k + "vel": vel, k + "u_new": cn,
                    k + "u_old": co, k + "alpha": alpha, k + "dt": dt, k + "vel_out": v_out, k + "pos_out": x_out})
    np.savez_compressed(os.path.join(outdir, "ref_transfer.npz"), **out)


def main(outdir, only=None):
    L = load()
    assert L.ref_device_ok(), "needs a CUDA device"
    os.makedirs(outdir, exist_ok=True)
    if only == "transfer":
        transfer_fixtures(L, outdir)
        print("transfer fixtures written to", outdir)
        return
    const = np.zeros(2, np.int32)
    L.ref_constants(const)
    R0, ML = int(const[0]), int(const[1])
    rng = np.random.default_rng(2024)

    # --- layouts, Morton, block info ------------------------------------------------------
    lay = np.zeros((ML, 6), np.uint32)
    for lvl in range(ML):
        L.ref_layout(lvl, lay[lvl])
    mort_in = rng.integers(0, 1024, size=(256, 3)).astype(np.uint32)
    mort = np.array([L.ref_morton(int(x), int(y), int(z)) for x, y, z in mort_in], np.uint32)
    dims_bi = np.array([5, 4, 3], np.int32)
    bi = np.zeros(5 * 60, np.uint32)
    assert L.ref_block_info(dims_bi, bi) == 0
    np.savez_compressed(os.path.join(outdir, "ref_layout.npz"), R0=R0, MAX_LEVELS=ML, layouts=lay, morton_in=mort_in,
                        morton=mort, block_info_dims=dims_bi, block_info=bi.reshape(-1, 5))

    # --- grading and offsets ----------------------------------------------------------------
    cases = {}
    for i, dims in enumerate([(6, 5, 4), (7, 3, 5), (4, 4, 4)]):
        d = np.array(dims, np.int32)
        nb = int(np.prod(dims))
        lv_in = rng.integers(0, ML + 1, size=nb).astype(np.uint32)  # value ML = inactive
        lv = lv_in.copy()
        passes = np.zeros(1, np.int32)
        assert L.ref_grading(d, lv, passes) == 0
        off = np.zeros(4 * nb, np.uint32)
        tot = np.zeros(4, np.uint32)
        assert L.ref_offsets(d, lv, off, tot) == 0
        cases[f"g{i}_dims"] = d
        cases[f"g{i}_in"] = lv_in
        cases[f"g{i}_out"] = lv
        cases[f"g{i}_passes"] = passes
        cases[f"g{i}_offsets"] = off.reshape(4, nb)
        cases[f"g{i}_totals"] = tot
        # coarse offsets on the same map with inactive blocks replaced by the coarsest level
        lv_act = np.where(lv == ML, ML - 1, lv).astype(np.uint32)
        lv_act2 = lv_act.copy()
        L.ref_grading(d, lv_act2, passes)
        cases[f"g{i}_active"] = lv_act2
        for m in range(ML + 1):
            o, t = coarse_offsets(L, dims, lv_act2, m)
            cases[f"g{i}_coarse{m}"] = o
            cases[f"g{i}_coarse{m}_tot"] = t
    # Galerkin coefficients, dest 1 and 2, random fine coefficients, on a small graded
    # three-level map (every block active)
    gd = np.array([3, 2, 2], np.int32)
    glv = np.array([0, 1, 1, 2, 1, 2, 2, 2, 1, 2, 2, 2], np.uint32)
    passes = np.zeros(1, np.int32)
    L.ref_grading(gd, glv, passes)
    cases["gal_dims"] = gd
    cases["gal_levels"] = glv
    for dest in (1, 2):
        fo, ft = coarse_offsets(L, tuple(gd), glv, dest - 1)
        co, ct = coarse_offsets(L, tuple(gd), glv, dest)
        fine = [(0.5 + rng.random(int(ft[1 + a]))).astype(np.float32) for a in range(3)]
        coarse = [np.zeros(max(1, int(ct[1 + a])), np.float32) for a in range(3)]
        assert L.ref_galerkin(gd, glv, dest, ptrs(fine), ptrs(coarse)) == 0
        for a in range(3):
            cases[f"gal{dest}_fine{a}"] = fine[a]
            cases[f"gal{dest}_coarse{a}"] = coarse[a][: int(ct[1 + a])]
    np.savez_compressed(os.path.join(outdir, "ref_grid.npz"), **cases)

    # --- multigrid kernels on single-level maps ----------------------------------------------
    mg = {}
    dims = np.array([2, 1, 1], np.int32)
    nb = 2
    lv0 = np.zeros(nb, np.uint32)
    off0, tot0 = coarse_offsets(L, tuple(dims), lv0, 0)
    for variant, beta_fn in (("unit", lambda n: np.ones(n, np.float32)),
                             ("rand", lambda n: (0.5 + rng.random(n)).astype(np.float32))):
        beta = [beta_fn(int(tot0[1 + a])) for a in range(3)]
        for a in range(3):
            mg[f"{variant}_beta{a}"] = beta[a]
        for lvl in (1, 2):
            _, t = coarse_offsets(L, tuple(dims), lv0, lvl)
            out = [np.zeros(int(t[1 + a]), np.float32) for a in range(3)]
            assert L.ref_level_beta(dims, lv0, ptrs(beta), lvl, ptrs(out)) == 0
            for a in range(3):
                mg[f"{variant}_level{lvl}_beta{a}"] = out[a]
        for lvl in (0, 1, 2):
            _, t = coarse_offsets(L, tuple(dims), lv0, lvl)
            n0 = int(t[0])
            n1 = int(coarse_offsets(L, tuple(dims), lv0, lvl + 1)[1][0]) if lvl + 1 < ML else 0
            x = rng.standard_normal(n0).astype(np.float32)
            b = rng.standard_normal(n0).astype(np.float32)
            xin1 = rng.standard_normal(max(n1, 1)).astype(np.float32)
            for op, name in ((0, "residual"), (1, "restrict"), (2, "prolong"), (3, "smooth"), (4, "vcycle")):
                if op in (1, 2) and lvl + 1 >= ML:
                    continue
                if op == 4 and lvl != 0:
                    continue
                xo, bo = x.copy(), b.copy()
                r = np.zeros(n0, np.float32)
                x1 = np.zeros(max(n1, 1), np.float32)
                b1 = np.zeros(max(n1, 1), np.float32)
                it = 2
                assert L.ref_mg_op(dims, lv0, ptrs(beta), lvl, op, it, xo, bo, r.ctypes.data, x1.ctypes.data,
                                   b1.ctypes.data, xin1.ctypes.data if n1 else None) == 0
                key = f"{variant}_L{lvl}_{name}"
                mg[key + "_x_in"] = x
                mg[key + "_b_in"] = b
                mg[key + "_x"] = xo
                mg[key + "_r"] = r
                if n1:
                    mg[key + "_x1_in"] = xin1[:n1]
                    mg[key + "_x1"] = x1[:n1]
                    mg[key + "_b1"] = b1[:n1]
    mg["dims"] = dims
    np.savez_compressed(os.path.join(outdir, "ref_mg.npz"), **mg)

    # --- normalizeVelocity ------------------------------------------------------------------
    dims = np.array([3, 2, 2], np.int32)
    lvn = np.array([0, 1, 1, 2, 0, 1, 2, 2, 1, 0, 1, 2], np.uint32)
    passes = np.zeros(1, np.int32)
    L.ref_grading(dims, lvn, passes)
    _, t = coarse_offsets(L, tuple(dims), lvn, 0)
    mom = [rng.standard_normal(int(t[1 + a])).astype(np.float32) for a in range(3)]
    mass = [np.where(rng.random(int(t[1 + a])) < 0.2, rng.random(int(t[1 + a])) * 2e-6,
                     rng.random(int(t[1 + a])) * 3).astype(np.float32) for a in range(3)]
    vel = [np.zeros(int(t[1 + a]), np.float32) for a in range(3)]
    assert L.ref_normalize(dims, lvn, ptrs(mom), ptrs(mass), ptrs(vel)) == 0
    np.savez_compressed(os.path.join(outdir, "ref_normalize.npz"), dims=dims, levels=lvn,
                        **{f"mom{a}": mom[a] for a in range(3)}, **{f"mass{a}": mass[a] for a in range(3)},
                        **{f"vel{a}": vel[a] for a in range(3)})
    transfer_fixtures(L, outdir)
    print("golden fixtures written to", outdir)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--only=")]
    only = next((a.split("=", 1)[1] for a in sys.argv[1:] if a.startswith("--only=")), None)
    main(args[0] if args else HERE, only)
