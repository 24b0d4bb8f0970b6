"""Time the reference's own CUDA kernels (oracle/_ref/libawref.so) beside this library on the
same B200, on a grid where the reference is memory-safe: 128^3 effective as 8^3 blocks of 16^3
cells, one level (the reference's constants), with the dam_drop_128 particles.

Reference kernels: P2GTransfer::run (P2G.cuh:173-195; its inverted weight test makes it deposit
nothing, so it is timed but its output is not used), G2PManager::backupGridVelocity +
performG2P (G2P.cuh:189-211), G2PManager::advect (G2P.cuh:216-227), and one runCycle from level 0
with the smoother in 1-thread CTAs (the only launch shape free of its divergent barrier).

Test/measurement infrastructure: prints one JSON line.  Usage: python oracle/ref_timing.py
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)


def main():
    import torch
    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import scenes

    L = C.CDLL(os.path.join(HERE, "_ref", "libawref.so"))
    L.ref_time_kernels.argtypes = [np.ctypeslib.ndpointer(np.int32), C.c_uint32, np.ctypeslib.ndpointer(np.float32),
                                   np.ctypeslib.ndpointer(np.float32), C.c_uint32, C.c_int,
                                   np.ctypeslib.ndpointer(np.float32)]
    S = scenes.config("dam_drop_128")
    dims = np.array([8, 8, 8], np.int32)
    ms = np.zeros(4, np.float32)
    t0 = time.perf_counter()
    # the reference grid has blockSize 1.0 (8 blocks per axis span [0, 8]); scale the unit-cube
    # scene by 8 so that its particles cover the same cells as on this library's 128^3 grid
    rc = L.ref_time_kernels(dims, 0, np.ascontiguousarray(8.0 * S.pos, np.float32),
                            np.ascontiguousarray(8.0 * S.vel, np.float32), S.n, 5, ms)
    ref_wall = time.perf_counter() - t0
    out = {"grid": "8^3 blocks x 16^3 cells, 1 level (128^3)", "particles": S.n, "ref_status": rc,
           "ref_ms": {"p2g": float(ms[0]), "g2p": float(ms[1]), "advect": float(ms[2]), "vcycle_1thread": float(ms[3])},
           "ref_wall_s": ref_wall}
    # this library on the same uniform grid through the drop-in calls
    g = aw.MSBG((8, 8, 8), 1.0 / 8, (0, 0, 0), 16, 3)
    g.init_refinement_map(0)
    g.enforce_grading()
    g.allocate()
    pos = torch.as_tensor(S.pos, device="cuda")
    vel = torch.as_tensor(S.vel, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ours = {"p2g_incl_sort": timed(lambda: g.p2g(pos, vel))}
    v2 = vel.clone()
    ours["g2p"] = timed(lambda: (g.backup_grid_velocity(), g.g2p(v2, pos, 0.95)))
    p2 = pos.clone()
    ours["advect"] = timed(lambda: g.advect(p2, 1.0 / 240))
    sv = aw.Solver(g, operator_mode=aw.OPERATOR_REFERENCE)
    sv.level_array(0, 1).normal_()
    ours["vcycle_reference_mode"] = timed(lambda: sv.vcycle(), reps=3)
    out["ours_ms"] = ours
    out["speedup"] = {"p2g": float(ms[0]) / ours["p2g_incl_sort"], "g2p": float(ms[1]) / ours["g2p"],
                      "advect": float(ms[2]) / ours["advect"], "vcycle": float(ms[3]) / ours["vcycle_reference_mode"]}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
