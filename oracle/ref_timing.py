"""Time the reference's own CUDA kernels (oracle/_ref/libawref.so) beside this library on the same
B200, on a grid where the reference is memory-safe: 128^3 effective as 8^3 blocks of 16^3 cells,
one level (the reference's constants), with the dam_drop_128 particles.

Reference kernels, launched directly in its managers' launch shapes (ref_time_kernels):
  p2g + 3 normalizeVelocity (P2GTransfer::run, P2G.cuh:175-195).  Its inverted weight test (D1)
    makes every weight zero, so it deposits nothing: the time is its weight evaluation and loads
    without any atomics, a lower bound on a working version of the same kernel.
  3 backup copies + g2pUpdateKernel (G2PManager, G2P.cuh:192-211), AoS float3 particles.
  advectParticlesKernel (G2P.cuh:216-227).
  one runCycle from level 0 with the smoother in 1-thread CTAs: its shipped 256-thread launch has a
    divergent barrier (D9), so 1-thread CTAs are the only shape that is safe to run; the figure is
    not its shipped speed.
This library: aw_p2g (sort + P2G), aw_backup_grid_velocity + aw_g2p, aw_advect, and one
reference-mode V-cycle, on the same grid and particles (CUDA events, after one warm-up call).

The reference leg runs in a child process that imports neither torch nor this library, so only one
CUDA runtime besides the driver is in it.  Test/measurement infrastructure; prints one JSON line.

    python oracle/ref_timing.py            # both legs
    python oracle/ref_timing.py --ref      # the reference leg alone (used by the above)
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
SCALE = 8.0  # the reference grid has block size 1: 8 blocks per axis span [0, 8]


def scene():
    from anitowave_adaptive_b200 import scenes  # numpy only
    return scenes.config("dam_drop_128")


def ref_leg(reps=5):
    L = C.CDLL(os.path.join(HERE, "_ref", "libawref.so"))
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
    L.ref_time_kernels.argtypes = [np.ctypeslib.ndpointer(np.int32, flags="C"), C.c_uint32, f32p, f32p, C.c_uint32,
                                   C.c_int, f32p]
    S = scene()
    dims = np.array([8, 8, 8], np.int32)
    ms = np.zeros(4, np.float32)
    pos = np.ascontiguousarray(SCALE * S.pos, np.float32)
    vel = np.ascontiguousarray(SCALE * S.vel, np.float32)
    t0 = time.perf_counter()
    rc = L.ref_time_kernels(dims, 0, pos, vel, S.n, reps, ms)
    return {"grid": "8^3 blocks x 16^3 cells, 1 level (128^3)", "particles": S.n, "ref_status": rc,
            "ref_ms": {"p2g_normalize": float(ms[0]), "backup_g2p": float(ms[1]), "advect": float(ms[2]),
                       "vcycle_1thread_smoother": float(ms[3])},
            "ref_wall_s": time.perf_counter() - t0}


def our_leg(reps=5):
    import torch
    import anitowave_adaptive_b200 as aw
    S = scene()
    g = aw.MSBG((8, 8, 8), 1.0 / 8, (0, 0, 0), 16, 3)
    g.init_refinement_map(0)
    g.enforce_grading()
    g.allocate()
    pos = torch.as_tensor(S.pos, device="cuda")
    vel = torch.as_tensor(S.vel, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, r=reps):
        fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(r):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / r

    out = {"p2g_with_sort": timed(lambda: g.p2g(pos, vel))}
    v2 = vel.clone()
    out["backup_g2p"] = timed(lambda: (g.backup_grid_velocity(), g.g2p(v2, pos, 0.95)))
    p2 = pos.clone()
    out["advect"] = timed(lambda: g.advect(p2, 1.0 / 240))
    sv = aw.Solver(g, operator_mode=aw.OPERATOR_REFERENCE)
    sv.level_array(0, 1).normal_()
    out["vcycle_reference_mode"] = timed(lambda: sv.vcycle(), r=3)
    sv.close()
    g.close()
    return out


def main():
    if "--ref" in sys.argv:
        print(json.dumps(ref_leg()), flush=True)
        return
    res = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref"], capture_output=True, text=True)
    sys.stderr.write(res.stderr)
    if res.returncode != 0:
        print(json.dumps({"ref_rc": res.returncode, "ref_stderr_tail": res.stderr[-2000:]}), flush=True)
        return
    out = json.loads(res.stdout.strip().splitlines()[-1])
    ours = our_leg()
    out["ours_ms"] = ours
    r = out["ref_ms"]
    out["speedup"] = {"p2g": r["p2g_normalize"] / ours["p2g_with_sort"], "g2p": r["backup_g2p"] / ours["backup_g2p"],
                      "advect": r["advect"] / ours["advect"]}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
