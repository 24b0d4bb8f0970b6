"""Full-size validation of the GPU adjoint on the differentiable rollout (the dam_break_64 layout,
505,856 particles, 50 steps, checkpoints every 10).  Needs a GPU and the
oracle; prints one JSON object (and writes it to --out when given).

  --mode along   GPU VJP (aw_vjp_rollout) against the FP64 adjoint evaluated along the GPU's own
                 trajectory (oracle.pyoracle.grad_along_states on the per-step states of
                 aw_flip_step): checks the adjoint arithmetic.
  --mode oracle  GPU VJP against the FP64 oracle's own rollout gradient, and FP64 central
                 differences (eps = 1e-4, 16 unit directions, seed 6, fluid flags held) against the
                 FP64 adjoint.

Test infrastructure (not collected by pytest): python tests/adjoint_validation.py --mode along
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def setup(steps, every=10):
    import torch

    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import scenes
    from oracle import pyoracle as po

    S = scenes.config("dam_break_64")
    g = aw.build_grid(S)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, g.refinement_map())
    rng = np.random.default_rng(5)
    target = (S.pos.astype(np.float64) + np.array([0.1, 0, 0]) + 0.01 * rng.standard_normal(S.pos.shape)).astype(np.float32)
    R = aw.Rollout(g, S.pos, steps, S.dt, S.alpha, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-8,
                   checkpoint_every=every)
    u0 = torch.zeros(R.nfaces, device="cuda")
    t = time.time()
    L = R.forward(u0, torch.as_tensor(target, device="cuda"))
    torch.cuda.synchronize()
    tf = time.time() - t
    t = time.time()
    G = R.vjp().double().cpu().numpy()
    torch.cuda.synchronize()
    tb = time.time() - t
    nfaces = R.nfaces
    R.close()
    return aw, po, S, g, O, target, L, G, nfaces, tf, tb


def mode_along(steps):
    aw, po, S, g, O, target, L, G, nfaces, tf, tb = setup(steps)
    F = aw.Flip(g, S.pos, np.zeros_like(S.pos), S.dt, S.alpha, (0, S.gravity, 0), precision=aw.PRECISION_MIXED,
                tolerance=1e-8)
    xs, vs = [S.pos.astype(np.float64)], [np.zeros(S.pos.shape)]
    for _ in range(steps):
        F.step()
        p, v = F.particles()
        xs.append(p.astype(np.float64))
        vs.append(v.astype(np.float64))
    F.close()
    t = time.time()
    go = np.concatenate(po.grad_along_states(O, xs, vs, O._faces(), target.astype(np.float64), S.dt, S.alpha,
                                             (0, S.gravity, 0)))
    return dict(mode="along", steps=steps, n=S.n, faces=nfaces, loss_rollout=L,
                loss_flip=float(((xs[-1] - target) ** 2).sum(1).mean()),
                grad_rel_l2=float(np.linalg.norm(G - go) / np.linalg.norm(go)),
                cosine=float(G @ go / np.linalg.norm(G) / np.linalg.norm(go)), gnorm_gpu=float(np.linalg.norm(G)),
                gnorm_fp64_along_gpu=float(np.linalg.norm(go)), t_gpu_forward_s=tf, t_gpu_vjp_s=tb,
                t_oracle_s=time.time() - t)


def mode_oracle(steps, ndirs=16, eps=1e-4):
    aw, po, S, g, O, target, L, G, nfaces, tf, tb = setup(steps)
    x0, tg = S.pos.astype(np.float64), target.astype(np.float64)
    grav = (0, S.gravity, 0)
    t = time.time()
    Lo, xN, recs = po.rollout64(O, x0, O._faces(), steps, S.dt, S.alpha, grav, tg, tol=1e-12)
    go = np.concatenate(po.rollout64_grad(O, x0, O._faces(), recs, xN, tg, S.dt, S.alpha, tol=1e-12))
    to = time.time() - t
    fluids = [r["fluid"] for r in recs]
    del recs
    out = dict(mode="oracle", steps=steps, n=S.n, faces=nfaces, loss_gpu=L, loss_oracle=Lo,
               grad_rel_l2_gpu_vs_oracle=float(np.linalg.norm(G - go) / np.linalg.norm(go)),
               t_gpu_forward_s=tf, t_gpu_vjp_s=tb, t_oracle_fwd_bwd_s=to, oracle_threads=po.num_threads())
    rng = np.random.default_rng(6)
    nf = [len(a) for a in O._faces()]
    rows = []
    for _ in range(ndirs):
        d = rng.standard_normal(nfaces)
        d /= np.linalg.norm(d)
        ds = np.split(d, np.cumsum(nf)[:-1])
        Lp, _, _ = po.rollout64(O, x0, [eps * a for a in ds], steps, S.dt, S.alpha, grav, tg, tol=1e-12, fluids=fluids)
        Lm, _, _ = po.rollout64(O, x0, [-eps * a for a in ds], steps, S.dt, S.alpha, grav, tg, tol=1e-12, fluids=fluids)
        fd = (Lp - Lm) / (2 * eps)
        rows.append(dict(fd=fd, oracle_vjp=float(go @ d), gpu_vjp=float(G @ d),
                         rel_oracle=abs(fd - float(go @ d)) / abs(fd)))
    out["directions"] = rows
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", choices=["along", "oracle"], default="along")
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    res = mode_along(a.steps) if a.mode == "along" else mode_oracle(a.steps)
    s = json.dumps(res)
    print(s)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s + "\n")


if __name__ == "__main__":
    main()
