"""One FLIP step of dam_drop2_256 (256^3 effective, 4 levels, 34,678,688 particles) on the GPU against
the FP64 oracle's step from the same particle state: relative L2 of the projected grid velocity and
of the particle velocities, and max |div u| dt of the GPU's projected field evaluated in FP64.  The
oracle solves with V-cycle-preconditioned CG.  The GPU runs the mixed solve to 1e-6 and the plain
FP32 V-cycle iteration to 1e-6 and to 1e-5.
Needs a GPU and the oracle; prints one JSON object.

Test infrastructure (not collected by pytest): python tests/flip256_validation.py
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    import torch

    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import scenes
    from oracle import pyoracle as po

    S = scenes.config("dam_drop2_256")
    grav = (0.0, S.gravity, 0.0)
    g = aw.build_grid(S)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, g.refinement_map())
    out = {"workload": "dam_drop2_256", "particles": S.n, "cells": int(O.tot0[0])}
    t = time.time()
    xo, vo, perm, det = po.flip_step(O, S.pos, S.vel, S.dt, S.alpha, grav, tol=1e-12, method="pcg")
    out["t_oracle_s"] = time.time() - t
    out["oracle_pcg_iterations"] = int(len(det["hist"]) - 1)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    un_o = np.concatenate(det["u_new"])
    for name, prec, tol in (("mixed", aw.PRECISION_MIXED, 1e-6), ("fp32", aw.PRECISION_FP32, 1e-6),
                            ("fp32_1e-5", aw.PRECISION_FP32, 1e-5)):
        F = aw.Flip(g, S.pos, S.vel, S.dt, S.alpha, grav, precision=prec, tolerance=tol, max_cycles=100)
        res = {"tolerance": tol}
        try:
            F.step()
            st = F.stats()
            u = [g.channel(aw.VELOCITY_X + a).double().cpu().numpy() for a in range(3)]
            fluid = (g.channel(aw.CELL_TYPE) > 0).to(torch.uint8).cpu().numpy()
            # FP64 net volume flux out of each fluid cell (sum of u.n A over its faces), GPU field
            flux = O.divergence(u, fluid, S.dt) * S.dt
            res.update(converged=True, cycles=st["cycles"], residual=st["residual"],
                       gpu_max_abs_div_per_volume=st["div_after"],
                       fp64_max_abs_cell_flux_of_gpu_field=float(np.abs(flux).max()),
                       grid_velocity_rel_l2=float(np.linalg.norm(np.concatenate(u) - un_o) / np.linalg.norm(un_o)))
            p, v = F.particles()
            res["particle_velocity_rel_l2"] = float(np.linalg.norm(v - vo[inv]) / np.linalg.norm(vo[inv]))
            res["particle_position_rel_l2"] = float(np.linalg.norm(p - xo[inv]) / np.linalg.norm(xo[inv]))
        except aw.AWError as err:
            res.update(converged=False, error=str(err))
        F.close()
        out[name] = res
    flux_o = O.divergence(det["u_new"], det["fluid"], S.dt) * S.dt
    out["oracle_fp64_max_abs_cell_flux"] = float(np.abs(flux_o).max())
    print(json.dumps(out))


if __name__ == "__main__":
    main()
