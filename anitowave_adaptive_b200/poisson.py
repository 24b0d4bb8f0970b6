"""The projection-only Poisson workload (poisson_256 and smaller variants).

Closed unit box (solid walls, every cell fluid), level map from the distance to the union of 32
seeded spheres (thresholds 8/24/56 finest cells), right-hand side = divergence of a field of 64
seeded Gaussian velocity blobs sampled at the face centres, made consistent at level interfaces
and projected to zero mean.  Built on the device through the C ABI.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import MSBG, VELOCITY_X, scenes


@dataclass
class PoissonProblem:
    grid: MSBG
    b: object          # torch float32 right-hand side (level-0 cells)
    fluid: object      # torch uint8 (all ones)
    N: int

    def divergence_after(self, solver, p, fp64=False):
        """max |div u| per unit volume after the pressure-gradient update with p (dt = 1); with fp64
        the face sums of the FP32 field are taken in FP64."""
        import torch
        g = self.grid
        saved = [g.channel(VELOCITY_X + a).clone() for a in range(3)]
        g.pressure_gradient(solver, p, self.fluid, 1.0)
        g.face_sync(VELOCITY_X)
        g.wall_bc(VELOCITY_X)
        if fp64:
            val = g.divergence_max64(self.fluid)
        else:
            _, mx = g.divergence(self.fluid, 1.0)
            val = float(mx.item())
        for a in range(3):
            g.channel(VELOCITY_X + a).copy_(saved[a])
        torch.cuda.synchronize()
        return val


def blob_velocity_torch(X, c, sig, amp):
    import torch
    out = torch.zeros_like(X, dtype=torch.float64)
    Xd = X.double()
    for k in range(c.shape[0]):
        d2 = ((Xd - torch.as_tensor(c[k], device=X.device)) ** 2).sum(-1)
        gk = torch.exp(-d2 / (2 * float(sig[k]) ** 2))
        out += gk[:, None] * torch.as_tensor(amp[k], device=X.device)[None, :]
    return out


def build_problem(N=256, base_res=8, levels=4, thresholds=(8, 24, 56)):
    import torch
    dims = (N // base_res,) * 3
    c, r = scenes.poisson_spheres()
    pts = torch.as_tensor(scenes.sphere_surface_points(N, c, r), device="cuda")
    g = MSBG(dims, base_res / N, (0.0, 0.0, 0.0), base_res, levels)
    g.levels_from_particles(pts, thresholds)
    g.enforce_grading()
    g.allocate()
    bc, bsig, bamp = scenes.poisson_blobs()
    for a in range(3):
        X = g.face_positions(a)
        u = blob_velocity_torch(X, bc, bsig, bamp)[:, a]
        g.channel(VELOCITY_X + a).copy_(u.float())
    g.face_sync(VELOCITY_X)
    g.wall_bc(VELOCITY_X)
    ncell = g.totals()[0]
    fluid = torch.ones(ncell, dtype=torch.uint8, device="cuda")
    b, _ = g.divergence(fluid, 1.0)
    b = (b.double() - b.double().mean()).float()
    torch.cuda.synchronize()
    return PoissonProblem(g, b, fluid, N)


__all__ = ["PoissonProblem", "build_problem", "np"]
