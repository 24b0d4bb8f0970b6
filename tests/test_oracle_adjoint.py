"""The FP64 oracle's adjoint of the FLIP step, pinned by FP64 central differences.

The oracle's hand-written VJPs (P2G, G2P, RK3, T-junction sync, walls, divergence, pressure
gradient and the solve, which reuses the symmetric operator) are chained through a rollout whose
initial particle velocities are the MAC sample of a face field u0 (the differentiable rollout of
the library).  d loss / d u0 along random unit directions must match central differences
(eps = 1e-4) to 1e-6 relative: in FP64, with every discrete decision of the forward held, the
difference quotient is exact up to O(eps^2) and rounding.
"""
import numpy as np


def test_oracle_rollout_gradient_matches_central_differences():
    from anitowave_adaptive_b200 import scenes
    from oracle import pyoracle as po

    S = scenes.config("dam_break_16")
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    x0 = S.pos.astype(np.float64)
    rng = np.random.default_rng(5)
    target = x0 + np.array([0.1, 0.0, 0.0]) + 0.01 * rng.standard_normal(x0.shape)
    u0 = O._faces()
    steps = 5
    grav = (0.0, S.gravity, 0.0)
    L, xN, recs = po.rollout64(O, x0, u0, steps, S.dt, S.alpha, grav, target)
    g = po.rollout64_grad(O, x0, u0, recs, xN, target, S.dt, S.alpha)
    fluids = [r["fluid"] for r in recs]
    rng = np.random.default_rng(6)
    eps = 1e-4
    for _ in range(4):
        d = [rng.standard_normal(len(a)) for a in g]
        nrm = np.sqrt(sum((a * a).sum() for a in d))
        d = [a / nrm for a in d]
        Lp, _, _ = po.rollout64(O, x0, [u0[a] + eps * d[a] for a in range(3)], steps, S.dt, S.alpha, grav, target,
                                fluids=fluids)
        Lm, _, _ = po.rollout64(O, x0, [u0[a] - eps * d[a] for a in range(3)], steps, S.dt, S.alpha, grav, target,
                                fluids=fluids)
        fd = (Lp - Lm) / (2 * eps)
        ad = sum(float((g[a] * d[a]).sum()) for a in range(3))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)


def test_oracle_projection_adjoint_is_transpose():
    """<P u, w> = <u, P^T w> for the oracle's projection and its VJP (one solve each way)."""
    from anitowave_adaptive_b200 import scenes
    from oracle import pyoracle as po

    S = scenes.config("dam_break_16")
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    _, _, cnt = O.p2g(S.pos, S.vel)
    fluid = (cnt > 0).astype(np.uint8)
    O.set_params(mode=0)
    O.build(fluid=fluid)
    rng = np.random.default_rng(3)
    u = [rng.standard_normal(len(a)) for a in O._faces()]
    w = [rng.standard_normal(len(a)) for a in O._faces()]
    p, _ = O.solve(O.divergence(u, fluid, S.dt), tol=1e-13)
    Pu = O.wall_bc(O.face_sync(O.gradient_update(p, S.dt, u)))
    gb = O.face_sync_vjp(O.wall_bc(w))
    pbar = np.zeros(int(O.tot0[0]))
    O.gradient_vjp(S.dt, gb, pbar)
    bbar, _ = O.solve(pbar * fluid, tol=1e-13)
    O.divergence_vjp(bbar, fluid, S.dt, gb)
    lhs = sum(float((Pu[a] * w[a]).sum()) for a in range(3))
    rhs = sum(float((u[a] * gb[a]).sum()) for a in range(3))
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs)
