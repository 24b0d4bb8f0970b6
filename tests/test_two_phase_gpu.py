"""GPU parity of the two-phase (variable density) path: aw_p2g_phase, the T-junction coefficient
sync, aw_solver_update_coefficients and the two-phase FLIP step, against the FP64 oracle.

Bars as in test_gpu_parity.py: 1e-5 relative L2 for FP32 results.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import anitowave_adaptive_b200 as aw  # noqa: E402
from anitowave_adaptive_b200 import scenes  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-5
RHO = (1.0, 3.0)
# a blob of the heavy phase inside each scene's fluid (both layouts have level-1 blocks in the fluid)
BLOB = {"dam_break_64": ((0.2, 0.3, 0.5), 0.12), "dam_drop_128": ((0.7, 0.8, 0.5), 0.12)}


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


@pytest.fixture(scope="module", params=sorted(BLOB))
def case(request):
    S = scenes.config(request.param)
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    g = aw.build_grid(S)
    c, r = BLOB[request.param]
    ph = scenes.phase_sphere(S.pos, c, r)
    assert 0 < ph.sum() < S.n
    return S, O, g, ph


def test_p2g_phase_matches_oracle(case):
    S, O, g, ph = case
    rng = np.random.default_rng(21)
    vel = (rng.standard_normal((S.n, 3)) * 0.5).astype(np.float32)
    u, m, cnt, phi = O.p2g_phase(S.pos, vel, ph)
    beta = O.phase_beta(phi, *RHO)
    dev = lambda x: torch.as_tensor(np.ascontiguousarray(x), device="cuda")  # noqa: E731
    g.p2g_phase(dev(S.pos), dev(vel), dev(ph), *RHO)
    torch.cuda.synchronize()
    for a in range(3):
        assert rel_l2(g.channel(aw.MASS_DENSITY_X + a).cpu().numpy(), m[a]) < RTOL
        assert rel_l2(g.channel(aw.VELOCITY_X + a).cpu().numpy(), u[a]) < RTOL
        assert rel_l2(g.channel(aw.PHASE_FIELD_X + a).cpu().numpy(), phi[a]) < RTOL
        assert rel_l2(g.channel(aw.BETA_COEFF_X + a).cpu().numpy(), beta[a]) < RTOL
        assert np.any(beta[a] < 0.5)  # the heavy phase reaches faces of every axis


def _step_pair(S, O, g, ph):
    xo, vo, perm, d = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), tol=1e-12, phase=ph, rho=RHO)
    F = aw.Flip(g, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-10,
                max_cycles=80)
    F.set_phase(ph, *RHO)
    F.step()
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    return F, xo[inv], vo[inv], d


def test_two_phase_flip_step_matches_oracle(case):
    S, O, g, ph = case
    F, x_ref, v_ref, d = _step_pair(S, O, g, ph)
    pos, vel = F.particles()
    # the bar is relative to the gravity increment each particle receives (FP32 rounding of u*)
    scale = abs(S.gravity) * S.dt * np.sqrt(vel.size)
    assert np.linalg.norm(vel - v_ref) / scale < RTOL
    for a in range(3):
        assert rel_l2(g.channel(aw.BETA_COEFF_X + a).cpu().numpy(), d["beta"][a]) < RTOL
        un = g.channel(aw.VELOCITY_X + a).cpu().numpy()
        assert np.linalg.norm(un - d["u_new"][a]) / (abs(S.gravity) * S.dt * np.sqrt(un.size)) < RTOL
    disp = np.abs(x_ref - S.pos).max()
    assert np.abs(pos.astype(np.float64) - x_ref).max() < 1e-5 * disp + 4 * np.spacing(np.float32(1.0))
    st = F.stats()
    assert st["div_after"] < 1e-4 * max(st["div_before"], 1e-30)
    # the heavy blob falls faster than the light fluid around it
    blob = ph > 0.5
    assert vel[blob, 1].mean() < vel[~blob, 1].mean()
    F.close()


def test_clearing_the_phase_restores_one_phase(case):
    S, O, g, ph = case
    xo, vo, perm, d = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), tol=1e-12)
    F = aw.Flip(g, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-10,
                max_cycles=60)
    F.set_phase(ph, *RHO)
    F.set_phase(None)
    F.step()
    _, vel = F.particles()
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    scale = abs(S.gravity) * S.dt * np.sqrt(vel.size)
    assert np.linalg.norm(vel - vo[inv]) / scale < RTOL
    for a in range(3):
        assert np.all(g.channel(aw.BETA_COEFF_X + a).cpu().numpy() == 1.0)
    F.close()


def test_phase_arguments_are_checked(case):
    S, O, g, ph = case
    F = aw.Flip(g, S.pos[:100], S.vel[:100], S.dt, 0.95, (0, S.gravity, 0))
    with pytest.raises(aw.AWError):
        F.set_phase(np.full(100, 1.5, np.float32), *RHO)
    with pytest.raises(aw.AWError):
        F.set_phase(np.zeros(100, np.float32), 0.0, 1.0)
    with pytest.raises(ValueError):
        F.set_phase(np.zeros(99, np.float32), *RHO)
    F.close()
