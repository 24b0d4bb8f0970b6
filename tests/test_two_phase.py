"""Two-phase (variable density) projection in the FP64 oracle: beta = 1/rho from the P2G face phase.

The reference allocates PHASE_FIELD_* and BETA_COEFF_* (MSBG.cuh:21-29) and leaves their
accumulation commented out (P2G.cuh:94-97); these cases pin the restatement with properties that
hold for any correct variable-coefficient projection.
"""
import numpy as np
import pytest

from anitowave_adaptive_b200 import scenes
from oracle import pyoracle as po


def small_scene(N=32):
    S = scenes.config(f"dam_break_{N}")
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    return S, lv, po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)


def test_phase_zero_is_the_single_phase_step():
    S, _, O = small_scene(32)
    g = (0, S.gravity, 0)
    x1, v1, _, d1 = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, g, tol=1e-12)
    x2, v2, _, d2 = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, g, tol=1e-12, phase=np.zeros(S.n), rho=(1.0, 5.0))
    for b in d2["beta"]:
        assert np.all(b == 1.0)
    np.testing.assert_allclose(v2, v1, rtol=0, atol=1e-12)
    np.testing.assert_allclose(x2, x1, rtol=0, atol=1e-12)


def test_uniform_density_scales_pressure_only():
    """rho = 4 everywhere: the pressure is 4x the rho = 1 pressure and the velocities are unchanged."""
    S, _, O = small_scene(32)
    g = (0, S.gravity, 0)
    _, v1, _, d1 = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, g, tol=1e-13)
    _, v4, _, d4 = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, g, tol=1e-13, phase=np.ones(S.n), rho=(4.0, 4.0))
    np.testing.assert_allclose(d4["p"], 4.0 * d1["p"], rtol=0, atol=1e-9 * np.abs(d1["p"]).max())
    np.testing.assert_allclose(v4, v1, rtol=0, atol=1e-9 * max(np.abs(v1).max(), 1.0))


def test_face_phase_is_a_weighted_average():
    S, _, O = small_scene(32)
    ph = scenes.phase_sphere(S.pos, (0.2, 0.3, 0.5), 0.12)
    assert 0 < ph.sum() < S.n
    _, perm = O.particle_keys(S.pos)
    u, m, cnt, phi = O.p2g_phase(S.pos[perm], S.vel[perm], ph[perm])
    u0, m0, _ = O.p2g(S.pos[perm], S.vel[perm])
    for a in range(3):
        np.testing.assert_array_equal(m[a], m0[a])
        np.testing.assert_array_equal(u[a], u0[a])
        assert phi[a].min() >= 0.0 and phi[a].max() <= 1.0
        assert np.any(phi[a] == 1.0) and np.any((phi[a] > 0) & (phi[a] < 1))
        assert np.all(phi[a][m[a] <= 1e-6] == 0.0)


@pytest.mark.parametrize("sync", [True, False])
def test_beta_sync_keeps_the_operator_symmetric(sync):
    """Coefficients from random particle phases (density ratio 10): with the T-junction sync A stays
    symmetric; without it the coarse and fine sides of a T-junction disagree and A is not
    symmetric (the sync is needed)."""
    S, lv, O = small_scene(64)  # 64^3 has level-1 blocks inside the fluid, so T-junctions carry mass
    assert len(np.unique(lv)) == 2
    rng = np.random.default_rng(3)
    _, perm = O.particle_keys(S.pos)
    _, _, _, phi = O.p2g_phase(S.pos[perm], S.vel[perm], rng.random(S.n).astype(np.float32))
    beta = [1.0 / ((1.0 - f) * 1.0 + f * 10.0) for f in phi]
    if sync:
        beta = O.beta_sync(beta)
    n = int(O.tot0[0])
    fluid = np.ones(n, np.uint8)
    O.set_params(mode=0)
    O.build(bbar=beta, fluid=fluid)
    x = rng.standard_normal(n)
    y = rng.standard_normal(n)
    asym = abs(y @ O.apply(0, x) - x @ O.apply(0, y)) / abs(y @ O.apply(0, x))
    if sync:
        assert asym < 1e-12
    else:
        assert asym > 1e-6


def test_heavy_blob_falls_through_a_resting_column():
    """A full-width resting column with a heavy spherical blob (rho 3 vs 1): after one step the light
    fluid stays near rest while the blob accelerates downward."""
    S = scenes.dam_break(32, 8, 2, (8,), 0, 1.0 / 240, box=(1.0, 0.6, 1.0))
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    ph = scenes.phase_sphere(S.pos, (0.5, 0.3, 0.5), 0.12)
    x, v, perm, d = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), tol=1e-12, phase=ph,
                                 rho=(1.0, 3.0))
    blob = ph[perm] > 0.5
    far = np.abs(S.pos[perm][:, 1] - 0.3) > 0.25
    vy_blob = v[blob, 1].mean()
    vy_far = v[far & ~blob, 1].mean()
    # free fall would be g dt; the blob gets a sizeable share of it, the far light fluid almost none
    assert vy_blob < 0.2 * S.gravity * S.dt
    assert abs(vy_far) < 0.5 * abs(vy_blob)
    assert d["hist"][-1] < 1e-12
