"""The RK3 advection's fallback for a stage point that lands in a block whose u_new tile G2P did not
write this step.

G2P builds no tile for a block with no particle in itself or its 26 neighbours; a stage point of a
particle more than a block away that lands there samples the face arrays (the same MAC stencil and
ghost rule as the tiles) instead.  Such points are rare, so AW_TEST_UNTILED makes G2P report every
tile as not written: every stage point outside its own block then takes the fallback.  The step
must agree with the step through the tiles, and both with the FP64 oracle.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import anitowave_adaptive_b200 as aw  # noqa: E402
from anitowave_adaptive_b200 import scenes  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

pytestmark = pytest.mark.gpu


def _steps(S, untiled, nsteps):
    g = aw.build_grid(S)
    F = aw.Flip(g, S.pos, S.vel, S.dt, S.alpha, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-10)
    if untiled:
        os.environ["AW_TEST_UNTILED"] = "1"
    try:
        for _ in range(nsteps):
            F.step()
        torch.cuda.synchronize()
    finally:
        os.environ.pop("AW_TEST_UNTILED", None)
    pos, vel = F.particles()
    F.close()
    g.close()
    return pos, vel


@pytest.mark.parametrize("name", ["dam_break_16", "dam_drop_128"])
def test_face_array_fallback_matches_tiles(name):
    S = scenes.config(name)
    p1, v1 = _steps(S, False, 1)
    p0, v0 = _steps(S, True, 1)
    # the fallback samples the same faces with the same weights: positions agree to the rounding of
    # an FP32 position (and the last-bit differences of P2G's atomic sums)
    assert np.abs(p0 - p1).max() <= 4 * np.spacing(np.float32(1.0)), np.abs(p0 - p1).max()
    # G2P itself is the same; two runs differ only by the order of P2G's float atomics
    assert np.linalg.norm(v0 - v1) <= 1e-6 * np.linalg.norm(v1), np.linalg.norm(v0 - v1) / np.linalg.norm(v1)


def test_face_array_fallback_matches_oracle():
    S = scenes.config("dam_break_16")
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    xo, vo, perm, _ = po.flip_step(O, S.pos, S.vel, S.dt, S.alpha, (0, S.gravity, 0), tol=1e-12)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    pos, vel = _steps(S, True, 1)
    err_v = np.linalg.norm(vel - vo[inv]) / np.linalg.norm(vo[inv])
    assert err_v < 1e-5, err_v
    # positions: 1e-5 of the displacement plus the rounding of an FP32 position (as the parity tests)
    disp = np.abs(xo[inv] - S.pos).max()
    err_x = np.abs(pos.astype(np.float64) - xo[inv]).max()
    assert err_x < 1e-5 * disp + 4 * np.spacing(np.float32(1.0)), (err_x, disp)
