"""The bounded wait of the TMA-staged G2P runs out without any fault.

aw_test_arm_copy_timeout makes the next G2P arm its first particle-copy barrier (expect_tx) without
issuing the copy, with a short poll limit: a flag that nothing sets.  The CTAs give up, wait for the
copies they did issue, and return; the FLIP step reports AW_ERR_STATE (its particle state is then
partly updated); the next steps run normally.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import anitowave_adaptive_b200 as aw  # noqa: E402
from anitowave_adaptive_b200 import scenes  # noqa: E402

pytestmark = pytest.mark.gpu
AW_ERR_STATE = 6


def test_g2p_copy_wait_runs_out_and_next_step_recovers():
    S = scenes.config("dam_break_64")
    g = aw.build_grid(S)
    F = aw.Flip(g, S.pos, S.vel, S.dt, S.alpha, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-8)
    F.step()
    assert aw.lib().aw_test_arm_copy_timeout(g.h) == aw.AW_OK
    with pytest.raises(aw.AWError) as e:
        F.step()
    assert e.value.status == AW_ERR_STATE
    assert "timed out" in str(e.value)
    # the context is usable and the flag was cleared: the next steps succeed
    F.step()
    F.step()
    torch.cuda.synchronize()
    pos, vel = F.particles()
    assert np.isfinite(pos).all() and np.isfinite(vel).all()
    F.close()
    g.close()
