"""aw_g2p_noalloc (G2P with a fixed static device scratch array) against aw_g2p, through the C ABI.

Collected last on purpose: it must pass both alone in a fresh process and after every other test
has run in the same process.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import anitowave_adaptive_b200 as aw  # noqa: E402
from anitowave_adaptive_b200 import scenes  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-5  # relative L2 bar for FP32 results, as in the other parity tests
AW_ERR_INVALID_ARGUMENT = 1


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)


def g2p_noalloc(g, vel, pos, alpha):
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return aw.lib().aw_g2p_noalloc(g.h, C.c_void_p(vel.data_ptr()), C.c_void_p(pos.data_ptr()),
                                   C.c_int64(pos.shape[0]), C.c_float(alpha), stream)


def _fresh_fields(g, rng):
    for a in range(3):
        for ch in (aw.VELOCITY_X + a, aw.VELOCITY_OLD_X + a):
            g.channel(ch).copy_(torch.as_tensor(rng.standard_normal(g.channel(ch).numel()), dtype=torch.float32))


def test_g2p_noalloc_matches_g2p_on_two_calls():
    S = scenes.config("dam_break_64")
    g = aw.build_grid(S)
    rng = np.random.default_rng(7)
    pos = torch.as_tensor(S.pos, device="cuda")
    for call, alpha in enumerate((0.95, 0.6)):
        # fresh fields and velocities on each call, so the second call cannot pass on what the
        # first one left in the shared scratch array; the allocation-free call runs first, on a grid
        # whose own G2P buffers aw_g2p has not allocated yet
        _fresh_fields(g, rng)
        vel0 = torch.as_tensor(rng.standard_normal((S.n, 3)).astype(np.float32), device="cuda")
        ref = vel0.clone()
        got = vel0.clone()
        st = g2p_noalloc(g, got, pos, alpha)
        assert st == aw.AW_OK, aw.lib().aw_last_error().decode()
        g.g2p(ref, pos, alpha)
        torch.cuda.synchronize()
        err = rel_l2(got.cpu().numpy(), ref.cpu().numpy())
        assert err < RTOL, (call, err)


def test_g2p_noalloc_takes_no_device_memory():
    # after a first call has set the device up, a call on a new grid leaves the free device memory
    # exactly as it was
    S = scenes.config("dam_break_32")
    g0 = aw.build_grid(S)
    pos = torch.as_tensor(S.pos, device="cuda")
    vel = torch.zeros((S.n, 3), device="cuda")
    assert g2p_noalloc(g0, vel, pos, 0.95) == aw.AW_OK
    g = aw.build_grid(S)
    _fresh_fields(g, np.random.default_rng(3))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = g2p_noalloc(g, vel, pos, 0.95)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert st == aw.AW_OK, aw.lib().aw_last_error().decode()
    assert free1 == free0, (free0, free1)


def test_g2p_noalloc_rejects_grid_beyond_its_scratch():
    # 128 blocks of 16^3 cells need 128 * 16524 > 2,097,152 tile floats per field
    g = aw.MSBG((8, 4, 4), 1.0 / 8, (0, 0, 0), 16, 1)
    g.init_refinement_map(0)
    g.enforce_grading()
    g.allocate()
    pos = torch.full((4, 3), 0.5, device="cuda")
    vel = torch.zeros((4, 3), device="cuda")
    st = g2p_noalloc(g, vel, pos, 0.95)
    assert st == AW_ERR_INVALID_ARGUMENT
    assert "static scratch" in aw.lib().aw_last_error().decode()
