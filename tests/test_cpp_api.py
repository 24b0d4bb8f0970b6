"""The C++ host classes with the reference's names (include/anitowave.hpp).

CPU: tests/cpp/reference_api.cpp — a caller written in the reference's call order (MSBGManager,
P2GTransfer, G2PManager, VCycleSolver) — compiles against the header and links against the
library.  GPU: it runs, and its results equal the same sequence issued through the Python
binding of the C ABI (bit-exact except P2G's shared-memory float sums, 1e-6 relative).
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "reference_api.cpp")


def _build(tmp_path):
    exe = str(tmp_path / "reference_api")
    lib = os.path.join(ROOT, "anitowave_adaptive_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", SRC,
           "-L", lib, "-lanitowave", "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{lib}", "-o", exe]
    subprocess.check_call(cmd)
    return exe


def test_reference_named_classes_compile_and_link(tmp_path):
    if not os.path.exists(os.path.join(ROOT, "anitowave_adaptive_b200", "libanitowave.so")):
        pytest.skip("library not built")
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_reference_named_classes_match_the_c_abi(tmp_path):
    import torch

    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import scenes

    exe = _build(tmp_path)
    S = scenes.config("dam_break_16")
    rng = np.random.default_rng(4)
    vel = (0.3 * rng.standard_normal(S.pos.shape)).astype(np.float32)
    data = str(tmp_path / "particles.bin")
    np.concatenate([S.pos, vel], 1).astype(np.float32).tofile(data)
    th = list(S.thresholds) + [0]
    subprocess.check_call([exe, data, str(S.dims[0]), repr(S.block_size), str(S.base_res), str(S.num_levels),
                           str(th[0]), str(th[1])])
    out = np.fromfile(data + ".out", np.float32)
    # the same sequence through the Python binding
    g = aw.build_grid(S)
    tot = g.totals()
    pos = torch.as_tensor(S.pos, device="cuda")
    v = torch.as_tensor(vel, device="cuda")
    g.p2g(pos, v)
    u = [g.channel(aw.VELOCITY_X + a).cpu().numpy() for a in range(3)]
    g.backup_grid_velocity()
    g.g2p(v, pos, 0.95)
    g.advect(pos, 1.0 / 240)
    sv = aw.Solver(g, operator_mode=aw.OPERATOR_REFERENCE)
    nc = tot[0]
    k = 0
    for a in range(3):
        got = out[k:k + tot[1 + a]]
        k += tot[1 + a]
        assert np.allclose(got, u[a], rtol=1e-6, atol=1e-7)
    n = S.n
    got_v = out[k:k + 3 * n].reshape(n, 3)
    k += 3 * n
    got_p = out[k:k + 3 * n].reshape(n, 3)
    k += 3 * n
    assert np.allclose(got_v, v.cpu().numpy(), rtol=1e-5, atol=1e-6)
    assert np.allclose(got_p, pos.cpu().numpy(), rtol=1e-6, atol=1e-6)
    got_x = out[k:k + nc]
    b = out[k + nc:k + 2 * nc]
    sv.level_array(0, 1).copy_(torch.as_tensor(b, device="cuda"))
    sv.vcycle()
    sv.vcycle()
    assert np.array_equal(got_x, sv.level_array(0, 0).cpu().numpy())
    sv.close()
