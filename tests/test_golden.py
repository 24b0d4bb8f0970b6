"""Pin the oracle against fixtures produced by the reference's own CUDA build.

tests/golden/ref_*.npz were generated by tests/golden/make_ref_golden.py, which runs the
reference's kernels (compiled from its own headers by oracle/build_ref.py) on a B200.  Reference
constants: 16^3 base blocks, 3 levels.  Bars: bit-exact for integer maps, offsets and the
Galerkin coefficients (same single-precision formula); 1e-5 relative L2 for the multigrid
kernels (FP32 reference vs FP64 oracle).
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as po

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        pytest.skip(f"fixture {name} missing")
    return np.load(path)


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)


def test_layout_morton_block_info():
    f = load("ref_layout.npz")
    R0, ML = int(f["R0"]), int(f["MAX_LEVELS"])
    assert (R0, ML) == (16, 3)
    for lvl in range(ML):
        assert np.array_equal(po.block_layout(R0, lvl), f["layouts"][lvl])
    for (x, y, z), m in zip(f["morton_in"], f["morton"]):
        assert po.morton3d(int(x), int(y), int(z)) == m
    dims = f["block_info_dims"]
    bi = f["block_info"]
    for b in range(bi.shape[0]):
        x, y, z = b % dims[0], (b // dims[0]) % dims[1], b // (dims[0] * dims[1])
        assert list(bi[b]) == [x, y, z, 0, po.morton3d(x, y, z)]


def cases(f):
    i = 0
    while f"g{i}_dims" in f:
        yield i
        i += 1


def test_grading_and_offsets_bit_exact():
    f = load("ref_grid.npz")
    n = 0
    for i in cases(f):
        dims = tuple(int(v) for v in f[f"g{i}_dims"])
        out, _ = po.enforce_grading(dims, 3, f[f"g{i}_in"])
        assert np.array_equal(out, f[f"g{i}_out"])
        O = po.Oracle(dims, 1.0, (0, 0, 0), 16, 3, f[f"g{i}_out"])
        off, tot = O.offsets(0, vanish=True)
        assert np.array_equal(off, f[f"g{i}_offsets"]) and np.array_equal(tot, f[f"g{i}_totals"])
        n += 1
    assert n >= 3


def test_coarse_offsets_bit_exact():
    f = load("ref_grid.npz")
    for i in cases(f):
        dims = tuple(int(v) for v in f[f"g{i}_dims"])
        O = po.Oracle(dims, 1.0, (0, 0, 0), 16, 3, f[f"g{i}_active"])
        for m in range(4):
            off, tot = O.offsets(m, vanish=True)
            assert np.array_equal(off, f[f"g{i}_coarse{m}"]), (i, m)
            assert np.array_equal(tot, f[f"g{i}_coarse{m}_tot"])


def test_galerkin_bit_exact():
    f = load("ref_grid.npz")
    dims = tuple(int(v) for v in f["gal_dims"])
    O = po.Oracle(dims, 1.0, (0, 0, 0), 16, 3, f["gal_levels"])
    for dest in (1, 2):
        fine = [f[f"gal{dest}_fine{a}"] for a in range(3)]
        got = O.galerkin_ref(dest, fine)
        for a in range(3):
            ref = f[f"gal{dest}_coarse{a}"]
            assert np.array_equal(got[a].view(np.uint32), ref.view(np.uint32)), (dest, a)


def mg_oracle(f, variant):
    dims = tuple(int(v) for v in f["dims"])
    nb = int(np.prod(dims))
    O = po.Oracle(dims, 1.0, (0, 0, 0), 16, 3, np.zeros(nb, np.uint32))
    O.set_params(mode=1)
    beta = [f[f"{variant}_beta{a}"].astype(np.float64) for a in range(3)]
    O.build(bbar=beta)
    return O


@pytest.mark.parametrize("variant", ["unit", "rand"])
def test_reference_hierarchy_coefficients(variant):
    f = load("ref_mg.npz")
    O = mg_oracle(f, variant)
    for lvl in (1, 2):
        for a in range(3):
            assert rel_l2(O.get(lvl, 3 + a), f[f"{variant}_level{lvl}_beta{a}"]) < 1e-6


@pytest.mark.parametrize("variant", ["unit", "rand"])
@pytest.mark.parametrize("lvl", [0, 1, 2])
def test_reference_residual_restrict_prolong(variant, lvl):
    f = load("ref_mg.npz")
    O = mg_oracle(f, variant)
    key = f"{variant}_L{lvl}_residual"
    O.set(lvl, 0, f[key + "_x_in"].astype(np.float64))
    O.set(lvl, 1, f[key + "_b_in"].astype(np.float64))
    O.residual(lvl)
    assert rel_l2(O.get(lvl, 2), f[key + "_r"]) < 1e-5
    key = f"{variant}_L{lvl}_restrict"
    if key + "_b1" in f:
        O.set(lvl, 0, f[key + "_x_in"].astype(np.float64))
        O.set(lvl, 1, f[key + "_b_in"].astype(np.float64))
        O.residual(lvl)
        O.restrict(lvl)
        assert rel_l2(O.get(lvl + 1, 1), f[key + "_b1"]) < 1e-5
    key = f"{variant}_L{lvl}_prolong"
    if key + "_x" in f:
        O.set(lvl, 0, f[key + "_x_in"].astype(np.float64))
        O.set(lvl + 1, 0, f[key + "_x1_in"].astype(np.float64))
        O.prolong(lvl)
        assert rel_l2(O.get(lvl, 0), f[key + "_x"]) < 1e-6


@pytest.mark.parametrize("variant", ["unit", "rand"])
@pytest.mark.parametrize("lvl", [0, 1, 2])
def test_reference_smoother(variant, lvl):
    f = load("ref_mg.npz")
    O = mg_oracle(f, variant)
    key = f"{variant}_L{lvl}_smooth"
    O.set(lvl, 0, f[key + "_x_in"].astype(np.float64))
    O.set(lvl, 1, f[key + "_b_in"].astype(np.float64))
    O.smooth(lvl, 2)
    assert rel_l2(O.get(lvl, 0), f[key + "_x"]) < 1e-5


@pytest.mark.parametrize("variant", ["unit", "rand"])
def test_reference_vcycle(variant):
    f = load("ref_mg.npz")
    O = mg_oracle(f, variant)
    key = f"{variant}_L0_vcycle"
    O.set(0, 0, f[key + "_x_in"].astype(np.float64))
    O.set(0, 1, f[key + "_b_in"].astype(np.float64))
    O.vcycle()
    assert rel_l2(O.get(0, 0), f[key + "_x"]) < 1e-5


def test_normalize_velocity_rule():
    # normalizeVelocity (P2G.cuh:163-170): u = P / m where m > 1e-6, else 0 (FP32)
    f = load("ref_normalize.npz")
    for a in range(3):
        m, p = f[f"mass{a}"], f[f"mom{a}"]
        u = np.where(m > np.float32(1e-6), p / np.where(m > 0, m, 1), np.float32(0)).astype(np.float32)
        assert np.array_equal(u.view(np.uint32), f[f"vel{a}"].view(np.uint32))


def transfer_cases(f):
    i = 0
    while f"c{i}_dims" in f:
        yield i
        i += 1


def uniform_fields(tot, values):
    return [np.full(int(tot[1 + a]), float(values[a])) for a in range(3)]


def test_flip_blend_and_rk3_match_reference_kernels():
    # g2pUpdateKernel (G2P.cuh:87-128) and advectParticlesKernel (G2P.cuh:131-173) run on a B200:
    # single-level maps, velocity uniform per axis, particles two cells from the walls.  Bars: the
    # blended velocity to 1e-5 relative L2 (FP32 reference vs FP64 oracle); positions to 1e-6 and the
    # RK3 displacement to 1e-4 (the FP32 sum x + dt v rounds at 6e-8 against a 5e-3 displacement).
    f = load("ref_transfer.npz")
    n = 0
    for i in transfer_cases(f):
        k = f"c{i}_"
        dims = tuple(int(v) for v in f[k + "dims"])
        O = po.Oracle(dims, 1.0, (0, 0, 0), 16, 3, np.full(int(np.prod(dims)), int(f[k + "level"]), np.uint32))
        _, tot = O.offsets(0)
        un, uo = uniform_fields(tot, f[k + "u_new"]), uniform_fields(tot, f[k + "u_old"])
        pos = f[k + "pos"]
        v = O.g2p(pos, un, uo, float(f[k + "alpha"]), f[k + "vel"])
        assert rel_l2(v, f[k + "vel_out"]) < 1e-5, i
        x = O.advect(un, float(f[k + "dt"]), pos)
        assert rel_l2(x, f[k + "pos_out"]) < 1e-6, i
        assert rel_l2(x - pos, f[k + "pos_out"].astype(np.float64) - pos) < 1e-4, i
        n += 1
    assert n >= 2
