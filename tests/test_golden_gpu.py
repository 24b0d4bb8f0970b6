"""The library's reference-operator mode against fixtures from the reference's own CUDA build
(tests/golden/ref_*.npz; reference constants 16^3 base blocks, 3 levels), through the C ABI."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import anitowave_adaptive_b200 as aw  # noqa: E402

pytestmark = pytest.mark.gpu
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


def grid(dims, levels):
    g = aw.MSBG(dims, 1.0, (0, 0, 0), 16, 3)
    g.set_refinement_map(np.asarray(levels, np.uint32))
    return g


def cases(f):
    i = 0
    while f"g{i}_dims" in f:
        yield i
        i += 1


def test_grading_offsets_galerkin_bit_exact():
    f = load("ref_grid.npz")
    for i in cases(f):
        dims = tuple(int(v) for v in f[f"g{i}_dims"])
        g = grid(dims, f[f"g{i}_in"])
        g.enforce_grading()
        assert np.array_equal(g.refinement_map(), f[f"g{i}_out"])
        g.allocate()
        assert g.totals() == list(f[f"g{i}_totals"])
        for k in range(4):
            assert np.array_equal(g.offsets(k), f[f"g{i}_offsets"][k])
        g2 = grid(dims, f[f"g{i}_active"])
        g2.enforce_grading()
        g2.allocate()
        for m in range(4):
            for k in range(4):
                off, tot = g2.coarse_offsets(m, k)
                assert np.array_equal(off, f[f"g{i}_coarse{m}"][k]) and tot == f[f"g{i}_coarse{m}_tot"][k]
    dims = tuple(int(v) for v in f["gal_dims"])
    g3 = grid(dims, f["gal_levels"])
    g3.enforce_grading()
    g3.allocate()
    for dest in (1, 2):
        fine = [torch.as_tensor(f[f"gal{dest}_fine{a}"], device="cuda") for a in range(3)]
        coarse = [torch.zeros(max(1, f[f"gal{dest}_coarse{a}"].size), device="cuda") for a in range(3)]
        g3.run_galerkin(fine, coarse, dest)
        for a in range(3):
            ref = f[f"gal{dest}_coarse{a}"]
            got = coarse[a].cpu().numpy()[: ref.size]
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (dest, a)


def ref_solver(f, variant):
    dims = tuple(int(v) for v in f["dims"])
    g = grid(dims, np.zeros(int(np.prod(dims)), np.uint32))
    g.enforce_grading()
    g.allocate()
    for a in range(3):
        g.channel(aw.BETA_COEFF_X + a).copy_(torch.as_tensor(f[f"{variant}_beta{a}"]))
    return g, aw.Solver(g, operator_mode=aw.OPERATOR_REFERENCE)


@pytest.mark.parametrize("variant", ["unit", "rand"])
def test_reference_mode_kernels(variant):
    f = load("ref_mg.npz")
    g, sv = ref_solver(f, variant)
    for lvl in (1, 2):
        for a in range(3):
            assert rel_l2(sv.level_array(lvl, 3 + a).cpu().numpy(), f[f"{variant}_level{lvl}_beta{a}"]) < 1e-6
    for lvl in (0, 1, 2):
        X, B, R = sv.level_array(lvl, 0), sv.level_array(lvl, 1), sv.level_array(lvl, 2)
        key = f"{variant}_L{lvl}_residual"
        X.copy_(torch.as_tensor(f[key + "_x_in"]))
        B.copy_(torch.as_tensor(f[key + "_b_in"]))
        sv.residual(lvl)
        torch.cuda.synchronize()
        assert rel_l2(R.cpu().numpy(), f[key + "_r"]) < 1e-5
        key = f"{variant}_L{lvl}_restrict"
        if key + "_b1" in f:
            X.copy_(torch.as_tensor(f[key + "_x_in"]))
            B.copy_(torch.as_tensor(f[key + "_b_in"]))
            sv.residual(lvl)
            sv.restrict(lvl)
            torch.cuda.synchronize()
            assert rel_l2(sv.level_array(lvl + 1, 1).cpu().numpy(), f[key + "_b1"]) < 1e-5
        key = f"{variant}_L{lvl}_prolong"
        if key + "_x" in f:
            X.copy_(torch.as_tensor(f[key + "_x_in"]))
            sv.level_array(lvl + 1, 0).copy_(torch.as_tensor(f[key + "_x1_in"]))
            sv.prolongate(lvl)
            torch.cuda.synchronize()
            assert rel_l2(X.cpu().numpy(), f[key + "_x"]) < 1e-6
        key = f"{variant}_L{lvl}_smooth"
        X.copy_(torch.as_tensor(f[key + "_x_in"]))
        B.copy_(torch.as_tensor(f[key + "_b_in"]))
        sv.smooth(lvl, 2)
        torch.cuda.synchronize()
        assert rel_l2(X.cpu().numpy(), f[key + "_x"]) < 1e-5
    key = f"{variant}_L0_vcycle"
    X, B = sv.level_array(0, 0), sv.level_array(0, 1)
    X.copy_(torch.as_tensor(f[key + "_x_in"]))
    B.copy_(torch.as_tensor(f[key + "_b_in"]))
    sv.vcycle()
    torch.cuda.synchronize()
    assert rel_l2(X.cpu().numpy(), f[key + "_x"]) < 1e-5


def test_flip_blend_and_rk3_match_reference_kernels():
    # aw_g2p / aw_advect against g2pUpdateKernel / advectParticlesKernel (G2P.cuh:87-173) run on a
    # B200, on single-level maps with a velocity uniform per axis and particles two cells from the
    # walls.  Bars: velocity 1e-5 relative L2; positions 1e-6 and the RK3 displacement 1e-4 (both
    # sides FP32: x + dt v rounds at 6e-8 against a 5e-3 displacement).
    f = load("ref_transfer.npz")
    n = 0
    i = 0
    while f"c{i}_dims" in f:
        k = f"c{i}_"
        dims = tuple(int(v) for v in f[k + "dims"])
        g = aw.MSBG(dims, 1.0, (0, 0, 0), 16, 3)
        g.init_refinement_map(int(f[k + "level"]))
        g.enforce_grading()
        g.allocate()
        for a in range(3):
            g.channel(aw.VELOCITY_X + a).fill_(float(f[k + "u_new"][a]))
            g.channel(aw.VELOCITY_OLD_X + a).fill_(float(f[k + "u_old"][a]))
        pos = torch.as_tensor(f[k + "pos"], device="cuda")
        vel = torch.as_tensor(f[k + "vel"], device="cuda")
        g.g2p(vel, pos, float(f[k + "alpha"]))
        torch.cuda.synchronize()
        assert rel_l2(vel.cpu().numpy(), f[k + "vel_out"]) < 1e-5, i
        x = pos.clone()
        g.advect(x, float(f[k + "dt"]))
        torch.cuda.synchronize()
        x = x.cpu().numpy().astype(np.float64)
        p0 = f[k + "pos"].astype(np.float64)
        assert rel_l2(x, f[k + "pos_out"]) < 1e-6, i
        assert rel_l2(x - p0, f[k + "pos_out"].astype(np.float64) - p0) < 1e-4, i
        g.close()
        n += 1
        i += 1
    assert n >= 2
