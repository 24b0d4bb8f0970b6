"""GPU parity: the sm_100a library (through its C ABI) against the FP64 oracle.

Bars: bit-exact for level maps, grading, offsets, sort keys and order, cell counts; 1e-5
relative L2 for FP32 floating-point results (grid velocities, residuals, V-cycle, particle
velocities); the Galerkin coefficients of the reference formula bit-exact.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import anitowave_adaptive_b200 as aw  # noqa: E402
from anitowave_adaptive_b200 import scenes  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-5  # relative L2 bar for FP32 results


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def oracle_grid(S):
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, passes = po.enforce_grading(S.dims, S.num_levels, lv)
    return lv, passes, po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)


SCENES = ["dam_break_32", "dam_break_64", "dam_drop_128"]


@pytest.fixture(scope="module", params=SCENES)
def case(request):
    S = scenes.config(request.param)
    lv, passes, O = oracle_grid(S)
    g = aw.build_grid(S)
    return S, lv, O, g


def test_level_map_and_offsets_bit_exact(case):
    S, lv, O, g = case
    assert np.array_equal(g.refinement_map(), lv)
    assert g.totals() == [int(t) for t in O.tot0]
    for k in range(4):
        assert np.array_equal(g.offsets(k), O.off0[k])


def test_coarse_offsets_bit_exact(case):
    S, lv, O, g = case
    for m in range(S.num_levels + 1):
        off, tot = O.offsets(m, vanish=True)
        for k in range(4):
            got, t = g.coarse_offsets(m, k)
            assert np.array_equal(got, off[k]) and t == tot[k]


def test_block_info_morton(case):
    S, lv, O, g = case
    info = g.block_info()
    for b in range(0, g.nb, max(1, g.nb // 97)):
        x, y, z = b % S.dims[0], (b // S.dims[0]) % S.dims[1], b // (S.dims[0] * S.dims[1])
        assert list(info[b]) == [x, y, z, po.morton3d(x, y, z)]


def test_sort_bit_exact(case):
    S, lv, O, g = case
    rng = np.random.default_rng(11)
    idx = rng.permutation(S.n)
    pos = np.ascontiguousarray(S.pos[idx])
    keys_o, perm_o = O.particle_keys(pos)
    keys, perm = g.sort_particles(torch.as_tensor(pos, device="cuda"))
    assert np.array_equal(perm.cpu().numpy().astype(np.int64), perm_o)
    assert np.array_equal(keys.cpu().numpy().view(np.uint32), keys_o[perm_o])


def test_p2g_matches_oracle(case):
    S, lv, O, g = case
    rng = np.random.default_rng(12)
    vel = (rng.standard_normal((S.n, 3)) * 0.5).astype(np.float32)
    u, m, cnt = O.p2g(S.pos, vel)
    g.p2g(torch.as_tensor(S.pos, device="cuda"), torch.as_tensor(vel, device="cuda"))
    torch.cuda.synchronize()
    for a in range(3):
        assert rel_l2(g.channel(aw.MASS_DENSITY_X + a).cpu().numpy(), m[a]) < RTOL
        assert rel_l2(g.channel(aw.VELOCITY_X + a).cpu().numpy(), u[a]) < RTOL
    assert np.array_equal(g.channel(aw.CELL_TYPE).cpu().numpy().astype(np.int64), cnt.astype(np.int64))


def _random_fields(O, rng):
    t = O.tot0
    return [rng.standard_normal(int(t[1 + a])) for a in range(3)]


def test_g2p_and_advect_match_oracle(case):
    S, lv, O, g = case
    rng = np.random.default_rng(13)
    un = _random_fields(O, rng)
    uo = _random_fields(O, rng)
    for a in range(3):
        g.channel(aw.VELOCITY_X + a).copy_(torch.as_tensor(un[a], dtype=torch.float32))
        g.channel(aw.VELOCITY_OLD_X + a).copy_(torch.as_tensor(uo[a], dtype=torch.float32))
    un32 = [x.astype(np.float32).astype(np.float64) for x in un]
    uo32 = [x.astype(np.float32).astype(np.float64) for x in uo]
    vel = (rng.standard_normal((S.n, 3))).astype(np.float32)
    ref = O.g2p(S.pos, un32, uo32, 0.95, vel)
    pos_t = torch.as_tensor(S.pos, device="cuda")
    vel_t = torch.as_tensor(vel, device="cuda")
    g.g2p(vel_t, pos_t, 0.95)
    assert rel_l2(vel_t.cpu().numpy(), ref) < RTOL
    dt = S.dt * 0.05
    xr = O.advect(un32, dt, S.pos.astype(np.float64))
    g.advect(pos_t, dt)
    check_positions(pos_t.cpu().numpy(), xr, S.pos)


def test_dropin_g2p_advect_after_p2g_match_oracle(case):
    # aw_g2p / aw_advect on the arrays the preceding aw_p2g sorted take the block-sorted kernels
    # (the caller's arrays hash as they did at the sort); once the arrays change, the general path.
    S, lv, O, g = case
    rng = np.random.default_rng(17)
    vel = (rng.standard_normal((S.n, 3))).astype(np.float32)
    pos_t = torch.as_tensor(S.pos, device="cuda")
    vel_t = torch.as_tensor(vel, device="cuda")
    g.p2g(pos_t, vel_t)
    un = _random_fields(O, rng)
    uo = _random_fields(O, rng)
    for a in range(3):
        g.channel(aw.VELOCITY_X + a).copy_(torch.as_tensor(un[a], dtype=torch.float32))
        g.channel(aw.VELOCITY_OLD_X + a).copy_(torch.as_tensor(uo[a], dtype=torch.float32))
    un32 = [x.astype(np.float32).astype(np.float64) for x in un]
    uo32 = [x.astype(np.float32).astype(np.float64) for x in uo]
    g.g2p(vel_t, pos_t, 0.95)  # sorted path
    v1 = vel_t.cpu().numpy()
    assert rel_l2(v1, O.g2p(S.pos, un32, uo32, 0.95, vel)) < RTOL
    g.g2p(vel_t, pos_t, 0.6)  # the velocities changed: general path
    assert rel_l2(vel_t.cpu().numpy(), O.g2p(S.pos, un32, uo32, 0.6, v1)) < RTOL
    g.p2g(pos_t, vel_t)
    for a in range(3):
        g.channel(aw.VELOCITY_X + a).copy_(torch.as_tensor(un[a], dtype=torch.float32))
    dt = S.dt * 0.05
    xr = O.advect(un32, dt, S.pos.astype(np.float64))
    g.advect(pos_t, dt)  # sorted path
    check_positions(pos_t.cpu().numpy(), xr, S.pos)
    # a position moved in place after the sort: the general path, still exact
    g.p2g(pos_t, vel_t)
    for a in range(3):
        g.channel(aw.VELOCITY_X + a).copy_(torch.as_tensor(un[a], dtype=torch.float32))
    x1 = pos_t.cpu().numpy().astype(np.float64)
    pos_t[0, 0] += 1e-3
    x1[0, 0] = float(pos_t[0, 0])
    v2 = vel_t.cpu().numpy()
    g.g2p(vel_t, pos_t, 0.95)
    assert rel_l2(vel_t.cpu().numpy(), O.g2p(x1.astype(np.float32), un32, uo32, 0.95, v2)) < RTOL


def check_positions(x_gpu, x_ref, x0):
    """Positions are FP32: compare per particle with a bound of 1e-5 of the displacement plus the
    rounding of an FP32 position (4 ulps of the domain extent 1.0)."""
    disp = np.abs(x_ref - x0).max()
    err = np.abs(x_gpu.astype(np.float64) - x_ref).max()
    assert err < 1e-5 * disp + 4 * np.spacing(np.float32(1.0)), (err, disp)


def _fv_solver_pair(S, O, g, fluid, **kw):
    O.set_params(mode=0)
    O.build(fluid=fluid)
    sv = aw.Solver(g, **kw)
    sv.setup(torch.as_tensor(fluid, device="cuda"))
    return sv


def test_fv_hierarchy_matches_oracle(case):
    S, lv, O, g = case
    u, m, cnt = O.p2g(S.pos, S.vel)
    fluid = (cnt > 0).astype(np.uint8)
    sv = _fv_solver_pair(S, O, g, fluid)
    assert sv.num_levels() == O.num_levels()
    for lvl in range(O.num_levels()):
        info = O.level_info(lvl)
        assert np.array_equal(sv.level_array(lvl, 6).cpu().numpy(), O.get(lvl, 6).astype(np.uint8))
        for a in range(3):
            assert rel_l2(sv.level_array(lvl, 3 + a).cpu().numpy(), O.get(lvl, 3 + a)) < 1e-6
        if not info[0]:
            off, _ = O.offsets(lvl, vanish=False)
            for k in range(4):
                assert np.array_equal(sv.level_array(lvl, 7 + k).cpu().numpy().view(np.uint32), off[k])


def test_fv_residual_smoother_vcycle_match_oracle(case):
    S, lv, O, g = case
    u, m, cnt = O.p2g(S.pos, S.vel)
    fluid = (cnt > 0).astype(np.uint8)
    sv = _fv_solver_pair(S, O, g, fluid, target_reduction=0.0)
    O.set_params(mode=0, target=0.0)
    O.build(fluid=fluid)
    rng = np.random.default_rng(14)
    n = int(O.tot0[0])
    x = (rng.standard_normal(n) * fluid).astype(np.float32)
    b = (rng.standard_normal(n) * fluid).astype(np.float32)
    X, B, R = sv.level_array(0, 0), sv.level_array(0, 1), sv.level_array(0, 2)
    # residual
    X.copy_(torch.as_tensor(x)); B.copy_(torch.as_tensor(b))
    O.set(0, 0, x.astype(np.float64)); O.set(0, 1, b.astype(np.float64))
    sv.residual(0); O.residual(0)
    torch.cuda.synchronize()
    assert rel_l2(R.cpu().numpy(), O.get(0, 2)) < RTOL
    # smoother (2 iterations, early exit disabled so both run the same sweeps)
    sv.smooth(0, 2); O.smooth(0, 2)
    torch.cuda.synchronize()
    assert rel_l2(X.cpu().numpy(), O.get(0, 0)) < RTOL
    # one V-cycle from zero
    X.zero_(); O.set(0, 0, np.zeros(n))
    sv.vcycle(); O.vcycle()
    torch.cuda.synchronize()
    assert rel_l2(X.cpu().numpy(), O.get(0, 0)) < RTOL


@pytest.mark.parametrize("precision", [aw.PRECISION_FP32, aw.PRECISION_MIXED, aw.PRECISION_FP32_PCG])
def test_fv_solve_reaches_tolerance(case, precision):
    S, lv, O, g = case
    x, v, perm, d = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), tol=1e-12)
    fluid = d["fluid"]
    b = d["b"].astype(np.float32)
    # plain FP32 stalls near 5e-6 on these problems: the rounding of an FP32 pressure alone
    # leaves a relative residual of that order; the mixed form carries the pressure in FP64
    # FP32 conjugate gradients carry the same FP32 rounding floor as the plain FP32 iteration
    tol = 1e-9 if precision == aw.PRECISION_MIXED else 2e-5
    sv = _fv_solver_pair(S, O, g, fluid, precision=precision, tolerance=tol, max_cycles=60)
    bt = torch.as_tensor(b, device="cuda")
    pt = torch.zeros(b.shape[0], dtype=torch.float64 if precision == aw.PRECISION_MIXED else torch.float32,
                     device="cuda")
    cyc, rel, st = sv.solve(bt, pt)
    assert rel < tol
    p = pt.cpu().numpy().astype(np.float64)
    # residual of the GPU pressure under the FP64 operator
    r = b.astype(np.float64) - O.apply(0, p)
    # under the FP64 oracle operator (FP64 conductances): FP32 storage of W and b bounds the mixed
    # result near 1e-8
    assert np.linalg.norm(r * fluid) / np.linalg.norm(b * fluid) < (1e-7 if precision == aw.PRECISION_MIXED else 5e-5)


def swirl(pos):
    """smooth divergent initial velocity (O(1) everywhere) for the parity of moving particles"""
    x, y, z = (pos[:, 0] - 0.5), (pos[:, 1] - 0.5), (pos[:, 2] - 0.5)
    return np.stack([-y + 0.3 * np.sin(6 * z), x + 0.2 * np.cos(5 * x), 0.5 * np.sin(4 * y)], -1).astype(np.float32)


@pytest.mark.parametrize("init", ["swirl", "rest"])
def test_flip_step_matches_oracle(case, init):
    S, lv, O, g = case
    vel0 = swirl(S.pos) if init == "swirl" else S.vel
    xo, vo, perm, d = po.flip_step(O, S.pos, vel0, S.dt, 0.95, (0, S.gravity, 0), tol=1e-12)
    F = aw.Flip(g, S.pos, vel0, S.dt, 0.95, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-10,
                max_cycles=60)
    F.step()
    pos, vel = F.particles()
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    v_ref = vo[inv]
    x_ref = xo[inv]
    if init == "swirl":
        assert rel_l2(vel, v_ref) < RTOL
        for a in range(3):
            assert rel_l2(g.channel(aw.VELOCITY_X + a).cpu().numpy(), d["u_new"][a]) < RTOL
    else:
        # from rest the step's velocities are ~1e-3 of the gravity increment that the projection
        # cancels; the bar is relative to that increment (FP32 rounding of u* = -g dt)
        scale = abs(S.gravity) * S.dt * np.sqrt(vel.size)
        assert np.linalg.norm(vel - v_ref) / scale < RTOL
    check_positions(pos, x_ref, S.pos)
    st = F.stats()
    assert st["div_after"] < 1e-4 * max(st["div_before"], 1e-30)
    F.close()


def test_reference_mode_galerkin_bit_exact():
    # reference constants: 16^3 base blocks, 3 levels, single-level map (the demo's layout)
    dims, R0, L = (4, 3, 5), 16, 3
    g = aw.MSBG(dims, 1.0, (0, 0, 0), R0, L)
    g.init_refinement_map(0)
    g.allocate()
    lv = np.zeros(int(np.prod(dims)), np.uint32)
    O = po.Oracle(dims, 1.0, (0, 0, 0), R0, L, lv)
    rng = np.random.default_rng(15)
    for dest in (1, 2):
        _, totf = O.offsets(dest - 1, True)
        _, totc = O.offsets(dest, True)
        fine = [rng.random(int(totf[1 + a])).astype(np.float32) + 0.5 for a in range(3)]
        ref = O.galerkin_ref(dest, fine)
        ft = [torch.as_tensor(f, device="cuda") for f in fine]
        ct = [torch.zeros(int(totc[1 + a]), device="cuda") for a in range(3)]
        g.run_galerkin(ft, ct, dest)
        for a in range(3):
            assert np.array_equal(ct[a].cpu().numpy().view(np.uint32), ref[a].view(np.uint32))


def test_reference_mode_vcycle_matches_oracle():
    dims, R0, L = (3, 3, 3), 16, 3
    g = aw.MSBG(dims, 1.0, (0, 0, 0), R0, L)
    g.init_refinement_map(0)
    g.allocate()
    lv = np.zeros(27, np.uint32)
    O = po.Oracle(dims, 1.0, (0, 0, 0), R0, L, lv)
    O.set_params(mode=1, pre=2, post=2, coarsest_iters=50, block_iters=10, omega=0.85714, target=0.0, theta=1e-4)
    O.build()
    sv = aw.Solver(g, operator_mode=aw.OPERATOR_REFERENCE, target_reduction=0.0)
    rng = np.random.default_rng(16)
    n = int(O.tot0[0])
    b = rng.standard_normal(n).astype(np.float32)
    sv.level_array(0, 1).copy_(torch.as_tensor(b))
    sv.level_array(0, 0).zero_()
    O.set(0, 1, b.astype(np.float64))
    for lvl in range(1, 3):
        for a in range(3):
            assert rel_l2(sv.level_array(lvl, 3 + a).cpu().numpy(), O.get(lvl, 3 + a)) < 1e-6
    sv.vcycle()
    O.vcycle()
    torch.cuda.synchronize()
    assert rel_l2(sv.level_array(0, 0).cpu().numpy(), O.get(0, 0)) < RTOL


def test_error_paths_return_status():
    with pytest.raises(aw.AWError) as e:
        aw.MSBG((0, 1, 1), 1.0, (0, 0, 0), 8, 2)
    assert e.value.status == 1
    with pytest.raises(aw.AWError):
        aw.MSBG((2, 2, 2), 1.0, (0, 0, 0), 6, 2)
    g = aw.MSBG((2, 2, 2), 1.0, (0, 0, 0), 8, 2)
    with pytest.raises(aw.AWError):
        g.totals()  # not allocated


@pytest.mark.gpu
def test_rebuild_levels_between_steps_matches_oracle():
    """aw_flip_rebuild_levels, every 10 steps over 160 steps: the level map re-derived from the moving
    particles (on the device, graded to its fixpoint there) is bit-exact with the oracle's at every
    rebuild, the grid is laid out again when it changes, and the step after the first change matches
    the FP64 oracle's step from the same particle state on the new layout."""
    import anitowave_adaptive_b200 as aw
    from anitowave_adaptive_b200 import scenes
    from oracle import pyoracle as po

    S = scenes.config("dam_break_16")
    grav = (0.0, S.gravity, 0.0)
    g = aw.build_grid(S)
    F = aw.Flip(g, S.pos, S.vel, S.dt, S.alpha, grav, precision=aw.PRECISION_MIXED, tolerance=1e-10)
    changes, unchanged, stepped = 0, 0, False
    for k in range(160):
        F.step()
        if (k + 1) % 10:
            continue
        pos, vel = F.particles()
        changed = F.rebuild_levels(S.thresholds)
        lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, pos, S.thresholds)
        lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
        assert np.array_equal(g.refinement_map(), lv), k
        changes += int(changed)
        unchanged += int(not changed)
        if changed and not stepped:
            stepped = True
            O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
            assert np.array_equal(O.tot0, np.asarray(g.totals(), np.uint32))
            xo, vo, perm, _ = po.flip_step(O, pos, vel, S.dt, S.alpha, grav, tol=1e-12)
            F.step()
            p2, v2 = F.particles()
            inv = np.empty_like(perm)
            inv[perm] = np.arange(perm.size)
            assert np.linalg.norm(v2 - vo[inv]) <= 1e-5 * np.linalg.norm(vo[inv])
            assert np.linalg.norm(p2 - xo[inv]) <= 1e-6 * np.linalg.norm(xo[inv])
    assert changes >= 1 and unchanged >= 1, (changes, unchanged)
    F.close()
