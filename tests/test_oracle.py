"""CPU tests of the FP64 oracle: index maps, grading, offsets, transfers and the projection.

These pin the oracle with known-answer and analytic cases (the reference ships no tests or
fixtures); tests/test_golden.py pins it against fixtures produced by the reference's own CUDA
build.
"""
import numpy as np
import pytest

from anitowave_adaptive_b200 import scenes
from oracle import pyoracle as po


def interleave(x, y, z):
    m = 0
    for i in range(10):
        m |= ((x >> i) & 1) << (3 * i)
        m |= ((y >> i) & 1) << (3 * i + 1)
        m |= ((z >> i) & 1) << (3 * i + 2)
    return m


def test_morton_matches_bit_interleave():
    rng = np.random.default_rng(0)
    for x, y, z in rng.integers(0, 1024, size=(200, 3)):
        assert po.morton3d(int(x), int(y), int(z)) == interleave(int(x), int(y), int(z))


@pytest.mark.parametrize("R0,levels", [(16, 3), (8, 4)])
def test_block_layout(R0, levels):
    for lv in range(levels):
        r = R0 >> lv
        out = po.block_layout(R0, lv)
        assert list(out) == [r ** 3, (r + 1) * r * r, r * (r + 1) * r, r * r * (r + 1), r ** 3 + 3 * (r + 1) * r * r, r]


def graded(levels, dims, L):
    lv = levels.reshape(dims[2], dims[1], dims[0])
    for z in range(dims[2]):
        for y in range(dims[1]):
            for x in range(dims[0]):
                a = lv[z, y, x]
                if a == L:
                    continue
                for dz in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dx in (-1, 0, 1):
                            zz, yy, xx = z + dz, y + dy, x + dx
                            if 0 <= zz < dims[2] and 0 <= yy < dims[1] and 0 <= xx < dims[0]:
                                b = lv[zz, yy, xx]
                                if b != L and abs(int(a) - int(b)) > 1:
                                    return False
    return True


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_grading_fixpoint(seed):
    rng = np.random.default_rng(seed)
    dims, L = (7, 5, 6), 4
    lv = rng.integers(0, L + 1, size=int(np.prod(dims))).astype(np.uint32)
    out, passes = po.enforce_grading(dims, L, lv)
    assert graded(out, dims, L)
    assert np.all(out <= lv)
    assert np.all((out == L) == (lv == L))
    again, p2 = po.enforce_grading(dims, L, out)
    assert p2 == 1 and np.array_equal(again, out)
    # maximality: raising any active block by one breaks grading or exceeds the input
    for b in rng.choice(np.nonzero(out < lv)[0], size=min(20, int((out < lv).sum())), replace=False):
        t = out.copy()
        t[b] += 1
        assert not graded(t, dims, L)


def test_offsets_are_exclusive_scan():
    dims, R0, L = (5, 4, 3), 8, 3
    rng = np.random.default_rng(3)
    lv, _ = po.enforce_grading(dims, L, rng.integers(0, L + 1, size=60).astype(np.uint32))
    O = po.Oracle(dims, 1.0, (0, 0, 0), R0, L, lv)
    for m in range(4):
        off, tot = O.offsets(m, vanish=True)
        r = np.where(lv < L, (R0 >> np.minimum(lv, 31)) >> m, 0)
        cells = r ** 3
        faces = np.where(r > 0, (r + 1) * r * r, 0)
        assert np.array_equal(off[0], np.concatenate([[0], np.cumsum(cells)[:-1]]))
        assert tot[0] == cells.sum()
        for k in (1, 2, 3):
            assert np.array_equal(off[k], np.concatenate([[0], np.cumsum(faces)[:-1]]))


def small_scene(N=32):
    S = scenes.config(f"dam_break_{N}")
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    return S, lv, po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)


def test_level_map_marks_surface_blocks():
    S, lv, O = small_scene(32)
    assert set(np.unique(lv)) == {0, 1}
    # the block holding the column's top surface is level 0; a far corner block is level 1
    dims = S.dims
    def b(x, y, z):
        return x + dims[0] * (y + dims[1] * z)
    assert lv[b(0, 2, 0)] == 0
    assert lv[b(3, 3, 3)] == 1 or lv[b(3, 3, 3)] == 0


def test_sort_is_stable_by_cell_key():
    S, lv, O = small_scene(32)
    rng = np.random.default_rng(5)
    idx = rng.permutation(S.n)
    keys, perm = O.particle_keys(S.pos[idx])
    ks = keys[perm]
    assert np.all(np.diff(ks.astype(np.int64)) >= 0)
    # ties in input order
    same = np.diff(ks.astype(np.int64)) == 0
    assert np.all(np.diff(perm)[same] > 0)


def test_p2g_uniform_velocity_is_reproduced():
    S, lv, O = small_scene(32)
    v = np.array([0.3, -1.25, 0.7], np.float32)
    vel = np.tile(v, (S.n, 1))
    u, m, cnt = O.p2g(S.pos, vel)
    for a in range(3):
        sel = m[a] > 1e-6
        assert sel.sum() > 1000
        np.testing.assert_allclose(u[a][sel], v[a], rtol=1e-12)
        assert np.all(u[a][~sel] == 0)
    assert cnt.sum() == S.n


def test_p2g_single_particle_weights():
    dims, R0, L = (2, 2, 2), 4, 1
    lv = np.zeros(8, np.uint32)
    O = po.Oracle(dims, 1.0, (0, 0, 0), R0, L, lv)
    p = np.array([[0.9, 1.1, 0.6]], np.float32)
    vel = np.array([[1.0, 2.0, 3.0]], np.float32)
    u, m, _ = O.p2g(p, vel)
    h = 0.25
    off, _ = O.offsets(0)
    # x-face (i, j, k) of block (bx, by, bz) sits at (bx + i h, by + (j+.5) h, bz + (k+.5) h)
    tot = 0.0
    for b in range(8):
        bc = np.array([b % 2, (b // 2) % 2, b // 4], float)
        for k in range(4):
            for j in range(4):
                for i in range(5):
                    xf = bc + h * np.array([i, j + 0.5, k + 0.5])
                    d2 = ((p[0].astype(float) - xf) ** 2).sum()
                    w = (1 - d2 / h ** 2) ** 3 if d2 < h * h else 0.0
                    got = m[0][off[1][b] + i + 5 * (j + 4 * k)]
                    assert abs(got - w) < 1e-12
                    tot += w
    assert tot > 0


def uniform_oracle(D=4, R0=8, L=1, bs=1.0):
    dims = (D, D, D)
    lv = np.zeros(D ** 3, np.uint32)
    return po.Oracle(dims, bs, (0, 0, 0), R0, L, lv)


def test_fv_operator_is_symmetric_multilevel():
    S, lv, O = small_scene(32)
    assert len(np.unique(lv)) == 2
    rng = np.random.default_rng(1)
    n = int(O.tot0[0])
    fluid = (rng.random(n) < 0.8).astype(np.uint8)
    O.set_params(mode=0)
    O.build(fluid=fluid)
    x = rng.standard_normal(n) * fluid
    y = rng.standard_normal(n) * fluid
    Ax, Ay = O.apply(0, x), O.apply(0, y)
    assert abs(y @ Ax - x @ Ay) < 1e-12 * np.abs(y @ Ax)
    assert x @ Ax < 0  # negative definite with Dirichlet air


def test_manufactured_poisson_dirichlet():
    O = uniform_oracle(4, 8, 1, 1.0)
    n = int(O.tot0[0])
    rng = np.random.default_rng(2)
    fluid = np.ones(n, np.uint8)
    fluid[rng.choice(n, 200, replace=False)] = 0  # air cells -> Dirichlet
    O.set_params(mode=0)
    O.build(fluid=fluid)
    p_true = rng.standard_normal(n) * fluid
    b = O.apply(0, p_true)
    p, hist = O.solve(b, tol=1e-12, max_cycles=80)
    assert hist[-1] < 1e-12
    np.testing.assert_allclose(p, p_true, atol=1e-9 * np.abs(p_true).max())


def test_projection_makes_velocity_divergence_free():
    S, lv, O = small_scene(32)
    x, v, perm, d = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), tol=1e-12)
    div = O.divergence(d["u_new"], d["fluid"], S.dt)
    assert np.abs(div).max() * S.dt < 1e-10 * np.abs(d["b"]).max() * S.dt + 1e-14
    assert d["hist"][-1] < 1e-12
    # convergence factor of the V-cycle (FV operator, all-children coarsening)
    rates = d["hist"][2:] / d["hist"][1:-1]
    assert np.median(rates) < 0.3


def test_hydrostatic_column_stays_at_rest():
    # a full-width column: the pressure balances gravity exactly, particles stay at rest
    S = scenes.dam_break(32, 8, 2, (8,), 0, 1.0 / 240, box=(1.0, 0.5, 1.0))
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    x, v, perm, d = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), tol=1e-13)
    assert np.abs(v).max() < 1e-9 * abs(S.gravity) * S.dt
    # pressure increases linearly with depth (fine level-0 cells: p = rho g (y_air - y))
    p = d["p"]
    assert p.max() > 0


def test_closed_box_poisson_converges():
    N, R0, L = 64, 8, 4
    dims = (N // R0,) * 3
    bs = R0 / N
    c, r = scenes.poisson_spheres()
    pts = scenes.sphere_surface_points(N, c, r)
    lv = po.levels_from_particles(dims, bs, (0, 0, 0), R0, L, pts, (8, 24, 56))
    lv, _ = po.enforce_grading(dims, L, lv)
    O = po.Oracle(dims, bs, (0, 0, 0), R0, L, lv)
    n = int(O.tot0[0])
    rng = np.random.default_rng(4)
    b = rng.standard_normal(n)
    b -= b.mean()
    O.set_params(mode=0)
    O.build(fluid=np.ones(n, np.uint8))
    p, hist = O.solve(b, tol=1e-10, max_cycles=40)
    assert hist[-1] < 1e-10
    assert len(hist) <= 15


def test_pcg_and_defect_correction_agree():
    """The oracle's two FP64 solves (V-cycle defect correction and V-cycle-preconditioned CG) reach
    the same pressure on a free-surface layout."""
    from anitowave_adaptive_b200 import scenes
    from oracle import pyoracle as po

    S = scenes.config("dam_break_16")
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    _, _, cnt = O.p2g(S.pos, S.vel)
    fluid = (cnt > 0).astype(np.uint8)
    rng = np.random.default_rng(1)
    b = rng.standard_normal(int(O.tot0[0])) * fluid
    O.set_params(mode=0)
    O.build(fluid=fluid)
    p1, h1 = O.solve(b, tol=1e-12, max_cycles=200)
    p2, h2 = O.solve(b, tol=1e-12, max_cycles=200, method="pcg")
    assert h1[-1] < 1e-12 and h2[-1] < 1e-12
    assert len(h2) <= len(h1)
    assert np.linalg.norm((p1 - p2) * fluid) <= 1e-9 * np.linalg.norm(p1 * fluid)


def test_fv_vcycle_is_a_symmetric_preconditioner():
    """With zero initial guess and no early exit the FV V-cycle is a linear map b -> x.  Post-smoothing
    in the adjoint order (colours black before red) makes that map symmetric, as conjugate gradients
    needs of its preconditioner: <V b1, b2> = <b1, V b2>."""
    S, lv, O = small_scene(64)
    assert len(np.unique(lv)) == 2
    rng = np.random.default_rng(7)
    n = int(O.tot0[0])
    _, _, cnt = O.p2g(S.pos, S.vel)
    fluid = (cnt > 0).astype(np.uint8)
    O.set_params(mode=0, target=0.0)
    O.build(fluid=fluid)

    def V(b):
        O.set(0, 0, np.zeros(n))
        O.set(0, 1, b)
        O.vcycle()
        return O.get(0, 0)

    b1 = rng.standard_normal(n) * fluid
    b2 = rng.standard_normal(n) * fluid
    x1, x2 = V(b1), V(b2)
    assert abs(x1 @ b2 - b1 @ x2) < 1e-10 * abs(x1 @ b2)
    assert x1 @ b1 < 0  # negative definite like A
