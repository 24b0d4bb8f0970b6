"""Edge cases of the particle transfers against the FP64 oracle: an empty particle set, one particle,
particles exactly on cell, block and domain boundaries, particles outside the domain or inside an
inactive block, and tens of thousands of particles in one coarse cell (the contended path of P2G,
where each warp deposits into a private copy of the block's tile)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import anitowave_adaptive_b200 as aw  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def make(levels, dims, R0=8, L=4, bs=1.0, dmin=(0.0, 0.0, 0.0)):
    g = aw.MSBG(dims, bs, dmin, R0, L)
    g.set_refinement_map(np.asarray(levels, np.uint32))
    g.enforce_grading()
    g.allocate()
    lv = g.refinement_map()
    return g, po.Oracle(dims, bs, dmin, R0, L, lv), lv


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x, np.float32), device="cuda")


def check_p2g(g, O, pos, vel):
    u, m, cnt = O.p2g(pos, vel)
    g.p2g(dev(pos), dev(vel))
    torch.cuda.synchronize()
    for a in range(3):
        assert rel_l2(g.channel(aw.MASS_DENSITY_X + a).cpu().numpy(), m[a]) < RTOL
        assert rel_l2(g.channel(aw.VELOCITY_X + a).cpu().numpy(), u[a]) < RTOL
    assert np.array_equal(g.channel(aw.CELL_TYPE).cpu().numpy().astype(np.int64), cnt.astype(np.int64))
    return u, m, cnt


# blocks along x at levels 0..3 (resolutions 8, 4, 2, 1), graded; 4 x 2 x 2 blocks of size 1
DIMS = (4, 2, 2)
LEVELS = [x for z in range(2) for y in range(2) for x in range(4)]


@pytest.fixture(scope="module")
def grid():
    g, O, lv = make(LEVELS, DIMS)
    assert list(lv[:4]) == [0, 1, 2, 3]
    return g, O


def test_empty_particle_set(grid):
    g, O = grid
    pos = np.zeros((0, 3), np.float32)
    g.p2g(dev(pos), dev(pos))
    torch.cuda.synchronize()
    for a in range(3):
        assert not np.any(g.channel(aw.VELOCITY_X + a).cpu().numpy())
        assert not np.any(g.channel(aw.MASS_DENSITY_X + a).cpu().numpy())
    assert not np.any(g.channel(aw.CELL_TYPE).cpu().numpy())
    g.g2p(dev(pos), dev(pos), 0.95)
    torch.cuda.synchronize()


def test_single_particle(grid):
    g, O = grid
    pos = np.array([[1.37, 0.61, 1.22]], np.float32)
    vel = np.array([[0.5, -1.0, 2.0]], np.float32)
    u, m, _ = check_p2g(g, O, pos, vel)
    assert sum(float(x.sum()) for x in m) > 0


@pytest.mark.parametrize("block", [(2, 0, 0), (3, 1, 1)])
def test_crowded_coarse_cell(grid, block):
    """40,000 particles inside one cell of a 2^3 block, or of a one-cell block: every particle of the
    block deposits on the same few faces."""
    g, O = grid
    rng = np.random.default_rng(11)
    lo = np.array(block, np.float64)
    pos = (lo + 0.05 + 0.4 * rng.random((40000, 3))).astype(np.float32)  # inside the first cell of the block
    vel = rng.standard_normal((40000, 3)).astype(np.float32)
    check_p2g(g, O, pos, vel)


@pytest.mark.parametrize("level", [0, 2])
def test_cell_beyond_the_slice_cap(level):
    """9,000,000 particles in one cell: more than 2^19 slices of 16 particles, so P2G lengthens its
    slices (to 18 particles) to keep the task count below 2^31.  The grid is uniform (8^3-cell blocks,
    or 2^3-cell blocks with per-warp tiles), so every face is summed by the own-particle pass from
    per-slice partial sums: each face adds some 10^5 FP32 partial sums, hence 1e-4 relative L2.
    (With another resolution within reach, each of the millions of particles would add its own weight
    to the neighbour's faces with a global FP32 atomic, and those sums stagnate once their spacing
    reaches the size of one weight.)"""
    g, O, _ = make([level] * 8, (2, 2, 2))
    rng = np.random.default_rng(12)
    n = 9_000_000
    h = 1.0 / (8 >> level)
    pos = (np.array([1.0, 1.0, 1.0]) + h * (0.1 + 0.8 * rng.random((n, 3)))).astype(np.float32)
    vel = rng.standard_normal((n, 3)).astype(np.float32)
    u, m, cnt = O.p2g(pos, vel)
    g.p2g(dev(pos), dev(vel))
    torch.cuda.synchronize()
    for a in range(3):
        assert rel_l2(g.channel(aw.MASS_DENSITY_X + a).cpu().numpy(), m[a]) < 1e-4
        assert rel_l2(g.channel(aw.VELOCITY_X + a).cpu().numpy(), u[a]) < 1e-4
    assert np.array_equal(g.channel(aw.CELL_TYPE).cpu().numpy().astype(np.int64), cnt.astype(np.int64))
    assert int(cnt.max()) == n
    g.close()


def test_boundary_positions(grid):
    """Particles exactly on cell faces, block faces and the domain's faces (including its far faces,
    which clamp into the last cell), sorted bit-exactly and transferred like the oracle's."""
    g, O = grid
    rng = np.random.default_rng(12)
    ticks = np.array([0.0, 0.125, 0.25, 0.5, 1.0, 1.5, 1.75, 2.0, 2.5, 3.0, 3.875, 4.0], np.float32)
    n = 6000
    pos = np.stack([rng.choice(ticks, n), rng.choice(ticks[ticks <= 2.0], n), rng.choice(ticks[ticks <= 2.0], n)], 1)
    vel = rng.standard_normal((n, 3)).astype(np.float32)
    keys_o, perm_o = O.particle_keys(pos)
    keys, perm = g.sort_particles(dev(pos))
    assert np.array_equal(perm.cpu().numpy().astype(np.int64), perm_o)
    assert np.array_equal(keys.cpu().numpy().view(np.uint32), keys_o[perm_o])
    check_p2g(g, O, pos, vel)
    # G2P from the resulting grid velocities, FLIP blend against the oracle's
    g.backup_grid_velocity()
    un = [g.channel(aw.VELOCITY_X + a).double().cpu().numpy() for a in range(3)]
    v_ref = O.g2p(pos, un, un, 0.95, vel)
    v = dev(vel)
    g.g2p(v, dev(pos), 0.95)
    torch.cuda.synchronize()
    assert rel_l2(v.cpu().numpy(), v_ref) < RTOL


def test_outside_domain_and_inactive_block():
    """Particles beyond the domain are clamped into its boundary blocks (worldToBlockCoord); a
    particle in an inactive block has no cell and deposits nothing of its own."""
    lv = [0, 0, 1, 4, 0, 0, 1, 1]  # 4 x 2 x 1 blocks, block 3 inactive (level >= L)
    g, O, lvg = make(lv, (4, 2, 1))
    assert lvg[3] >= 4
    rng = np.random.default_rng(13)
    inside = rng.random((3000, 3)) * np.array([4.0, 2.0, 1.0])
    outside = np.array([[-0.3, 0.5, 0.5], [4.2, 1.5, 0.5], [1.5, -0.01, 0.2], [2.5, 2.3, 1.4]])
    in_inactive = np.array([[3.5, 0.5, 0.5], [3.2, 0.2, 0.9]])
    pos = np.concatenate([inside, outside, in_inactive]).astype(np.float32)
    vel = rng.standard_normal(pos.shape).astype(np.float32)
    keys_o, perm_o = O.particle_keys(pos)
    keys, perm = g.sort_particles(dev(pos))
    assert np.array_equal(perm.cpu().numpy().astype(np.int64), perm_o)
    _, _, cnt = check_p2g(g, O, pos, vel)
    assert cnt.sum() < pos.shape[0]  # the inactive block's particles have no cell
    g.close()
