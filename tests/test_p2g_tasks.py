"""Index arithmetic of P2G's own-particle tasks (`k_p2g_own` in anitowave_adaptive_b200/csrc/
aw_particles.cu), restated in numpy and checked on the CPU: for every kind of task, each particle of
each cell falls in exactly one (cell, slice) task; the task count stays below 2^31 and the slice
offsets below 2^32, up to the largest cell counts the uint32 cell starts can hold.

The restatement follows the kernel line for line:
    mc = max particles in one of the block's r^3 cells
    nsl = min(ceil(mc / P2G_SLICE), P2G_MAX_SLICES);  slice = ceil(mc / nsl)
    ntask = NK * r^3 * nsl  (NK = 3, or 6 with phases)
    task -> kind = task // (r^3 nsl), c = rem % r^3, sl = rem // r^3
    skip when sl * slice >= count[c]; else particles [sl * slice, min(count[c], (sl + 1) * slice))
"""
import numpy as np
import pytest

P2G_SLICE = 16
P2G_MAX_SLICES = 1 << 19
INT32_MAX = 2**31 - 1


def plan(mc):
    nsl = min(-(-mc // P2G_SLICE), P2G_MAX_SLICES)
    slice_ = -(-mc // nsl) if nsl else 0
    return nsl, slice_


def coverage(counts, nk):
    """Per kind, how many tasks cover each particle of each cell (must be exactly 1)."""
    counts = np.asarray(counts, np.int64)
    nc3 = counts.size
    nsl, slice_ = plan(int(counts.max()))
    ntask = nk * nc3 * nsl
    task = np.arange(ntask, dtype=np.int64)
    kind = task // (nc3 * nsl)
    rem = task - kind * nc3 * nsl
    c, sl = rem % nc3, rem // nc3
    lo = sl * slice_
    live = lo < counts[c]
    hi = np.minimum(counts[c], lo + slice_)
    cover = []
    for k in range(nk):
        sel = live & (kind == k)
        hits = np.zeros(int(counts.sum()) + 1, np.int64)
        base = np.concatenate([[0], np.cumsum(counts)])[c[sel]]
        np.add.at(hits, base + lo[sel], 1)
        np.add.at(hits, base + hi[sel], -1)
        cover.append(np.cumsum(hits)[:-1])
    return cover, ntask, nsl, slice_


@pytest.mark.parametrize("r", [1, 2, 4, 8])
@pytest.mark.parametrize("nk", [3, 6])
def test_every_particle_in_exactly_one_task(r, nk):
    rng = np.random.default_rng(r * 10 + nk)
    for counts in (rng.integers(0, 40, r**3), rng.poisson(8, r**3), np.zeros(r**3, np.int64) + 16,
                   np.r_[np.zeros(r**3 - 1, np.int64), 1000]):
        if counts.max() == 0:
            continue
        cover, ntask, nsl, slice_ = coverage(counts, nk)
        assert ntask <= INT32_MAX
        for cv in cover:
            assert np.all(cv == 1)


@pytest.mark.parametrize("r", [1, 2])
def test_slices_lengthen_past_the_cap(r):
    """9,000,000 particles in one cell: 2^19 slices of 18 particles."""
    counts = np.zeros(r**3, np.int64)
    counts[-1] = 9_000_000
    cover, ntask, nsl, slice_ = coverage(counts, 6)
    assert (nsl, slice_) == (P2G_MAX_SLICES, 18)
    assert ntask <= INT32_MAX
    for cv in cover:
        assert np.all(cv == 1)


def test_bounds_at_the_largest_counts():
    """The largest block (8^3 cells) with phases, and cells up to the uint32 limit of the starts."""
    for mc in (1, 16, 17, P2G_SLICE * P2G_MAX_SLICES, P2G_SLICE * P2G_MAX_SLICES + 1, 2**31, 2**32 - 1):
        nsl, slice_ = plan(mc)
        assert 6 * 8**3 * nsl <= INT32_MAX
        assert nsl * slice_ >= mc                  # the slices cover the fullest cell
        assert (nsl - 1) * slice_ < 2**32          # sl * slice fits the kernel's uint32
        # slices that start past a cell's count are skipped before any index is formed, and
        # i0 + slice is only taken when it stays below the cell's end
