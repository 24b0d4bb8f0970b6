"""Dense resampling for inspection (sampleMSBG, vtx_visualization.cuh:8-62) and the block VTK
writer (exportMultigrid_VTK, :129-195) against the oracle's lookups.

The lattice points are computed here in float32 with the library's rule
domain_min + (i + 0.5) * spacing; the cell lookup is then bit-exact (same keys as the oracle's
particle sort), the velocity within FP32 rounding of the oracle's FP64 MAC sample.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import anitowave_adaptive_b200 as aw  # noqa: E402
from anitowave_adaptive_b200 import scenes  # noqa: E402
from oracle import pyoracle as po  # noqa: E402
from tests.vtk_read import read_vtk  # noqa: E402

pytestmark = pytest.mark.gpu


def lattice_points(g, dims):
    origin, sp = g.resample_lattice(dims)
    sp = np.asarray(sp, np.float32)
    ii = [np.arange(d, dtype=np.float32) for d in dims]
    z, y, x = np.meshgrid(ii[2], ii[1], ii[0], indexing="ij")
    half = np.float32(0.5)
    pts = np.stack([(x + half) * sp[0], (y + half) * sp[1], (z + half) * sp[2]], -1).reshape(-1, 3)
    return pts, np.asarray(origin, np.float32), sp


@pytest.fixture(scope="module")
def setup():
    S = scenes.config("dam_break_64")
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    g = aw.build_grid(S)
    return S, O, g


@pytest.mark.parametrize("dims", [(64, 64, 64), (37, 5, 101), (1, 1, 1)])
def test_resample_cells_bit_exact(setup, dims):
    S, O, g = setup
    pos = torch.as_tensor(S.pos, device="cuda")
    g.p2g(pos, torch.as_tensor(S.vel, device="cuda"))  # CELL_TYPE = particles per cell
    out = g.resample_cells(aw.CELL_TYPE, dims).cpu().numpy().reshape(-1)
    pts, origin, sp = lattice_points(g, dims)
    pts += np.asarray(S.domain_min, np.float32)
    np.testing.assert_array_equal(origin, pts[0])
    keys, _ = O.particle_keys(pts)
    ch = g.channel(aw.CELL_TYPE).cpu().numpy()
    ref = np.where(keys == 0xFFFFFFFF, 0.0, ch[np.minimum(keys, ch.size - 1)]).astype(np.float32)
    np.testing.assert_array_equal(out, ref)
    assert out.sum() > 0 or dims == (1, 1, 1)


def test_resample_velocity_matches_oracle_sample(setup):
    S, O, g = setup
    rng = np.random.default_rng(4)
    u = []
    for a in range(3):
        ch = g.channel(aw.VELOCITY_X + a)
        v = rng.standard_normal(ch.numel()).astype(np.float32)
        ch.copy_(torch.as_tensor(v, device="cuda"))
        u.append(v.astype(np.float64))
    dims = (48, 40, 33)
    out = g.resample_velocity(dims).cpu().numpy().reshape(-1, 3)
    pts, _, _ = lattice_points(g, dims)
    pts += np.asarray(S.domain_min, np.float32)
    ref = O.sample(pts.astype(np.float64), u)
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err < 1e-6, err


def test_flip_step_leaves_its_pressure(setup):
    S, O, g = setup
    xo, vo, perm, d = po.flip_step(O, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), tol=1e-12)
    F = aw.Flip(g, S.pos, S.vel, S.dt, 0.95, (0, S.gravity, 0), precision=aw.PRECISION_MIXED, tolerance=1e-10,
                max_cycles=60)
    F.step()
    p = g.channel(aw.PRESSURE).cpu().numpy().astype(np.float64)
    ref = d["p"] * d["fluid"]
    assert np.linalg.norm(p - ref) / np.linalg.norm(ref) < 1e-5
    assert np.all(p[d["fluid"] == 0] == 0)
    dense = g.resample_cells(aw.PRESSURE, (64, 64, 64)).cpu().numpy()
    assert dense.max() > 0
    F.close()


def test_vtk_blocks_and_dense_field_files(setup, tmp_path):
    S, O, g = setup
    g.vtk_write_blocks(tmp_path / "blocks.vtk")
    h, arr = read_vtk(tmp_path / "blocks.vtk")
    nb = int(np.prod(S.dims))
    assert h["dataset"] == "UNSTRUCTURED_GRID" and arr["CELL_TYPES"].size == nb and np.all(arr["CELL_TYPES"] == 12)
    lv = g.refinement_map().astype(np.int64)
    np.testing.assert_array_equal(arr["refineLevel"], np.where(lv < S.num_levels, lv, -1))
    # block b's first corner is domain_min + its coordinate * block size
    b = nb - 1
    c = np.array([b % S.dims[0], (b // S.dims[0]) % S.dims[1], b // (S.dims[0] * S.dims[1])], np.float32)
    np.testing.assert_allclose(arr["POINTS"][8 * b], np.asarray(S.domain_min, np.float32) + c * S.block_size)
    dims = (16, 16, 16)
    field = g.resample_cells(aw.CELL_TYPE, dims).cpu().numpy()
    origin, sp = g.resample_lattice(dims)
    aw.vtk_write_structured_points(tmp_path / "cells.vtk", field, origin, sp, name="count")
    h, arr = read_vtk(tmp_path / "cells.vtk")
    np.testing.assert_array_equal(arr["count"], field.reshape(-1))


def test_resample_rejects_bad_arguments(setup):
    S, O, g = setup
    with pytest.raises(aw.AWError):
        g.resample_cells(aw.VELOCITY_X, (4, 4, 4))
    with pytest.raises(aw.AWError):
        g.resample_cells(aw.PRESSURE, (0, 4, 4))


def test_resample_honours_domain_min():
    """sampleMSBG places lattice points from the origin 0 and ignores domain_min; the library
    offsets the lattice by domain_min (corrected)."""
    import dataclasses
    S0 = scenes.config("dam_break_32")
    shift = np.array([0.25, -0.5, 1.0], np.float32)
    S = dataclasses.replace(S0, domain_min=tuple(float(x) for x in shift), pos=(S0.pos + shift).astype(np.float32))
    lv = po.levels_from_particles(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, S.pos, S.thresholds)
    lv, _ = po.enforce_grading(S.dims, S.num_levels, lv)
    O = po.Oracle(S.dims, S.block_size, S.domain_min, S.base_res, S.num_levels, lv)
    g = aw.build_grid(S)
    g.p2g(torch.as_tensor(S.pos, device="cuda"), torch.as_tensor(S.vel, device="cuda"))
    dims = (40, 24, 32)
    out = g.resample_cells(aw.CELL_TYPE, dims).cpu().numpy().reshape(-1)
    pts, origin, sp = lattice_points(g, dims)
    pts += shift
    np.testing.assert_array_equal(origin, pts[0])
    keys, _ = O.particle_keys(pts)
    ch = g.channel(aw.CELL_TYPE).cpu().numpy()
    ref = np.where(keys == 0xFFFFFFFF, 0.0, ch[np.minimum(keys, ch.size - 1)]).astype(np.float32)
    np.testing.assert_array_equal(out, ref)
    assert out.sum() > 0
    g.close()
