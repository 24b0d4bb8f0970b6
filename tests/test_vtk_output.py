"""Binary legacy-VTK writers (exportUniformPressure_VTK / exportParticles_VTK,
vtx_visualization.cuh:64-127,197-218, written as BINARY instead of ASCII): host code, no GPU."""
import os

import numpy as np
import pytest

import anitowave_adaptive_b200 as aw
from tests.vtk_read import read_vtk


def test_structured_points_scalars_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    a = rng.standard_normal((2, 3, 4)).astype(np.float32)  # (nz, ny, nx)
    p = tmp_path / "s.vtk"
    aw.vtk_write_structured_points(p, a, (0.5, 0.25, 0.125), (1.0, 0.5, 0.25), name="pressure")
    h, arr = read_vtk(p)
    assert h["encoding"] == "BINARY" and h["dataset"] == "STRUCTURED_POINTS"
    assert h["DIMENSIONS"] == [4, 3, 2] and h["POINT_DATA"] == 24
    assert h["ORIGIN"] == [0.5, 0.25, 0.125] and h["SPACING"] == [1.0, 0.5, 0.25]
    np.testing.assert_array_equal(arr["pressure"], a.reshape(-1))


def test_structured_points_vectors_round_trip(tmp_path):
    a = np.arange(5 * 1 * 3 * 3, dtype=np.float32).reshape(5, 1, 3, 3) - 7.5
    p = tmp_path / "v.vtk"
    aw.vtk_write_structured_points(p, a, (0, 0, 0), (1, 1, 1), name="velocity")
    h, arr = read_vtk(p)
    assert h["DIMENSIONS"] == [3, 1, 5]
    np.testing.assert_array_equal(arr["velocity"], a.reshape(-1, 3))


@pytest.mark.parametrize("with_scalar", [True, False])
def test_particles_round_trip(tmp_path, with_scalar):
    rng = np.random.default_rng(1)
    pos = rng.random((37, 3)).astype(np.float32)
    s = rng.random(37).astype(np.float32) if with_scalar else None
    p = tmp_path / "p.vtk"
    aw.vtk_write_particles(p, pos, s, name="speed")
    h, arr = read_vtk(p)
    assert h["dataset"] == "POLYDATA"
    np.testing.assert_array_equal(arr["POINTS"], pos)
    v = arr["VERTICES"].reshape(-1, 2)
    assert np.all(v[:, 0] == 1) and np.array_equal(v[:, 1], np.arange(37))
    if with_scalar:
        np.testing.assert_array_equal(arr["speed"], s)
    else:
        assert "speed" not in arr


def test_empty_particle_set(tmp_path):
    p = tmp_path / "e.vtk"
    aw.vtk_write_particles(p, np.zeros((0, 3), np.float32))
    h, arr = read_vtk(p)
    assert arr["POINTS"].shape == (0, 3)


def test_writer_errors_are_statuses(tmp_path):
    a = np.zeros((2, 2, 2), np.float32)
    with pytest.raises(aw.AWError) as e:
        aw.vtk_write_structured_points(tmp_path / "x.vtk", a, (0, 0, 0), (1, 1, 1), name="two words")
    assert e.value.status == 1
    with pytest.raises(aw.AWError) as e:
        aw.vtk_write_structured_points(os.path.join(str(tmp_path), "missing_dir", "x.vtk"), a, (0, 0, 0), (1, 1, 1))
    assert e.value.status == 8
    with pytest.raises(ValueError):
        aw.vtk_write_particles(tmp_path / "y.vtk", np.zeros((3, 3), np.float32), np.zeros(2, np.float32))
