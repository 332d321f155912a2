"""Mitosius frame-bin storage (bmMitosius_create.m / _load.m / _nCell.m):
cell folders named by 1-based column-major multi-index, round trips through
MAT v5 and .npy files, sub-mitosius edge selection and MATLAB's squeeze, and
the refusal of MAT v7.3 (HDF5) files with an explanation.
"""
import os

import numpy as np
import pytest

from monalisa_b200 import mitosius as M


def _cells(shape, seed=0):
    rng = np.random.default_rng(seed)
    c = np.empty(shape, dtype=object)
    for i in range(c.size):
        n = 5 + i
        c[np.unravel_index(i, shape, order="F")] = (rng.standard_normal((n, 2)) +
                                                    1j * rng.standard_normal((n, 2))).astype(np.complex64)
    return c


@pytest.mark.parametrize("fmt", ["mat", "npy"])
def test_round_trip_column_cell(tmp_path, fmt):
    y = [c for c in _cells((3, 1)).ravel()]
    t = [np.random.default_rng(i).standard_normal((2, yy.shape[0])) for i, yy in enumerate(y)]
    ve = [np.full(yy.shape[0], 0.5 + i, np.float32) for i, yy in enumerate(y)]
    d = str(tmp_path / "m")
    M.bmMitosius_create(d, y, t, ve, fmt=fmt)
    assert sorted(os.listdir(d))[:3] == ["cell_1_1", "cell_2_1", "cell_3_1"]
    assert M.bmMitosius_nCell(d) == 3
    out = M.bmMitosius_load(d, "y")
    assert out.shape == (3, 1)
    for a, b in zip(out.ravel(), y):
        assert np.array_equal(np.asarray(a), b)
    yy, tt, vv = M.load_frame_bins(d)
    for f in range(3):
        assert np.array_equal(yy[f], y[f]) and np.array_equal(tt[f], t[f]) and np.array_equal(vv[f], ve[f])


def test_multi_index_edges_and_squeeze(tmp_path):
    c = _cells((2, 3))
    d = str(tmp_path / "m2")
    M.bmMitosius_create(d, c)
    assert os.path.isdir(os.path.join(d, "cell_2_3")) and M.bmMitosius_nCell(d) == 6
    row = M.bmMitosius_load(d, "y", [2], "all")  # a 1 x 3 sub-mitosius stays 2-D
    assert row.shape == (1, 3)
    for j in range(3):
        assert np.array_equal(row[0, j], c[1, j])
    sub = M.bmMitosius_load(d, "y", [2, 1], [3])
    assert sub.shape == (2, 1) and np.array_equal(sub[0, 0], c[1, 2]) and np.array_equal(sub[1, 0], c[0, 2])
    with pytest.raises(ValueError):
        M.bmMitosius_load(d, "y", [1])  # one edge per dimension


def test_three_dimensional_cells_squeeze(tmp_path):
    c = _cells((2, 1, 3), seed=3)
    d = str(tmp_path / "m3")
    M.bmMitosius_create(d, c)
    assert os.path.isdir(os.path.join(d, "cell_2_1_3"))
    out = M.bmMitosius_load(d, "y")
    assert out.shape == (2, 3)  # the singleton middle dimension is squeezed out
    assert np.array_equal(out[1, 2], c[1, 0, 2])


def test_v73_files_are_refused(tmp_path):
    d = tmp_path / "m4"
    M.bmMitosius_create(str(d), [np.zeros((2, 1), np.complex64)])
    (d / "cell_1_1" / "y.mat").write_bytes(b"MATLAB 7.3 MAT-file, Platform: GLNXA64" + bytes(200))
    with pytest.raises(ValueError, match="v7.3"):
        M.bmMitosius_load(str(d), "y")
