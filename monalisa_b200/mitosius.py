"""Mitosius frame-bin storage (src/mitosius/bmMitosius_create.m,
bmMitosius_load.m, bmMitosius_nCell.m) and its ingest into the frame-bin
solvers.

A mitosius is a directory holding ``mitosius_size.mat`` (variable
``mitosius_size``, the size of the cell array) and one folder per cell,
``cell_i_j...`` with the cell's 1-based multi-index in column-major order
(bmIndex2MultiIndex.m), each with ``y.mat``, ``t.mat`` and ``ve.mat`` (one
variable each: k-space [nPt, nCh], trajectory [imDim, nPt], volume
elements [nPt]).

Files: the reference saves with ``-v7.3`` (HDF5).  This module reads and
writes MAT v5 / v7 through scipy (MATLAB reads and writes them natively,
``save(..., '-v7')``) and NumPy ``.npy`` files beside or instead of the
``.mat`` ones.  A v7.3 file is recognised by its header and rejected with
an error saying so: no HDF5 reader is part of this package's dependencies.
"""
from __future__ import annotations

import os

import numpy as np

_V73 = b"MATLAB 7.3"


def _multi_index(i: int, size) -> tuple:
    """bmIndex2MultiIndex.m: 1-based linear index -> 1-based multi-index,
    first index fastest."""
    return tuple(int(v) + 1 for v in np.unravel_index(i - 1, tuple(int(s) for s in size), order="F"))


def _cell_dir(mitosius_dir: str, idx: tuple) -> str:
    return os.path.join(mitosius_dir, "cell" + "".join(f"_{k}" for k in idx))


def _read_var(path_noext: str):
    """The single variable of <path>.mat (MAT v5/v7) or <path>.npy."""
    npy = path_noext + ".npy"
    if os.path.exists(npy):
        return np.load(npy, allow_pickle=False)
    mat = path_noext + ".mat"
    with open(mat, "rb") as f:
        head = f.read(len(_V73))
    if head == _V73:
        raise ValueError(f"{mat} is a MAT v7.3 (HDF5) file; re-save it with save(..., '-v7') or as .npy "
                         "(no HDF5 reader is available here)")
    import scipy.io

    d = scipy.io.loadmat(mat)
    names = [k for k in d if not k.startswith("__")]
    if len(names) != 1:
        raise ValueError(f"{mat} must hold one variable, found {names}")
    return d[names[0]]


def _write_var(path_noext: str, name: str, value, fmt: str):
    if fmt == "npy":
        np.save(path_noext + ".npy", np.asarray(value))
    else:
        import scipy.io

        scipy.io.savemat(path_noext + ".mat", {name: np.asarray(value)}, format="5")


def bmMitosius_create(mitosius_dir: str, y_cell=None, t_cell=None, ve_cell=None, mitosius_length=None,
                      fmt: str = "mat"):
    """bmMitosius_create.m: one folder per cell with y / t / ve.  The cell
    arrays may be lists (a column cell array [n, 1]) or object ndarrays whose
    shape is the cell array's size; with only mitosius_length the folders
    are made empty.  fmt 'mat' (MAT v5) or 'npy'."""
    def as_cells(c):
        if c is None:
            return None
        if isinstance(c, np.ndarray) and c.dtype == object:
            return c
        arr = np.empty((len(c), 1), dtype=object)
        for k, v in enumerate(c):
            arr[k, 0] = v
        return arr

    y_cell, t_cell, ve_cell = as_cells(y_cell), as_cells(t_cell), as_cells(ve_cell)
    ref = next((c for c in (y_cell, t_cell, ve_cell) if c is not None), None)
    if ref is not None:
        size = tuple(ref.shape) if ref.ndim >= 2 else (ref.shape[0], 1)
        length = int(np.prod(size))
    elif mitosius_length is not None:
        size, length = (int(mitosius_length), 1), int(mitosius_length)
    else:
        raise ValueError("give the cell arrays or mitosius_length")
    os.makedirs(mitosius_dir, exist_ok=True)
    for i in range(1, length + 1):
        idx = _multi_index(i, size)
        d = _cell_dir(mitosius_dir, idx)
        os.makedirs(d, exist_ok=True)
        for name, c in (("y", y_cell), ("t", t_cell), ("ve", ve_cell)):
            if c is not None:
                _write_var(os.path.join(d, name), name, c.reshape(-1, order="F")[i - 1], fmt)
    if ref is not None:
        _write_var(os.path.join(mitosius_dir, "mitosius_size"), "mitosius_size", np.asarray(size, np.float64), fmt)


def bmMitosius_nCell(mitosius_dir: str) -> int:
    """bmMitosius_nCell.m: the folders whose name begins with 'cell_'."""
    return sum(1 for e in os.listdir(mitosius_dir)
               if e.startswith("cell_") and os.path.isdir(os.path.join(mitosius_dir, e)))


def _matlab_squeeze(a: np.ndarray) -> np.ndarray:
    """MATLAB squeeze: arrays of two dimensions stay as they are; higher
    ones lose their singleton dimensions (down to two)."""
    if a.ndim <= 2:
        return a
    shape = [s for s in a.shape if s != 1]
    while len(shape) < 2:
        shape.append(1)
    return a.reshape(shape, order="F")


def bmMitosius_load(mitosius_dir: str, arg_name: str, *edges) -> np.ndarray:
    """bmMitosius_load.m: the cells' `arg_name` variables as an object
    array of the (sub-)mitosius size, column-major, MATLAB-squeezed.  Each
    edge (one per mitosius dimension) is 'all' or a list of 1-based
    indices."""
    size = [int(v) for v in np.ravel(_read_var(os.path.join(mitosius_dir, "mitosius_size")))]
    if edges and len(edges) != len(size):
        raise ValueError("The number of edges not compatible with mitosius_ndims. ")
    edge_list = []
    for k, n in enumerate(size):
        e = edges[k] if edges else "all"
        if isinstance(e, str):
            if e != "all":
                raise ValueError("Wrong input arguments. ")
            e = range(1, n + 1)
        edge_list.append([int(v) for v in np.ravel(e)])
    out_size = [len(e) for e in edge_list]
    n_out = int(np.prod(out_size))
    out = np.empty(n_out, dtype=object)
    for i in range(1, n_out + 1):
        o = _multi_index(i, out_size)
        idx = tuple(edge_list[j][o[j] - 1] for j in range(len(size)))
        out[i - 1] = _read_var(os.path.join(_cell_dir(mitosius_dir, idx), arg_name))
    return _matlab_squeeze(out.reshape(out_size, order="F"))


def load_frame_bins(mitosius_dir: str):
    """The cells' (y, t, ve) in linear (column-major) cell order, as lists:
    y [nPt, nCh] complex64, t [imDim, nPt] float64, ve [nPt] float32."""
    ys = bmMitosius_load(mitosius_dir, "y").reshape(-1, order="F")
    ts = bmMitosius_load(mitosius_dir, "t").reshape(-1, order="F")
    ves = bmMitosius_load(mitosius_dir, "ve").reshape(-1, order="F")
    y = [np.asarray(v, np.complex64).reshape(np.asarray(v).shape[0], -1) for v in ys]
    t = [np.asarray(v, np.float64) for v in ts]
    ve = [np.asarray(v, np.float32).ravel() for v in ves]
    return y, t, ve


def frame_bin_chain(mitosius_dir: str, C, n_u, N_u, dK_u, kernelType=None, nWin=None, kernelParam=None,
                    autotune=False):
    """Ingest into the temporal-TV path: loads every cell, builds each bin's
    Gu / Gut on the device (bmTraj2SparseMat) and returns
    (chain, y, ve) with chain a TevaMorphosiaChain over the bins in linear
    cell order (chain.run_host(y, ve, ...) runs bmTevaMorphosia_chain)."""
    from .solvers import TevaMorphosiaChain
    from .sparsemat import bmTraj2SparseMat

    y, t, ve = load_frame_bins(mitosius_dir)
    mats = [bmTraj2SparseMat(tt, vv, N_u, dK_u, kernelType, nWin, kernelParam) for tt, vv in zip(t, ve)]
    chain = TevaMorphosiaChain([m[0] for m in mats], [m[1] for m in mats], C, n_u, dK_u, autotune=autotune)
    return chain, y, ve
