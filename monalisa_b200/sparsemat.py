"""Sparse gridding matrices: the reference's ``bmSparseMat`` data class,
device-resident matrices, ``bmTraj2SparseMat`` on the GPU and
``bmSparseMat_vec``.

Reference: src/sparseMat/m/bmSparseMat.m (format, lines 15-47 and
cpp_prepare 100-188), src/gridding123/m/bmTraj2SparseMat.m (builder),
src/sparseMat/m/bmSparseMat_vec.m (product dispatch).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


def kernel_defaults(kernelType=None, nWin=None, kernelParam=None):
    """src/varargin/bmVarargin_kernelType_nWin_kernelParam.m:15-40."""
    if not kernelType:
        kernelType = "gauss"
    if kernelType not in ("gauss", "kaiser"):
        raise ValueError(f"unknown kernel type {kernelType!r}")
    if nWin is None:
        nWin = 3
    if kernelParam is None:
        kernelParam = [0.61, 10] if kernelType == "gauss" else [1.95, 10, 10]
    kp = np.asarray(np.ravel(kernelParam), np.float32).astype(np.float64)
    if kernelType == "gauss" and kp.size == 3:
        raise ValueError("Wrong list of gridding kernel parameters. ")
    if kernelType == "kaiser" and kp.size == 2:
        raise ValueError("Wrong list of gridding kernel parameters. ")
    return kernelType, int(np.float32(nWin)), kp


def kernel_code(kernelType: str) -> int:
    return N.MLG_KERNEL_GAUSS if kernelType == "gauss" else N.MLG_KERNEL_KAISER


@dataclass
class bmSparseMat:
    """A cpp_prepared 'one_block' jump-coded CSR (bmSparseMat.m:15-47):
    ``r_jump`` holds column deltas (first entry absolute, 0-based),
    ``r_nJump`` entries per stored row, ``l_jump`` row deltas of the stored
    rows when rows are squeezed (empty otherwise)."""

    r_size: int
    r_jump: np.ndarray
    r_nJump: np.ndarray
    m_val: np.ndarray
    l_size: int
    l_jump: np.ndarray
    l_nJump: int
    N_u: np.ndarray | None = None
    d_u: np.ndarray | None = None
    kernel_type: str = "void"
    nWin: int = 0
    kernelParam: np.ndarray | None = None
    block_type: str = "one_block"
    type: str = "cpp_prepared"
    extra: dict = field(default_factory=dict)

    @property
    def l_squeeze_flag(self) -> bool:
        return self.l_jump is not None and self.l_jump.size > 0

    def jump_arrays(self):
        c = lambda a, t: np.ascontiguousarray(np.ravel(a), t)
        lj = c(self.l_jump, np.int32) if self.l_squeeze_flag else None
        return (int(self.r_size), c(self.r_jump, np.int32), c(self.r_nJump, np.int32), c(self.m_val, np.float32),
                int(self.l_size), lj, int(self.l_nJump))

    def to_device(self) -> "DeviceMatrix":
        return DeviceMatrix.from_bm(self)

    def to_csr(self):
        """Standard CSR arrays (indptr int64 [l_size + 1], indices int32
        [nnz], data float32 [nnz]) of this [l_size, r_size] matrix: columns
        are the running sum of r_jump, stored rows the running sum of l_jump
        (or every row when rows are not squeezed), r_nJump entries each
        (bmSparseMat.m:100-188, bmSparseMat_r_nJump2index_mex.cpp:12-80)."""
        r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump = self.jump_arrays()
        cols = np.cumsum(r_jump.astype(np.int64))
        if cols.size and (cols.min() < 0 or cols.max() >= r_size):
            raise ValueError("column index outside the matrix")
        counts = np.zeros(l_size, np.int64)
        if l_jump is not None:
            rows = np.cumsum(l_jump.astype(np.int64))
            if rows.size and (rows.min() < 0 or rows.max() >= l_size):
                raise ValueError("row index outside the matrix")
            counts[rows] = r_nJump[:rows.size]
        else:
            counts[:] = r_nJump[:l_size]
        indptr = np.zeros(l_size + 1, np.int64)
        np.cumsum(counts, out=indptr[1:])
        if indptr[-1] != cols.size:
            raise ValueError("r_nJump does not add up to the number of entries")
        return indptr, cols.astype(np.int32), m_val.copy()


class DeviceMatrix:
    """A bmSparseMat resident in device memory (mlg_matrix_t)."""

    def __init__(self, handle, meta: dict, squeezed: bool):
        self._h = handle
        self.meta = meta
        self.squeezed = squeezed
        nnz, r, l = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
        N.call("mlg_matrix_info", self._h, ctypes.byref(nnz), ctypes.byref(r), ctypes.byref(l))
        self.nnz, self.r_size, self.l_size = nnz.value, r.value, l.value

    @property
    def handle(self):
        return self._h

    def row_stats(self):
        """(non-empty rows, rows longer than 256 entries)."""
        a, b = ctypes.c_int(), ctypes.c_int()
        N.call("mlg_matrix_row_stats", self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    @classmethod
    def from_bm(cls, G: bmSparseMat) -> "DeviceMatrix":
        r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump = G.jump_arrays()
        h = ctypes.c_void_p()
        nb = int(G.extra.get("nBlock", 0) or 0)
        if nb > 1:  # multi-block preparation
            N.call("mlg_matrix_create_blocks", r_size, N.iptr(r_jump), N.iptr(r_nJump), N.fptr(m_val), l_size,
                   N.iptr(l_jump), l_nJump, nb, N.iptr(np.ascontiguousarray(G.extra["block_length"], np.int32)),
                   N.iptr(np.ascontiguousarray(G.extra["l_block_start"], np.int32)),
                   N.llptr(np.ascontiguousarray(G.extra["m_block_start"], np.int64)), ctypes.byref(h))
        else:
            N.call("mlg_matrix_create", r_size, N.iptr(r_jump), N.iptr(r_nJump), N.fptr(m_val), l_size,
                   N.iptr(l_jump), l_nJump, ctypes.byref(h))
        meta = dict(N_u=G.N_u, d_u=G.d_u, kernel_type=G.kernel_type, nWin=G.nWin, kernelParam=G.kernelParam)
        return cls(h, meta, G.l_squeeze_flag)

    def download(self) -> bmSparseMat:
        r_jump = np.zeros(self.nnz, np.int32)
        r_nJump = np.zeros(self.l_size, np.int32)
        m_val = np.zeros(self.nnz, np.float32)
        l_jump = np.zeros(self.l_size, np.int32) if self.squeezed else None
        n = ctypes.c_int()
        N.call("mlg_matrix_download", self._h, N.iptr(r_jump), N.iptr(r_nJump), N.fptr(m_val),
               N.iptr(l_jump) if l_jump is not None else None, ctypes.byref(n))
        if self.squeezed:
            r_nJump, l_jump = r_nJump[:n.value].copy(), l_jump[:n.value].copy()
        return bmSparseMat(r_size=self.r_size, r_jump=r_jump, r_nJump=r_nJump, m_val=m_val, l_size=self.l_size,
                           l_jump=l_jump if l_jump is not None else np.zeros(0, np.int32),
                           l_nJump=n.value if self.squeezed else self.l_size,
                           type="l_squeezed_cpp_prepared" if self.squeezed else "cpp_prepared", **self.meta)

    def spmm(self, v, out=None):
        """w = M v for complex64 CUDA tensors in point layout [rows, nVec]."""
        import torch

        nVec = v.shape[1] if v.dim() == 2 else 1
        assert v.dtype == torch.complex64 and v.shape[0] == self.r_size
        if out is None:
            out = torch.empty((self.l_size, nVec), dtype=torch.complex64, device=v.device)
        N.call("mlg_matrix_spmm_dev", self._h, N.tptr(v.contiguous()), nVec, N.tptr(out), N.stream_ptr())
        return out

    def close(self):
        if self._h:
            N.lib().mlg_matrix_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bmTraj2SparseMat(t, v, N_u, dK_u, kernelType=None, nWin=None, kernelParam=None, nargout=2):
    """GPU form of src/gridding123/m/bmTraj2SparseMat.m: returns
    device-resident (Gu, Gut) (nargout 2), Gn (nargout 1) or (Gn, Gu, Gut)
    (nargout 3).  t [imDim, nPt] physical units, v volume elements (they
    cancel in the row-normalised Gu/Gut; Gn carries them, :245-256)."""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    t = np.asarray(t, np.float64)
    if t.ndim == 1:
        t = t[None, :]
    imDim, nPt = t.shape
    tt = np.ascontiguousarray(t.T)  # column-major [imDim, nPt]
    Nu = np.ascontiguousarray(np.ravel(N_u), np.int32)
    dK = np.ascontiguousarray(np.ravel(dK_u), np.float64)
    kp3 = np.zeros(3)
    kp3[:kp.size] = kp
    if nargout not in (1, 2, 3):
        raise ValueError("nargout must be 1, 2 or 3")
    want_n, want_u = nargout in (1, 3), nargout in (2, 3)
    ve = np.ascontiguousarray(np.ravel(v), np.float64) if want_n else None
    hn, hu, ht = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    N.call("mlg_traj2sparsemat3", imDim, nPt, N.dptr(tt), N.dptr(ve), N.iptr(Nu), N.dptr(dK),
           kernel_code(kernelType), nWin, N.dptr(kp3), ctypes.byref(hn) if want_n else None,
           ctypes.byref(hu) if want_u else None, ctypes.byref(ht) if want_u else None)
    meta = dict(N_u=Nu.copy(), d_u=dK.astype(np.float32), kernel_type=kernelType, nWin=nWin,
                kernelParam=kp.astype(np.float32))
    Gn = DeviceMatrix(hn, meta, True) if want_n else None
    if nargout == 1:
        return Gn
    Gu, Gut = DeviceMatrix(hu, meta, False), DeviceMatrix(ht, meta, True)
    return (Gn, Gu, Gut) if nargout == 3 else (Gu, Gut)


def bmImDeformField2SparseMat(v, N_u, Dn=None, torus_flag=False, nargout=2):
    """GPU form of src/gridding123/m/bmImDeformField2SparseMat.m for one
    displacement field v [imDim, prod(N_u)] (pixel units): device-resident
    (Tu, Tut) (nargout 2), Gn (nargout 1, needs Dn) or (Gn, Tu, Tut)
    (nargout 3).  Each pixel's row holds bump weights on the 2^imDim cells
    around its displaced position, normalised to sum 1; pixels displaced
    outside the image keep empty rows unless torus_flag."""
    v = np.asarray(v, np.float64)
    if v.ndim == 1:
        v = v[None, :]
    N_u = np.ascontiguousarray(np.ravel(N_u), np.int32)
    imDim = N_u.size
    v = v.reshape(imDim, -1, order="F")
    if v.shape[1] != int(np.prod(N_u)):
        raise ValueError("the deformation field must have as many vectors as the number of pixels in the image")
    if nargout not in (1, 2, 3):
        raise ValueError("nargout must be 1, 2 or 3")
    want_n, want_u = nargout in (1, 3), nargout in (2, 3)
    if want_n and Dn is None:
        raise ValueError("Gn needs Dn")
    vv = np.ascontiguousarray(v.T)  # column-major [imDim, nPt]
    dn = np.ascontiguousarray(np.ravel(Dn), np.float64) if want_n else None
    hn, hu, ht = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    N.call("mlg_deform2sparsemat", imDim, N.iptr(N_u), N.dptr(vv), N.dptr(dn), int(bool(torus_flag)),
           ctypes.byref(hn) if want_n else None, ctypes.byref(hu) if want_u else None,
           ctypes.byref(ht) if want_u else None)
    meta = dict(N_u=N_u.copy(), d_u=np.ones(imDim, np.float32), kernel_type="bump", nWin=2,
                kernelParam=np.zeros(0, np.float32))
    Gn = DeviceMatrix(hn, meta, False) if want_n else None
    if nargout == 1:
        return Gn
    Tu, Tut = DeviceMatrix(hu, meta, False), DeviceMatrix(ht, meta, False)
    return (Gn, Tu, Tut) if nargout == 3 else (Tu, Tut)


def bmSparseMat_vec(G: bmSparseMat, v, layout: str = "column"):
    """bmSparseMat_vec (src/sparseMat/m/bmSparseMat_vec.m:11-243) for a
    cpp_prepared matrix, one block or multi-block (G.extra['nBlock'],
    'block_length', 'l_block_start', 'm_block_start'): complex or real v.

    layout 'column': v [r_size, nVec] -> w [l_size, nVec] (the cC / rC MEX);
    layout 'row': v [nVec, r_size] -> w [nVec, l_size] (the cR / rR MEX)."""
    r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump = G.jump_arrays()
    nb = int(G.extra.get("nBlock", 0) or 0)
    if nb > 1:
        bl = np.ascontiguousarray(G.extra["block_length"], np.int32)
        ls = np.ascontiguousarray(G.extra["l_block_start"], np.int32)
        ms = np.ascontiguousarray(G.extra["m_block_start"], np.int64)
    else:
        nb, bl, ls, ms = 0, None, None, None
    v = np.asarray(v)
    if v.ndim == 1:
        v = v[:, None] if layout == "column" else v[None, :]
    cplx = np.iscomplexobj(v)
    if layout == "column":
        nVec = v.shape[1]
        code = N.MLG_LAYOUT_CC if cplx else N.MLG_LAYOUT_RC
        vR = np.ascontiguousarray(np.real(v).T, np.float32)  # [nVec][r_size]: column layout
        vI = np.ascontiguousarray(np.imag(v).T, np.float32) if cplx else None
        wR = np.zeros((nVec, l_size), np.float32)
        wI = np.zeros((nVec, l_size), np.float32) if cplx else None
    else:
        nVec = v.shape[0]
        code = N.MLG_LAYOUT_CR if cplx else N.MLG_LAYOUT_RR
        # column-major [nVec, r_size] == C-order [r_size][nVec]
        vR = np.ascontiguousarray(np.real(v).T, np.float32)
        vI = np.ascontiguousarray(np.imag(v).T, np.float32) if cplx else None
        wR = np.zeros((l_size, nVec), np.float32)
        wI = np.zeros((l_size, nVec), np.float32) if cplx else None
    N.call("mlg_sparsemat_vec", code, r_size, N.iptr(r_jump), N.iptr(r_nJump), N.fptr(m_val), l_size,
           N.iptr(l_jump), l_nJump, nb, N.iptr(bl), N.iptr(ls), N.llptr(ms), N.fptr(vR), N.fptr(vI), nVec,
           N.fptr(wR), N.fptr(wI))
    w = (wR + 1j * wI) if cplx else wR
    return w.T.astype(np.complex64 if cplx else np.float32)
