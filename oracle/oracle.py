"""ORACLE -- test infrastructure, not product code.

CPU restatement of the Monalisa reference's gridding hot path, used only as
the checker by ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg.  Nothing in ``monalisa_b200`` imports it.

Two layers:

* the native kernels: either the reference's own C++ MEX files compiled from
  source against the project's MEX-API shim (``oracle/_ref``, built by
  ``make -C oracle ref``) or the plain-C restatement
  (``oracle/_lib/liboracle.so``, ``make -C oracle port``).  The restatement is
  pinned bit-for-bit against the compiled reference by
  ``tests/test_oracle_pinning.py`` and against the committed golden fixtures
  (``tests/golden``, produced by the compiled reference kernels);
* the MATLAB layers, restated in numpy/scipy line by line from the cited
  ``.m`` files.  MATLAB itself is not available, so its built-ins are replaced
  by stand-ins: ``fft``/``ifft`` -> ``scipy.fft`` (pocketfft), ``sparse`` ->
  ``scipy.sparse`` (duplicates summed, zeros dropped), ``besseli(0, .)`` ->
  ``scipy.special.i0``, ``normpdf`` -> its defining formula.  At the MATLAB
  boundary parity is therefore pinned only through these stand-ins.

Conventions: MATLAB column-major data are held as numpy arrays indexed in
MATLAB order; "column" vectors of images are Fortran-order flattenings.
k-space data are ``[nPt, nCh]`` (MATLAB column layout).
"""
from __future__ import annotations

import ctypes
import os
import sys
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft
import scipy.sparse as sp
import scipy.special as sspec

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(ORACLE_DIR)
REF_DIR = os.path.join(ORACLE_DIR, "_ref")
LIB_PATH = os.path.join(ORACLE_DIR, "_lib", "liboracle.so")

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int)


# --------------------------------------------------------------------------
# compiled checkers
# --------------------------------------------------------------------------
def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "bmSparseMat_cC_oBlock_omp_mex.so"))


def ref_mex(name: str):
    """The reference's own MEX kernel ``name`` compiled against the shim."""
    if REPO_DIR not in sys.path:
        sys.path.insert(0, REPO_DIR)
    from monalisa_b200.mexcall import MexFunction

    return MexFunction(os.path.join(REF_DIR, name + ".so"))


_port = None


def port():
    """ctypes handle on the plain-C restatement (liboracle.so)."""
    global _port
    if _port is None:
        lib = ctypes.CDLL(LIB_PATH)
        lib.oracle_gridder_leight.argtypes = [ctypes.c_int] + [_f32p] * 6 + [ctypes.c_int] * 6 + \
            [ctypes.c_float, ctypes.c_float, _f32p, _f32p]
        lib.oracle_gridder_n2u.argtypes = [_f32p, _f32p, _f32p, _i32p] + [ctypes.c_int] * 4 + [_f32p, _f32p]
        for n in ("oracle_spmv_cC", "oracle_spmv_cR"):
            getattr(lib, n).argtypes = [ctypes.c_int, _i32p, _i32p, _f32p, ctypes.c_int, _i32p,
                                        ctypes.c_int, _f32p, _f32p, ctypes.c_int, _f32p, _f32p]
        lib.oracle_spmv_rC.argtypes = [ctypes.c_int, _i32p, _i32p, _f32p, ctypes.c_int, _i32p,
                                       ctypes.c_int, _f32p, ctypes.c_int, _f32p]
        lib.oracle_r_nJump2index.argtypes = [_i32p, ctypes.c_int, _i32p]
        lib.oracle_r_nJump2index.restype = ctypes.c_longlong
        _port = lib
    return _port


def _fp(a):
    return a.ctypes.data_as(_f32p) if a is not None and a.size else None


def _ip(a):
    return a.ctypes.data_as(_i32p) if a is not None and a.size else None


def port_gridder_leight(imDim, aReal, aImag, tx, ty, tz, Dn, nCh, nPt, Nx, Ny, Nz, nWin, kp1, kp2):
    """Restated bmGridder_n2u_leight{1,2,3}_mex (split [nCh,nPt] -> [nCh,Nu])."""
    nu = int(Nx) * (int(Ny) if imDim > 1 else 1) * (int(Nz) if imDim > 2 else 1)
    bR = np.zeros(nu * nCh, np.float32)
    bI = np.zeros(nu * nCh, np.float32)
    c = lambda a: None if a is None else np.ascontiguousarray(a, np.float32).ravel(order="F")
    aR, aI, x, y, z, d = c(aReal), c(aImag), c(tx), c(ty), c(tz), c(Dn)
    port().oracle_gridder_leight(imDim, _fp(aR), _fp(aI), _fp(x), _fp(y), _fp(z), _fp(d), nCh, nPt,
                                 int(Nx), int(Ny or 1), int(Nz or 1), int(nWin), float(kp1), float(kp2),
                                 _fp(bR), _fp(bI))
    return bR.reshape(nCh, nu, order="F"), bI.reshape(nCh, nu, order="F")


def port_gridder_n2u(aReal, aImag, w, nJump, nCh, nNb, nPt, Nu_tot):
    bR = np.zeros(Nu_tot * nCh, np.float32)
    bI = np.zeros(Nu_tot * nCh, np.float32)
    aR = np.asfortranarray(aReal, np.float32).ravel(order="F")
    aI = np.asfortranarray(aImag, np.float32).ravel(order="F")
    w = np.ascontiguousarray(w, np.float32).ravel()
    nJ = np.ascontiguousarray(nJump, np.int32).ravel()
    port().oracle_gridder_n2u(_fp(aR), _fp(aI), _fp(w), _ip(nJ), nNb, nCh, nPt, Nu_tot, _fp(bR), _fp(bI))
    return bR.reshape(nCh, Nu_tot, order="F"), bI.reshape(nCh, Nu_tot, order="F")


def port_spmv(G: "SparseMat", v: np.ndarray, layout: str = "C") -> np.ndarray:
    """Restated bmSparseMat_c{C,R}_oBlock: complex v -> complex w.

    layout "C": v [r_size, nVec] -> w [l_size, nVec]; "R": v [nVec, r_size] ->
    w [nVec, l_size].
    """
    v = np.asarray(v)
    if v.ndim == 1:
        v = v[:, None] if layout == "C" else v[None, :]
    nVec = v.shape[1] if layout == "C" else v.shape[0]
    vR = np.asfortranarray(v.real, np.float32).ravel(order="F")
    vI = np.asfortranarray(v.imag, np.float32).ravel(order="F")
    n = int(G.l_size) * nVec
    wR = np.zeros(n, np.float32)
    wI = np.zeros(n, np.float32)
    fn = port().oracle_spmv_cC if layout == "C" else port().oracle_spmv_cR
    fn(int(G.r_size), _ip(G.r_jump), _ip(G.r_nJump), _fp(G.m_val), int(G.l_size),
       _ip(G.l_jump) if G.l_jump is not None and G.l_jump.size else None, int(G.l_nJump),
       _fp(vR), _fp(vI), nVec, _fp(wR), _fp(wI))
    shape = (int(G.l_size), nVec) if layout == "C" else (nVec, int(G.l_size))
    return (wR + 1j * wI).astype(np.complex64).reshape(shape, order="F")


# --------------------------------------------------------------------------
# kernel parameters and window geometry
# --------------------------------------------------------------------------
def single(x):
    """MATLAB's double(single(x))."""
    return np.asarray(x, np.float64).astype(np.float32).astype(np.float64)


def kernel_defaults(kernelType=None, nWin=None, kernelParam=None):
    """bmVarargin_kernelType_nWin_kernelParam.m:15-40."""
    if not kernelType:
        kernelType = "gauss"
    if nWin is None:
        nWin = 3
    if kernelParam is None:
        kernelParam = [0.61, 10] if kernelType == "gauss" else [1.95, 10, 10]
    kp = single(np.ravel(kernelParam))
    if kernelType == "gauss" and kp.size == 3:
        raise ValueError("Wrong list of gridding kernel parameters. ")
    if kernelType == "kaiser" and kp.size == 2:
        raise ValueError("Wrong list of gridding kernel parameters. ")
    return kernelType, float(single(nWin)), kp


def normpdf(d, sigma):
    """MATLAB normpdf(d, 0, sigma) by its definition."""
    return np.exp(-0.5 * (d / sigma) ** 2) / (np.sqrt(2 * np.pi) * sigma)


def kernel_weight(d, kernelType, kp):
    """bmTraj2SparseMat.m:191-204 / bmK.m:70-83 (no cutoff, KB floor 1/I0(a))."""
    if kernelType == "gauss":
        return normpdf(d, kp[0])
    tau, alpha = kp[0], kp[1]
    w = np.maximum(1 - (d / tau) ** 2, 0)
    w = alpha * np.sqrt(w)
    return sspec.i0(w) / sspec.i0(alpha)


def window_offsets(imDim: int, nWin: int):
    """Offsets c [imDim, nNb] in MATLAB ndgrid order (x fastest) and the
    floor shift (bmTraj2SparseMat.m:134-164)."""
    nWin = int(nWin)
    if nWin % 2 == 0:
        rng = np.arange(-nWin // 2 - 1, nWin // 2 + 1)
        shift = 0.0
    else:
        h = nWin // 2
        rng = np.arange(-h, h + 1)
        shift = 0.5
    grids = np.meshgrid(*([rng] * imDim), indexing="ij")
    c = np.stack([g.ravel(order="F") for g in grids], 0).astype(np.float64)
    return c, shift


def to_grid_units(t, Dn, N_u, dK_u):
    """t/dK_u + fix(N/2+1) and Dn/prod(dK_u); out-of-grid mask
    (bmTraj2SparseMat.m:81-126, bmGridder_n2u_leight.m:40-81)."""
    t = np.array(t, np.float64, copy=True)
    imDim = t.shape[0]
    Dn = None if Dn is None else np.array(Dn, np.float64).ravel()
    mask = np.zeros(t.shape[1], bool)
    for i in range(imDim):
        t[i] = t[i] / dK_u[i]
        if Dn is not None:
            Dn = Dn / dK_u[i]
        t[i] = t[i] + np.fix(N_u[i] / 2 + 1)
    for i in range(imDim):
        mask |= (t[i] < 1) | (t[i] > N_u[i])
    return t, Dn, mask


# --------------------------------------------------------------------------
# bmSparseMat (jump-coded CSR)
# --------------------------------------------------------------------------
@dataclass
class SparseMat:
    r_size: int
    l_size: int
    r_nJump: np.ndarray
    m_val: np.ndarray
    r_jump: np.ndarray | None = None
    l_jump: np.ndarray | None = None
    l_nJump: int = 0
    r_ind: np.ndarray | None = None  # 1-based, before cpp_prepare
    l_ind: np.ndarray | None = None
    N_u: np.ndarray | None = None
    d_u: np.ndarray | None = None
    kernel_type: str = "void"
    nWin: int = 0
    kernelParam: np.ndarray | None = None
    type: str = "void"
    block_type: str = "void"
    extra: dict = field(default_factory=dict)

    def to_scipy(self) -> sp.csr_matrix:
        """Decodes the jump format into a scipy CSR [l_size, r_size]; running
        sums restart at every block's first entry / first stored row."""
        def seg_cumsum(jump, starts):
            out = np.empty(jump.size, np.int64)
            bounds = list(np.ravel(starts).astype(np.int64)) + [jump.size]
            for s, e in zip(bounds[:-1], bounds[1:]):
                out[s:e] = np.cumsum(jump[s:e].astype(np.int64))
            return out

        m_starts = self.extra.get("m_block_start", [0])
        l_starts = self.extra.get("l_block_start", [0])
        cols = seg_cumsum(self.r_jump, m_starts)
        if self.l_jump is not None and self.l_jump.size:
            rows_nz = seg_cumsum(self.l_jump, l_starts)
        else:
            rows_nz = np.arange(self.l_size)
        rows = np.repeat(rows_nz, self.r_nJump.astype(np.int64))
        return sp.csr_matrix((self.m_val.astype(np.float32), (rows, cols)),
                             shape=(int(self.l_size), int(self.r_size)))


def matlab_sparse_to_bm(a: sp.spmatrix, N_u, d_u, kernelType, nWin, kernelParam) -> SparseMat:
    """bmSparseMat_matlabSparse2bmSparseMat.m:6-40: row-major nnz, columns
    ascending within a row, 1-based r_ind."""
    a = sp.csr_matrix(a)
    a.sort_indices()
    return SparseMat(r_size=a.shape[1], l_size=a.shape[0], l_nJump=a.shape[0],
                     r_nJump=np.diff(a.indptr).astype(np.int32),
                     r_ind=(a.indices + 1).astype(np.int32),
                     m_val=a.data.astype(np.float32),
                     N_u=np.asarray(N_u, np.int32), d_u=np.asarray(d_u, np.float32),
                     kernel_type=kernelType, nWin=int(nWin),
                     kernelParam=np.asarray(kernelParam, np.float32), type="matlab_ind")


def l_squeeze(G: SparseMat) -> SparseMat:
    """bmSparseMat.m:62-94: drop empty rows, remember their 1-based indices."""
    keep = G.r_nJump != 0
    G.r_nJump = G.r_nJump[keep].astype(np.int32)
    G.l_ind = (np.nonzero(keep)[0] + 1).astype(np.int32)
    G.l_nJump = int(G.l_ind.size)
    G.type = "l_squeezed_matlab_ind"
    return G


def block_partition(r_nJump, nJumpPerBlock_factor=None, blockLengthMax_factor=None, one=False):
    """bmSparseMat_blockPartition.m:6-181: greedy blocks of consecutive stored
    rows; a block grows while its entry count stays below
    fix(f1 * max(r_nJump)) + 1 and its length below fix(f2 * max(r_nJump)).
    Returns (l_block_start, block_length) as int32 arrays."""
    r_nJump = np.ravel(r_nJump).astype(np.int64)
    if r_nJump.sum() <= 0:
        raise ValueError("The sparse matrix got a zero block. Preparation aborted.")
    if one:
        return np.zeros(1, np.int32), np.array([r_nJump.size], np.int32)
    l_nJump = r_nJump.size
    mx = int(r_nJump.max())
    per_block = int(np.fix(nJumpPerBlock_factor * mx)) + 1
    len_max = int(np.fix(blockLengthMax_factor * mx))
    starts, lengths = [], []
    start = 0
    while start < l_nJump:
        length, nxt = 1, start + 1
        if nxt < l_nJump:
            acc = int(r_nJump[start])
            while nxt < l_nJump:
                acc += int(r_nJump[nxt])
                if acc < per_block and length < len_max:
                    length += 1
                    nxt += 1
                else:
                    break
        starts.append(start)
        lengths.append(length)
        start += length
    return np.array(starts, np.int32), np.array(lengths, np.int32)


def cpp_prepare(G: SparseMat, argMode="one_block", nJumpPerBlock_factor=None, blockLengthMax_factor=None) -> SparseMat:
    """bmSparseMat.m:100-188: r_jump = deltas of r_ind and l_jump = deltas of
    l_ind, except that the first entry and the first stored row of every
    block are absolute 0-based (:135-168); m_block_start = entries before
    each block (int64)."""
    if argMode == "one_block":
        l_block_start, block_length = block_partition(G.r_nJump, one=True)
    elif argMode == "multi_block":
        l_block_start, block_length = block_partition(G.r_nJump, nJumpPerBlock_factor, blockLengthMax_factor)
    else:
        raise ValueError("Wrong list of arguments. ")
    r_ind = G.r_ind.astype(np.int64)
    r_jump = np.diff(np.concatenate([[0], r_ind]))
    csum = np.concatenate([[0], np.cumsum(G.r_nJump.astype(np.int64))])
    m_block_start = csum[l_block_start.astype(np.int64)].astype(np.int64)
    for m in m_block_start:
        r_jump[m] = r_ind[m] - 1
    G.r_jump = r_jump.astype(np.int32)
    if G.type == "l_squeezed_matlab_ind":
        l_ind = G.l_ind.astype(np.int64)
        l_jump = np.diff(np.concatenate([[0], l_ind]))
        for s in l_block_start:
            l_jump[s] = l_ind[s] - 1
        G.l_jump = l_jump.astype(np.int32)
        G.l_nJump = int(G.l_jump.size)
        G.type = "l_squeezed_cpp_prepared"
    else:
        G.l_jump = np.zeros(0, np.int32)
        G.l_nJump = int(G.l_size)
        G.type = "cpp_prepared"
    G.r_ind = None
    G.l_ind = None
    G.block_type = argMode
    G.extra.update(nBlock=int(l_block_start.size), l_block_start=l_block_start, block_length=block_length,
                   m_block_start=m_block_start)
    return G


def traj2sparsemat(t, v, N_u, dK_u, kernelType=None, nWin=None, kernelParam=None,
                   want=("Gu", "Gut")):
    """bmTraj2SparseMat.m:12-314 for one trajectory.  Returns a dict with the
    requested 'Gn', 'Gu', 'Gut' (cpp_prepared bmSparseMat)."""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    t = np.asarray(t, np.float64)
    if t.ndim == 1:
        t = t[None, :]
    imDim, nPt = t.shape
    N_u = single(np.ravel(N_u))
    dK_u = single(np.ravel(dK_u))
    Nu_tot = int(np.prod(N_u))
    Du = 1.0
    for i in range(imDim):
        Du *= (1 / dK_u[i]) / N_u[i]
    tg, Dn, deleteMask = to_grid_units(t, v, N_u, dK_u)

    c, shift = window_offsets(imDim, nWin)
    nNb = c.shape[1]
    t_floor = np.floor(tg + shift)
    t_rest = tg - t_floor
    d2 = np.zeros((nNb, nPt))
    for i in range(imDim):
        d2 = d2 + (t_rest[i][None, :] - c[i][:, None]) ** 2
    d = np.sqrt(d2)  # [nNb, nPt]
    weight = kernel_weight(d, kernelType, kp)

    n = t_floor[:, None, :] + c[:, :, None]  # [imDim, nNb, nPt]
    lin = np.zeros((nNb, nPt))
    stride = 1.0
    for i in range(imDim):
        ni = np.mod(n[i] - 1, N_u[i]) + 1
        lin = lin + (ni - 1) * stride
        stride *= N_u[i]
    lin = lin + 1  # 1-based linear cell index
    keep = ~deleteMask
    rows = np.repeat(np.arange(nPt)[keep], nNb)
    cols = (lin[:, keep].T.ravel() - 1).astype(np.int64)
    w = weight[:, keep].T.ravel()
    dn = Dn[keep].repeat(nNb) if Dn is not None else None
    out = {}
    if "Gn" in want:
        vals = w * dn
        A = sp.coo_matrix((vals, (rows, cols)), shape=(nPt, Nu_tot)).tocsr().T.tocsr()
        A.sum_duplicates()
        A.eliminate_zeros()
        s = np.asarray(A.sum(axis=1)).ravel()
        inv = np.zeros_like(s)
        inv[s != 0] = 1.0 / s[s != 0]
        A = sp.diags(inv) @ A
        G = matlab_sparse_to_bm(A, N_u, dK_u, kernelType, nWin, kp)
        out["Gn"] = cpp_prepare(l_squeeze(G))
    if "Gu" in want or "Gut" in want:
        A = sp.coo_matrix((w * Du, (rows, cols)), shape=(nPt, Nu_tot)).tocsr()
        A.sum_duplicates()
        A.eliminate_zeros()
        A.sort_indices()
        # row sums in ascending column order (MATLAB's sum(A, 2) over CSC)
        row_of = np.repeat(np.arange(nPt), np.diff(A.indptr))
        s = np.bincount(row_of, weights=A.data, minlength=nPt)
        inv = np.zeros_like(s)
        inv[s != 0] = 1.0 / s[s != 0]
        A = sp.csr_matrix((A.data * np.repeat(inv, np.diff(A.indptr)), A.indices, A.indptr), shape=A.shape)
        if "Gu" in want:
            out["Gu"] = cpp_prepare(matlab_sparse_to_bm(A, N_u, dK_u, kernelType, nWin, kp))
        if "Gut" in want:
            out["Gut"] = cpp_prepare(l_squeeze(matlab_sparse_to_bm(A.T.tocsr(), N_u, dK_u, kernelType, nWin, kp)))
    return out


def deform2sparsemat(v, N_u, Dn=None, torus_flag=False, want=("Gu", "Gut")):
    """bmImDeformField2SparseMat.m:14-146 with the weights of
    bmImDeformField2sparseMat_ind_weight.m:6-150 for one displacement field
    v [imDim, prod(N_u)] (pixel units).  Returns a dict with the requested
    'Gn', 'Gu', 'Gut' (cpp_prepared bmSparseMat, not squeezed)."""
    v = np.asarray(v, np.float64)
    if v.ndim == 1:
        v = v[None, :]
    imDim, nPt = v.shape
    N_u = np.ravel(N_u).astype(np.float64)
    Nu_tot = int(np.prod(N_u))
    if nPt != Nu_tot:
        raise ValueError("the deformation field must have as many vectors as pixels")
    # t = ndgrid(1:N) + v, x fastest (ind_weight.m:30-51)
    grids = np.meshgrid(*[np.arange(1, int(n) + 1, dtype=np.float64) for n in N_u[:imDim]], indexing="ij")
    t = np.stack([g.ravel(order="F") for g in grids]) + v
    deleteMask = np.zeros(nPt, bool)
    for i in range(imDim):  # :56-67
        deleteMask |= (t[i] < 1) | (t[i] > N_u[i])
    c = np.stack([g.ravel(order="F") for g in np.meshgrid(*[np.arange(2.0)] * imDim, indexing="ij")])  # [imDim, nNb]
    nNb = c.shape[1]
    t_floor = np.floor(t)
    t_rest = t - t_floor
    d2 = np.zeros((nNb, nPt))
    for i in range(imDim):
        d2 = d2 + (t_rest[i][None, :] - c[i][:, None]) ** 2
    d = np.sqrt(d2)
    with np.errstate(divide="ignore", over="ignore"):
        w = np.exp(-1.0 / (1.0 - d ** 2))  # bump function (:97-99)
    w[np.isinf(w)] = 0.0
    w = w * (np.abs(d) < 1)
    lin = np.zeros((nNb, nPt))
    stride = 1.0
    for i in range(imDim):  # periodic wrap (:105-118)
        ni = np.mod(t_floor[i][None, :] + c[i][:, None] - 1, N_u[i]) + 1
        lin = lin + (ni - 1) * stride
        stride *= N_u[i]
    keep = np.ones(nPt, bool) if torus_flag else ~deleteMask  # :122-130
    rows = np.repeat(np.arange(nPt)[keep], nNb)
    cols = lin[:, keep].T.ravel().astype(np.int64)
    ww = w[:, keep].T.ravel()
    out = {}
    bump = ("bump", 2, [])
    if "Gn" in want:
        if Dn is None:
            raise ValueError("Gn needs Dn")
        dn = np.asarray(Dn, np.float64).ravel()[keep].repeat(nNb)
        A = sp.coo_matrix((ww * dn, (rows, cols)), shape=(nPt, Nu_tot)).tocsr().T.tocsr()
        A.sum_duplicates()
        A.eliminate_zeros()
        s = np.asarray(A.sum(axis=1)).ravel()
        inv = np.zeros_like(s)
        inv[s != 0] = 1.0 / s[s != 0]
        out["Gn"] = cpp_prepare(matlab_sparse_to_bm(sp.diags(inv) @ A, N_u, [1, 1, 1], *bump))
    if "Gu" in want or "Gut" in want:
        A = sp.coo_matrix((ww, (rows, cols)), shape=(nPt, Nu_tot)).tocsr()
        A.sum_duplicates()
        A.eliminate_zeros()
        A.sort_indices()
        row_of = np.repeat(np.arange(nPt), np.diff(A.indptr))
        s = np.bincount(row_of, weights=A.data, minlength=nPt)
        inv = np.zeros_like(s)
        inv[s != 0] = 1.0 / s[s != 0]
        A = sp.csr_matrix((A.data * np.repeat(inv, np.diff(A.indptr)), A.indices, A.indptr), shape=A.shape)
        if "Gu" in want:
            out["Gu"] = cpp_prepare(matlab_sparse_to_bm(A, N_u, [1, 1, 1], *bump))
        if "Gut" in want:
            out["Gut"] = cpp_prepare(matlab_sparse_to_bm(A.T.tocsr(), N_u, [1, 1, 1], *bump))
    return out


def gridder_n2u_weights(t, Dn, N_u, dK_u, kernelType=None, nWin=None, kernelParam=None):
    """The argument preparation of bmGridder_n2u.m:22-211: returns the kept
    sample mask, weights w [nNb*nPt] (single) and jump-coded cells nJump."""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    t = np.asarray(t, np.float64)
    imDim = t.shape[0]
    N_u = np.asarray(np.ravel(N_u), np.float64)
    dK_u = np.asarray(np.ravel(dK_u), np.float64)
    tg, Dn, mask = to_grid_units(t, Dn, N_u, dK_u)
    keep = ~mask
    tg, Dn = tg[:, keep], Dn[keep]
    c, shift = window_offsets(imDim, nWin)
    t_floor = np.floor(tg + shift)
    t_rest = tg - t_floor
    d2 = 0
    for i in range(imDim):
        d2 = d2 + (t_rest[i][None, :] - c[i][:, None]) ** 2
    w = kernel_weight(np.sqrt(d2), kernelType, kp) * Dn[None, :]  # [nNb, nPt]
    n = t_floor[:, None, :] + c[:, :, None]
    lin = np.zeros(w.shape)
    stride = 1.0
    for i in range(imDim):
        lin = lin + (np.mod(n[i] - 1, N_u[i])) * stride
        stride *= N_u[i]
    lin = lin.T.ravel() + 1  # 1-based, point-major order
    nJump = np.diff(np.concatenate([[0], lin]))
    nJump[0] = lin[0] - 1
    return keep, w.T.ravel().astype(np.float32), nJump.astype(np.int32), int(c.shape[1])


# --------------------------------------------------------------------------
# deapodisation
# --------------------------------------------------------------------------
def _shift_fft(x, axes, inverse=False, workers=None):
    for ax in axes:
        x = sfft.ifftshift(x, axes=ax)
        x = (sfft.ifft if inverse else sfft.fft)(x, axis=ax, workers=workers)
        x = sfft.fftshift(x, axes=ax)
    return x


def bmK(N_u, dK_u, nCh, kernelType=None, nWin=None, kernelParam=None):
    """bmK.m:6-156: deapodisation on the N_u grid, [prod(N_u), nCh] single.
    (The 1D branch keeps the reference's mask expression, bmK.m:88.)"""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    osf = 2
    N_u = np.asarray(np.ravel(N_u), np.int64)
    imDim = N_u.size
    N_os = N_u * osf
    axes1d = [np.arange(-N_os[i] // 2, N_os[i] // 2) / osf for i in range(imDim)]
    grids = np.meshgrid(*axes1d, indexing="ij")
    d = np.sqrt(sum(g ** 2 for g in grids))
    w = kernel_weight(d, kernelType, kp)
    K_max = kp[1] if kernelType == "gauss" else kp[2]
    h = np.fix(nWin / 2)
    if imDim == 1:
        w[(grids[0] < h) | (grids[0] > h)] = 0
    else:
        for g in grids:
            w[(g < -h) | (g > h)] = 0
    K = _shift_fft(w.astype(np.complex128), range(imDim))
    K = K / (np.prod(N_os) * np.prod(1.0 / N_u))
    sl = tuple(slice(N_os[i] // 2 - N_u[i] // 2, N_os[i] // 2 + N_u[i] // 2) for i in range(imDim))
    K = np.abs(np.real(K[sl]))
    K = K / np.max(np.abs(K))
    K = np.minimum(1.0 / K, K_max)
    col = K.ravel(order="F")
    return np.repeat(col[:, None], int(nCh), axis=1).astype(np.float32)


def crop_index(N_u, n_u):
    """bmImCrope.m / bmImZeroFill.m: the n_u block sits at N/2-n/2 .. N/2+n/2-1."""
    return tuple(slice(int(N) // 2 - int(n) // 2, int(N) // 2 + int(n) // 2) for N, n in zip(N_u, n_u))


def crop_col(x, N_u, n_u):
    """Crops column data [prod(N_u), nCh] to [prod(n_u), nCh]."""
    nCh = x.shape[1]
    blk = x.reshape(tuple(int(v) for v in N_u) + (nCh,), order="F")
    return blk[crop_index(N_u, n_u)].reshape(-1, nCh, order="F")


def zerofill_col(x, N_u, n_u):
    nCh = x.shape[1]
    out = np.zeros(tuple(int(v) for v in N_u) + (nCh,), x.dtype)
    out[crop_index(N_u, n_u)] = x.reshape(tuple(int(v) for v in n_u) + (nCh,), order="F")
    return out.reshape(-1, nCh, order="F")


def bmKF(C, N_u, n_u, dK_u, nCh, kernelType=None, nWin=None, kernelParam=None):
    """bmKF.m:6-36: K * (1/prod(N_u)/prod(dK_u)) * C, single [prod(n_u), nCh]."""
    K = bmK(single(N_u), single(dK_u), nCh, kernelType, nWin, kernelParam)
    K = crop_col(K, np.ravel(N_u).astype(int), np.ravel(n_u).astype(int))
    F = np.float32(1 / np.prod(single(N_u)) / np.prod(single(dK_u)))
    if C is None:
        return (K * F).astype(np.float32)
    C = np.asarray(C).reshape(K.shape[0], -1, order="F").astype(np.complex64)
    return (K * F * C).astype(np.complex64)


def bmKF_conj(C_conj, N_u, n_u, dK_u, nCh, kernelType=None, nWin=None, kernelParam=None):
    """bmKF_conj.m:6-39: K * (1/prod(dK_u)) * conj(C) (caller passes conj(C))."""
    K = bmK(single(N_u), single(dK_u), nCh, kernelType, nWin, kernelParam)
    K = crop_col(K, np.ravel(N_u).astype(int), np.ravel(n_u).astype(int))
    F = np.float32(1 / np.prod(single(dK_u)))
    if C_conj is None:
        return (K * F).astype(np.float32)
    C_conj = np.asarray(C_conj).reshape(K.shape[0], -1, order="F").astype(np.complex64)
    return (K * F * C_conj).astype(np.complex64)


# --------------------------------------------------------------------------
# operators
# --------------------------------------------------------------------------
class SpMV:
    """The sparse product used by the restated operators: the compiled
    reference MEX (kind 'reference') or the C restatement ('port')."""

    def __init__(self, kind: str = "port"):
        self.kind = kind
        self._mex = ref_mex("bmSparseMat_cC_oBlock_omp_mex") if kind == "reference" else None

    def __call__(self, G: SparseMat, v: np.ndarray) -> np.ndarray:
        if self.kind == "fp64":  # float64 product of the same float32 matrix
            S = G.to_scipy().astype(np.float64)
            v = np.asarray(v, np.complex128)
            return np.asarray(S @ (v[:, None] if v.ndim == 1 else v), np.complex128)
        v = np.asarray(v, np.complex64)
        if v.ndim == 1:
            v = v[:, None]
        if self._mex is None:
            return port_spmv(G, v, "C")
        wR, wI = self._mex(np.int32(G.r_size), G.r_jump, G.r_nJump, G.m_val, np.int32(G.l_size),
                           G.l_jump if G.l_jump is not None and G.l_jump.size else None,
                           np.int32(G.l_nJump), np.int32(1 if G.l_jump is not None and G.l_jump.size else 0),
                           np.ascontiguousarray(v.real, np.float32), np.ascontiguousarray(v.imag, np.float32),
                           np.int32(v.shape[1]), nlhs=2)
        return (wR + 1j * wI).astype(np.complex64)


_default_spmv = None


def _spmv(kind=None):
    global _default_spmv
    if kind is not None:
        return SpMV(kind)
    if _default_spmv is None:
        _default_spmv = SpMV("port")
    return _default_spmv


def bmShanna(x, G: SparseMat, KFC, n_u=None, spmv=None, workers=None, dtype=np.complex64):
    """bmShanna_MATLAB.m:6-56: y = Gu * FFT(ZF(x .* KFC)), y [nPt, nCh].
    dtype complex128 (with spmv 'fp64') gives the FP64 restatement."""
    N_u = np.ravel(G.N_u).astype(int)
    n_u = N_u if n_u is None else np.ravel(n_u).astype(int)
    x = np.asarray(x, dtype)
    if x.ndim == 1:
        x = x[:, None]
    KFC = np.asarray(KFC)
    nCh = KFC.shape[1] if x.shape[1] == 1 else x.shape[1]
    if x.shape[1] < nCh:
        x = np.repeat(x, nCh, axis=1)
    x = (x * KFC).astype(dtype)
    if not np.array_equal(N_u, n_u):
        x = zerofill_col(x, N_u, n_u)
    blk = x.reshape(tuple(N_u) + (nCh,), order="F")
    blk = _shift_fft(blk, range(len(N_u)), workers=workers).astype(dtype)
    x = blk.reshape(-1, nCh, order="F")
    return (spmv or _spmv())(G, x)


def bmNakatsha(y, Gut: SparseMat, KFC_conj, C_flag=True, n_u=None, spmv=None, workers=None, dtype=np.complex64):
    """bmNakatsha_MATLAB.m:6-58: x = sum_c KFC_conj .* Crop(IFFT(Gut * y))."""
    N_u = np.ravel(Gut.N_u).astype(int)
    n_u = N_u if n_u is None else np.ravel(n_u).astype(int)
    y = np.asarray(y, dtype)
    if y.ndim == 1:
        y = y[:, None]
    nCh = y.shape[1]
    x = (spmv or _spmv())(Gut, y)
    blk = x.reshape(tuple(N_u) + (nCh,), order="F")
    blk = _shift_fft(blk, range(len(N_u)), inverse=True, workers=workers).astype(dtype)
    x = blk.reshape(-1, nCh, order="F")
    if not np.array_equal(N_u, n_u):
        x = crop_col(x, N_u, n_u)
    x = (x * KFC_conj).astype(dtype)
    if C_flag:
        x = x.sum(axis=1, dtype=dtype)[:, None]
    return x


def gridder_n2u_leight(data_n, t, Dn, N_u, dK_u, kernelType=None, nWin=None, kernelParam=None,
                       impl="port"):
    """bmGridder_n2u_leight.m:15-141 -> [nCh, prod(N_u)] complex single."""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    t = np.asarray(t, np.float32).astype(np.float64)
    data_n = np.asarray(data_n, np.complex64)
    imDim = t.shape[0]
    N_u = np.ravel(N_u).astype(np.float64)
    dK_u = np.ravel(dK_u).astype(np.float64)
    Dn = np.asarray(Dn, np.float32).astype(np.float64).ravel()
    # single-precision arithmetic of the wrapper (t and Dn are single there)
    ts = np.asarray(t, np.float32).copy()
    Dns = Dn.astype(np.float32)
    for i in range(imDim):
        ts[i] = ts[i] / np.float32(dK_u[i])
        Dns = Dns / np.float32(dK_u[i])
    shift = np.array([np.fix(N_u[i] / 2 + 1) for i in range(imDim)], np.float32)
    ts = ts + shift[:, None]
    mask = np.zeros(ts.shape[1], bool)
    for i in range(imDim):
        mask |= (ts[i] < 1) | (ts[i] > N_u[i])
    ts, Dns, a = ts[:, ~mask], Dns[~mask], data_n[:, ~mask]
    nCh, nPt = a.shape
    args = [ts[0], ts[1] if imDim > 1 else None, ts[2] if imDim > 2 else None]
    Ns = [int(N_u[0]), int(N_u[1]) if imDim > 1 else 1, int(N_u[2]) if imDim > 2 else 1]
    if impl == "reference":
        name = f"bmGridder_n2u_leight{imDim}_mex"
        m = ref_mex(name)
        aR = np.ascontiguousarray(a.real, np.float32)
        aI = np.ascontiguousarray(a.imag, np.float32)
        tt = [np.ascontiguousarray(v, np.float32)[None, :] for v in args[:imDim]]
        NN = [np.int32(v) for v in Ns[:imDim]]
        bR, bI = m(aR, aI, *tt, Dns[None, :], np.int32(nCh), np.int32(nPt), *NN, np.int32(nWin),
                   np.float32(kp[0]), np.float32(kp[1]), nlhs=2)
    else:
        bR, bI = port_gridder_leight(imDim, a.real, a.imag, args[0], args[1], args[2], Dns, nCh, nPt,
                                     Ns[0], Ns[1], Ns[2], int(nWin), kp[0], kp[1])
    return (bR + 1j * bI).astype(np.complex64)


def bmIDF(x, N_u, dK_u):
    """bmIDF{1,2,3}.m: fftshift(ifft(ifftshift)) * single(prod(N_u)*prod(dK_u))."""
    N_u = np.ravel(N_u).astype(int)
    x = np.asarray(x, np.complex64)
    y = _shift_fft(x, range(len(N_u)), inverse=True).astype(np.complex64)
    return (y * np.float32(np.prod(N_u) * np.prod(np.ravel(dK_u)))).astype(np.complex64)


def coil_pinv(C, x0):
    """bmCoilSense_pinv.m:10: sum(conj(C).*x0, 2) ./ sum(|C|^2, 2)."""
    C = np.asarray(C, np.complex64)
    return (np.sum(np.conj(C) * x0, axis=1) / np.sum(np.abs(C) ** 2, axis=1)).astype(np.complex64)


def bmMathilda(y, t, v, C, N_u, n_u, dK_u, kernelType=None, nWin=None, kernelParam=None,
               leight=True):
    """bmMathilda.m:14-125 (MATLAB FFT branch).  y [nPt, nCh] -> x [prod(n_u)]
    (coil-combined when C is given, else [prod(n_u), nCh])."""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    y = np.asarray(y, np.complex64)
    if y.ndim == 1:
        y = y[:, None]
    yt = y.T  # [nCh, nPt]
    N_u = np.ravel(N_u).astype(int)
    n_u = np.ravel(n_u).astype(int)
    dK_u = single(np.ravel(dK_u))
    nCh = yt.shape[0]
    if leight:
        xg = gridder_n2u_leight(yt, t, v, N_u, dK_u, kernelType, nWin, kp)
    else:
        keep, w, nJump, nNb = gridder_n2u_weights(t, v, N_u, dK_u, kernelType, nWin, kp)
        a = yt[:, keep]
        bR, bI = port_gridder_n2u(a.real, a.imag, w, nJump, nCh, nNb, a.shape[1], int(np.prod(N_u)))
        xg = (bR + 1j * bI).astype(np.complex64)
    x = xg.reshape(nCh, -1).T.reshape(tuple(N_u) + (nCh,), order="F")
    x = bmIDF(x, N_u, dK_u)
    K = bmK(N_u, dK_u, nCh, kernelType, nWin, kp).reshape(tuple(N_u) + (nCh,), order="F")
    x = (x * K).astype(np.complex64)
    x = x[crop_index(N_u, n_u)]
    x = x.reshape(-1, nCh, order="F")
    if C is not None:
        return coil_pinv(np.asarray(C).reshape(x.shape[0], -1, order="F"), x)
    return x


def bmNasha(y, Gn: SparseMat, n_u, C=None, K=None, spmv=None):
    """bmNasha.m:6-91 (MATLAB FFT branch): x = Gn y (the complex column
    product, :45), reshape to N_u, bmIDF, .* K (:77), crop (:80-82), coil
    pinv (:85-88).  y [nPt, nCh] -> x [prod(n_u)] (C given) or
    [prod(n_u), nCh]."""
    y = np.asarray(y, np.complex64)
    if y.ndim == 1:
        y = y[:, None]
    nCh = y.shape[1]
    N_u = np.ravel(Gn.N_u).astype(int)
    n_u = N_u if n_u is None else np.ravel(n_u).astype(int)
    dK_u = single(np.ravel(Gn.d_u))
    if K is None:
        K = bmK(N_u, dK_u, nCh, Gn.kernel_type, Gn.nWin, Gn.kernelParam)
    x = _spmv(spmv)(Gn, y)  # [prod(N_u), nCh]
    x = x.reshape(tuple(N_u) + (nCh,), order="F")
    x = bmIDF(x, N_u, dK_u)
    x = (x * np.asarray(K, np.float32).reshape(tuple(N_u) + (-1,), order="F")).astype(np.complex64)
    x = x[crop_index(N_u, n_u)].reshape(-1, nCh, order="F")
    if C is not None:
        return coil_pinv(np.asarray(C).reshape(x.shape[0], -1, order="F"), x)
    return x


# --------------------------------------------------------------------------
# solvers (FP32 data, FP64 scalars)
# --------------------------------------------------------------------------
def _dot(a, b, h=None):
    """real(a' * (h .* b)) accumulated in float64 (bmEuclideProd.m:6-45)."""
    a = np.asarray(a).ravel().astype(np.complex128)
    b = np.asarray(b).ravel().astype(np.complex128)
    if h is None:
        return float(np.real(np.vdot(a, b)))
    h = np.asarray(h).ravel().astype(np.float64)
    return float(np.real(np.vdot(a, h * b)))


def bmSensa(x, y, ve, C, Gu, Gut, n_u, nCGD, ve_max=None, nIter=1, spmv=None, dtype=np.complex64,
            workers=None, history=None):
    """bmSensa.m:6-96 CG-SENSE.  x [prod(n_u)] initial image, y [nPt, nCh],
    ve [nPt] (or [nPt, nCh]), C [prod(n_u), nCh].  ``nIter`` outer
    iterations (convCond), ``nCGD`` inner CG steps.  Scalars in FP64."""
    myEps = 10 * np.finfo(np.float32).eps
    y = np.asarray(y, np.complex64)
    nCh = y.shape[1]
    N_u = np.ravel(Gu.N_u).astype(int)
    n_u = np.ravel(n_u).astype(int)
    dK_u = single(np.ravel(Gu.d_u))
    KFC = bmKF(C, N_u, n_u, dK_u, nCh, Gu.kernel_type, Gu.nWin, Gu.kernelParam)
    KFC_conj = bmKF_conj(np.conj(C), N_u, n_u, dK_u, nCh, Gu.kernel_type, Gu.nWin, Gu.kernelParam)
    x = np.asarray(x, dtype).ravel()[:, None]
    dX_u = (np.float32(1) / dK_u.astype(np.float32)) / N_u.astype(np.float32)
    HX = float(np.prod(dX_u.astype(np.float32)))
    ve = np.asarray(ve, np.float32)
    ve = np.broadcast_to(ve.reshape(-1, 1) if ve.ndim == 1 else ve, y.shape)
    if ve_max is None:
        ve_max = float(np.max(ve))
    HY = np.minimum(ve, np.float32(ve_max)).astype(np.float32)

    if dtype == np.complex128 and spmv is None:
        spmv = SpMV("fp64")  # the FP64 restatement: products in double too
    M = lambda v: bmShanna(v, Gu, KFC, n_u, spmv, workers, dtype).astype(dtype)
    dagM = lambda r: ((1 / HX) * bmNakatsha((HY * r).astype(dtype), Gut, KFC_conj, True, n_u, spmv,
                                            workers, dtype)).astype(dtype)
    for _ in range(nIter):
        res_next = y - M(x)
        dagM_res_next = dagM(res_next)
        sqn_next = HX * _dot(dagM_res_next, dagM_res_next)
        p_next = dagM_res_next
        for i in range(1, nCGD + 1):
            res_curr, sqn_curr, p_curr = res_next, sqn_next, p_next
            if sqn_curr < myEps:
                break
            Mp = M(p_curr)
            sqn_Mp = _dot(Mp, Mp, HY)
            a = sqn_curr / sqn_Mp
            x = (x + dtype(a) * p_curr).astype(dtype)
            if i == nCGD:
                break
            res_next = (res_curr - dtype(a) * Mp).astype(dtype)
            dagM_res_next = dagM(res_next)
            sqn_next = HX * _dot(dagM_res_next, dagM_res_next)
            b = sqn_next / sqn_curr
            p_next = (dagM_res_next + dtype(b) * p_curr).astype(dtype)
        temp_r = y - M(x)
        R = _dot(temp_r, temp_r, HY)
        if history is not None:
            history.append(R)
    return x.ravel()


def prox_one_norm(w, s):
    """bmProx_oneNorm.m:6-35: soft threshold of real and imaginary parts."""
    s = np.float32(abs(s))
    w = np.asarray(w)
    def st(v):
        return ((v > s) * (v - s) + (v < -s) * (v + s)).astype(np.float32)
    if np.iscomplexobj(w):
        return (st(w.real) + 1j * st(w.imag)).astype(np.complex64)
    return st(w)


def back_gradient(x, n_u, dX_u):
    """bmBackGradient.m:6-17 / bmBackGradient_n.m:6-51: per axis n,
    (x - circshift(x, e_n)) / dX_u(n) with the first slice along n zeroed.
    x [prod(n_u)] -> [prod(n_u), imDim] (single)."""
    n_u = [int(v) for v in np.ravel(n_u)]
    dX_u = np.ravel(dX_u).astype(np.float32)
    xb = np.asarray(x, np.complex64).reshape(n_u, order="F")
    out = np.zeros((xb.size, len(n_u)), np.complex64)
    for n in range(len(n_u)):
        g = ((xb - np.roll(xb, 1, axis=n)) / dX_u[n]).astype(np.complex64)
        idx = [slice(None)] * len(n_u)
        idx[n] = 0
        g[tuple(idx)] = 0
        out[:, n] = g.ravel(order="F")
    return out


def back_gradient_T(g, n_u, dX_u):
    """bmBackGradientT.m:6-17 / bmBackGradient_nT.m:6-47: sum over axes of
    (g_n with its first slice zeroed - circshift(g_n, -e_n)) / dX_u(n); the
    shifted term uses g_n before zeroing.  [prod(n_u), imDim] -> [prod(n_u)]."""
    n_u = [int(v) for v in np.ravel(n_u)]
    dX_u = np.ravel(dX_u).astype(np.float32)
    g = np.asarray(g, np.complex64)
    x = np.zeros(int(np.prod(n_u)), np.complex64)
    for n in range(len(n_u)):
        xb = g[:, n].reshape(n_u, order="F")
        gz = xb.copy()
        idx = [slice(None)] * len(n_u)
        idx[n] = 0
        gz[tuple(idx)] = 0
        t = ((gz - np.roll(xb, -1, axis=n)) / dX_u[n]).astype(np.complex64)
        x = (x + t.ravel(order="F")).astype(np.complex64)
    return x


def bmSteva(x, y, ve, C, Gu, Gut, n_u, delta, rho, nCGD, ve_max=None, nIter=1, spmv=None, workers=None,
            history=None):
    """bmSteva.m:6-138, spatial-TV ADMM with z, u initialised as in :40-45.
    delta, rho: scalars or (first, last) of their per-iteration linspace
    (private_init_delta_rho, :140-157).  history receives (R, TV) per
    iteration (:117-125)."""
    myEps = 10 * np.finfo(np.float32).eps
    y = np.asarray(y, np.complex64)
    nCh = y.shape[1]
    N_u = np.ravel(Gu.N_u).astype(int)
    n_u = np.ravel(n_u).astype(int)
    imDim = N_u.size
    dK_u = single(np.ravel(Gu.d_u)).astype(np.float64)
    dX_u = ((np.float32(1) / dK_u.astype(np.float32)) / N_u.astype(np.float32)).astype(np.float32)
    ve = np.asarray(ve, np.float32)
    ve = np.broadcast_to(ve.reshape(-1, 1) if ve.ndim == 1 else ve, y.shape)
    if ve_max is None:
        ve_max = float(np.max(ve))
    lin = lambda v: (np.full(nIter, np.float32(abs(v)), np.float32) if np.isscalar(v) else
                     np.linspace(abs(v[0]), abs(v[1]), nIter).astype(np.float32))
    dl, rl = lin(delta), lin(rho)
    HX = np.float32(np.prod(dX_u))
    HZ = HX
    HY = np.minimum(ve, np.float32(ve_max)).astype(np.float32)
    KFC = bmKF(C, N_u, n_u, dK_u, nCh, Gu.kernel_type, Gu.nWin, Gu.kernelParam)
    KFC_conj = bmKF_conj(np.conj(C), N_u, n_u, dK_u, nCh, Gu.kernel_type, Gu.nWin, Gu.kernelParam)
    x = np.asarray(x, np.complex64).ravel()
    M = lambda v: bmShanna(v, Gu, KFC, n_u, spmv, workers)[:, :]
    G = lambda v: back_gradient(v, n_u, dX_u)
    GT = lambda g: back_gradient_T(g, n_u, dX_u)
    dagM = lambda r: (np.float32(1 / HX) * bmNakatsha((HY * r).astype(np.complex64), Gut, KFC_conj, True, n_u,
                                                       spmv, workers).ravel()).astype(np.complex64)
    z = G(x)
    u = np.zeros((x.size, imDim), np.complex64)
    for c in range(nIter):
        r = np.float32(rl[c])
        s = np.float32(r * np.float32(1 / HX))
        res_y = (y - M(x)).astype(np.complex64)
        res_z = ((z - u) - G(x)).astype(np.complex64)
        dA = (dagM(res_y) + s * GT((HZ * res_z).astype(np.complex64))).astype(np.complex64)
        p = dA
        sq_next = float(HX) * _dot(dA, dA)
        for i in range(1, nCGD + 1):
            res_y_c, res_z_c, sq_c, p_c = res_y, res_z, sq_next, p
            if sq_c < myEps:
                break
            Mp = M(p_c)
            Fp = G(p_c)
            a = sq_c / (_dot(Mp, Mp, HY) + float(np.float32(r * HZ)) * _dot(Fp, Fp))
            x = (x + np.float32(a) * p_c).astype(np.complex64)
            if i == nCGD:
                break
            res_y = (res_y_c - np.float32(a) * Mp).astype(np.complex64)
            res_z = (res_z_c - np.float32(a) * Fp).astype(np.complex64)
            dA = (dagM(res_y) + s * GT((HZ * res_z).astype(np.complex64))).astype(np.complex64)
            sq_next = float(HX) * _dot(dA, dA)
            b = sq_next / sq_c
            p = (dA + np.float32(b) * p_c).astype(np.complex64)
        bGu = (G(x) + u).astype(np.complex64)
        z = prox_one_norm(bGu, float(np.float32(dl[c] / r)))
        u = (bGu - z).astype(np.complex64)
        if history is not None:
            tr = y - M(x)
            R = _dot(tr, tr, HY)
            g = G(x)
            TV = float(HZ) * float(np.sum(np.abs(g.real), dtype=np.float64) + np.sum(np.abs(g.imag), dtype=np.float64))
            history.append((R, TV))
    return x


def bmTevaMorphosia_chain(x, y, ve, C, Gu, Gut, n_u, delta, rho, nCGD, ve_max, nIter, spmv=None,
                          workers=None, history=None, regul_mode="normal", Tu=None, Tut=None):
    """bmTevaMorphosia_chain.m:6-291, z and u initialised as in :75-81.  x, y,
    ve, Gu, Gut are lists over frames.  regul_mode 'normal' takes delta / rho
    from their lists (:104-106); 'adapt' sets delta = delta_list(c) * regul /
    dafi and rho = rho_list(c) * delta from the latest monitoring (:107-109,
    private_adapt_delta_rho :240-248), the first one taken on the initial x
    (:86).  Tu, Tut: per-frame deformation matrices (None, or None entries:
    identity); F x_i = Tu_i x_i - x_{i-1} (private_F :262-269, bmImDeform.m
    with K = []), F* z_i = (1/HX)(Tut_i (HZ z_i) - HZ z_{i+1}) (private_dagF
    :282-289, bmImDeformT.m)."""
    myEps = 10 * np.finfo(np.float32).eps
    nFr = len(y)
    nCh = y[0].shape[1]
    N_u = np.ravel(Gu[0].N_u).astype(int)
    n_u = np.ravel(n_u).astype(int)
    dK_u = np.ravel(Gu[0].d_u).astype(np.float32)
    dX_u = (np.float32(1) / dK_u) / N_u.astype(np.float32)
    HX = float(np.float32(np.prod(dX_u)))
    HZ = HX
    HY = [np.minimum(np.broadcast_to(np.asarray(v, np.float32).reshape(-1, 1), yy.shape), np.float32(ve_max))
          for v, yy in zip(ve, y)]
    KFC = bmKF(C, N_u, n_u, dK_u, nCh, Gu[0].kernel_type, Gu[0].nWin, Gu[0].kernelParam)
    KFC_conj = bmKF_conj(np.conj(C), N_u, n_u, dK_u, nCh, Gu[0].kernel_type, Gu[0].nWin, Gu[0].kernelParam)
    x = [np.asarray(xi, np.complex64).ravel()[:, None] for xi in x]
    Tu = Tu if Tu is not None else [None] * nFr
    Tut = Tut if Tut is not None else [None] * nFr
    sm = spmv or _spmv()

    def deform(T, v):  # bmImDeform / bmImDeformT with K = []: T v in FP32, or v
        return v if T is None else np.asarray(sm(T, v), np.complex64).reshape(v.shape)

    Mop = lambda v: [bmShanna(v[i], Gu[i], KFC, n_u, spmv, workers) for i in range(nFr)]
    Fop = lambda v: [(deform(Tu[i], v[i]) - v[(i - 1) % nFr]).astype(np.complex64) for i in range(nFr)]
    dagM = lambda r: [((1 / HX) * bmNakatsha((HY[i] * r[i]).astype(np.complex64), Gut[i], KFC_conj, True, n_u,
                                             spmv, workers)).astype(np.complex64) for i in range(nFr)]
    dagF = lambda z: [((1 / HX) * (deform(Tut[i], (np.float32(HZ) * z[i]).astype(np.complex64))
                                   - np.float32(HZ) * z[(i + 1) % nFr])).astype(np.complex64) for i in range(nFr)]
    sqn = lambda v, h: sum(_dot(v[i], v[i], h[i] if isinstance(h, list) else None) * (1 if isinstance(h, list) else h)
                           for i in range(nFr))
    z = Fop(x)
    u = [np.zeros_like(xi) for xi in x]
    dl = np.full(nIter, np.float32(abs(delta)), np.float32) if np.isscalar(delta) else \
        np.linspace(abs(delta[0]), abs(delta[1]), nIter).astype(np.float32)
    rl = np.full(nIter, np.float32(abs(rho)), np.float32) if np.isscalar(rho) else \
        np.linspace(abs(rho[0]), abs(rho[1]), nIter).astype(np.float32)

    def dafi_regul(x):  # private_dafi_regul (:211-224)
        dafi = sum(_dot(yy - m, yy - m, HY[i]) for i, (yy, m) in enumerate(zip(y, Mop(x))))
        regul = 0.0
        for i in range(nFr):
            tr = x[(i - 1) % nFr] - deform(Tu[i], x[i])
            regul += HZ * float(np.sum(np.abs(tr.real), dtype=np.float64) + np.sum(np.abs(tr.imag), dtype=np.float64))
        return dafi, regul

    dafi, regul = dafi_regul(x) if regul_mode == "adapt" else (None, None)
    for c in range(nIter):
        dlt, r = float(dl[c]), float(rl[c])
        if regul_mode == "adapt":
            dlt = float(np.float32(dlt * regul / dafi))
            r = float(np.float32(r * dlt))
        res_y = [y[i] - m for i, m in enumerate(Mop(x))]
        Fx = Fop(x)
        res_z = [(z[i] - u[i]) - Fx[i] for i in range(nFr)]
        dMy = dagM(res_y)
        dFz = dagF(res_z)
        dA = [(dMy[i] + np.float32(r) * dFz[i]).astype(np.complex64) for i in range(nFr)]
        p = dA
        sq_next = sqn(dA, HX)
        for j in range(1, nCGD + 1):
            res_y_c, res_z_c, sq_c, p_c = res_y, res_z, sq_next, p
            if sq_c < myEps:
                break
            Mp = Mop(p_c)
            Fp = Fop(p_c)
            a = sq_c / (sqn(Mp, HY) + sqn(Fp, r * HZ))
            x = [(x[i] + np.float32(a) * p_c[i]).astype(np.complex64) for i in range(nFr)]
            if j == nCGD:
                break
            res_y = [(res_y_c[i] - np.float32(a) * Mp[i]).astype(np.complex64) for i in range(nFr)]
            res_z = [(res_z_c[i] - np.float32(a) * Fp[i]).astype(np.complex64) for i in range(nFr)]
            dMy = dagM(res_y)
            dFz = dagF(res_z)
            dA = [(dMy[i] + np.float32(r) * dFz[i]).astype(np.complex64) for i in range(nFr)]
            sq_next = sqn(dA, HX)
            b = sq_next / sq_c
            p = [(dA[i] + np.float32(b) * p_c[i]).astype(np.complex64) for i in range(nFr)]
        Fx = Fop(x)
        Fxu = [(u[i] + Fx[i]).astype(np.complex64) for i in range(nFr)]
        z = [prox_one_norm(v, dlt / r) for v in Fxu]
        u = [(Fxu[i] - z[i]).astype(np.complex64) for i in range(nFr)]
        if history is not None or regul_mode == "adapt":
            dafi, regul = dafi_regul(x)
            if history is not None:
                history.append((0.5 * dafi + 0.5 * dlt * regul, dafi, regul))
    return [xi.ravel() for xi in x]


# --------------------------------------------------------------------------
# FP64 direct NUDFT with Monalisa's scaling
# --------------------------------------------------------------------------
def nudft_fp64(x, C, t, n_u, dK_u, N_u=None):
    """y_j = sum_r C(r) x(r) exp(-2 pi i k_j . r) / prod(N_u)/prod(dK_u)...

    The image grid r follows the reference's conventions: image index i
    (0-based) of an n_u image with pixel size dX = 1/(dK_u*N_u) has position
    (i - n_u/2)*dX; k_j are the trajectory points t (physical units).  The
    scaling is that of the forward operator (KFC's 1/prod(N_u)/prod(dK_u)
    times the unnormalised FFT sum), without deapodisation or gridding, so the
    result is what the gridded forward operator approximates."""
    t = np.asarray(t, np.float64)
    imDim, nPt = t.shape
    n_u = np.ravel(n_u).astype(int)
    N_u = n_u if N_u is None else np.ravel(N_u).astype(int)
    dK_u = np.ravel(dK_u).astype(np.float64)
    dX = 1.0 / (dK_u * N_u)
    coords = np.meshgrid(*[(np.arange(n) - n // 2) * dX[i] for i, n in enumerate(n_u)], indexing="ij")
    r = np.stack([c.ravel(order="F") for c in coords], 0)  # [imDim, nPix]
    x = np.asarray(x, np.complex128).ravel()
    C = np.asarray(C, np.complex128).reshape(x.size, -1, order="F")
    scale = 1.0 / np.prod(N_u) / np.prod(dK_u)
    out = np.zeros((nPt, C.shape[1]), np.complex128)
    for j0 in range(0, nPt, 256):
        ph = np.exp(-2j * np.pi * (t[:, j0:j0 + 256].T @ r))  # [b, nPix]
        out[j0:j0 + 256] = ph @ (C * x[:, None]) * scale
    return out
