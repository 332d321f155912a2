"""Iterative reconstructions on the device.

bmSensa: src/fourier123/solver_function/imDim/nonCartesian/bmSensa.m:6-96
(CG-SENSE).  ``convCond`` is the outer iteration cap (an int, or an object
with ``nIter_max`` like the reference's bmConvergeCondition).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .operators import NufftPlan, bmKF, bmKF_conj
from .sparsemat import DeviceMatrix, bmSparseMat


def _niter(convCond) -> int:
    if convCond is None:
        return 1
    if isinstance(convCond, (int, np.integer)):
        return int(convCond)
    return int(getattr(convCond, "nIter_max"))


class SensaRecon:
    """CG-SENSE with everything resident on the device: Gu/Gut, KFC,
    KFC_conj, cuFFT plans and work vectors (one per trajectory/coil set)."""

    def __init__(self, Gu, Gut, C, n_u, dK_u=None, autotune=False):
        if isinstance(Gu, bmSparseMat):
            Gu = Gu.to_device()
        if isinstance(Gut, bmSparseMat):
            Gut = Gut.to_device()
        meta = Gu.meta
        self.N_u = np.ravel(meta["N_u"]).astype(np.int64)
        self.n_u = np.ravel(n_u).astype(np.int64)
        self.dK_u = np.ravel(meta["d_u"] if dK_u is None else dK_u).astype(np.float32).astype(np.float64)
        C = np.asarray(C, np.complex64).reshape(int(np.prod(self.n_u)), -1, order="F")
        self.nCh = C.shape[1]
        kt, nw, kp = meta["kernel_type"], meta["nWin"], meta["kernelParam"]
        KFC = bmKF(C, self.N_u, self.n_u, self.dK_u, self.nCh, kt, nw, kp)
        KFC_conj = bmKF_conj(np.conj(C), self.N_u, self.n_u, self.dK_u, self.nCh, kt, nw, kp)
        self.plan = NufftPlan(self.N_u, self.n_u, self.nCh, Gu, Gut, KFC, KFC_conj, self.dK_u)
        self.nPt = self.plan.nPt
        self._mats = (Gu, Gut)
        self.tuning = self.plan.autotune() if autotune else None

    def run_dev(self, y, ve, x, nIter=1, nCGD=20, ve_max=None, residual=None):
        """y [nPt, nCh], ve [nPt] float32, x [prod(n_u)] (in/out) CUDA tensors."""
        res = np.zeros(max(1, nIter), np.float64) if residual is not None else None
        N.call("mlg_sensa_dev", self.plan.handle, N.tptr(y), N.tfptr(ve), float(ve_max or 0.0), int(nIter),
               int(nCGD), N.tptr(x), N.dptr(res) if res is not None else None, N.stream_ptr())
        if residual is not None:
            residual.extend(res[:nIter].tolist())
        return x

    def run_host(self, y, ve, x0=None, nIter=1, nCGD=20, ve_max=None, residual=None):
        """Host arrays in, host image out (copies inside the call)."""
        y = np.asarray(y, np.complex64)
        nu = int(np.prod(self.n_u))
        yR = np.ascontiguousarray(y.real.T)  # column-major [nPt, nCh]
        yI = np.ascontiguousarray(y.imag.T)
        x = np.zeros(nu, np.complex64) if x0 is None else np.asarray(x0, np.complex64).ravel(order="F")
        xR = np.ascontiguousarray(x.real)
        xI = np.ascontiguousarray(x.imag)
        res = np.zeros(max(1, nIter), np.float64)
        N.call("mlg_sensa", self.plan.handle, N.fptr(yR), N.fptr(yI),
               N.fptr(np.ascontiguousarray(np.ravel(ve), np.float32)), float(ve_max or 0.0), int(nIter), int(nCGD),
               N.fptr(xR), N.fptr(xI), N.dptr(res))
        if residual is not None:
            residual.extend(res[:nIter].tolist())
        return (xR + 1j * xI).astype(np.complex64)


def bmSensa(x, y, ve, C, Gu, Gut, n_u, nCGD, ve_max=None, convCond=None, witnessInfo=None):
    """CG-SENSE (bmSensa.m).  x initial image [prod(n_u)], y [nPt, nCh],
    ve [nPt], C [prod(n_u), nCh]; returns the image as an n_u block (MATLAB
    order).  ``witnessInfo`` may be a list that receives the residuals
    ||y - Mx||^2_HY of each outer iteration (bmSensa.m:82-84)."""
    r = SensaRecon(Gu, Gut, C, n_u)
    nIter = _niter(convCond)
    hist = witnessInfo if isinstance(witnessInfo, list) else None
    out = r.run_host(y, ve, x, nIter=nIter, nCGD=int(nCGD), ve_max=ve_max, residual=hist)
    return out.reshape(tuple(int(v) for v in np.ravel(n_u)), order="F")
