"""Iterative reconstructions on the device.

bmSensa: src/fourier123/solver_function/imDim/nonCartesian/bmSensa.m:6-96
(CG-SENSE).  bmTevaMorphosia_chain:
src/fourier123/solver_function/imDim_morphosia/nonCartesian/
bmTevaMorphosia_chain.m:6-195 (temporal-TV ADMM over frame bins).
``convCond`` is the outer iteration cap (an int, or an object with
``nIter_max`` like the reference's bmConvergeCondition).
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
    KFC_conj, FFT pass tables and work vectors (one per trajectory/coil
    set)."""

    def __init__(self, Gu, Gut, C, n_u, dK_u=None, autotune=False, precision="fp32"):
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
        self.KFC, self.KFC_conj = KFC, KFC_conj  # host copies, [prod(n_u), nCh]
        self.nPt = self.plan.nPt
        self._mats = (Gu, Gut)
        if precision != "fp32":
            self.plan.precision = precision
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


class TevaMorphosiaChain:
    """Temporal-TV ADMM over frame bins with everything resident on the
    device.  Frame f has its own Gu{f}, Gut{f}; all frames share N_u, n_u,
    the coil maps and KFC.  Frame 0's plan owns the grid buffers and KFC, the
    others borrow them (NufftPlan.sharing); the chain (mlg_chain_t) holds the
    solver's work arrays over all frames."""

    REGUL_MODES = ("normal", "adapt")

    def __init__(self, Gu, Gut, C, n_u, dK_u=None, autotune=False):
        Gu = [g.to_device() if isinstance(g, bmSparseMat) else g for g in Gu]
        Gut = [g.to_device() if isinstance(g, bmSparseMat) else g for g in Gut]
        if len(Gu) != len(Gut) or not Gu:
            raise ValueError("Gu and Gut must be non-empty lists of the same length")
        self.nFr = len(Gu)
        first = SensaRecon(Gu[0], Gut[0], C, n_u, dK_u, autotune=autotune)
        self.N_u, self.n_u, self.dK_u, self.nCh = first.N_u, first.n_u, first.dK_u, first.nCh
        self.plans = [first.plan] + [NufftPlan.sharing(first.plan, Gu[f], Gut[f]) for f in range(1, self.nFr)]
        if autotune:
            for p in self.plans[1:]:
                p.autotune()
        self._first = first
        self.nPt = [p.nPt for p in self.plans]
        arr = (ctypes.c_void_p * self.nFr)(*[p.handle.value for p in self.plans])
        h = ctypes.c_void_p()
        N.call("mlg_chain_create", self.nFr, arr, ctypes.byref(h))
        self._h = h

    @property
    def handle(self):
        return self._h

    def set_deform(self, Tu=None, Tut=None):
        """Deformation fields of the temporal sparsifier: lists over frames
        of [prod(n_u), prod(n_u)] matrices (DeviceMatrix, bmSparseMat or
        None = identity), e.g. from bmImDeformField2SparseMat.  F x_f =
        Tu_f x_f - x_{f-1}; the adjoint applies Tut_f.  The matrices are kept
        alive by the chain."""
        def handles(T):
            if T is None or len(T) == 0:
                return None, []
            if len(T) != self.nFr:
                raise ValueError(f"need one deformation matrix (or None) per frame ({self.nFr})")
            mats = [None if m is None else (m.to_device() if isinstance(m, bmSparseMat) else m) for m in T]
            arr = (ctypes.c_void_p * self.nFr)(*[None if m is None else m.handle.value for m in mats])
            return arr, mats

        tu, mu = handles(Tu)
        tut, mut = handles(Tut)
        N.call("mlg_chain_set_deform", self._h, tu, tut)
        self._deform = mu + mut  # the chain reads them on every run

    @staticmethod
    def _pair(v):
        v = np.abs(np.ravel(np.asarray(v, np.float32)))
        return np.ascontiguousarray([v[0], v[-1]], np.float32)

    def run_dev(self, y, ve, x, z, u, delta, rho, nIter, nCGD, ve_max, regul_mode="normal", init_zu=True,
                history=None):
        """y [sum nPt, nCh], ve [sum nPt] float32, x/z/u [nFr, prod(n_u)]
        complex64 CUDA tensors (x, z, u in/out)."""
        hist = np.zeros(3 * max(1, nIter), np.float64)
        N.call("mlg_tevamorphosia_dev", self._h, N.tptr(y), N.tfptr(ve), float(ve_max), N.fptr(self._pair(delta)),
               N.fptr(self._pair(rho)), self.REGUL_MODES.index(regul_mode), int(nIter), int(nCGD), N.tptr(x),
               N.tptr(z), N.tptr(u), int(bool(init_zu)), N.dptr(hist), N.stream_ptr())
        if history is not None:
            history.extend(tuple(hist[3 * c:3 * c + 3]) for c in range(nIter))
        return x

    def run_host(self, y, ve, x0, delta, rho, nIter, nCGD, ve_max, regul_mode="normal", history=None):
        """y, ve: lists over frames ([nPt_f, nCh], [nPt_f]); x0: list of
        images or None (zeros).  Returns the list of frame images (flat)."""
        nu = int(np.prod(self.n_u))
        yR = np.concatenate([np.asarray(yy, np.complex64).real.T.ravel() for yy in y]).astype(np.float32)
        yI = np.concatenate([np.asarray(yy, np.complex64).imag.T.ravel() for yy in y]).astype(np.float32)
        vv = np.concatenate([np.ravel(v) for v in ve]).astype(np.float32)
        x = np.zeros((self.nFr, nu), np.complex64) if x0 is None else \
            np.stack([np.asarray(xi, np.complex64).ravel(order="F") for xi in x0])
        xR = np.ascontiguousarray(x.real, np.float32)
        xI = np.ascontiguousarray(x.imag, np.float32)
        hist = np.zeros(3 * max(1, nIter), np.float64)
        N.call("mlg_tevamorphosia", self._h, N.fptr(yR), N.fptr(yI), N.fptr(vv), float(ve_max),
               N.fptr(self._pair(delta)), N.fptr(self._pair(rho)), self.REGUL_MODES.index(regul_mode), int(nIter),
               int(nCGD), N.fptr(xR), N.fptr(xI), N.dptr(hist))
        if history is not None:
            history.extend(tuple(hist[3 * c:3 * c + 3]) for c in range(nIter))
        return [(xR[f] + 1j * xI[f]).astype(np.complex64) for f in range(self.nFr)]

    def close(self):
        if getattr(self, "_h", None):
            N.lib().mlg_chain_destroy(self._h)
            self._h = None
        for p in reversed(getattr(self, "plans", [])[1:]):
            p.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bmTevaMorphosia_chain(x, z, u, y, ve, C, Gu, Gut, n_u, Tu, Tut, delta, rho, regul_mode, nCGD, ve_max,
                          convCond=None, witnessInfo=None):
    """Temporal-TV ADMM (bmTevaMorphosia_chain.m).  x, y, ve, Gu, Gut are
    lists over frames; z, u must be empty (None / []) -- they start as F x
    and 0 as in the reference (:75-81).  Tu / Tut: empty, or lists over
    frames of deformation matrices (None entries = identity), as from
    bmImDeformField2SparseMat.  Returns the frame images as n_u blocks
    (MATLAB order).  ``witnessInfo`` may be a list that receives (objective,
    dafi, regul) per iteration (:172-178)."""
    if (z is not None and len(z)) or (u is not None and len(u)):
        raise NotImplementedError("z / u start values are taken from x (pass empty z and u)")
    r = TevaMorphosiaChain(Gu, Gut, C, n_u)
    r.set_deform(Tu, Tut)
    nIter = _niter(convCond)
    hist = witnessInfo if isinstance(witnessInfo, list) else None
    n_u = tuple(int(v) for v in np.ravel(n_u))
    out = r.run_host(y, ve, x, delta, rho, nIter, int(nCGD), ve_max, regul_mode, hist)
    r.close()
    return [o.reshape(n_u, order="F") for o in out]


def bmSteva(x, z, u, y, ve, C, Gu, Gut, n_u, delta, rho, nCGD, ve_max=None, convCond=None, witnessInfo=None):
    """Spatial-TV ADMM (bmSteva.m): a chain of one frame whose sparsifier is
    the backward gradient.  x initial image [prod(n_u)], y [nPt, nCh], ve
    [nPt]; z, u must be empty (they start as G x and 0, :40-45); delta, rho
    scalars or (first, last) pairs.  Returns the image as an n_u block
    (MATLAB order).  ``witnessInfo`` may be a list that receives (R, TV) per
    iteration (:117-125)."""
    if (z is not None and len(z)) or (u is not None and len(u)):
        raise NotImplementedError("z / u start values are taken from x (pass empty z and u)")
    r = TevaMorphosiaChain([Gu], [Gut], C, n_u)
    nIter = _niter(convCond)
    nu = int(np.prod(r.n_u))
    y = np.asarray(y, np.complex64)
    yR = np.ascontiguousarray(y.real.T, np.float32)
    yI = np.ascontiguousarray(y.imag.T, np.float32)
    xx = np.zeros(nu, np.complex64) if x is None else np.asarray(x, np.complex64).ravel(order="F")
    xR = np.ascontiguousarray(xx.real, np.float32)
    xI = np.ascontiguousarray(xx.imag, np.float32)
    hist = np.zeros(2 * max(1, nIter), np.float64)
    N.call("mlg_steva", r.handle, N.fptr(yR), N.fptr(yI), N.fptr(np.ascontiguousarray(np.ravel(ve), np.float32)),
           float(ve_max or 0.0), N.fptr(r._pair(delta)), N.fptr(r._pair(rho)), int(nIter), int(nCGD), N.fptr(xR),
           N.fptr(xI), N.dptr(hist))
    r.close()
    if isinstance(witnessInfo, list):
        witnessInfo.extend(tuple(hist[2 * c:2 * c + 2]) for c in range(nIter))
    return (xR + 1j * xI).astype(np.complex64).reshape(tuple(int(v) for v in np.ravel(n_u)), order="F")
