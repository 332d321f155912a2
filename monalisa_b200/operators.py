"""Non-Cartesian Fourier operators.

bmK / bmKF / bmKF_conj: src/fourier123/prep_function/bmK.m, bmKF.m, bmKF_conj.m
bmShanna:   src/fourier123/map_function/nonCartesian/bmShanna.m (forward)
bmNakatsha: src/fourier123/map_function/nonCartesian/bmNakatsha.m (adjoint)
bmIDF:      src/fourier3/bmIDF3.m (and 1/2-D)
bmMathilda: src/fourier123/map_function/nonCartesian/bmMathilda.m

Array conventions follow the reference: images are column vectors
[prod(n_u), nCol] in MATLAB (x fastest) order, k-space data [nPt, nCh].
NufftPlan is the device-resident form used by the solvers and the serving
loop; the bmShanna / bmNakatsha functions take host arrays like the MATLAB
functions and run through the stateless CUDA entry points.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .gridding import bmGridder_n2u, bmGridder_n2u_leight
from .sparsemat import DeviceMatrix, bmSparseMat, kernel_code, kernel_defaults


def _ints(v):
    return np.ascontiguousarray(np.ravel(v), np.int32)


def bmK(N_u, dK_u, nCh, kernelType=None, nWin=None, kernelParam=None):
    """Deapodisation [prod(N_u), nCh] float32 (bmK.m:6-156)."""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    Nu = _ints(N_u)
    dK = np.ascontiguousarray(np.ravel(dK_u), np.float64)
    kp3 = np.zeros(3)
    kp3[:kp.size] = kp
    K = np.zeros(int(np.prod(Nu)), np.float32)
    N.call("mlg_deapodization", Nu.size, N.iptr(Nu), N.dptr(dK), kernel_code(kernelType), nWin, N.dptr(kp3),
           N.fptr(K))
    return np.repeat(K[:, None], int(nCh), axis=1)


def bmK_dev(N_u, dK_u, kernelType=None, nWin=None, kernelParam=None):
    """One column of bmK computed on the device (mlg_deapodization_dev): a
    CUDA float32 tensor [prod(N_u)], bit-identical to bmK's column."""
    import torch

    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    Nu = _ints(N_u)
    dK = np.ascontiguousarray(np.ravel(dK_u), np.float64)
    kp3 = np.zeros(3)
    kp3[:kp.size] = kp
    K = torch.empty(int(np.prod(Nu)), dtype=torch.float32, device="cuda")
    N.call("mlg_deapodization_dev", Nu.size, N.iptr(Nu), N.dptr(dK), kernel_code(kernelType), nWin, N.dptr(kp3),
           N.tptr(K), N.stream_ptr())
    return K


def crop_index(N_u, n_u):
    """bmImCrope.m: the n_u block occupies N/2-n/2 .. N/2+n/2-1 of N_u."""
    return tuple(slice(int(a) // 2 - int(b) // 2, int(a) // 2 + int(b) // 2) for a, b in zip(N_u, n_u))


def _crop_col(x, N_u, n_u):
    nc = x.shape[1]
    blk = x.reshape(tuple(int(v) for v in N_u) + (nc,), order="F")
    return blk[crop_index(N_u, n_u)].reshape(-1, nc, order="F")


_K_CACHE = {}
_K_LOCK = __import__("threading").Lock()


def _cropped_K(N_u, n_u, dK_u, kernelType, nWin, kernelParam):
    """One column of bmK cropped to n_u, [prod(n_u), 1] float32.  Every coil
    column of bmK is the same (bmK.m:148-152), so one is computed; it is
    cached per grid, image and kernel (read-only, shared)."""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    key = (tuple(np.ravel(N_u).astype(int)), tuple(np.ravel(n_u).astype(int)),
           tuple(np.ravel(dK_u).astype(np.float32)), kernelType, int(nWin), tuple(kp))
    with _K_LOCK:
        K = _K_CACHE.get(key)
    if K is None:
        import torch

        if torch.cuda.is_available():  # the device computation, bit-identical to the host one
            col = bmK_dev(N_u, dK_u, kernelType, nWin, kp).cpu().numpy()[:, None]
        else:
            col = bmK(N_u, dK_u, 1, kernelType, nWin, kp)
        K = _crop_col(col, N_u, n_u)
        K.setflags(write=False)
        with _K_LOCK:
            if len(_K_CACHE) > 16:
                _K_CACHE.clear()
            _K_CACHE[key] = K
    return K


def bmKF(C, N_u, n_u, dK_u, nCh, kernelType=None, nWin=None, kernelParam=None):
    """K * (1/prod(N_u)/prod(dK_u)) * C cropped to n_u (bmKF.m:6-36)."""
    N_u = np.ravel(N_u).astype(np.float32)
    n_u = np.ravel(n_u).astype(np.float32)
    dK_u = np.ravel(dK_u).astype(np.float32)
    K = _cropped_K(N_u, n_u, dK_u, kernelType, nWin, kernelParam)
    F = np.float32(1 / np.prod(N_u) / np.prod(dK_u))
    if C is None:
        return np.repeat((K * F).astype(np.float32), int(nCh), axis=1)
    C = np.asarray(C, np.complex64).reshape(K.shape[0], -1, order="F")
    return (K * F * C).astype(np.complex64)


def bmKF_conj(C_conj, N_u, n_u, dK_u, nCh, kernelType=None, nWin=None, kernelParam=None):
    """K * (1/prod(dK_u)) * conj(C) cropped to n_u (bmKF_conj.m:6-39); the
    caller passes conj(C), as in the reference."""
    N_u = np.ravel(N_u).astype(np.float32)
    n_u = np.ravel(n_u).astype(np.float32)
    dK_u = np.ravel(dK_u).astype(np.float32)
    K = _cropped_K(N_u, n_u, dK_u, kernelType, nWin, kernelParam)
    F = np.float32(1 / np.prod(dK_u))
    if C_conj is None:
        return np.repeat((K * F).astype(np.float32), int(nCh), axis=1)
    C_conj = np.asarray(C_conj, np.complex64).reshape(K.shape[0], -1, order="F")
    return (K * F * C_conj).astype(np.complex64)


def _split(a, shape2):
    a = np.asarray(a, np.complex64).reshape(shape2, order="F")
    return np.ascontiguousarray(a.real.T), np.ascontiguousarray(a.imag.T)  # column-major


class NufftPlan:
    """Device-resident Shanna / Nakatsha operator pair (mlg_plan_t).

    Gu, Gut: DeviceMatrix (or bmSparseMat, uploaded); KFC / KFC_conj:
    [prod(n_u), nCh] complex.  Device tensors are complex64 CUDA tensors:
    images [prod(n_u)], k-space [nPt, nCh] (point layout)."""

    def __init__(self, N_u, n_u, nCh, Gu, Gut, KFC, KFC_conj, dK_u=None):
        self.N_u = _ints(N_u)
        self.n_u = _ints(n_u if n_u is not None else N_u)
        self.imDim = self.N_u.size
        self.nCh = int(nCh)
        self._keep = []
        if isinstance(Gu, bmSparseMat):
            Gu = Gu.to_device()
        if isinstance(Gut, bmSparseMat):
            Gut = Gut.to_device()
        self._keep = [Gu, Gut]
        self.nPt = Gu.l_size if Gu is not None else Gut.r_size
        nu = int(np.prod(self.n_u))
        kr, ki = _split(KFC, (nu, self.nCh)) if KFC is not None else (None, None)
        cr, ci = _split(KFC_conj, (nu, self.nCh)) if KFC_conj is not None else (None, None)
        h = ctypes.c_void_p()
        N.call("mlg_plan_create", self.imDim, N.iptr(self.N_u), N.iptr(self.n_u), self.nCh,
               Gu.handle if Gu is not None else None, Gut.handle if Gut is not None else None,
               N.fptr(kr), N.fptr(ki), N.fptr(cr), N.fptr(ci), ctypes.byref(h))
        self._h = h
        if dK_u is not None:
            N.call("mlg_plan_set_dk", self._h, N.dptr(np.ascontiguousarray(np.ravel(dK_u), np.float64)))

    @classmethod
    def sharing(cls, base: "NufftPlan", Gu, Gut):
        """A plan over other matrices on base's grid that borrows base's KFC,
        grid buffers, FFT tables and stream (mlg_plan_create_sharing)."""
        if isinstance(Gu, bmSparseMat):
            Gu = Gu.to_device()
        if isinstance(Gut, bmSparseMat):
            Gut = Gut.to_device()
        self = cls.__new__(cls)
        self.N_u, self.n_u, self.imDim, self.nCh = base.N_u, base.n_u, base.imDim, base.nCh
        self._keep = [Gu, Gut]
        self._base = base  # outlives this plan
        self.nPt = Gu.l_size if Gu is not None else Gut.r_size
        h = ctypes.c_void_p()
        N.call("mlg_plan_create_sharing", base.handle, Gu.handle if Gu is not None else None,
               Gut.handle if Gut is not None else None, ctypes.byref(h))
        self._h = h
        return self

    @property
    def handle(self):
        return self._h

    ADJOINT_MODES = ("full_grid", "fused", "masked")

    @property
    def adjoint_mode(self) -> str:
        m = ctypes.c_int()
        N.call("mlg_plan_get_adjoint", self._h, ctypes.byref(m))
        return self.ADJOINT_MODES[m.value]

    @adjoint_mode.setter
    def adjoint_mode(self, name: str):
        N.call("mlg_plan_set_adjoint", self._h, self.ADJOINT_MODES.index(name))

    PRECISIONS = ("fp32", "mixed", "fp16_values")

    @property
    def precision(self) -> str:
        m = ctypes.c_int()
        N.call("mlg_plan_get_precision", self._h, ctypes.byref(m))
        return self.PRECISIONS[m.value]

    @precision.setter
    def precision(self, name: str):
        """'fp32', 'mixed' (FP16 matrix values and, where the plan supports
        it, the 3-D transforms' intermediate stored in scaled FP16 inside the
        CG-SENSE solver's steps; FP32 k-space vectors, sums and FFT
        arithmetic, FP64 scalars) or 'fp16_values' (FP16 matrix values
        only)."""
        N.call("mlg_plan_set_precision", self._h, self.PRECISIONS.index(name))

    @property
    def half_intermediate(self) -> bool:
        """Whether the CG steps of a mixed solve keep the intermediate of the
        3-D transforms (after the y pass of the forward, the z pass of the
        adjoint) in scaled FP16: mixed precision on a plan whose passes support
        it (3-D, a multiple of 4 coils, TMA line passes)."""
        m = ctypes.c_int()
        N.call("mlg_plan_get_half_intermediate", self._h, ctypes.byref(m))
        return bool(m.value & 1)

    @property
    def half_grid(self) -> bool:
        """Whether the CG steps of a mixed solve also store the forward grid
        in scaled FP16 (written by the last forward pass, read by Gu)."""
        m = ctypes.c_int()
        N.call("mlg_plan_get_half_intermediate", self._h, ctypes.byref(m))
        return bool(m.value & 2)

    def autotune(self, reps: int = 3, variants: bool = True) -> dict:
        """Times the valid adjoint strategies and keeps the fastest, then (with
        `variants`) the kernel variants of that strategy (TMA or cp.async
        line-FFT passes, Gut rows from the CSR or from row records); returns
        {name: ms} (what the plan cannot run is omitted)."""
        ms = np.zeros(3)
        N.call("mlg_plan_autotune", self._h, int(reps), N.dptr(ms))
        out = {n: float(t) for n, t in zip(self.ADJOINT_MODES, ms) if t >= 0}
        if variants and self.nPt > 0:
            mv = np.zeros(6)
            N.call("mlg_plan_autotune_variants", self._h, int(reps), N.dptr(mv))
            names = ("passes_tma_2buf", "passes_tma_3buf", "passes_cp_async", "gut_csr", "gut_records",
                     "fwd_full_store")
            out.update({n: float(t) for n, t in zip(names, mv) if t >= 0})
        return out

    @property
    def variant(self) -> dict:
        """The plan's kernel variants: {'pass_buffers': 0 (cp.async passes),
        2 or 3 (TMA passes with that many bundle buffers), 'gut_records': 0 (CSR
        rows) or 1 (row records), 'fwd_masked_store': 1 (the last forward pass
        stores only the grid chunks holding cells Gu reads) or 0}."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        N.call("mlg_plan_get_variant", self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return {"pass_buffers": a.value, "gut_records": b.value, "fwd_masked_store": c.value}

    @variant.setter
    def variant(self, v: dict):
        cur = self.variant
        cur.update(v)
        N.call("mlg_plan_set_variant", self._h, int(cur["pass_buffers"]), int(cur["gut_records"]),
               int(cur["fwd_masked_store"]))

    def status(self) -> None:
        """Synchronises the plan's stream; raises MonalisaError (timeout) when
        a bounded wait inside a device pass ran out since the last check."""
        N.call("mlg_plan_status", self._h)

    def device_bytes(self) -> int:
        b = ctypes.c_longlong()
        N.call("mlg_plan_device_bytes", self._h, ctypes.byref(b))
        return b.value

    def shanna(self, x, out=None, per_coil=False):
        import torch

        if out is None:
            out = torch.empty((self.nPt, self.nCh), dtype=torch.complex64, device=x.device)
        N.call("mlg_shanna_dev", self._h, N.tptr(x), int(per_coil), N.tptr(out), N.stream_ptr())
        return out

    def nakatsha(self, y, HY=None, scale=1.0, out=None):
        import torch

        if out is None:
            out = torch.empty(int(np.prod(self.n_u)), dtype=torch.complex64, device=y.device)
        N.call("mlg_nakatsha_dev", self._h, N.tptr(y), N.tfptr(HY), float(scale), N.tptr(out), N.stream_ptr())
        return out

    def close(self):
        if getattr(self, "_h", None):
            N.lib().mlg_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bmShanna(x, G: bmSparseMat, KFC, n_u=None):
    """y = Gu * FFT(ZF(x .* KFC)) with host arrays (bmShanna.m /
    bmShanna_MATLAB.m).  x [prod(n_u)] or [prod(n_u), nCh] -> y [nPt, nCh]."""
    N_u = _ints(G.N_u)
    n_u = _ints(n_u if n_u is not None else G.N_u)
    KFC = np.asarray(KFC)
    nu = int(np.prod(n_u))
    nCh = KFC.reshape(nu, -1, order="F").shape[1]
    x = np.asarray(x, np.complex64).reshape(nu, -1, order="F")
    kr, ki = _split(KFC, (nu, nCh))
    xr, xi = _split(x, x.shape)
    r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump = G.jump_arrays()
    yR = np.zeros((nCh, l_size), np.float32)
    yI = np.zeros((nCh, l_size), np.float32)
    N.call("mlg_shanna", N_u.size, N.iptr(N_u), N.iptr(n_u), nCh, N.fptr(xr), N.fptr(xi), x.shape[1], N.fptr(kr),
           N.fptr(ki), r_size, N.iptr(r_jump), N.iptr(r_nJump), N.fptr(m_val), l_size, N.iptr(l_jump), l_nJump,
           N.fptr(yR), N.fptr(yI))
    return (yR + 1j * yI).T.astype(np.complex64)


def bmNakatsha(y, Gut: bmSparseMat, KFC_conj, C_flag=True, n_u=None):
    """x = sum_c KFC_conj .* Crop(IFFT(Gut * y)) with host arrays
    (bmNakatsha.m).  As in the reference's GPU branch, C_flag must be true."""
    if not C_flag:
        raise ValueError(" 'C_flag' must be 'true' for the CUFFT version of bmNakatsha. ")
    N_u = _ints(Gut.N_u)
    n_u = _ints(n_u if n_u is not None else Gut.N_u)
    y = np.asarray(y, np.complex64)
    if y.ndim == 1:
        y = y[:, None]
    nPt, nCh = y.shape
    nu = int(np.prod(n_u))
    cr, ci = _split(KFC_conj, (nu, nCh))
    yr, yi = _split(y, y.shape)
    r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump = Gut.jump_arrays()
    xR = np.zeros(nu, np.float32)
    xI = np.zeros(nu, np.float32)
    N.call("mlg_nakatsha", N_u.size, N.iptr(N_u), N.iptr(n_u), nCh, N.fptr(yr), N.fptr(yi), N.fptr(cr), N.fptr(ci),
           r_size, N.iptr(r_jump), N.iptr(r_nJump), N.fptr(m_val), l_size, N.iptr(l_jump), l_nJump, N.fptr(xR),
           N.fptr(xI))
    return (xR + 1j * xI).astype(np.complex64)[:, None]


def bmIDF(x, N_u, dK_u):
    """fftshift(ifft(ifftshift(x))) * prod(N_u)*prod(dK_u) over the first
    len(N_u) dimensions of x (block [N_u..., nCol], MATLAB order)."""
    N_u = _ints(N_u)
    x = np.asarray(x, np.complex64)
    nu = int(np.prod(N_u))
    shape = x.shape
    xc = x.reshape(nu, -1, order="F")
    nCol = xc.shape[1]
    xr = np.ascontiguousarray(xc.real.T)
    xi = np.ascontiguousarray(xc.imag.T)
    yR = np.zeros((nCol, nu), np.float32)
    yI = np.zeros((nCol, nu), np.float32)
    N.call("mlg_idf", N_u.size, N.iptr(N_u), N.fptr(np.ascontiguousarray(np.ravel(dK_u), np.float32)), nCol,
           N.fptr(xr), N.fptr(xi), N.fptr(yR), N.fptr(yI))
    return (yR + 1j * yI).T.reshape(shape, order="F").astype(np.complex64)


def bmCoilSense_pinv(C, x0):
    """src/coilSense/map/bmCoilSense_pinv.m:10."""
    C = np.asarray(C, np.complex64)
    return (np.sum(np.conj(C) * x0, axis=1) / np.sum(np.abs(C) ** 2, axis=1)).astype(np.complex64)


def bmMathilda(y, t, v, C, N_u, n_u, dK_u, kernelType=None, nWin=None, kernelParam=None, leight_flag=True):
    """Gridded reconstruction (bmMathilda.m:14-125, CUFFT branch): adjoint
    gridding -> bmIDF -> deapodisation -> crop -> coil pinv.
    y [nPt, nCh] -> x [prod(n_u)] (or [prod(n_u), nCh] without C)."""
    import torch

    from .gridding import bmGridder_n2u_leight_dev

    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    y = np.asarray(y, np.complex64)
    if y.ndim == 1:
        y = y[:, None]
    if y.shape[0] < y.shape[1]:
        y = y.T  # bmMathilda.m:35-37 expects more points than coils
    N_u = _ints(N_u)
    dK_u = np.ravel(dK_u).astype(np.float32).astype(np.float64)
    nCh = y.shape[1]
    dev = torch.device("cuda", torch.cuda.current_device())
    if leight_flag:
        bR, bI = bmGridder_n2u_leight_dev(y.T, t, v, N_u, dK_u, kernelType, nWin, kp)
    else:  # precomputed-weight gridder (host arguments), result moved to the device
        xg = bmGridder_n2u(y.T, t, v, N_u, dK_u, kernelType, nWin, kp)  # [nCh, prod(N_u)]
        bR = torch.from_numpy(np.ascontiguousarray(xg.real.T, np.float32)).to(dev)
        bI = torch.from_numpy(np.ascontiguousarray(xg.imag.T, np.float32)).to(dev)
    return _gridded_tail(bR, bI, N_u, n_u, dK_u, nCh, C, kernelType, nWin, kp)


def _gridded_tail(ga, gb, N_u, n_u, dK_u, nCh, C, kernelType, nWin, kp, K=None):
    """coil_pinv(crop(K .* bmIDF(grid))) on the device (mlg_gridded_tail_dev);
    ga, gb: split [prod(N_u)][nCh] float32 CUDA tensors, or ga an interleaved
    complex64 one and gb None.  Returns host x [prod(n_u)] with C, else
    [prod(n_u), nCh]."""
    import torch

    N_u = _ints(N_u)
    n_u = _ints(n_u if n_u is not None else N_u)
    dev = ga.device
    if K is None:
        Kv = bmK(N_u, dK_u, 1, kernelType, nWin, kp)[:, 0]
    else:  # [prod(N_u)] or [prod(N_u), nCh] (identical columns)
        Kv = np.asarray(K, np.float32).reshape(int(np.prod(N_u)), -1, order="F")[:, 0]
    Kd = torch.from_numpy(np.ascontiguousarray(Kv, np.float32)).to(dev)
    nu = int(np.prod(n_u))
    Cd = None
    if C is not None:
        Cd = torch.from_numpy(np.ascontiguousarray(np.asarray(C, np.complex64).reshape(nu, -1, order="F"))).to(dev)
        if Cd.shape[1] != nCh:
            raise ValueError("C must be [prod(n_u), nCh]")
    x = torch.empty((nu if C is not None else nCh * nu,), dtype=torch.complex64, device=dev)
    N.call("mlg_gridded_tail_dev", N_u.size, N.iptr(N_u), N.iptr(n_u),
           N.fptr(np.ascontiguousarray(np.ravel(dK_u), np.float32)), nCh, 1 if gb is not None else 0, N.tptr(ga),
           N.tptr(gb), N.tptr(Kd), N.tptr(Cd), N.tptr(x), N.stream_ptr())
    out = x.cpu().numpy()
    return out if C is not None else out.reshape(nCh, nu).T.copy()


def bmNasha(y, G, n_u=None, C=None, K=None):
    """Gridded reconstruction with the Gn matrix (src/fourier123/
    map_function/nonCartesian/bmNasha.m:6-91): x = Gn y, bmIDF, .* K, crop,
    coil pinv (C given) -- all on the device.  y [nPt, nCh]; G the Gn
    bmSparseMat or DeviceMatrix ([prod(N_u), nPt], from bmTraj2SparseMat
    with nargout 1 or 3); K optional ([prod(N_u)] or [prod(N_u), nCh]),
    computed from G's kernel when absent (:25-28)."""
    import torch

    Gd = G.to_device() if isinstance(G, bmSparseMat) else G
    meta = Gd.meta
    N_u = _ints(meta["N_u"])
    dK_u = np.ravel(meta["d_u"]).astype(np.float32).astype(np.float64)
    y = np.asarray(y, np.complex64)
    if y.ndim == 1:
        y = y[:, None]
    nPt, nCh = y.shape
    if nPt != Gd.r_size:  # bmNasha.m:117-120
        raise ValueError("The data matrix 'y' is not in the correct size. ")
    if np.any(N_u % 2):  # bmNasha.m:137-140
        raise ValueError("N_u must have all components even for the Fourier transform. ")
    dev = torch.device("cuda", torch.cuda.current_device())
    g = Gd.spmm(torch.from_numpy(np.ascontiguousarray(y)).to(dev))  # [prod(N_u)][nCh]
    return _gridded_tail(g, None, N_u, n_u, dK_u, nCh, C, meta["kernel_type"], int(meta["nWin"]),
                         np.ravel(meta["kernelParam"]).astype(np.float64), K)
