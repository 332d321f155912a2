"""Adjoint gridding wrappers with the reference's argument preparation.

bmGridder_n2u_leight: src/gridding123/m/bmGridder_n2u_leight.m:15-141
bmGridder_n2u:        src/gridding123/m/bmGridder_n2u.m:15-216
Both prepare the trajectory on the host exactly as the MATLAB wrappers do and
call the CUDA library's MEX-equivalent entry points.
"""
from __future__ import annotations

import numpy as np
import scipy.special as sspec

from . import _native as N
from .sparsemat import kernel_defaults


def _point(a, dtype):
    a = np.asarray(a, dtype)
    return a[None, :] if a.ndim == 1 else a


def _leight_prepare(data_n, t, Dn, N_u, dK_u):
    """Argument preparation of bmGridder_n2u_leight.m:40-87 (single
    precision): grid units, Dn / prod(dK_u), samples outside the grid box
    deleted.  Returns aR, aI [nPt][nCh], the per-axis t, Dn, nCh, nPt and the
    three grid extents."""
    t = _point(t, np.float32).copy()
    data_n = _point(data_n, np.complex64)
    Dn = np.asarray(Dn, np.float32).ravel().copy()
    imDim = t.shape[0]
    N_u = np.ravel(N_u).astype(np.float64)
    dK_u = np.ravel(dK_u).astype(np.float64)
    for i in range(imDim):
        t[i] = t[i] / np.float32(dK_u[i])
        Dn = Dn / np.float32(dK_u[i])
    t = t + np.array([np.fix(N_u[i] / 2 + 1) for i in range(imDim)], np.float32)[:, None]
    mask = np.zeros(t.shape[1], bool)
    for i in range(imDim):
        mask |= (t[i] < 1) | (t[i] > N_u[i])
    t, Dn, a = t[:, ~mask], Dn[~mask], data_n[:, ~mask]
    nCh, nPt = a.shape
    aR = np.ascontiguousarray(a.real.T, np.float32)
    aI = np.ascontiguousarray(a.imag.T, np.float32)
    tx = [np.ascontiguousarray(t[i]) for i in range(imDim)] + [None] * (3 - imDim)
    Ns = [int(N_u[i]) if i < imDim else 1 for i in range(3)]
    return aR, aI, tx, np.ascontiguousarray(Dn), nCh, nPt, Ns


def bmGridder_n2u_leight_dev(data_n, t, Dn, N_u, dK_u, kernelType=None, nWin=None, kernelParam=None):
    """The leight gridder with its output left on the device: returns CUDA
    float32 tensors (bR, bI), each [prod(N_u)][nCh] (point layout)."""
    import torch

    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    aR, aI, tx, Dn, nCh, nPt, Ns = _leight_prepare(data_n, t, Dn, N_u, dK_u)
    imDim = np.ravel(N_u).size
    dev = torch.device("cuda", torch.cuda.current_device())
    up = lambda a: torch.from_numpy(a).to(dev) if a is not None else None
    dA, dI, dD = up(aR), up(aI), up(Dn)
    dT = [up(v) for v in tx]
    nu = int(np.prod(Ns))
    bR = torch.empty((nu, nCh), dtype=torch.float32, device=dev)
    bI = torch.empty((nu, nCh), dtype=torch.float32, device=dev)
    N.call("mlg_gridder_n2u_leight_dev", imDim, N.tptr(dA), N.tptr(dI), N.tptr(dT[0]), N.tptr(dT[1]),
           N.tptr(dT[2]), N.tptr(dD), nCh, nPt, Ns[0], Ns[1], Ns[2], nWin, float(kp[0]), float(kp[1]), N.tptr(bR),
           N.tptr(bI), N.stream_ptr())
    return bR, bI


def bmGridder_n2u_leight(data_n, t, Dn, N_u, dK_u, kernelType=None, nWin=None, kernelParam=None):
    """data_n [nCh, nPt] (point layout), t [imDim, nPt], Dn [nPt] ->
    data_u [nCh, prod(N_u)] complex64 (column order of N_u)."""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    t = _point(t, np.float32).copy()
    data_n = _point(data_n, np.complex64)
    Dn = np.asarray(Dn, np.float32).ravel().copy()
    imDim = t.shape[0]
    N_u = np.ravel(N_u).astype(np.float64)
    dK_u = np.ravel(dK_u).astype(np.float64)
    # single-precision scaling and shift, bmGridder_n2u_leight.m:40-67
    for i in range(imDim):
        t[i] = t[i] / np.float32(dK_u[i])
        Dn = Dn / np.float32(dK_u[i])
    t = t + np.array([np.fix(N_u[i] / 2 + 1) for i in range(imDim)], np.float32)[:, None]
    # samples outside the grid box are deleted, :71-87
    mask = np.zeros(t.shape[1], bool)
    for i in range(imDim):
        mask |= (t[i] < 1) | (t[i] > N_u[i])
    t, Dn, a = t[:, ~mask], Dn[~mask], data_n[:, ~mask]
    nCh, nPt = a.shape
    # [nCh, nPt] column-major == C-order [nPt][nCh]
    aR = np.ascontiguousarray(a.real.T, np.float32)
    aI = np.ascontiguousarray(a.imag.T, np.float32)
    tx = [np.ascontiguousarray(t[i]) for i in range(imDim)] + [None] * (3 - imDim)
    Ns = [int(N_u[i]) if i < imDim else 1 for i in range(3)]
    nu = int(np.prod(Ns))
    bR = np.zeros((nu, nCh), np.float32)
    bI = np.zeros((nu, nCh), np.float32)
    N.call("mlg_gridder_n2u_leight", imDim, N.fptr(aR), N.fptr(aI), N.fptr(tx[0]),
           N.fptr(tx[1]), N.fptr(tx[2]), N.fptr(np.ascontiguousarray(Dn)), nCh, nPt, Ns[0], Ns[1], Ns[2], nWin,
           float(kp[0]), float(kp[1]), N.fptr(bR), N.fptr(bI))
    return (bR + 1j * bI).T.astype(np.complex64)


def _n2u_weights(t, Dn, N_u, dK_u, kernelType, nWin, kp):
    """Argument preparation of bmGridder_n2u.m:22-199 (FP64)."""
    t = np.asarray(t, np.float64)
    imDim, nPt = t.shape
    Dn = np.asarray(Dn, np.float64).ravel().copy()
    t = t.copy()
    for i in range(imDim):
        t[i] = t[i] / dK_u[i]
        Dn = Dn / dK_u[i]
        t[i] = t[i] + np.fix(N_u[i] / 2 + 1)
    mask = np.zeros(nPt, bool)
    for i in range(imDim):
        mask |= (t[i] < 1) | (t[i] > N_u[i])
    keep = ~mask
    t, Dn = t[:, keep], Dn[keep]
    if nWin % 2 == 0:
        rng, shift = np.arange(-nWin // 2 - 1, nWin // 2 + 1), 0.0
    else:
        rng, shift = np.arange(-(nWin // 2), nWin // 2 + 1), 0.5
    grids = np.meshgrid(*([rng] * imDim), indexing="ij")
    c = np.stack([g.ravel(order="F") for g in grids], 0).astype(np.float64)
    t_floor = np.floor(t + shift)
    t_rest = t - t_floor
    d2 = 0
    for i in range(imDim):
        d2 = d2 + (t_rest[i][None, :] - c[i][:, None]) ** 2
    d = np.sqrt(d2)
    if kernelType == "gauss":
        w = np.exp(-0.5 * (d / kp[0]) ** 2) / (np.sqrt(2 * np.pi) * kp[0])
    else:
        u = np.maximum(1 - (d / kp[0]) ** 2, 0)
        w = sspec.i0(kp[1] * np.sqrt(u)) / sspec.i0(kp[1])
    w = w * Dn[None, :]
    n = t_floor[:, None, :] + c[:, :, None]
    lin = np.zeros(w.shape)
    stride = 1.0
    for i in range(imDim):
        lin = lin + np.mod(n[i] - 1, N_u[i]) * stride
        stride *= N_u[i]
    lin = lin.T.ravel() + 1
    nJump = np.diff(np.concatenate([[0], lin]))
    nJump[0] = lin[0] - 1
    return keep, np.ascontiguousarray(w.T.ravel(), np.float32), np.ascontiguousarray(nJump, np.int32), c.shape[1]


def bmGridder_n2u(data_n, t, Dn, N_u, dK_u, kernelType=None, nWin=None, kernelParam=None):
    """Adjoint gridding with precomputed weights and periodic wrap ->
    [nCh, prod(N_u)] complex64."""
    kernelType, nWin, kp = kernel_defaults(kernelType, nWin, kernelParam)
    t = _point(t, np.float64)
    data_n = _point(data_n, np.complex64)
    N_u = np.ravel(N_u).astype(np.float64)
    dK_u = np.ravel(dK_u).astype(np.float64)
    keep, w, nJump, nNb = _n2u_weights(t, Dn, N_u, dK_u, kernelType, nWin, kp)
    a = data_n[:, keep]
    nCh, nPt = a.shape
    Nu = int(np.prod(N_u))
    aR = np.ascontiguousarray(a.real.T, np.float32)  # column-major [nCh, nPt]
    aI = np.ascontiguousarray(a.imag.T, np.float32)
    bR = np.zeros((Nu, nCh), np.float32)
    bI = np.zeros((Nu, nCh), np.float32)
    N.call("mlg_gridder_n2u", N.fptr(aR), N.fptr(aI), N.fptr(w), N.iptr(nJump), nCh, nNb, nPt, Nu, N.fptr(bR),
           N.fptr(bI))
    return (bR + 1j * bI).T.astype(np.complex64)
