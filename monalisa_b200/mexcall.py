"""Call a MEX gateway compiled against the project's MEX-API shim.

MATLAB is not present on the build/test machines, so MEX files (this
project's drop-in gateways in ``monalisa_b200/_lib/mex`` and, for tests only,
the reference's kernels) are shared objects exporting ``mexFunction`` and
linked with ``libmexshim.so``.  :class:`MexFunction` marshals numpy values to
``mxArray`` the way MATLAB would hand them to the gateway:

* ``numpy`` arrays keep their dtype (``float32`` -> single, ``int32`` -> int32,
  ``float64`` -> double, ``int64`` -> int64) and are passed column-major;
  complex arrays use MATLAB's separate real/imaginary storage;
* Python ``int``/``float`` become 1x1 double scalars (``mxGetScalar`` reads
  them like MATLAB does);
* ``None`` or a zero-size array becomes an empty array (NULL data pointer).

Outputs come back as numpy arrays in MATLAB's column-major shape.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

# mxClassID values of mex.h
_CLS = {
    np.dtype(np.float64): 6,
    np.dtype(np.float32): 7,
    np.dtype(np.int8): 8,
    np.dtype(np.uint8): 9,
    np.dtype(np.int16): 10,
    np.dtype(np.uint16): 11,
    np.dtype(np.int32): 12,
    np.dtype(np.uint32): 13,
    np.dtype(np.int64): 14,
    np.dtype(np.uint64): 15,
}
_DT = {v: k for k, v in _CLS.items()}
_COMPLEX = {np.dtype(np.complex64): np.dtype(np.float32), np.dtype(np.complex128): np.dtype(np.float64)}


class MexError(RuntimeError):
    """Raised when a gateway calls mexErrMsgTxt / mexErrMsgIdAndTxt."""


class _Shim:
    _cache: dict = {}

    def __new__(cls, path: str):
        path = os.path.realpath(path)
        if path in cls._cache:
            return cls._cache[path]
        self = super().__new__(cls)
        lib = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
        lib.mxshim_wrap.restype = ctypes.c_void_p
        lib.mxshim_wrap.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                                    ctypes.c_void_p, ctypes.c_void_p]
        lib.mxshim_call.restype = ctypes.c_int
        lib.mxshim_call.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        lib.mxshim_last_error.restype = ctypes.c_char_p
        lib.mxDestroyArray.argtypes = [ctypes.c_void_p]
        lib.mxGetData.restype = ctypes.c_void_p
        lib.mxGetData.argtypes = [ctypes.c_void_p]
        lib.mxGetImagData.restype = ctypes.c_void_p
        lib.mxGetImagData.argtypes = [ctypes.c_void_p]
        lib.mxGetNumberOfDimensions.restype = ctypes.c_size_t
        lib.mxGetNumberOfDimensions.argtypes = [ctypes.c_void_p]
        lib.mxGetDimensions.restype = ctypes.POINTER(ctypes.c_size_t)
        lib.mxGetDimensions.argtypes = [ctypes.c_void_p]
        lib.mxGetClassID.restype = ctypes.c_int
        lib.mxGetClassID.argtypes = [ctypes.c_void_p]
        self.lib = lib
        cls._cache[path] = self
        return self


class MexFunction:
    """A MEX gateway loaded from ``so_path`` (shim looked up beside it)."""

    def __init__(self, so_path: str, shim_path: str | None = None):
        if not os.path.exists(so_path):
            raise FileNotFoundError(so_path)
        shim_path = shim_path or os.path.join(os.path.dirname(so_path), "libmexshim.so")
        if not os.path.exists(shim_path):
            shim_path = os.path.join(os.path.dirname(os.path.dirname(so_path)), "libmexshim.so")
        self._shim = _Shim(shim_path)
        self._lib = ctypes.CDLL(os.path.realpath(so_path))
        self._fn = ctypes.cast(self._lib.mexFunction, ctypes.c_void_p)
        self.name = os.path.splitext(os.path.basename(so_path))[0]

    # -- marshalling -------------------------------------------------------
    def _wrap(self, v, keep: list):
        lib = self._shim.lib
        if v is None:
            v = np.zeros((0, 0), np.float64)
        if isinstance(v, (bool, int, float)) and not isinstance(v, np.generic):
            v = np.array([[float(v)]], np.float64)
        v = np.asarray(v)
        if v.ndim == 0:
            v = v.reshape(1, 1)
        if v.ndim == 1:
            v = v.reshape(1, -1)  # MATLAB row vector
        imag = None
        if v.dtype in _COMPLEX:
            base = _COMPLEX[v.dtype]
            real = np.asfortranarray(v.real.astype(base))
            imag = np.asfortranarray(v.imag.astype(base))
        else:
            real = np.asfortranarray(v)
        if real.dtype not in _CLS:
            raise TypeError(f"unsupported dtype {real.dtype}")
        keep.append(real)
        if imag is not None:
            keep.append(imag)
        dims = (ctypes.c_size_t * real.ndim)(*real.shape)
        return lib.mxshim_wrap(_CLS[real.dtype], real.ndim, dims,
                               real.ctypes.data if real.size else None,
                               imag.ctypes.data if (imag is not None and imag.size) else None)

    def _unwrap(self, a) -> np.ndarray:
        lib = self._shim.lib
        nd = lib.mxGetNumberOfDimensions(a)
        dp = lib.mxGetDimensions(a)
        shape = tuple(dp[i] for i in range(nd))
        dt = _DT[lib.mxGetClassID(a)]
        n = int(np.prod(shape)) if shape else 0
        def grab(ptr):
            if not ptr or n == 0:
                return np.zeros(shape, dt, order="F")
            buf = (ctypes.c_char * (n * dt.itemsize)).from_address(ptr)
            return np.frombuffer(buf, dtype=dt).copy().reshape(shape, order="F")
        re = grab(lib.mxGetData(a))
        ip = lib.mxGetImagData(a)
        if ip:
            return re + 1j * grab(ip)
        return re

    def __call__(self, *args, nlhs: int = 1):
        lib = self._shim.lib
        keep: list = []
        wrapped = [self._wrap(a, keep) for a in args]
        prhs = (ctypes.c_void_p * max(1, len(wrapped)))(*wrapped)
        plhs = (ctypes.c_void_p * max(1, nlhs))()
        try:
            rc = lib.mxshim_call(self._fn, nlhs, plhs, len(wrapped), prhs)
            if rc != 0:
                raise MexError(f"{self.name}: {lib.mxshim_last_error().decode()}")
            outs = []
            for i in range(nlhs):
                if plhs[i]:
                    outs.append(self._unwrap(plhs[i]))
                    lib.mxDestroyArray(plhs[i])
                else:
                    outs.append(None)
        finally:
            for w in wrapped:
                lib.mxDestroyArray(w)
        return outs[0] if nlhs == 1 else tuple(outs)


def load_dir(directory: str, names: Sequence[str] | None = None) -> dict:
    """Loads every ``<name>.so`` MEX file of a directory into a dict."""
    out = {}
    for fn in sorted(os.listdir(directory)):
        if not fn.endswith(".so") or fn.startswith("lib"):
            continue
        name = fn[:-3]
        if names is None or name in names:
            out[name] = MexFunction(os.path.join(directory, fn))
    return out
