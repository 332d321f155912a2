"""ctypes binding of libmonalisa_gpu.so (include/monalisa_gpu.h).

The library is built in-tree by ``monalisa_b200.build`` into
``monalisa_b200/_lib``.  There is no CPU fallback: if the library is missing
or no CUDA device is present, calls raise.
"""
from __future__ import annotations

import ctypes
import os

_LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib")
LIB_PATH = os.path.join(_LIB_DIR, "libmonalisa_gpu.so")

MLG_OK = 0
MLG_KERNEL_GAUSS = 0
MLG_KERNEL_KAISER = 1
MLG_LAYOUT_CC, MLG_LAYOUT_CR, MLG_LAYOUT_RC, MLG_LAYOUT_RR = 0, 1, 2, 3

c_int, c_float, c_double, c_ll, c_vp = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_longlong, ctypes.c_void_p
P_f = ctypes.POINTER(ctypes.c_float)
P_i = ctypes.POINTER(ctypes.c_int)
P_d = ctypes.POINTER(ctypes.c_double)
P_ll = ctypes.POINTER(ctypes.c_longlong)

# name -> argtypes (all return int unless listed in _RESTYPE)
SIGNATURES = {
    "mlg_version": [],
    "mlg_status_string": [c_int],
    "mlg_last_error": [],
    "mlg_set_device": [c_int],
    "mlg_kernel_launch_count": [],
    "mlg_gridder_n2u_leight": [c_int, P_f, P_f, P_f, P_f, P_f, P_f, c_int, c_int, c_int, c_int, c_int, c_int,
                               c_float, c_float, P_f, P_f],
    "mlg_gridder_n2u": [P_f, P_f, P_f, P_i, c_int, c_int, c_int, c_int, P_f, P_f],
    "mlg_gridder_n2u_leight_noalloc": [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int,
                                       c_int, c_float, c_float, c_vp, c_vp, c_vp],
    "mlg_sparsemat_vec_cC": [c_int, P_i, P_i, P_f, c_int, P_i, c_int, P_f, P_f, c_int, P_f, P_f],
    "mlg_sparsemat_vec_cR": [c_int, P_i, P_i, P_f, c_int, P_i, c_int, P_f, P_f, c_int, P_f, P_f],
    "mlg_sparsemat_vec_rC": [c_int, P_i, P_i, P_f, c_int, P_i, c_int, P_f, c_int, P_f],
    "mlg_sparsemat_r_nJump2index": [c_int, P_i, c_ll, P_i],
    "mlg_sparsemat_vec_rR": [c_int, P_i, P_i, P_f, c_int, P_i, c_int, P_f, c_int, P_f],
    "mlg_sparsemat_vec": [c_int, c_int, P_i, P_i, P_f, c_int, P_i, c_int, c_int, P_i, P_i, P_ll, P_f, P_f, c_int, P_f,
                          P_f],
    "mlg_matrix_create_blocks": [c_int, P_i, P_i, P_f, c_int, P_i, c_int, c_int, P_i, P_i, P_ll,
                                 ctypes.POINTER(c_vp)],
    "mlg_matrix_create": [c_int, P_i, P_i, P_f, c_int, P_i, c_int, ctypes.POINTER(c_vp)],
    "mlg_matrix_destroy": [c_vp],
    "mlg_matrix_info": [c_vp, P_ll, P_i, P_i],
    "mlg_matrix_row_stats": [c_vp, P_i, P_i],
    "mlg_plan_profile": [c_vp, c_int, P_d],
    "mlg_plan_set_adjoint": [c_vp, c_int],
    "mlg_plan_get_adjoint": [c_vp, P_i],
    "mlg_plan_autotune": [c_vp, c_int, P_d],
    "mlg_plan_set_variant": [c_vp, c_int, c_int, c_int],
    "mlg_plan_get_variant": [c_vp, P_i, P_i, P_i],
    "mlg_plan_autotune_variants": [c_vp, c_int, P_d],
    "mlg_plan_set_precision": [c_vp, c_int],
    "mlg_plan_get_precision": [c_vp, P_i],
    "mlg_plan_get_half_intermediate": [c_vp, P_i],
    "mlg_matrix_download": [c_vp, P_i, P_i, P_f, P_i, P_i],
    "mlg_matrix_spmm_dev": [c_vp, c_vp, c_int, c_vp, c_vp],
    "mlg_traj2sparsemat": [c_int, c_int, P_d, P_d, P_i, P_d, c_int, c_int, P_d, ctypes.POINTER(c_vp),
                           ctypes.POINTER(c_vp)],
    "mlg_deapodization": [c_int, P_i, P_d, c_int, c_int, P_d, P_f],
    "mlg_deapodization_dev": [c_int, P_i, P_d, c_int, c_int, P_d, c_vp, c_vp],
    "mlg_volume_element_radial_dev": [c_int, c_int, c_int, c_vp, c_vp, c_vp],
    "mlg_plan_create": [c_int, P_i, P_i, c_int, c_vp, c_vp, P_f, P_f, P_f, P_f, ctypes.POINTER(c_vp)],
    "mlg_plan_destroy": [c_vp],
    "mlg_plan_set_dk": [c_vp, P_d],
    "mlg_plan_device_bytes": [c_vp, P_ll],
    "mlg_plan_status": [c_vp],
    "mlg_shanna_dev": [c_vp, c_vp, c_int, c_vp, c_vp],
    "mlg_nakatsha_dev": [c_vp, c_vp, P_f, c_float, c_vp, c_vp],
    "mlg_shanna": [c_int, P_i, P_i, c_int, P_f, P_f, c_int, P_f, P_f, c_int, P_i, P_i, P_f, c_int, P_i, c_int,
                   P_f, P_f],
    "mlg_nakatsha": [c_int, P_i, P_i, c_int, P_f, P_f, P_f, P_f, c_int, P_i, P_i, P_f, c_int, P_i, c_int, P_f, P_f],
    "mlg_idf": [c_int, P_i, P_f, c_int, P_f, P_f, P_f, P_f],
    "mlg_sensa_dev": [c_vp, c_vp, P_f, c_float, c_int, c_int, c_vp, P_d, c_vp],
    "mlg_sensa": [c_vp, P_f, P_f, P_f, c_float, c_int, c_int, P_f, P_f, P_d],
    "mlg_plan_create_sharing": [c_vp, c_vp, c_vp, ctypes.POINTER(c_vp)],
    "mlg_chain_create": [c_int, ctypes.POINTER(c_vp), ctypes.POINTER(c_vp)],
    "mlg_chain_destroy": [c_vp],
    "mlg_chain_info": [c_vp, P_i, P_ll, P_ll],
    "mlg_tevamorphosia_dev": [c_vp, c_vp, P_f, c_float, P_f, P_f, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_int, P_d,
                              c_vp],
    "mlg_tevamorphosia": [c_vp, P_f, P_f, P_f, c_float, P_f, P_f, c_int, c_int, c_int, P_f, P_f, P_d],
    "mlg_traj2sparsemat3": [c_int, c_int, P_d, P_d, P_i, P_d, c_int, c_int, P_d, ctypes.POINTER(c_vp),
                            ctypes.POINTER(c_vp), ctypes.POINTER(c_vp)],
    "mlg_gridder_n2u_leight_dev": [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int,
                                   c_int, c_float, c_float, c_vp, c_vp, c_vp],
    "mlg_gridded_tail_dev": [c_int, P_i, P_i, P_f, c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    "mlg_steva_dev": [c_vp, c_vp, P_f, c_float, P_f, P_f, c_int, c_int, c_vp, c_vp, c_vp, c_int, P_d, c_vp],
    "mlg_steva": [c_vp, P_f, P_f, P_f, c_float, P_f, P_f, c_int, c_int, P_f, P_f, P_d],
    "mlg_deform2sparsemat": [c_int, P_i, P_d, P_d, c_int, ctypes.POINTER(c_vp), ctypes.POINTER(c_vp),
                             ctypes.POINTER(c_vp)],
    "mlg_chain_set_deform": [c_vp, ctypes.POINTER(c_vp), ctypes.POINTER(c_vp)],
}
_RESTYPE = {"mlg_status_string": ctypes.c_char_p, "mlg_last_error": ctypes.c_char_p,
            "mlg_kernel_launch_count": c_ll}


class MonalisaError(RuntimeError):
    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} failed with status {status}: {msg}")
        self.status = status


_lib = None


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m monalisa_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, argt in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = argt
            f.restype = _RESTYPE.get(name, c_int)
        _lib = L
    return _lib


def call(name: str, *args) -> None:
    """Calls ``name`` and raises MonalisaError on a non-zero status."""
    st = getattr(lib(), name)(*args)
    if st != MLG_OK:
        raise MonalisaError(name, st, lib().mlg_last_error().decode(errors="replace"))


def launch_count() -> int:
    return int(lib().mlg_kernel_launch_count())


def fptr(a):
    """float* of a contiguous float32 numpy array (None for empty / None)."""
    if a is None or a.size == 0:
        return None
    assert a.dtype.name == "float32" and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(P_f)


def iptr(a):
    if a is None or a.size == 0:
        return None
    assert a.dtype.name == "int32" and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(P_i)


def dptr(a):
    if a is None or a.size == 0:
        return None
    assert a.dtype.name == "float64" and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(P_d)


def llptr(a):
    if a is None or a.size == 0:
        return None
    assert a.dtype.name == "int64" and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(P_ll)


def tptr(t):
    """Device pointer of a CUDA torch tensor (None for None)."""
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return ctypes.c_void_p(t.data_ptr())


def tfptr(t):
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous()
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), P_f)


def stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
