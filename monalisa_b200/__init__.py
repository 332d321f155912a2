"""monalisa_b200 -- B200 (sm_100a) implementation of Monalisa's
non-Cartesian gridding hot path: adjoint/forward gridding, the Gu/Gut
gridding-matrix products, the fused Shanna/Nakatsha operators around cuFFT
and the CG-SENSE reconstruction that calls them.

The compute runs in libmonalisa_gpu.so (include/monalisa_gpu.h); this package
mirrors the reference's MATLAB interface on top of it.
"""
from ._native import MonalisaError, launch_count  # noqa: F401
from .gridding import bmGridder_n2u, bmGridder_n2u_leight  # noqa: F401
from .operators import (NufftPlan, bmCoilSense_pinv, bmIDF, bmK, bmKF, bmKF_conj, bmMathilda,  # noqa: F401
                        bmNakatsha, bmNasha, bmShanna)
from .solvers import SensaRecon, TevaMorphosiaChain, bmSensa, bmSteva, bmTevaMorphosia_chain  # noqa: F401
from .sparsemat import (DeviceMatrix, bmImDeformField2SparseMat, bmSparseMat, bmSparseMat_vec,  # noqa: F401
                        bmTraj2SparseMat)

__all__ = [
    "MonalisaError", "bmGridder_n2u", "bmGridder_n2u_leight", "NufftPlan", "bmIDF", "bmK", "bmKF", "bmKF_conj",
    "bmMathilda", "bmNasha", "bmNakatsha", "bmShanna", "bmCoilSense_pinv", "SensaRecon", "bmSensa", "bmSteva", "TevaMorphosiaChain",
    "bmTevaMorphosia_chain", "DeviceMatrix", "bmSparseMat", "bmSparseMat_vec", "bmTraj2SparseMat",
    "bmImDeformField2SparseMat", "launch_count",
]
