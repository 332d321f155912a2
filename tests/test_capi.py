"""C ABI and host-side logic, no GPU needed (no compute entry point is
called): the library builds and exports every function include/*.h declares,
the MEX gateways load and validate their arguments before touching the GPU,
and the package's host-side helpers behave like the reference's MATLAB."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def built():
    from monalisa_b200 import build

    return build.build()


def _declared():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(mlg_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(built):
    lib = ctypes.CDLL(built)
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from monalisa_b200 import _native

    assert set(_declared()) <= set(_native.SIGNATURES), set(_declared()) - set(_native.SIGNATURES)


def test_library_identity_calls(built):
    from monalisa_b200 import _native as N

    assert N.lib().mlg_version() >= 10000
    assert N.lib().mlg_status_string(-1) == b"invalid argument"
    assert N.lib().mlg_kernel_launch_count() >= 0


def test_mex_gateways_export_mexFunction(built):
    mexdir = os.path.join(ROOT, "monalisa_b200", "_lib", "mex")
    from monalisa_b200.build import GATEWAYS

    for name in GATEWAYS:
        lib = ctypes.CDLL(os.path.join(mexdir, name + ".so"))
        assert hasattr(lib, "mexFunction"), name


def test_mex_gateway_rejects_bad_argument_lists(built):
    from monalisa_b200.mexcall import MexError, MexFunction

    mexdir = os.path.join(ROOT, "monalisa_b200", "_lib", "mex")
    m = MexFunction(os.path.join(mexdir, "bmGridder_n2u_mex.so"))
    with pytest.raises(MexError, match="wrong number of arguments"):
        m(np.zeros((1, 3), np.float32), nlhs=2)
    s = MexFunction(os.path.join(mexdir, "bmShanna3_CUFFT_omp_mex.so"))
    with pytest.raises(MexError, match="N_u must be int32"):
        s(*([np.zeros((8, 1), np.float32)] * 4), np.array([[2.0, 2.0, 2.0]]), *([np.int32(1)] * 7), nlhs=2)


def test_kernel_defaults_match_reference():
    from monalisa_b200.sparsemat import kernel_defaults

    kt, nw, kp = kernel_defaults()
    assert kt == "gauss" and nw == 3 and np.allclose(kp, [0.61, 10])
    assert kp[0] == np.float32(0.61)  # parameters pass through single precision
    kt, nw, kp = kernel_defaults("kaiser")
    assert nw == 3 and np.allclose(kp, [1.95, 10, 10])
    with pytest.raises(ValueError):
        kernel_defaults("gauss", 3, [1, 2, 3])


def test_trajectory_generators():
    from monalisa_b200 import traj

    t = traj.bmTraj_fullRadial3_phyllotaxis_lineAssym2(16, 20, 1, 1.0)
    assert t.shape == (3, 320)
    r = np.sqrt((t ** 2).sum(0)).reshape(16, 20, order="F")
    assert np.allclose(r[8], 0) and np.allclose(r[0], 8)  # lines through the centre, radius N/2
    t2 = traj.bmTraj_fullRadial2_lineAssym2(32, 10, 1.0)
    assert t2.shape == (2, 320) and np.isclose(np.abs(t2).max(), 16)
    ve = traj.bmVolumeElement_voronoi_full_radial2(t2, 32)
    assert ve.shape == (320,) and (ve > 0).all()
    ve3 = traj.bmVolumeElement_full_radial3(t)
    assert ve3.shape == (320,) and (ve3 > 0).all()


def test_volume_element_1d_matches_restatement():
    import sys

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from monalisa_b200 import traj

    x = np.sort(np.random.default_rng(1).uniform(-1, 1, 50))
    v = traj.bmVolumeElement1(x).ravel()
    mid = (x[1:] + x[:-1]) / 2
    edges = np.concatenate([[x[0] - (mid[0] - x[0])], mid, [x[-1] + (x[-1] - mid[-1])]])
    assert np.allclose(v, np.diff(edges))


def test_to_csr_decodes_the_jump_format():
    """bmSparseMat.to_csr (product) against the oracle's decoder, for a
    row-complete Gu and an l-squeezed Gut."""
    import oracle
    from monalisa_b200 import bmSparseMat

    rng = np.random.default_rng(17)
    t = rng.uniform(-6, 6, (2, 300))
    G = oracle.traj2sparsemat(t, np.ones(300), [12, 12], [1, 1], "gauss", 3, [0.61, 10])
    for name in ("Gu", "Gut"):
        M = G[name]
        ref = M.to_scipy()
        ref.sum_duplicates()
        b = bmSparseMat(r_size=M.r_size, r_jump=M.r_jump, r_nJump=M.r_nJump, m_val=M.m_val, l_size=M.l_size,
                        l_jump=M.l_jump, l_nJump=M.l_nJump)
        indptr, indices, data = b.to_csr()
        assert np.array_equal(indptr, ref.indptr) and np.array_equal(indices, ref.indices)
        assert np.array_equal(data, ref.data)
