"""Deformation fields on the GPU: the device builder of the
image-deformation matrices (mlg_deform2sparsemat, bmImDeformField2SparseMat.m)
against the oracle's restatement, and the temporal-TV chain with per-frame
Tu / Tut (bmTevaMorphosia_chain.m private_F / private_dagF) against the
oracle chain.

Tolerances: matrix structure identical, values within 1e-6 relative (FP64
weights rounded to FP32 on both sides; CUDA's and numpy's exp may differ in
the last bit of a double); chain images and monitoring history within 1e-4
relative L2 (as for the chain without deformation).  Identity deformation
matrices reproduce the undeformed chain bit for bit.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

from test_gpu_chain import _device_mats, _frames, rel  # noqa: E402


def _smooth_field(n_u, amp, seed):
    """A smooth random displacement field [imDim, prod(n_u)] (pixel units)."""
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.linspace(0, 2 * np.pi, n, endpoint=False) for n in n_u], indexing="ij")
    v = []
    for d in range(len(n_u)):
        f = np.zeros(grids[0].shape)
        for _ in range(3):
            k = rng.integers(0, 3, len(n_u))
            f += rng.standard_normal() * np.cos(sum(kk * g for kk, g in zip(k, grids)) + rng.uniform(0, 2 * np.pi))
        v.append(amp * f.ravel(order="F"))
    return np.stack(v)


def _csr_equal(dev, ref, rtol=1e-6):
    ip, ix, dv = dev.download().to_csr()
    R = ref.to_scipy()
    R.sort_indices()
    assert np.array_equal(ip, R.indptr) and np.array_equal(ix, R.indices)
    den = np.maximum(np.abs(R.data), 1e-30)
    assert np.all(np.abs(dv - R.data) <= rtol * den + 1e-38)


@pytest.mark.parametrize("n_u", [[40], [24, 20], [12, 10, 9]])
@pytest.mark.parametrize("torus", [False, True])
def test_device_builder_matches_oracle(n_u, torus):
    import monalisa_b200 as mb

    nPt = int(np.prod(n_u))
    v = _smooth_field(n_u, 1.7, 5 + len(n_u))
    Dn = np.random.default_rng(1).uniform(0.5, 2.0, nPt)
    ref = oracle.deform2sparsemat(v, n_u, Dn=Dn, torus_flag=torus, want=("Gn", "Gu", "Gut"))
    Gn, Tu, Tut = mb.bmImDeformField2SparseMat(v, n_u, Dn, torus, nargout=3)
    assert Tu.l_size == Tu.r_size == nPt
    _csr_equal(Tu, ref["Gu"])
    _csr_equal(Tut, ref["Gut"])
    _csr_equal(Gn, ref["Gn"])


@pytest.fixture(scope="module")
def case():
    return _frames()


def test_chain_with_deformation_matches_oracle(case):
    import monalisa_b200 as mb

    nFr, n_u = len(case["y"]), case["n_u"]
    nu = int(np.prod(n_u))
    fields = [_smooth_field(n_u, 0.8, 20 + f) for f in range(nFr)]
    T = [oracle.deform2sparsemat(fld, n_u, torus_flag=True) for fld in fields]
    delta, rho, nIter, nCGD, ve_max = 0.02, 0.2, 3, 4, 10.0
    x0 = [(0.9 * xt).astype(np.complex64) for xt in case["x_true"]]
    hist_o = []
    ref = oracle.bmTevaMorphosia_chain(x0, case["y"], case["ve"], case["C"], [g["Gu"] for g in case["G"]],
                                       [g["Gut"] for g in case["G"]], n_u, delta, rho, nCGD, ve_max, nIter,
                                       history=hist_o, Tu=[t["Gu"] for t in T], Tut=[t["Gut"] for t in T])
    Gu, Gut = _device_mats(case)
    Tu, Tut = zip(*[mb.bmImDeformField2SparseMat(fld, n_u, None, True) for fld in fields])
    hist = []
    out = mb.bmTevaMorphosia_chain(x0, None, None, case["y"], case["ve"], case["C"], Gu, Gut, n_u, list(Tu),
                                   list(Tut), delta, rho, "normal", nCGD, ve_max, nIter, hist)
    for f in range(nFr):
        assert rel(out[f].ravel(order="F"), ref[f]) <= 1e-4, f
    for c in range(nIter):
        for k in range(3):
            assert abs(hist[c][k] - hist_o[c][k]) <= 1e-4 * abs(hist_o[c][k]), (c, k)
    # the fields matter: without them the result differs
    plain = oracle.bmTevaMorphosia_chain(x0, case["y"], case["ve"], case["C"], [g["Gu"] for g in case["G"]],
                                         [g["Gut"] for g in case["G"]], n_u, delta, rho, nCGD, ve_max, nIter)
    assert max(rel(out[f].ravel(order="F"), plain[f]) for f in range(nFr)) > 1e-3
    assert nu == out[0].size


def test_identity_deformation_is_bit_identical(case):
    import monalisa_b200 as mb

    nFr, n_u = len(case["y"]), case["n_u"]
    nu = int(np.prod(n_u))
    eye = mb.bmImDeformField2SparseMat(np.zeros((2, nu)), n_u)
    Gu, Gut = _device_mats(case)
    args = ([np.zeros(nu, np.complex64)] * nFr, None, None, case["y"], case["ve"], case["C"], Gu, Gut, n_u)
    tail = (0.02, 0.2, "normal", 3, 10.0, 2)
    h0, h1 = [], []
    a = mb.bmTevaMorphosia_chain(*args, None, None, *tail, h0)
    b = mb.bmTevaMorphosia_chain(*args, [eye[0]] * nFr, [eye[1]] * nFr, *tail, h1)
    for f in range(nFr):
        assert np.array_equal(a[f], b[f])
    assert h0 == h1
