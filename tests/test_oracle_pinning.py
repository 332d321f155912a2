"""Pins the oracle before it is trusted as the checker.

* The plain-C restatement (oracle/_lib/liboracle.so) must reproduce the golden
  fixtures bit for bit; the fixtures were produced by the Monalisa reference's
  own C++ MEX kernels (tests/golden/make_golden.py).
* Where the compiled reference kernels are present (oracle/_ref), fresh
  random cases are compared live as well.
* The numpy restatement of the MATLAB layers is checked against the golden
  operator fixture (which used the reference's SpMV kernel) and against
  mathematical identities of the operators.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="session", autouse=True)
def _build_port():
    if not os.path.exists(oracle.LIB_PATH):
        subprocess.run(["make", "-C", oracle.ORACLE_DIR, "port"], check=True, capture_output=True)


def _load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def _sparse(g, tag):
    return oracle.SparseMat(r_size=int(g[f"{tag}_G_r_size"]), l_size=int(g[f"{tag}_G_l_size"]),
                            r_nJump=g[f"{tag}_G_r_nJump"], m_val=g[f"{tag}_G_m_val"],
                            r_jump=g[f"{tag}_G_r_jump"], l_jump=g[f"{tag}_G_l_jump"],
                            l_nJump=int(g[f"{tag}_G_l_nJump"]))


@pytest.mark.parametrize("name", ["leight1_gauss", "leight2_gauss", "leight2_even", "leight3_gauss"])
def test_port_leight_matches_golden_bitwise(name):
    g = _load(name)
    imDim, N, t = int(g["imDim"]), int(g["N"]), g["t"]
    bR, bI = oracle.port_gridder_leight(imDim, g["aR"], g["aI"], t[0], t[1] if imDim > 1 else None,
                                        t[2] if imDim > 2 else None, g["Dn"], int(g["nCh"]), int(g["nPt"]),
                                        N, N, N, int(g["nWin"]), float(g["sigma"]), 10.0)
    assert np.array_equal(bR, g["bR"]) and np.array_equal(bI, g["bI"])


def test_port_n2u_matches_golden_bitwise():
    g = _load("n2u_kaiser")
    bR, bI = oracle.port_gridder_n2u(g["aR"], g["aI"], g["w"], g["nJump"], int(g["nCh"]), int(g["nNb"]),
                                     int(g["nPt"]), int(g["Nu_tot"]))
    assert np.array_equal(bR, g["bR"]) and np.array_equal(bI, g["bI"])


@pytest.mark.parametrize("tag", ["u", "t"])
def test_port_spmv_matches_golden_bitwise(tag):
    g = _load("spmv")
    G = _sparse(g, tag)
    v = g["v_" + tag]
    w = oracle.port_spmv(G, v, "C")
    assert np.array_equal(w, g[f"{tag}_bmSparseMat_cC_oBlock_omp_mex"])
    assert np.array_equal(w, g[f"{tag}_bmSparseMat_cC_oBlock_mex"])
    assert np.array_equal(oracle.port_spmv(G, v.T, "R"), g[f"{tag}_bmSparseMat_cR_oBlock_mex"])


def test_r_nJump2index_golden():
    g = _load("spmv")
    G = _sparse(g, "u")
    out = np.zeros(int(G.r_nJump.sum()), np.int32)
    n = oracle.port().oracle_r_nJump2index(oracle._ip(G.r_nJump), int(G.l_nJump), oracle._ip(out))
    assert n == out.size
    assert np.array_equal(out, g["r_nJump2index"].ravel())


def test_restated_matrix_builder_matches_golden_matrix():
    """The numpy bmTraj2SparseMat reproduces the stored Gu/Gut exactly."""
    g = _load("spmv")
    G = oracle.traj2sparsemat(g["t"], g["ve"], [16, 16], [1, 1], "gauss", 3, [0.61, 10])
    for tag, key in (("u", "Gu"), ("t", "Gut")):
        ref = _sparse(g, tag)
        assert np.array_equal(G[key].r_jump, ref.r_jump)
        assert np.array_equal(G[key].r_nJump, ref.r_nJump)
        assert np.array_equal(G[key].m_val, ref.m_val)
        assert np.array_equal(G[key].l_jump, ref.l_jump)


def test_restated_operators_match_golden():
    """Shanna/Nakatsha/CG-SENSE restatements with the C-port SpMV reproduce
    the fixture made with the reference's SpMV kernel."""
    g = _load("operators2d")
    n_u, N_u = g["n_u"], g["N_u"]
    G = oracle.traj2sparsemat(g["t"], g["ve"], N_u, [1, 1], "kaiser", 3, [1.95, 10, 10])
    yS = oracle.bmShanna(g["x"], G["Gu"], g["KFC"], n_u)
    xN = oracle.bmNakatsha(g["y"], G["Gut"], g["KFC_conj"], True, n_u)
    assert np.array_equal(yS, g["shanna"])
    assert np.array_equal(xN, g["nakatsha"])
    hist = []
    xs = oracle.bmSensa(np.zeros(n_u.prod(), np.complex64), g["y"], g["ve"], g["C"], G["Gu"], G["Gut"], n_u,
                        5, 10.0, 1, history=hist)
    assert np.array_equal(xs, g["sensa"])
    assert np.allclose(hist, g["sensa_residual"], rtol=0, atol=0)


@pytest.mark.skipif(not oracle.ref_available(), reason="compiled reference kernels absent")
def test_port_matches_live_reference_random():
    rng = np.random.default_rng(7)
    for imDim, N, nCh, nWin in ((2, 24, 4, 3), (3, 10, 2, 3), (2, 20, 1, 5)):
        nPt = 200
        t = rng.uniform(0.5, N + 0.5, (imDim, nPt)).astype(np.float32)
        aR = rng.standard_normal((nCh, nPt)).astype(np.float32)
        aI = rng.standard_normal((nCh, nPt)).astype(np.float32)
        Dn = rng.uniform(0.1, 1, (1, nPt)).astype(np.float32)
        m = oracle.ref_mex(f"bmGridder_n2u_leight{imDim}_mex")
        ref = m(aR, aI, *[t[i][None] for i in range(imDim)], Dn, np.int32(nCh), np.int32(nPt),
                *[np.int32(N)] * imDim, np.int32(nWin), np.float32(0.61), np.float32(10), nlhs=2)
        got = oracle.port_gridder_leight(imDim, aR, aI, t[0], t[1], t[2] if imDim > 2 else None, Dn, nCh, nPt,
                                         N, N, N, nWin, 0.61, 10.0)
        assert np.array_equal(ref[0], got[0]) and np.array_equal(ref[1], got[1])


def test_matrix_rows_normalised_and_transpose():
    rng = np.random.default_rng(3)
    t = rng.uniform(-7.5, 7.5, (3, 300))
    G = oracle.traj2sparsemat(t, np.ones(300), [16, 16, 16], [1, 1, 1], "kaiser", 3, [1.95, 10, 10])
    A = G["Gu"].to_scipy().astype(np.float64)
    B = G["Gut"].to_scipy().astype(np.float64)
    s = np.asarray(A.sum(axis=1)).ravel()
    nonempty = np.diff(A.indptr) > 0
    assert np.allclose(s[nonempty], 1.0, atol=1e-6)  # samples outside the grid keep empty rows
    assert nonempty.sum() < 300
    assert abs(A - B.T).max() == 0


def test_operator_adjointness():
    """<Shanna x, y> == <x, Nakatsha y> (Gut = Gu^T, KFC_conj = conj(KFC)*prod(N_u))."""
    g = _load("operators2d")
    n_u, N_u = g["n_u"], g["N_u"]
    G = oracle.traj2sparsemat(g["t"], g["ve"], N_u, [1, 1], "kaiser", 3, [1.95, 10, 10])
    x = g["x"].astype(np.complex64)
    y = g["y"]
    lhs = np.vdot(oracle.bmShanna(x, G["Gu"], g["KFC"], n_u).astype(np.complex128), y)
    xn = oracle.bmNakatsha(y, G["Gut"], g["KFC_conj"], False, n_u)
    rhs = np.vdot(np.repeat(x[:, None], 2, 1).astype(np.complex128), xn)
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_deapodisation_is_inverse_kernel_transform():
    K = oracle.bmK([32, 32], [1, 1], 1, "gauss", 3, [0.61, 10])[:, 0].reshape(32, 32, order="F")
    assert K.min() >= 1.0 - 1e-6 and K.max() <= 10.0 + 1e-6
    assert abs(K[16, 16] - 1.0) < 1e-6  # kernel transform is maximal at the centre


def _random_bm(rng, l_size, r_size, density, squeeze, mode, f=(1.5, 6)):
    """A random sparse matrix with some empty rows, prepared as the reference
    does (matlabSparse2bmSparseMat, optional l_squeeze, cpp_prepare)."""
    import scipy.sparse as sp

    a = sp.random(l_size, r_size, density=density, random_state=np.random.RandomState(rng.integers(1 << 30)),
                  dtype=np.float32, format="csr")
    a = sp.csr_matrix(a.multiply(rng.random((l_size, 1)) > 0.2))  # empty rows
    a.eliminate_zeros()
    G = oracle.matlab_sparse_to_bm(a, [r_size], [1], "gauss", 3, [0.61, 10])
    if squeeze:
        G = oracle.l_squeeze(G)
    return oracle.cpp_prepare(G, mode, *f), a


def _block_args(G):
    e = G.extra
    return (np.int32(e["nBlock"]), e["block_length"][None], e["l_block_start"][None],
            e["m_block_start"].astype(np.int64)[None])


def _jump(G):
    lj = G.l_jump
    return (np.int32(G.r_size), G.r_jump[None], G.r_nJump[None], G.m_val[None], np.int32(G.l_size),
            lj[None] if lj.size else None, np.int32(G.l_nJump), np.int32(1 if lj.size else 0))


@pytest.mark.skipif(not oracle.ref_available(), reason="compiled reference kernels absent")
@pytest.mark.parametrize("squeeze", [False, True])
def test_multi_block_restatement_matches_reference(squeeze):
    """The multi-block cpp_prepare restatement (bmSparseMat.m:100-188 with
    bmSparseMat_blockPartition.m) fed to the reference's own nBlock kernels
    gives, bit for bit, its one-block kernels' products; and the products
    are the matrix's (float64 check)."""
    rng = np.random.default_rng(31 + squeeze)
    Gm, a = _random_bm(rng, 300, 400, 0.03, squeeze, "multi_block")
    G1, _ = _random_bm(np.random.default_rng(31 + squeeze), 300, 400, 0.03, squeeze, "one_block")
    assert Gm.extra["nBlock"] > 5 and np.array_equal(Gm.m_val, G1.m_val)
    nVec = 3
    v = (rng.standard_normal((nVec, 400)) + 1j * rng.standard_normal((nVec, 400))).astype(np.complex64)
    wm = oracle.ref_mex("bmSparseMat_cR_nBlock_omp_mex")(*_jump(Gm), *_block_args(Gm), v, np.int32(nVec))
    w1 = oracle.ref_mex("bmSparseMat_cR_oBlock_mex")(*_jump(G1), v, np.int32(nVec))
    assert np.array_equal(wm, w1)
    ref = (a.astype(np.float64) @ v.T.astype(np.complex128)).T
    assert np.allclose(wm, ref, rtol=1e-5, atol=1e-5)
    vr = rng.standard_normal((nVec, 400)).astype(np.float32)
    rm = oracle.ref_mex("bmSparseMat_rR_nBlock_omp_mex")(*_jump(Gm), *_block_args(Gm), vr, np.int32(nVec))
    r1 = oracle.ref_mex("bmSparseMat_rR_oBlock_mex")(*_jump(G1), vr, np.int32(nVec))
    assert np.array_equal(rm, r1)
    S = Gm.to_scipy()
    S.sum_duplicates()
    assert (S != a).nnz == 0
