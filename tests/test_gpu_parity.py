"""Parity of the CUDA path with the oracle (GPU tests).

Every call goes through libmonalisa_gpu.so: either the MEX gateways (the
drop-in boundary, called through the MEX-API shim) or the package API that
wraps the C ABI.  Tolerances:
* sparse products and the precomputed-weight gridder: bit-exact (the kernels
  keep the reference's per-row accumulation order, no FMA contraction);
* on-the-fly gridder (cell-binned gather: each cell sums its samples in its
  own fixed order, CUDA expf): relative L2 <= 1e-5;
* FFT-based operators: relative L2 <= 1e-5 against the FP32 oracle;
* CG-SENSE: relative L2 <= 1e-4 after 5 iterations (FP32 data, FP64 scalars
  on both sides).
"""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def mex():
    from monalisa_b200 import build
    from monalisa_b200.mexcall import load_dir

    build.build()
    return load_dir(os.path.join(os.path.dirname(build.__file__), "_lib", "mex"))


@pytest.fixture(scope="module", autouse=True)
def _port():
    import subprocess

    if not os.path.exists(oracle.LIB_PATH):
        subprocess.run(["make", "-C", oracle.ORACLE_DIR, "port"], check=True, capture_output=True)


def _g(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def _sparse_args(g, tag):
    lj = g[f"{tag}_G_l_jump"]
    return (np.int32(g[f"{tag}_G_r_size"]), g[f"{tag}_G_r_jump"][None], g[f"{tag}_G_r_nJump"][None],
            g[f"{tag}_G_m_val"][None], np.int32(g[f"{tag}_G_l_size"]), lj[None] if lj.size else None,
            np.int32(g[f"{tag}_G_l_nJump"]), np.int32(1 if lj.size else 0))


@pytest.mark.parametrize("tag", ["u", "t"])
def test_spmv_gateways_bitexact(mex, tag):
    g = _g("spmv")
    v = g["v_" + tag]
    args = _sparse_args(g, tag)
    for name in ("bmSparseMat_cC_oBlock_omp_mex", "bmSparseMat_cC_oBlock_mex"):
        wR, wI = mex[name](*args, np.ascontiguousarray(v.real), np.ascontiguousarray(v.imag), np.int32(v.shape[1]),
                           nlhs=2)
        assert np.array_equal(wR + 1j * wI, g[f"{tag}_{name}"]), name
    w = mex["bmSparseMat_cR_oBlock_mex"](*args, np.ascontiguousarray(v.T), np.int32(v.shape[1]), nlhs=1)
    assert np.array_equal(w, g[f"{tag}_bmSparseMat_cR_oBlock_mex"])
    w = mex["bmSparseMat_rC_oBlock_mex"](*args, np.ascontiguousarray(v.real), np.int32(v.shape[1]), nlhs=1)
    assert np.array_equal(w, g[f"{tag}_bmSparseMat_rC_oBlock_mex"])


def test_r_nJump2index_gateway(mex):
    g = _g("spmv")
    idx, chk = mex["bmSparseMat_r_nJump2index_mex"](np.int32(g["u_G_l_size"]), g["u_G_r_nJump"][None],
                                                     np.int64(g["u_G_r_nJump"].sum()), nlhs=2)
    assert np.array_equal(idx.ravel(), g["r_nJump2index"].ravel())
    assert int(chk.ravel()[0]) == g["u_G_r_nJump"].sum()


@pytest.mark.parametrize("name", ["leight1_gauss", "leight2_gauss", "leight2_even", "leight3_gauss"])
def test_leight_gateways_match_golden(mex, name):
    g = _g(name)
    imDim, N = int(g["imDim"]), int(g["N"])
    t = g["t"]
    nCh, nPt, nWin, sigma = int(g["nCh"]), int(g["nPt"]), int(g["nWin"]), float(g["sigma"])
    m = mex[f"bmGridder_n2u_leight{imDim}_mex"]
    ts = [t[i][None] for i in range(imDim)]
    bR, bI = m(g["aR"], g["aI"], *ts, g["Dn"], np.int32(nCh), np.int32(nPt), *[np.int32(N)] * imDim,
               np.int32(nWin), np.float32(sigma), np.float32(10), nlhs=2)
    assert rel(bR + 1j * bI, g["bR"] + 1j * g["bI"]) <= 1e-5
    if imDim == 1:  # the reference's own gapped 12-argument layout
        bR2, bI2 = m(g["aR"], g["aI"], ts[0], None, g["Dn"], np.int32(nCh), np.int32(nPt), np.int32(N), None,
                     np.int32(nWin), np.float32(sigma), np.float32(10), nlhs=2)
        assert rel(bR2 + 1j * bI2, g["bR"] + 1j * g["bI"]) <= 1e-5


def test_n2u_gateway_bitexact(mex):
    g = _g("n2u_kaiser")
    bR, bI = mex["bmGridder_n2u_mex"](g["aR"], g["aI"], g["w"][None], g["nJump"][None], np.int32(g["nCh"]),
                                      np.int32(g["nNb"]), np.int32(g["nPt"]), np.int32(g["Nu_tot"]), nlhs=2)
    assert np.array_equal(bR, g["bR"]) and np.array_equal(bI, g["bI"])


def _radial3(nSpoke, nRead, N, seed):
    from monalisa_b200 import traj

    return traj.bmTraj_fullRadial3_phyllotaxis_lineAssym2(nRead, nSpoke, 1, N / nRead)


def _dense_case(imDim, N, nCh, nPt, seed):
    rng = np.random.default_rng(seed)
    # half the points crowd the centre, half spread out, some outside
    t = np.concatenate([rng.normal(N / 2 + 1, 1.5, (imDim, nPt // 2)),
                        rng.uniform(-1, N + 2, (imDim, nPt - nPt // 2))], 1).astype(np.float32)
    aR = rng.standard_normal((nCh, nPt)).astype(np.float32)
    aI = rng.standard_normal((nCh, nPt)).astype(np.float32)
    Dn = rng.uniform(0.1, 1, nPt).astype(np.float32)
    return t, aR, aI, Dn


@pytest.mark.parametrize("imDim,N,nCh,nWin,nPt", [(3, 32, 4, 3, 60000), (2, 96, 3, 3, 120000), (3, 24, 1, 4, 8000),
                                                  (2, 40, 16, 5, 20000), (1, 64, 2, 3, 5000),
                                                  (3, 32, 16, 3, 60000), (3, 24, 12, 3, 30000),
                                                  (3, 32, 5, 3, 60000), (3, 24, 6, 3, 30000), (2, 64, 7, 3, 40000),
                                                  (3, 20, 8, 2, 20000)])
def test_leight_heavy_bins_match_port(imDim, N, nCh, nWin, nPt):
    """Dense central sampling: cells covered by more than 64 samples take a
    warp or (beyond 2048) a CTA each, the rest a thread per (cell, coil
    group) with 1 to 8 coils per thread; 3-wide windows in 2-D and 3-D have
    their own compiled forms.  Compared with the bit-exact C restatement."""
    from monalisa_b200 import _native as NN

    t, aR, aI, Dn = _dense_case(imDim, N, nCh, nPt, 11 + imDim)
    ref = oracle.port_gridder_leight(imDim, aR, aI, t[0], t[1] if imDim > 1 else None, t[2] if imDim > 2 else None,
                                     Dn, nCh, nPt, N, N, N, nWin, 0.61, 10.0)
    Ns = [N if d < imDim else 1 for d in range(3)]
    nu = int(np.prod(Ns))
    bR = np.zeros((nu, nCh), np.float32)
    bI = np.zeros((nu, nCh), np.float32)
    tt = [np.ascontiguousarray(t[d]) if d < imDim else None for d in range(3)]
    NN.call("mlg_gridder_n2u_leight", imDim, NN.fptr(np.ascontiguousarray(aR.T)), NN.fptr(np.ascontiguousarray(aI.T)),
            NN.fptr(tt[0]), NN.fptr(tt[1]), NN.fptr(tt[2]), NN.fptr(Dn), nCh, nPt, Ns[0], Ns[1], Ns[2], nWin,
            0.61, 10.0, NN.fptr(bR), NN.fptr(bI))
    assert rel(bR + 1j * bI, (ref[0] + 1j * ref[1]).T) <= 1e-5


@pytest.mark.parametrize("shift", [0, 1])
def test_leight_device_entry_deterministic_and_unaligned(shift):
    """The device-buffer entry: repeated calls give bit-identical grids (the
    samples are binned by a stable sort, each cell sums in a fixed order);
    buffers one float off 16-byte alignment fall back to scalar coil access
    with the same result."""
    import torch

    from monalisa_b200 import _native as NN

    imDim, N, nCh, nWin, nPt = 3, 32, 16, 3, 60000
    t, aR, aI, Dn = _dense_case(imDim, N, nCh, nPt, 21)
    ref = oracle.port_gridder_leight(imDim, aR, aI, t[0], t[1], t[2], Dn, nCh, nPt, N, N, N, nWin, 0.61, 10.0)

    def dev(a):  # a device copy starting `shift` floats into its allocation
        buf = torch.zeros(a.size + shift, dtype=torch.float32, device="cuda")
        buf[shift:] = torch.from_numpy(np.ascontiguousarray(a).ravel()).cuda()
        return buf, buf[shift:]

    keep = [dev(aR.T), dev(aI.T), dev(t[0]), dev(t[1]), dev(t[2]), dev(Dn)]
    d = [v for _, v in keep]
    nu = N ** 3
    outs = []
    for _ in range(2):
        bR, bI = dev(np.zeros(nu * nCh, np.float32))[1], dev(np.zeros(nu * nCh, np.float32))[1]
        NN.call("mlg_gridder_n2u_leight_dev", imDim, *[NN.tptr(x) for x in d], nCh, nPt, N, N, N, nWin, 0.61, 10.0,
                NN.tptr(bR), NN.tptr(bI), NN.stream_ptr())
        torch.cuda.synchronize()
        outs.append((bR.cpu().numpy().reshape(nu, nCh), bI.cpu().numpy().reshape(nu, nCh)))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    assert rel(outs[0][0] + 1j * outs[0][1], (ref[0] + 1j * ref[1]).T) <= 1e-5


def test_leight_empty_input():
    from monalisa_b200 import _native as NN

    bR = np.full((64, 2), 7, np.float32)
    bI = np.full((64, 2), 7, np.float32)
    NN.call("mlg_gridder_n2u_leight", 2, None, None, None, None, None, None, 2, 0, 8, 8, 1, 3, 0.61, 10.0,
            NN.fptr(bR), NN.fptr(bI))
    assert not bR.any() and not bI.any()


def test_sparse_long_rows_match_port():
    """Gut of a dense radial trajectory has centre rows with thousands of
    entries (CTA-split path); Gu rows stay short (bit-exact path)."""
    import monalisa_b200 as mb

    t = _radial3(400, 32, 32, 0)
    G = oracle.traj2sparsemat(t, np.ones(t.shape[1]), [32, 32, 32], [1, 1, 1], "gauss", 3, [0.61, 10])
    Gut = G["Gut"]
    assert Gut.r_nJump.max() > 256
    rng = np.random.default_rng(5)
    v = (rng.standard_normal((Gut.r_size, 3)) + 1j * rng.standard_normal((Gut.r_size, 3))).astype(np.complex64)
    w_ref = oracle.port_spmv(Gut, v, "C")
    Gb = mb.bmSparseMat(r_size=Gut.r_size, r_jump=Gut.r_jump, r_nJump=Gut.r_nJump, m_val=Gut.m_val,
                        l_size=Gut.l_size, l_jump=Gut.l_jump, l_nJump=Gut.l_nJump)
    w = mb.bmSparseMat_vec(Gb, v)
    assert rel(w, w_ref) <= 1e-6
    short = np.zeros(Gut.l_size, bool)
    rows = np.cumsum(Gut.l_jump.astype(np.int64))
    short[rows[Gut.r_nJump <= 256]] = True
    assert np.array_equal(w[short], w_ref[short])  # short rows bit-exact


def test_traj2sparsemat_gpu_matches_restatement():
    import monalisa_b200 as mb

    rng = np.random.default_rng(8)
    for imDim, N, kt, kp, nWin in ((2, [24, 20], "kaiser", [1.95, 10, 10], 3), (3, [12, 10, 14], "gauss", [0.61, 10], 3),
                                   (2, [16, 16], "gauss", [0.61, 10], 4)):
        nPt = 700
        t = rng.uniform(-0.6, 0.6, (imDim, nPt)) * np.array(N)[:, None]
        ve = rng.uniform(0.5, 1.5, nPt)
        ref = oracle.traj2sparsemat(t, ve, N, [1] * imDim, kt, nWin, kp)
        Gu, Gut = mb.bmTraj2SparseMat(t, ve, N, [1] * imDim, kt, nWin, kp)
        for dev, r in ((Gu.download(), ref["Gu"]), (Gut.download(), ref["Gut"])):
            assert np.array_equal(dev.r_nJump, r.r_nJump)
            assert np.array_equal(dev.r_jump, r.r_jump)
            assert np.array_equal(dev.l_jump, r.l_jump)
            assert np.allclose(dev.m_val, r.m_val, rtol=2e-7, atol=0)


def test_gn_builder_matches_restatement():
    """The Gn output of the GPU builder (nargout 3) against the restatement
    of bmTraj2SparseMat.m:245-264: same pattern, values within one float
    rounding (FP64 weights and cell sums on both sides)."""
    import monalisa_b200 as mb

    rng = np.random.default_rng(18)
    for imDim, N, kt, kp, nWin, dK in ((2, [24, 20], "kaiser", [1.95, 10, 10], 3, [1.0, 0.5]),
                                       (3, [12, 10, 14], "gauss", [0.61, 10], 3, [1.0, 1.0, 2.0])):
        nPt = 900
        t = rng.uniform(-0.6, 0.6, (imDim, nPt)) * (np.array(N) * np.array(dK))[:, None]
        ve = rng.uniform(0.5, 1.5, nPt)
        ref = oracle.traj2sparsemat(t, ve, N, dK, kt, nWin, kp, want=("Gn",))["Gn"]
        Gn, Gu, Gut = mb.bmTraj2SparseMat(t, ve, N, dK, kt, nWin, kp, nargout=3)
        dev = Gn.download()
        assert np.array_equal(dev.r_nJump, ref.r_nJump)
        assert np.array_equal(dev.r_jump, ref.r_jump)
        assert np.array_equal(dev.l_jump, ref.l_jump)
        assert np.allclose(dev.m_val, ref.m_val, rtol=2.5e-7, atol=0)
        assert mb.bmTraj2SparseMat(t, ve, N, dK, kt, nWin, kp, nargout=1).nnz == Gn.nnz


@pytest.mark.parametrize("with_C", [True, False])
def test_nasha_matches_oracle(with_C):
    """bmNasha (Gn product, IDF, K, crop, coil pinv on the device) against
    the restatement of bmNasha.m, relative L2 <= 1e-5."""
    import monalisa_b200 as mb
    from monalisa_b200 import traj

    rng = np.random.default_rng(19)
    N_u, n_u, nCh, kp = np.array([40, 32]), np.array([20, 16]), 3, [1.95, 10, 10]
    t = traj.golden_angle_radial2(40, 36, 1.0)
    ve = traj.bmVolumeElement_voronoi_full_radial2(t, 40)
    G = oracle.traj2sparsemat(t, ve, N_u, [1, 1], "kaiser", 3, kp, want=("Gn",))["Gn"]
    y = (rng.standard_normal((t.shape[1], nCh)) + 1j * rng.standard_normal((t.shape[1], nCh))).astype(np.complex64)
    C = traj.coil_maps(n_u, nCh, 4) if with_C else None
    Gb = mb.bmSparseMat(r_size=G.r_size, r_jump=G.r_jump, r_nJump=G.r_nJump, m_val=G.m_val, l_size=G.l_size,
                        l_jump=G.l_jump, l_nJump=G.l_nJump, N_u=N_u, d_u=np.array([1, 1], np.float32),
                        kernel_type="kaiser", nWin=3, kernelParam=np.array(kp, np.float32))
    x = mb.bmNasha(y, Gb, n_u, C)
    xo = oracle.bmNasha(y, G, n_u, C)
    assert x.shape == xo.shape and rel(x, xo) <= 1e-5


@pytest.fixture(scope="module")
def op2d():
    g = _g("operators2d")
    n_u, N_u = g["n_u"], g["N_u"]
    G = oracle.traj2sparsemat(g["t"], g["ve"], N_u, [1, 1], "kaiser", 3, [1.95, 10, 10])
    return g, G


def test_shanna_nakatsha_gateways(mex, op2d):
    g, G = op2d
    Gu, Gut = G["Gu"], G["Gut"]
    n_u = g["n_u"].astype(np.int32)
    N_u = g["N_u"].astype(np.int32)

    def margs(M):
        lj = M.l_jump
        return (np.int32(M.r_size), M.r_jump[None], M.r_nJump[None], M.m_val[None], np.int32(M.l_size),
                lj[None] if lj.size else None, np.int32(M.l_nJump))

    x, KFC = g["x"], g["KFC"]
    yR, yI = mex["bmShanna2_CUFFT_omp_mex"](np.ascontiguousarray(x.real)[:, None], np.ascontiguousarray(x.imag)[:, None],
                                            np.ascontiguousarray(KFC.real), np.ascontiguousarray(KFC.imag),
                                            N_u[None], *margs(Gu), n_u[None], nlhs=2)
    assert rel(yR + 1j * yI, g["shanna"]) <= 1e-5
    y, KFCc = g["y"], g["KFC_conj"]
    xR, xI = mex["bmNakatsha2_CUFFT_omp_mex"](np.ascontiguousarray(y.real), np.ascontiguousarray(y.imag),
                                              np.ascontiguousarray(KFCc.real), np.ascontiguousarray(KFCc.imag),
                                              N_u[None], *margs(Gut), n_u[None], nlhs=2)
    assert rel(xR + 1j * xI, g["nakatsha"]) <= 1e-5


@pytest.mark.parametrize("nCh", [3, 8, 16])
@pytest.mark.parametrize("N_u,n_u", [([16, 20, 12], [8, 10, 6]), ([48, 96, 16], [24, 48, 8]),
                                     ([192, 16, 24], [96, 8, 12])])
def test_operators_3d_and_per_coil(N_u, n_u, nCh):
    """3-D Shanna with per-coil x and Nakatsha, package API, vs oracle.
    Line lengths: 16, 32 (radix-2 passes), 20, 12, 24 (runtime DFT passes),
    48, 96, 192 (radix-3 x radix-2 passes).  Coil counts: odd (per-element
    passes), 8 and 16 (pipelined passes of 16 columns: 2 and 1 lines per
    bundle)."""
    import monalisa_b200 as mb

    rng = np.random.default_rng(3)
    N_u, n_u = np.array(N_u), np.array(n_u)
    t = rng.uniform(-0.5, 0.5, (3, 3000)) * N_u[:, None]
    G = oracle.traj2sparsemat(t, np.ones(3000), N_u, [1, 1, 1], "gauss", 3, [0.61, 10])
    C = (rng.standard_normal((n_u.prod(), nCh)) + 1j * rng.standard_normal((n_u.prod(), nCh))).astype(np.complex64)
    KFC = oracle.bmKF(C, N_u, n_u, [1, 1, 1], nCh, "gauss", 3, [0.61, 10])
    KFCc = oracle.bmKF_conj(np.conj(C), N_u, n_u, [1, 1, 1], nCh, "gauss", 3, [0.61, 10])
    x = (rng.standard_normal((n_u.prod(), nCh)) + 1j * rng.standard_normal((n_u.prod(), nCh))).astype(np.complex64)
    conv = lambda M: mb.bmSparseMat(r_size=M.r_size, r_jump=M.r_jump, r_nJump=M.r_nJump, m_val=M.m_val,
                                    l_size=M.l_size, l_jump=M.l_jump, l_nJump=M.l_nJump, N_u=N_u)
    y = mb.bmShanna(x, conv(G["Gu"]), KFC, n_u)
    assert rel(y, oracle.bmShanna(x, G["Gu"], KFC, n_u)) <= 1e-5
    x1 = np.ascontiguousarray(x[:, 0])  # one image shared by the coils (the solvers' form)
    assert rel(mb.bmShanna(x1, conv(G["Gu"]), KFC, n_u), oracle.bmShanna(x1, G["Gu"], KFC, n_u)) <= 1e-5
    yy = (rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape)).astype(np.complex64)
    xn = mb.bmNakatsha(yy, conv(G["Gut"]), KFCc, True, n_u)
    assert rel(xn, oracle.bmNakatsha(yy, G["Gut"], KFCc, True, n_u)) <= 1e-5


@pytest.mark.parametrize("nCh", [4, 3])
def test_adjoint_strategies_agree(nCh):
    """Every adjoint strategy of a plan gives the oracle's Nakatsha; the
    autotuner picks one of them."""
    import monalisa_b200 as mb
    import torch

    rng = np.random.default_rng(21)
    N_u, n_u = np.array([32, 32, 32]), np.array([16, 16, 16])
    t = _radial3(300, 32, 32, 2)  # dense centre: long rows exist
    Gu, Gut = mb.bmTraj2SparseMat(t, np.ones(t.shape[1]), N_u, [1, 1, 1])
    C = (rng.standard_normal((n_u.prod(), nCh)) + 1j * rng.standard_normal((n_u.prod(), nCh))).astype(np.complex64)
    KFC = oracle.bmKF(C, N_u, n_u, [1, 1, 1], nCh, "gauss", 3, [0.61, 10])
    KFCc = oracle.bmKF_conj(np.conj(C), N_u, n_u, [1, 1, 1], nCh, "gauss", 3, [0.61, 10])
    plan = mb.NufftPlan(N_u, n_u, nCh, Gu, Gut, KFC, KFCc)
    y = (rng.standard_normal((t.shape[1], nCh)) + 1j * rng.standard_normal((t.shape[1], nCh))).astype(np.complex64)
    gut_o = Gut.download()
    G = oracle.SparseMat(r_size=gut_o.r_size, l_size=gut_o.l_size, r_nJump=gut_o.r_nJump, m_val=gut_o.m_val,
                         r_jump=gut_o.r_jump, l_jump=gut_o.l_jump, l_nJump=gut_o.l_nJump, N_u=N_u)
    ref = oracle.bmNakatsha(y, G, KFCc, True, n_u).ravel()
    yd = torch.from_numpy(y).cuda()
    outs = {}
    for mode in mb.NufftPlan.ADJOINT_MODES:
        try:
            plan.adjoint_mode = mode
        except mb.MonalisaError:
            assert mode == "masked" and nCh % 2  # masked needs an even coil count
            continue
        outs[mode] = plan.nakatsha(yd).cpu().numpy()
        assert rel(outs[mode], ref) <= 1e-5, mode
    times = plan.autotune(2, variants=False)
    assert set(times) == set(outs) and plan.adjoint_mode in outs
    assert min(times.values()) > 0


def test_idf_gateway(mex):
    rng = np.random.default_rng(4)
    x = (rng.standard_normal((16, 12, 2)) + 1j * rng.standard_normal((16, 12, 2))).astype(np.complex64)
    ref = oracle.bmIDF(x, [16, 12], [0.5, 2.0])
    yR, yI = mex["bmIDF2_CUFFT_mex"](np.asfortranarray(x.real), np.asfortranarray(x.imag),
                                     np.array([[16, 12]], np.int32), np.array([[0.5, 2.0]], np.float32), nlhs=2)
    assert rel(yR + 1j * yI, ref) <= 1e-5


def test_sensa_matches_oracle(op2d):
    import monalisa_b200 as mb

    g, G = op2d
    n_u = g["n_u"]
    conv = lambda M: mb.bmSparseMat(r_size=M.r_size, r_jump=M.r_jump, r_nJump=M.r_nJump, m_val=M.m_val,
                                    l_size=M.l_size, l_jump=M.l_jump, l_nJump=M.l_nJump, N_u=g["N_u"],
                                    d_u=np.array([1, 1], np.float32), kernel_type="kaiser", nWin=3,
                                    kernelParam=np.array([1.95, 10, 10], np.float32))
    hist = []
    x = mb.bmSensa(np.zeros(n_u.prod(), np.complex64), g["y"], g["ve"], g["C"], conv(G["Gu"]), conv(G["Gut"]), n_u,
                   5, 10.0, 1, hist)
    assert rel(x.ravel(order="F"), g["sensa"]) <= 1e-4
    assert abs(hist[0] - g["sensa_residual"][0]) / g["sensa_residual"][0] <= 1e-4


def test_sensa_residual_decreases_and_restarts():
    """Two outer iterations (restarted CG): the HY-weighted residual decreases."""
    import monalisa_b200 as mb
    from monalisa_b200 import traj

    n_u, N_u, nCh = np.array([24, 24]), np.array([48, 48]), 4
    t = traj.golden_angle_radial2(48, 40, 1.0)
    ve = traj.bmVolumeElement_voronoi_full_radial2(traj.bmTraj_fullRadial2_lineAssym2(48, 40, 1.0), 48)
    Gu, Gut = mb.bmTraj2SparseMat(t, ve, N_u, [1, 1], "kaiser", 3, [1.95, 10, 10])
    C = traj.coil_maps(n_u, nCh, 1)
    x_true = traj.ellipsoid_phantom(n_u, 4, 2)
    rec = mb.SensaRecon(Gu, Gut, C, n_u)
    import torch

    xt = torch.from_numpy(x_true).cuda()
    y = rec.plan.shanna(xt)
    hist = []
    x = rec.run_host(y.cpu().numpy(), ve, None, nIter=3, nCGD=6, residual=hist)
    assert hist[1] < hist[0] and hist[2] <= hist[1] * 1.0001
    assert rel(x, x_true) < 0.5


def test_mathilda_matches_oracle():
    import monalisa_b200 as mb
    from monalisa_b200 import traj

    rng = np.random.default_rng(9)
    N_u, n_u, nCh = np.array([32, 32]), np.array([16, 16]), 2
    t = traj.golden_angle_radial2(32, 30, 1.0)
    ve = rng.uniform(0.5, 1.5, t.shape[1])
    y = (rng.standard_normal((t.shape[1], nCh)) + 1j * rng.standard_normal((t.shape[1], nCh))).astype(np.complex64)
    C = traj.coil_maps(n_u, nCh, 3)
    x = mb.bmMathilda(y, t, ve, C, N_u, n_u, [1, 1])
    xo = oracle.bmMathilda(y, t, ve, C, N_u, n_u, [1, 1])
    assert rel(x, xo) <= 1e-5
    # every coil's image (no C), and the precomputed-weight (Kaiser) gridder
    x = mb.bmMathilda(y, t, ve, None, N_u, n_u, [1, 1])
    xo = oracle.bmMathilda(y, t, ve, None, N_u, n_u, [1, 1])
    assert x.shape == xo.shape == (256, nCh) and rel(x, xo) <= 1e-5
    kp = [1.95, 10, 10]
    x = mb.bmMathilda(y, t, ve, C, N_u, n_u, [1, 1], "kaiser", 3, kp, leight_flag=False)
    xo = oracle.bmMathilda(y, t, ve, C, N_u, n_u, [1, 1], "kaiser", 3, kp, leight=False)
    assert rel(x, xo) <= 1e-5


def test_spmm_deterministic():
    import monalisa_b200 as mb
    import torch

    t = _radial3(300, 32, 32, 1)
    Gu, Gut = mb.bmTraj2SparseMat(t, np.ones(t.shape[1]), [32, 32, 32], [1, 1, 1])
    v = torch.randn(Gut.r_size, 4, dtype=torch.complex64, device="cuda")
    a = Gut.spmm(v)
    b = Gut.spmm(v)
    assert torch.equal(a, b)


def test_gateway_rejects_bad_matrix(mex):
    from monalisa_b200.mexcall import MexError

    g = _g("spmv")
    args = list(_sparse_args(g, "u"))
    bad = g["u_G_r_jump"].copy()
    bad[0] = 10 ** 6  # column outside r_size
    args[1] = bad[None]
    v = g["v_u"]
    with pytest.raises(MexError, match="column index"):
        mex["bmSparseMat_cC_oBlock_omp_mex"](*args, np.ascontiguousarray(v.real), np.ascontiguousarray(v.imag),
                                             np.int32(v.shape[1]), nlhs=2)


@pytest.mark.skipif(not oracle.ref_available(), reason="compiled reference kernels absent")
@pytest.mark.parametrize("squeeze", [False, True])
def test_block_and_real_row_gateways_bitexact(mex, squeeze):
    """bmSparseMat_{cR,rR}_nBlock_omp_mex, rR_oBlock_mex and
    cC_oBlock_2_omp_mex against the reference's own compiled kernels on the
    same multi-block / one-block matrices, bit for bit (short rows); the
    cR_nBlock gateway also takes the 15-argument form of
    bmSparseMat_vec.m:167-172 (real and imaginary parts apart)."""
    from test_oracle_pinning import _block_args, _jump, _random_bm

    rng = np.random.default_rng(50 + squeeze)
    Gm, _ = _random_bm(rng, 400, 500, 0.02, squeeze, "multi_block")
    G1, _ = _random_bm(np.random.default_rng(50 + squeeze), 400, 500, 0.02, squeeze, "one_block")
    nVec = 4
    v = (rng.standard_normal((nVec, 500)) + 1j * rng.standard_normal((nVec, 500))).astype(np.complex64)
    vr = rng.standard_normal((nVec, 500)).astype(np.float32)
    cases = [
        ("bmSparseMat_cR_nBlock_omp_mex", (*_jump(Gm), *_block_args(Gm), v, np.int32(nVec))),
        ("bmSparseMat_rR_nBlock_omp_mex", (*_jump(Gm), *_block_args(Gm), vr, np.int32(nVec))),
        ("bmSparseMat_rR_oBlock_mex", (*_jump(G1), vr, np.int32(nVec))),
        ("bmSparseMat_cC_oBlock_2_omp_mex", (*_jump(G1), np.asfortranarray(v.T), np.int32(nVec))),
    ]
    for name, args in cases:
        ref = oracle.ref_mex(name)(*args)
        got = mex[name](*args)
        assert got.shape == ref.shape and np.array_equal(got, ref), name
    split = mex["bmSparseMat_cR_nBlock_omp_mex"](*_jump(Gm), *_block_args(Gm), np.ascontiguousarray(v.real),
                                                 np.ascontiguousarray(v.imag), np.int32(nVec))
    assert np.array_equal(split, oracle.ref_mex("bmSparseMat_cR_nBlock_omp_mex")(*cases[0][1]))


def test_multi_block_matrix_on_device():
    """A multi-block bmSparseMat uploads (mlg_matrix_create_blocks) to the
    same device matrix as its one-block form."""
    import monalisa_b200 as mb
    import torch
    from test_oracle_pinning import _random_bm

    Gm, a = _random_bm(np.random.default_rng(61), 300, 350, 0.03, True, "multi_block")
    conv = lambda G: mb.bmSparseMat(r_size=G.r_size, r_jump=G.r_jump, r_nJump=G.r_nJump, m_val=G.m_val,
                                    l_size=G.l_size, l_jump=G.l_jump, l_nJump=G.l_nJump, extra=dict(G.extra))
    D = conv(Gm).to_device()
    v = torch.randn((350, 2), dtype=torch.complex64, device="cuda")
    got = D.spmm(v).cpu().numpy()
    ref = a.astype(np.float64) @ v.cpu().numpy().astype(np.complex128)
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-5)
    w = mb.bmSparseMat_vec(conv(Gm), v.cpu().numpy().T, layout="row")
    assert np.allclose(w.T, ref, rtol=1e-5, atol=1e-5)
