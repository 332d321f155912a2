"""Temporal-TV ADMM over frame bins (bmTevaMorphosia_chain) and the plans
that share one grid (mlg_plan_create_sharing): CUDA path vs the oracle.

Tolerances: relative L2 <= 1e-4 on every frame image and on the monitoring
history after 3 ADMM iterations of 4 CG steps (FP32 data, FP64 scalars on
both sides, operators within 1e-5 of each other).  Restarting from the
returned x, z, u is bit-identical to running on, since the kept monitoring
residual is recomputed bit for bit from the same x.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

KP = [0.61, 10]


def rel(a, b):
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _frames(nFr=3, N=48, n=24, nCh=4, seed=7):
    """Golden-angle radial frame bins of different sizes over one moving
    phantom; y simulated with the oracle's forward operator plus noise."""
    from monalisa_b200 import traj

    rng = np.random.default_rng(seed)
    N_u, n_u = np.array([N, N]), np.array([n, n])
    C = traj.coil_maps(n_u, nCh, seed)
    KFC = oracle.bmKF(C, N_u, n_u, [1, 1], nCh, "gauss", 3, KP)
    spokes = [20 + 8 * f for f in range(nFr)]
    t_all = traj.golden_angle_radial2(N, sum(spokes), 1.0)
    G, y, ve, x_true = [], [], [], []
    s0 = 0
    for f, ns in enumerate(spokes):
        t = t_all[:, s0 * N:(s0 + ns) * N]
        s0 += ns
        v = traj.bmVolumeElement_voronoi_full_radial2(t, N)
        g = oracle.traj2sparsemat(t, v, N_u, [1, 1], "gauss", 3, KP)
        xt = traj.ellipsoid_phantom(n_u, 4, 100) * (1 + 0.2 * f)
        yy = oracle.bmShanna(xt, g["Gu"], KFC, n_u)
        yy = (yy + 1e-3 * np.abs(yy).mean() * (rng.standard_normal(yy.shape) + 1j * rng.standard_normal(yy.shape)))
        G.append(g)
        y.append(yy.astype(np.complex64))
        ve.append(np.asarray(v, np.float32))
        x_true.append(xt)
    return dict(N_u=N_u, n_u=n_u, C=C, G=G, y=y, ve=ve, x_true=x_true, nCh=nCh)


def _device_mats(case):
    import monalisa_b200 as mb

    conv = lambda M: mb.bmSparseMat(r_size=M.r_size, r_jump=M.r_jump, r_nJump=M.r_nJump, m_val=M.m_val,
                                    l_size=M.l_size, l_jump=M.l_jump, l_nJump=M.l_nJump, N_u=case["N_u"],
                                    d_u=np.array([1, 1], np.float32), kernel_type="gauss", nWin=3,
                                    kernelParam=np.array(KP, np.float32))
    return [conv(g["Gu"]) for g in case["G"]], [conv(g["Gut"]) for g in case["G"]]


@pytest.fixture(scope="module")
def case():
    return _frames()


@pytest.mark.parametrize("mode", ["normal", "adapt"])
def test_chain_matches_oracle(case, mode):
    import monalisa_b200 as mb

    nFr = len(case["y"])
    delta, rho, nIter, nCGD, ve_max = 0.02, 0.2, 3, 4, 10.0
    x0 = [np.zeros(int(np.prod(case["n_u"])), np.complex64) for _ in range(nFr)]
    if mode == "adapt":
        delta, rho = 0.5, 10.0  # factors: delta = 0.5 regul/dafi, rho = 10 delta
        # a start with frame differences (x = 0 has regul = 0, so delta = rho = 0)
        x0 = [(0.8 * xt).astype(np.complex64) for xt in case["x_true"]]
    hist_o = []
    ref = oracle.bmTevaMorphosia_chain(x0, case["y"], case["ve"], case["C"], [g["Gu"] for g in case["G"]],
                                       [g["Gut"] for g in case["G"]], case["n_u"], delta, rho, nCGD, ve_max, nIter,
                                       history=hist_o, regul_mode=mode)
    Gu, Gut = _device_mats(case)
    hist = []
    out = mb.bmTevaMorphosia_chain(x0, None, None, case["y"], case["ve"], case["C"], Gu, Gut, case["n_u"], None, None,
                                   delta, rho, mode, nCGD, ve_max, nIter, hist)
    for f in range(nFr):
        assert rel(out[f].ravel(order="F"), ref[f]) <= 1e-4, f
    assert len(hist) == nIter
    for c in range(nIter):
        for k in range(3):
            assert abs(hist[c][k] - hist_o[c][k]) <= 1e-4 * abs(hist_o[c][k]), (c, k)
    if mode == "normal":  # from x = 0 the data term falls
        assert hist[-1][1] < hist[0][1]


def test_chain_one_frame_is_cg_sense(case):
    """With one frame F x = x - x = 0: the ADMM x-update is CG-SENSE."""
    import monalisa_b200 as mb
    import torch

    Gu, Gut = _device_mats(case)
    chain = mb.TevaMorphosiaChain(Gu[:1], Gut[:1], case["C"], case["n_u"])
    nu = int(np.prod(case["n_u"]))
    y = torch.from_numpy(case["y"][0]).cuda()
    ve = torch.from_numpy(case["ve"][0]).cuda()
    x = torch.zeros((1, nu), dtype=torch.complex64, device="cuda")
    z, u = torch.empty_like(x), torch.empty_like(x)
    chain.run_dev(y, ve, x, z, u, 0.01, 0.1, 2, 5, 10.0)
    xs = torch.zeros(nu, dtype=torch.complex64, device="cuda")
    res = []
    chain._first.run_dev(y, ve, xs, nIter=2, nCGD=5, ve_max=10.0, residual=res)
    assert rel(x.cpu().numpy()[0], xs.cpu().numpy()) <= 1e-5
    chain.close()


def test_chain_restart_is_bit_identical(case):
    """Running 2 + 2 iterations from the returned x, z, u equals running 4."""
    import monalisa_b200 as mb
    import torch

    Gu, Gut = _device_mats(case)
    chain = mb.TevaMorphosiaChain(Gu, Gut, case["C"], case["n_u"])
    nFr, nu = len(Gu), int(np.prod(case["n_u"]))
    y = torch.from_numpy(np.concatenate(case["y"])).cuda()
    ve = torch.from_numpy(np.concatenate(case["ve"])).cuda()

    def fresh():
        return [torch.zeros((nFr, nu), dtype=torch.complex64, device="cuda") for _ in range(3)]

    x, z, u = fresh()
    h4 = []
    chain.run_dev(y, ve, x, z, u, 0.02, 0.2, 4, 3, 10.0, history=h4)
    x2, z2, u2 = fresh()
    h22 = []
    chain.run_dev(y, ve, x2, z2, u2, 0.02, 0.2, 2, 3, 10.0, history=h22)
    chain.run_dev(y, ve, x2, z2, u2, 0.02, 0.2, 2, 3, 10.0, init_zu=False, history=h22)
    torch.cuda.synchronize()
    assert torch.equal(x, x2) and torch.equal(z, z2) and torch.equal(u, u2)
    assert h4 == h22
    chain.close()


def test_sharing_plans_match_own_plans(case):
    """A plan borrowing frame 0's buffers gives the operators of a plan of
    its own; the owner refuses to go while it is borrowed."""
    import monalisa_b200 as mb
    import torch

    Gu, Gut = _device_mats(case)
    nu, nCh = int(np.prod(case["n_u"])), case["nCh"]
    KFC = oracle.bmKF(case["C"], case["N_u"], case["n_u"], [1, 1], nCh, "gauss", 3, KP)
    KFCc = oracle.bmKF_conj(np.conj(case["C"]), case["N_u"], case["n_u"], [1, 1], nCh, "gauss", 3, KP)
    base = mb.NufftPlan(case["N_u"], case["n_u"], nCh, Gu[0], Gut[0], KFC, KFCc)
    own = mb.NufftPlan(case["N_u"], case["n_u"], nCh, Gu[1], Gut[1], KFC, KFCc)
    shared = mb.NufftPlan.sharing(base, Gu[1], Gut[1])
    rng = np.random.default_rng(9)
    x = torch.from_numpy((rng.standard_normal(nu) + 1j * rng.standard_normal(nu)).astype(np.complex64)).cuda()
    y1 = shared.shanna(x)
    y0 = base.shanna(x)  # interleaved use of the shared grid buffers
    assert torch.equal(y1, own.shanna(x))
    assert torch.equal(y0, base.shanna(x))
    yy = torch.from_numpy(case["y"][1]).cuda()
    assert torch.equal(shared.nakatsha(yy), own.nakatsha(yy))
    from monalisa_b200 import _native as N

    with pytest.raises(N.MonalisaError, match="borrow"):
        N.call("mlg_plan_destroy", base.handle)
    shared.close()
    base.close()
    own.close()


@pytest.mark.parametrize("dims", [2, 3])
def test_steva_matches_oracle(dims):
    """Spatial-TV ADMM (bmSteva) vs the oracle: 2-D golden-angle radial and
    3-D random samples, dK_u != 1 so the gradient's 1/dX_u scaling counts."""
    import monalisa_b200 as mb
    from monalisa_b200 import traj

    rng = np.random.default_rng(40 + dims)
    if dims == 2:
        N_u, n_u, dK = np.array([48, 40]), np.array([24, 20]), np.array([0.5, 0.5])
        t = traj.golden_angle_radial2(48, 40, 0.5)
        ve = traj.bmVolumeElement_voronoi_full_radial2(t, 48).astype(np.float32)
    else:
        N_u, n_u, dK = np.array([24, 16, 20]), np.array([12, 8, 10]), np.array([1.0, 2.0, 1.0])
        t = rng.uniform(-0.5, 0.5, (3, 6000)) * (N_u * dK)[:, None]
        ve = rng.uniform(0.5, 1.5, 6000).astype(np.float32)
    nCh = 4
    C = traj.coil_maps(n_u, nCh, 5)
    G = oracle.traj2sparsemat(t, ve, N_u, dK, "gauss", 3, KP)
    KFC = oracle.bmKF(C, N_u, n_u, dK, nCh, "gauss", 3, KP)
    xt = traj.ellipsoid_phantom(n_u, 3, 7)
    y = oracle.bmShanna(xt, G["Gu"], KFC, n_u)
    y = (y + 1e-2 * np.abs(y).mean() * (rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape))
         ).astype(np.complex64)
    delta, rho, nIter, nCGD = (1e-4, 1e-3), 1e-2, 3, 4
    ho = []
    ref = oracle.bmSteva(np.zeros(int(np.prod(n_u)), np.complex64), y, ve, C, G["Gu"], G["Gut"], n_u, delta, rho,
                         nCGD, None, nIter, history=ho)
    conv = lambda M: mb.bmSparseMat(r_size=M.r_size, r_jump=M.r_jump, r_nJump=M.r_nJump, m_val=M.m_val,
                                    l_size=M.l_size, l_jump=M.l_jump, l_nJump=M.l_nJump, N_u=N_u,
                                    d_u=dK.astype(np.float32), kernel_type="gauss", nWin=3,
                                    kernelParam=np.array(KP, np.float32))
    h = []
    out = mb.bmSteva(None, None, None, y, ve, C, conv(G["Gu"]), conv(G["Gut"]), n_u, delta, rho, nCGD, None, nIter, h)
    assert rel(out.ravel(order="F"), ref) <= 1e-4
    assert len(h) == nIter
    for c in range(nIter):
        for k in range(2):
            assert abs(h[c][k] - ho[c][k]) <= 1e-4 * abs(ho[c][k]), (c, k)
