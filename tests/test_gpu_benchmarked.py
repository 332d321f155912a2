"""Parity at the benchmarked configurations: the exact kernel instantiations
behind every bench number, against the oracle, at the bench's own sizes.

* c2 (3-D koosh 128^3 image / 256^3 grid, 4096 x 256 samples, 16 coils):
  the device-built Gu/Gut against the restatement of bmTraj2SparseMat.m
  (structure exact, values within 2.5e-7); one Shanna (bmShanna_MATLAB.m:28-54)
  and one Nakatsha (bmNakatsha_MATLAB.m:32-56) in every adjoint strategy --
  256-point lines, 16-column TMA passes (the default variant) -- relative L2 <= 1e-5 against
  the FP32 oracle on the same matrices; the leight gridder
  (bmGridder_n2u_leight3_mex.cpp:226-351) on the c2 samples against the
  bit-pinned C restatement, relative L2 <= 1e-5.
* c1 (2-D golden-angle radial 256^2 / 512^2, 1 coil, Kaiser-Bessel): Shanna
  and Nakatsha (512-point lines) <= 1e-5, and the 20-iteration CG-SENSE
  (bmSensa.m:39-85) against the FP32 oracle <= 1e-4 (FP64 scalars on both
  sides).
* c3 bins and the 3-D serving requests with 12 coils (96^3 / 192^3): the
  24-column passes on radix-3 192-point lines, <= 1e-5.
* 2-D serving requests (512^2 grid, 12 coils): 512-point lines in 24-column
  passes, <= 1e-5.

The oracle side runs on all host cores; the c2 cases take about a minute of
CPU time.
"""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

WORKERS = os.cpu_count() or 1


def rel(a, b):
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module", autouse=True)
def _port():
    import subprocess

    if not os.path.exists(oracle.LIB_PATH):
        subprocess.run(["make", "-C", oracle.ORACLE_DIR, "port"], check=True, capture_output=True)


def _to_oracle(D, w):
    """A device matrix as the oracle's jump-format matrix (same entries)."""
    b = D.download()
    return oracle.SparseMat(r_size=b.r_size, l_size=b.l_size, r_nJump=b.r_nJump, m_val=b.m_val, r_jump=b.r_jump,
                            l_jump=b.l_jump, l_nJump=b.l_nJump, N_u=w.N_u, d_u=w.dK_u, kernel_type=w.kernelType,
                            nWin=w.nWin, kernelParam=np.array(w.kernelParam))


class Case:
    """A workload with its device matrices, the same matrices in the
    oracle's format, and KFC / KFC_conj from the oracle (inputs of both
    sides)."""

    def __init__(self, w):
        import monalisa_b200 as mb

        self.w = w
        self.Gu, self.Gut = mb.bmTraj2SparseMat(w.t, w.ve, w.N_u, w.dK_u, w.kernelType, w.nWin, w.kernelParam)
        self.oGu, self.oGut = _to_oracle(self.Gu, w), _to_oracle(self.Gut, w)
        C = np.asarray(w.C, np.complex64)
        self.KFC = oracle.bmKF(C, w.N_u, w.n_u, w.dK_u, w.nCh, w.kernelType, w.nWin, w.kernelParam)
        self.KFCc = oracle.bmKF_conj(np.conj(C), w.N_u, w.n_u, w.dK_u, w.nCh, w.kernelType, w.nWin, w.kernelParam)

    def plan(self):
        import monalisa_b200 as mb

        return mb.NufftPlan(self.w.N_u, self.w.n_u, self.w.nCh, self.Gu, self.Gut, self.KFC, self.KFCc, self.w.dK_u)


def _operators_match(case, seed):
    """One Shanna and one Nakatsha per adjoint strategy against the oracle."""
    import torch

    w = case.w
    rng = np.random.default_rng(seed)
    nu = int(np.prod(w.n_u))
    x = (rng.standard_normal(nu) + 1j * rng.standard_normal(nu)).astype(np.complex64)
    y = (rng.standard_normal((case.Gu.l_size, w.nCh)) + 1j * rng.standard_normal((case.Gu.l_size, w.nCh))).astype(
        np.complex64)
    plan = case.plan()
    try:
        ys = plan.shanna(torch.from_numpy(x).cuda()).cpu().numpy()
        ref = oracle.bmShanna(x, case.oGu, case.KFC, w.n_u, workers=WORKERS)
        errs = {"shanna": rel(ys, ref)}
        del ref
        ref = oracle.bmNakatsha(y, case.oGut, case.KFCc, True, w.n_u, workers=WORKERS).ravel()
        yd = torch.from_numpy(y).cuda()
        for mode in plan.ADJOINT_MODES:
            if mode == "masked" and w.nCh % 2:
                continue  # the masked strategy needs an even coil count
            plan.adjoint_mode = mode
            errs[mode] = rel(plan.nakatsha(yd).cpu().numpy(), ref)
    finally:
        plan.close()
    return errs


# ---- c2 ---------------------------------------------------------------------
@pytest.fixture(scope="module")
def c2():
    from monalisa_b200.workloads import koosh3d

    return Case(koosh3d())


def test_c2_matrices_match_restatement(c2):
    """bmTraj2SparseMat on the device at full size: 1,048,576 samples x 27
    window cells onto 256^3."""
    w = c2.w
    ref = oracle.traj2sparsemat(w.t, w.ve, w.N_u, w.dK_u, w.kernelType, w.nWin, w.kernelParam)
    for dev, r in ((c2.oGu, ref["Gu"]), (c2.oGut, ref["Gut"])):
        assert np.array_equal(dev.r_nJump, r.r_nJump)
        assert np.array_equal(dev.r_jump, r.r_jump)
        assert np.array_equal(dev.l_jump, r.l_jump)
        assert np.allclose(dev.m_val, r.m_val, rtol=2.5e-7, atol=0)


def test_c2_operators_match_oracle(c2):
    errs = _operators_match(c2, 20)
    assert max(errs.values()) <= 1e-5, errs


def test_c2_leight_gridder_matches_oracle(c2):
    """The allocating leight gridder on the device (the bench's
    mlg_gridder_n2u_leight_dev call) against the C restatement that
    reproduces the reference's compiled kernel bit for bit."""
    import torch

    from monalisa_b200 import _native as N
    from monalisa_b200.gridding import _leight_prepare

    w = c2.w
    rng = np.random.default_rng(7)
    data = (rng.standard_normal((w.nCh, w.nPt)) + 1j * rng.standard_normal((w.nCh, w.nPt))).astype(np.complex64)
    aR, aI, tx, Dn, nCh, nPt, Ns = _leight_prepare(data, w.t, w.ve, w.N_u, w.dK_u)
    nu = int(np.prod(Ns))
    up = lambda a: torch.from_numpy(a).cuda() if a is not None else None
    dT = [up(v) for v in tx]
    dA, dI, dD = up(aR), up(aI), up(Dn)
    bR = torch.empty((nu, nCh), dtype=torch.float32, device="cuda")
    bI = torch.empty_like(bR)
    N.call("mlg_gridder_n2u_leight_dev", 3, N.tptr(dA), N.tptr(dI), N.tptr(dT[0]), N.tptr(dT[1]), N.tptr(dT[2]),
           N.tptr(dD), nCh, nPt, Ns[0], Ns[1], Ns[2], int(w.nWin), float(w.kernelParam[0]),
           float(w.kernelParam[1]), N.tptr(bR), N.tptr(bI), N.stream_ptr())
    got = bR.cpu().numpy() + 1j * bI.cpu().numpy()
    del bR, bI
    # the restatement takes the MEX layout [nCh, nPt] (coil fastest in memory)
    rR, rI = oracle.port_gridder_leight(3, aR.T, aI.T, tx[0], tx[1], tx[2], Dn, nCh, nPt, Ns[0], Ns[1], Ns[2],
                                        int(w.nWin), float(w.kernelParam[0]), float(w.kernelParam[1]))
    assert rel(got, (np.asarray(rR) + 1j * np.asarray(rI)).T) <= 1e-5  # [nCh, Nu] -> [Nu][nCh]


# ---- c1 ---------------------------------------------------------------------
@pytest.fixture(scope="module")
def c1():
    from monalisa_b200.workloads import radial2d

    return Case(radial2d())


def test_c1_operators_match_oracle(c1):
    errs = _operators_match(c1, 21)
    assert max(errs.values()) <= 1e-5, errs


def test_c1_sensa_20_iterations_matches_oracle(c1):
    """c1's reconstruction: 20 CG updates from x = 0 (bmSensa with nIter 1,
    nCGD 20), the device solver against the FP32 restatement."""
    import monalisa_b200 as mb

    w = c1.w
    rec = mb.SensaRecon(c1.Gu, c1.Gut, w.C, w.n_u)
    try:
        got = rec.run_host(w.y, w.ve, nIter=1, nCGD=w.nCGD)
    finally:
        rec.plan.close()
    ref = oracle.bmSensa(np.zeros(int(np.prod(w.n_u)), np.complex64), w.y, w.ve, w.C, c1.oGu, c1.oGut, w.n_u,
                         w.nCGD, workers=WORKERS)
    assert rel(got, np.asarray(ref).ravel(order="F")) <= 1e-4


# ---- 12-coil passes (c3 bins, serving requests) -------------------------------
def test_c3_bin_12_coil_operators_match_oracle():
    """One c3-shaped frame bin: 1500 koosh spokes x 256, 96^3 image on a
    192^3 grid (radix-3 192-point lines), 12 coils (24-column passes)."""
    from monalisa_b200 import traj as T
    from monalisa_b200.workloads import Workload

    w = Workload("c3_bin", 3, np.array([96] * 3), np.array([192] * 3), np.ones(3), 12, 5, "gauss", 3, [0.61, 10])
    w.t = T.bmTraj_fullRadial3_phyllotaxis_lineAssym2(256, 1500, 1, 192 / 256)
    w.ve = T.bmVolumeElement_full_radial3(w.t)
    w.C = T.coil_maps(w.n_u, 12, 3)
    errs = _operators_match(Case(w), 22)
    assert max(errs.values()) <= 1e-5, errs


def test_serving_2d_12_coil_operators_match_oracle():
    """A 2-D serving request: 256 golden-angle spokes x 512 on a 512^2 grid,
    12 coils (512-point lines in 24-column passes)."""
    from monalisa_b200 import traj as T
    from monalisa_b200.workloads import Workload

    w = Workload("serving_2d", 2, np.array([256] * 2), np.array([512] * 2), np.ones(2), 12, 20, "kaiser", 3,
                 [1.95, 10, 10])
    w.t = T.golden_angle_radial2(512, 256, 1.0)
    w.ve = T.bmVolumeElement_voronoi_full_radial2(T.bmTraj_fullRadial2_lineAssym2(512, 256, 1.0), 512)
    w.C = T.coil_maps(w.n_u, 12, 6)
    errs = _operators_match(Case(w), 23)
    assert max(errs.values()) <= 1e-5, errs
