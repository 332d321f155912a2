"""The coil-sharded CG-SENSE reconstruction (monalisa_b200.sharded) on one
GPU with the library's NUFFT plans as its coil-group engines: two coil
groups on one uploaded Gu / Gut pair (even 4 + 4 and uneven 3 + 5 splits of
8 coils), as one rank (no process group) and as a one-rank NCCL group (the
collective code path).  It must give the restatement of bmSensa.m within the
CG-SENSE tolerance (relative L2 1e-4, FP32 data with FP64 scalars on both
sides) and agree with the single-plan reconstruction over all coils
(SensaRecon.run_dev, relative L2 2e-5).  The multi-rank exchange itself is
covered on CPU ranks (tests/test_sharded_coils.py)."""
import datetime
import socket

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
N_CGD, N_ITER = 6, 2


def rel(a, b):
    a, b = np.ravel(a).astype(np.complex128), np.ravel(b).astype(np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.fixture(scope="module")
def case():
    from monalisa_b200 import traj

    n, N, nCh = 16, 32, 8
    rng = np.random.default_rng(21)
    C = traj.coil_maps([n] * 3, nCh, 5)
    t = traj.bmTraj_fullRadial3_phyllotaxis_lineAssym2(32, 400, 1, 1.0, counter_start=1, q_segments=800)
    ve = np.asarray(traj.bmVolumeElement_full_radial3(t), np.float32)
    G = oracle.traj2sparsemat(t, ve, [N] * 3, [1, 1, 1], "gauss", 3, [0.61, 10])
    KFC = oracle.bmKF(C, [N] * 3, [n] * 3, [1, 1, 1], nCh, "gauss", 3, [0.61, 10])
    xt = traj.ellipsoid_phantom([n] * 3, 3, 33)
    y = oracle.bmShanna(xt, G["Gu"], KFC, [n] * 3)
    y = (y + 0.01 * np.abs(y).mean() * rng.standard_normal(y.shape)).astype(np.complex64)
    x0 = (0.5 * xt).astype(np.complex64).ravel(order="F")
    return dict(n=n, N=N, nCh=nCh, C=C, t=t, ve=ve, G=G, y=y, x0=x0)


def _matrices(case):
    import monalisa_b200 as mb

    N = case["N"]
    return mb.bmTraj2SparseMat(case["t"], case["ve"], [N] * 3, [1, 1, 1], "gauss", 3, [0.61, 10])


def _sharded(case, groups, group):
    import torch

    from monalisa_b200.sharded import CoilPlanEngine, CoilShardedSensa

    Gu, Gut = _matrices(case)
    engines = [CoilPlanEngine(Gu, Gut, case["C"], [case["n"]] * 3, lo, hi) for lo, hi in groups]
    try:
        sh = CoilShardedSensa(engines, group=group)
        hist = []
        x = sh.run([torch.from_numpy(np.ascontiguousarray(case["y"][:, lo:hi])).cuda() for lo, hi in groups],
                   torch.from_numpy(case["ve"]).cuda(), torch.from_numpy(case["x0"].copy()).cuda(), nIter=N_ITER,
                   nCGD=N_CGD, history=hist)
        for e in engines:
            e.plan.status()
        return x.cpu().numpy(), hist
    finally:
        for e in engines:
            e.close()


@pytest.fixture(scope="module")
def reference(case):
    hist = []
    x = oracle.bmSensa(case["x0"].copy(), case["y"], case["ve"], case["C"], case["G"]["Gu"], case["G"]["Gut"],
                       [case["n"]] * 3, N_CGD, nIter=N_ITER, history=hist)
    return np.asarray(x, np.complex64).ravel(), np.array(hist)


@pytest.fixture(scope="module")
def single_plan(case):
    import torch

    from monalisa_b200.solvers import SensaRecon

    Gu, Gut = _matrices(case)
    r = SensaRecon(Gu, Gut, case["C"], [case["n"]] * 3)
    try:
        x = torch.from_numpy(case["x0"].copy()).cuda()
        res = []
        r.run_dev(torch.from_numpy(case["y"]).cuda(), torch.from_numpy(case["ve"]).cuda(), x, nIter=N_ITER,
                  nCGD=N_CGD, residual=res)
        r.plan.status()
        return x.cpu().numpy(), np.array(res)
    finally:
        r.plan.close()


@pytest.mark.parametrize("groups", [[(0, 4), (4, 8)], [(0, 3), (3, 8)]])
def test_coil_groups_match_restatement_and_single_plan(case, reference, single_plan, groups):
    x, hist = _sharded(case, groups, None)
    x_ref, hist_ref = reference
    assert rel(x, x_ref) <= 1e-4
    np.testing.assert_allclose(np.array(hist), hist_ref, rtol=1e-4)
    x_one, hist_one = single_plan
    assert rel(x, x_one) <= 2e-5
    np.testing.assert_allclose(np.array(hist), hist_one, rtol=2e-5)


def test_coil_groups_one_rank_nccl_group(case):
    import torch
    import torch.distributed as dist

    if dist.is_initialized():
        pytest.skip("a process group already exists in this process")
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        x, hist = _sharded(case, [(0, 4), (4, 8)], dist.group.WORLD)
        x1, hist1 = _sharded(case, [(0, 4), (4, 8)], None)
    finally:
        dist.destroy_process_group()
    assert rel(x, x1) <= 1e-6
    np.testing.assert_allclose(np.array(hist), np.array(hist1), rtol=1e-9)
