"""The frame-bin sharded temporal-TV reconstruction (monalisa_b200.sharded)
on one GPU with the library's NUFFT plans as its per-frame engine: as one
rank (no process group) and as a one-rank NCCL group (the collective code
path), it must give the restatement of bmTevaMorphosia_chain.m within the
chain tolerance (relative L2 1e-4, FP32 data with FP64 scalars on both
sides) and agree with the single-GPU chain (solvers.TevaMorphosiaChain).
The multi-rank exchange itself is covered on CPU ranks (tests/test_sharded.py)."""
import datetime
import os
import socket

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.concatenate([np.ravel(v) for v in a]).astype(np.complex128)
    b = np.concatenate([np.ravel(v) for v in b]).astype(np.complex128)
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

    n, N, nCh, nFr = 16, 32, 4, 4
    rng = np.random.default_rng(12)
    C = traj.coil_maps([n] * 3, nCh, 2)
    t, ve, G, y, x0 = [], [], [], [], []
    KFC = oracle.bmKF(C, [N] * 3, [n] * 3, [1, 1, 1], nCh, "gauss", 3, [0.61, 10])
    counter = 1
    for f in range(nFr):
        ns = int(rng.integers(120, 200))
        tf = traj.bmTraj_fullRadial3_phyllotaxis_lineAssym2(32, ns, 1, 1.0, counter_start=counter, q_segments=800)
        counter += ns
        vf = traj.bmVolumeElement_full_radial3(tf)
        Gf = oracle.traj2sparsemat(tf, vf, [N] * 3, [1, 1, 1], "gauss", 3, [0.61, 10])
        xt = traj.ellipsoid_phantom([n] * 3, 3, 40 + f)
        yf = oracle.bmShanna(xt, Gf["Gu"], KFC, [n] * 3)
        yf = (yf + 0.01 * np.abs(yf).mean() * rng.standard_normal(yf.shape)).astype(np.complex64)
        t.append(tf)
        ve.append(np.asarray(vf, np.float32))
        G.append(Gf)
        y.append(yf)
        x0.append((0.5 * xt).astype(np.complex64))
    return dict(n=n, N=N, nCh=nCh, nFr=nFr, C=C, t=t, ve=ve, G=G, y=y, x0=x0)


def _sharded(case, group):
    import torch

    import monalisa_b200 as mb
    from monalisa_b200.sharded import PlanEngine, ShardedTevaMorphosia

    n, N = case["n"], case["N"]
    mats = [mb.bmTraj2SparseMat(case["t"][f], case["ve"][f], [N] * 3, [1, 1, 1], "gauss", 3, [0.61, 10])
            for f in range(case["nFr"])]
    eng = PlanEngine([m[0] for m in mats], [m[1] for m in mats], case["C"], [n] * 3)
    try:
        sh = ShardedTevaMorphosia(eng, 0, case["nFr"], case["nFr"], group=group)
        hist = []
        x = sh.run([torch.from_numpy(v).cuda() for v in case["y"]], [torch.from_numpy(v).cuda() for v in case["ve"]],
                   [torch.from_numpy(v.copy()).cuda() for v in case["x0"]], 0.01, 0.1, 3, 4, 10.0, history=hist)
        for p in eng.plans:
            p.status()
        return [v.cpu().numpy() for v in x], hist
    finally:
        eng.close()


def test_sharded_one_rank_matches_restatement_and_chain(case):
    import monalisa_b200 as mb

    n, N = case["n"], case["N"]
    hist_ref = []
    ref = oracle.bmTevaMorphosia_chain([v.copy() for v in case["x0"]], case["y"], case["ve"], case["C"],
                                       [g["Gu"] for g in case["G"]], [g["Gut"] for g in case["G"]], [n] * 3, 0.01,
                                       0.1, 4, 10.0, 3, history=hist_ref)
    x, hist = _sharded(case, None)
    assert rel(x, ref) <= 1e-4
    np.testing.assert_allclose(np.array(hist), np.array(hist_ref), rtol=1e-4)
    mats = [mb.bmTraj2SparseMat(case["t"][f], case["ve"][f], [N] * 3, [1, 1, 1], "gauss", 3, [0.61, 10])
            for f in range(case["nFr"])]
    chain = mb.TevaMorphosiaChain([m[0] for m in mats], [m[1] for m in mats], case["C"], [n] * 3)
    try:
        xc = chain.run_host(case["y"], case["ve"], case["x0"], 0.01, 0.1, 3, 4, 10.0)
    finally:
        chain.close()
    assert rel(x, xc) <= 1e-4


def test_sharded_one_rank_nccl_group(case):
    import torch
    import torch.distributed as dist

    if dist.is_initialized():
        pytest.skip("a process group already exists in this process")
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        x, hist = _sharded(case, dist.group.WORLD)
        x1, hist1 = _sharded(case, None)
    finally:
        dist.destroy_process_group()
    assert rel(x, x1) <= 1e-6
    np.testing.assert_allclose(np.array(hist), np.array(hist1), rtol=1e-9)
