"""Coil sharding of one CG-SENSE reconstruction on CPU ranks (gloo): the
coils split over 2 and 3 ranks (one or two coil groups per rank, and two
coil groups in one process), with the adjoint's coil sum all-reduced as an
image and the k-space norms as FP64 scalars, give the single-process
restatement of bmSensa.m (oracle) --
image relative L2 <= 1e-5, monitored residuals within 1e-5 -- and every rank
ends with the same image.  The per-group operators are the restatement's
Shanna / Nakatsha over the group's columns of KFC / KFC_conj on CPU tensors
(the same engine interface the GPU plans implement)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_CGD, N_ITER = 6, 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _case(n=12, nCh=5, spokes=18, seed=7):
    import oracle
    from monalisa_b200 import traj

    N = 2 * n
    rng = np.random.default_rng(seed)
    t = traj.golden_angle_radial2(2 * n, spokes, 1.0)
    ve = np.asarray(traj.bmVolumeElement_voronoi_full_radial2(
        traj.bmTraj_fullRadial2_lineAssym2(2 * n, spokes, 1.0), 2 * n), np.float32)
    G = oracle.traj2sparsemat(t, ve, [N, N], [1, 1], "gauss", 3, [0.61, 10])
    C = traj.coil_maps([n, n], nCh, seed)
    KFC = oracle.bmKF(C, [N, N], [n, n], [1, 1], nCh, "gauss", 3, [0.61, 10])
    x_true = traj.ellipsoid_phantom([n, n], 3, seed)
    y = (oracle.bmShanna(x_true, G["Gu"], KFC, [n, n])
         + 0.01 * (rng.standard_normal((G["Gu"].l_size, nCh)) + 1j * rng.standard_normal((G["Gu"].l_size, nCh))))
    x0 = (0.5 * x_true + 0.05).astype(np.complex64).ravel(order="F")
    return dict(n_u=np.array([n, n]), N_u=np.array([N, N]), C=C, Gu=G["Gu"], Gut=G["Gut"],
                y=np.asarray(y, np.complex64), ve=ve, nCh=nCh, x0=x0)


class OracleCoilEngine:
    """The restatement's operators of the coils [lo, hi) on CPU tensors."""

    def __init__(self, case, lo, hi):
        import oracle

        self.o = oracle
        self.case = case
        n_u, N_u, nCh = case["n_u"], case["N_u"], case["nCh"]
        self.KFC = oracle.bmKF(case["C"], N_u, n_u, [1, 1], nCh, "gauss", 3, [0.61, 10])[:, lo:hi]
        self.KFCc = oracle.bmKF_conj(np.conj(case["C"]), N_u, n_u, [1, 1], nCh, "gauss", 3,
                                     [0.61, 10])[:, lo:hi]
        dX = (np.float32(1) / np.ones(2, np.float32)) / N_u.astype(np.float32)
        self.HX = float(np.prod(dX.astype(np.float32)))

    def M(self, x):
        import torch

        return torch.from_numpy(self.o.bmShanna(x.numpy(), self.case["Gu"], self.KFC, self.case["n_u"]))

    def MH(self, r, HY, scale):
        import torch

        rr = (HY.numpy()[:, None] * r.numpy()).astype(np.complex64)
        out = self.o.bmNakatsha(rr, self.case["Gut"], self.KFCc, True, self.case["n_u"])
        return torch.from_numpy((scale * out).astype(np.complex64).ravel())


def _reference(case):
    import oracle

    hist = []
    x = oracle.bmSensa(case["x0"].copy(), case["y"], case["ve"], case["C"], case["Gu"], case["Gut"], case["n_u"],
                       N_CGD, nIter=N_ITER, history=hist)
    return np.asarray(x, np.complex64).ravel(), np.array(hist)


def _check(x, hist, ref):
    x_ref, hist_ref = ref
    a, b = np.asarray(x, np.complex128), x_ref.astype(np.complex128)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5
    np.testing.assert_allclose(np.array(hist), hist_ref, rtol=1e-5)


def _rank(rank, world, port, out, split=False):
    import sys

    for p in (ROOT, os.path.join(ROOT, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch
    import torch.distributed as dist

    from monalisa_b200.sharded import CoilShardedSensa, shard_coils

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    case = _case()
    bounds = shard_coils(case["nCh"], world)
    lo, hi = bounds[rank], bounds[rank + 1]
    # split: the rank's coils as two groups (summed locally before the all-reduce)
    groups = [(lo, lo + 1), (lo + 1, hi)] if split and hi - lo > 1 else [(lo, hi)]
    sh = CoilShardedSensa([OracleCoilEngine(case, a, b) for a, b in groups], group=dist.group.WORLD)
    hist = []
    x = sh.run([torch.from_numpy(np.ascontiguousarray(case["y"][:, a:b])) for a, b in groups],
               torch.from_numpy(case["ve"]), torch.from_numpy(case["x0"].copy()), nIter=N_ITER, nCGD=N_CGD,
               history=hist)
    out[rank] = (lo, hi, x.numpy(), hist)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,split", [(2, False), (3, False), (2, True)])
def test_coil_sharded_sensa_matches_single_process_restatement(world, split):
    import sys

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    case = _case()
    ref = _reference(case)
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out, split)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    covered = []
    x0 = out[0][2]
    for r in range(world):
        lo, hi, x, hist = out[r]
        covered.extend(range(lo, hi))
        _check(x, hist, ref)
        np.testing.assert_array_equal(x, x0)  # the all-reduced image is the same on every rank
    assert covered == list(range(case["nCh"]))


def test_two_coil_groups_in_one_process():
    import sys

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch

    from monalisa_b200.sharded import CoilShardedSensa

    case = _case()
    groups = [(0, 2), (2, 5)]
    sh = CoilShardedSensa([OracleCoilEngine(case, lo, hi) for lo, hi in groups])
    hist = []
    x = sh.run([torch.from_numpy(np.ascontiguousarray(case["y"][:, lo:hi])) for lo, hi in groups],
               torch.from_numpy(case["ve"]), torch.from_numpy(case["x0"].copy()), nIter=N_ITER, nCGD=N_CGD,
               history=hist)
    _check(x.numpy(), hist, _reference(case))


def test_shard_coils_keeps_coil_pairs_together():
    from monalisa_b200.sharded import shard_coils

    assert shard_coils(16, 2) == [0, 8, 16]
    assert shard_coils(16, 3) == [0, 6, 12, 16]
    assert shard_coils(12, 4) == [0, 4, 8, 10, 12]
    assert shard_coils(5, 2) == [0, 2, 5]
    assert shard_coils(5, 3) == [0, 2, 4, 5]
    assert shard_coils(1, 1) == [0, 1]
    for nCh in range(1, 20):
        for world in range(1, nCh + 1):
            b = shard_coils(nCh, world)
            sizes = np.diff(b)
            assert b[0] == 0 and b[-1] == nCh and len(b) == world + 1 and sizes.min() >= 1
    with pytest.raises(ValueError):
        shard_coils(2, 3)
