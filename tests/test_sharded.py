"""Frame-bin sharding of the temporal-TV reconstruction on CPU ranks (gloo):
the frames split over 2 and 3 ranks, with the boundary images of F / F*
exchanged around the ring and the CG scalars all-reduced in FP64, give the
single-process restatement of bmTevaMorphosia_chain.m (oracle) -- image
relative L2 <= 1e-5 and monitoring history within 1e-6 -- in the 'normal'
and 'adapt' regularisation modes.  The per-frame operators are the
restatement's Shanna / Nakatsha on CPU tensors (the same engine interface
the GPU plans implement)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _case(nFr=5, n=12, nCh=2, seed=3):
    import oracle
    from monalisa_b200 import traj

    N = 2 * n
    rng = np.random.default_rng(seed)
    t, ve, Gu, Gut, x_true = [], [], [], [], []
    C = traj.coil_maps([n, n], nCh, seed)
    for f in range(nFr):
        ns = int(rng.integers(10, 20))
        tf = traj.golden_angle_radial2(2 * n, ns, 1.0)
        vf = traj.bmVolumeElement_voronoi_full_radial2(traj.bmTraj_fullRadial2_lineAssym2(2 * n, ns, 1.0), 2 * n)
        G = oracle.traj2sparsemat(tf, vf, [N, N], [1, 1], "gauss", 3, [0.61, 10])
        t.append(tf)
        ve.append(np.asarray(vf, np.float32))
        Gu.append(G["Gu"])
        Gut.append(G["Gut"])
        x_true.append(traj.ellipsoid_phantom([n, n], 3, seed + f))
    KFC = oracle.bmKF(C, [N, N], [n, n], [1, 1], nCh, "gauss", 3, [0.61, 10])
    y = [(oracle.bmShanna(x_true[f], Gu[f], KFC, [n, n])
          + 0.01 * (rng.standard_normal((Gu[f].l_size, nCh)) + 1j * rng.standard_normal((Gu[f].l_size, nCh))))
         .astype(np.complex64) for f in range(nFr)]
    # a non-zero start (the 'adapt' mode scales delta by the initial regulariser)
    x0 = [(0.5 * x_true[f] + 0.05).astype(np.complex64) for f in range(nFr)]
    return dict(n_u=np.array([n, n]), N_u=np.array([N, N]), C=C, Gu=Gu, Gut=Gut, y=y, ve=ve, nFr=nFr, nCh=nCh,
                x0=x0)


class OracleEngine:
    """Per-frame operators of the restatement on CPU tensors."""

    def __init__(self, case, frames):
        import oracle

        self.o = oracle
        self.case = case
        self.frames = frames
        n_u, N_u, nCh = case["n_u"], case["N_u"], case["nCh"]
        self.KFC = oracle.bmKF(case["C"], N_u, n_u, [1, 1], nCh, "gauss", 3, [0.61, 10])
        self.KFCc = oracle.bmKF_conj(np.conj(case["C"]), N_u, n_u, [1, 1], nCh, "gauss", 3, [0.61, 10])
        dX = (np.float32(1) / np.ones(2, np.float32)) / N_u.astype(np.float32)
        self.HX = float(np.float32(np.prod(dX)))

    def M(self, i, x):
        import torch

        f = self.frames[i]
        return torch.from_numpy(self.o.bmShanna(x.numpy(), self.case["Gu"][f], self.KFC, self.case["n_u"]))

    def MH(self, i, r, HY, scale):
        import torch

        f = self.frames[i]
        rr = (HY.numpy()[:, None] * r.numpy()).astype(np.complex64)
        out = self.o.bmNakatsha(rr, self.case["Gut"][f], self.KFCc, True, self.case["n_u"])
        return torch.from_numpy((scale * out).astype(np.complex64).ravel())


def _rank(rank, world, port, mode, out):
    import sys

    for p in (ROOT, os.path.join(ROOT, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch
    import torch.distributed as dist

    from monalisa_b200.sharded import ShardedTevaMorphosia, shard_frames

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    case = _case()
    bounds = shard_frames([g.l_size for g in case["Gu"]], world)
    lo, hi = bounds[rank], bounds[rank + 1]
    eng = OracleEngine(case, list(range(lo, hi)))
    sh = ShardedTevaMorphosia(eng, lo, hi, case["nFr"], group=dist.group.WORLD)
    hist = []
    x = sh.run([torch.from_numpy(case["y"][f]) for f in range(lo, hi)],
               [torch.from_numpy(case["ve"][f]) for f in range(lo, hi)],
               [torch.from_numpy(case["x0"][f].copy()) for f in range(lo, hi)], 0.01, 0.1, 3, 4, 10.0,
               regul_mode=mode, history=hist)
    out[rank] = (lo, hi, [v.numpy() for v in x], hist)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,mode", [(2, "normal"), (3, "adapt")])
def test_sharded_chain_matches_single_process_restatement(world, mode):
    import sys

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    case = _case()
    hist_ref = []
    ref = oracle.bmTevaMorphosia_chain([v.copy() for v in case["x0"]], case["y"],
                                       case["ve"], case["C"], case["Gu"], case["Gut"], case["n_u"], 0.01, 0.1, 4, 10.0,
                                       3, history=hist_ref, regul_mode=mode)
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, mode, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    got = [None] * case["nFr"]
    for r in range(world):
        lo, hi, xs, hist = out[r]
        for k, f in enumerate(range(lo, hi)):
            got[f] = xs[k]
        np.testing.assert_allclose(np.array(hist), np.array(hist_ref), rtol=1e-6)
    a = np.concatenate([np.ravel(v) for v in got]).astype(np.complex128)
    b = np.concatenate([np.ravel(v) for v in ref]).astype(np.complex128)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5


def test_shard_frames_balances_contiguous_runs():
    from monalisa_b200.sharded import shard_frames

    b = shard_frames([1, 1, 1, 1, 10, 1, 1, 1], 2)
    assert b[0] == 0 and b[-1] == 8 and len(b) == 3 and 1 <= b[1] <= 7
    assert abs(sum([1, 1, 1, 1, 10, 1, 1, 1][:b[1]]) - 8.5) <= 5.5
    assert shard_frames([3] * 6, 3) == [0, 2, 4, 6]
    with pytest.raises(ValueError):
        shard_frames([1, 1], 3)
