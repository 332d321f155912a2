"""Alternative device paths that must give identical results, each side in
a child process (the switches are read once per process):
* the line-FFT passes whose bundles the TMA unit moves (cp.async.bulk.tensor
  loads with out-of-bounds zero fill, natural-order transform, bulk tensor
  stores) against the passes that move them with per-thread cp.async copies
  (MLG_FFT_TMA=0): the arithmetic is the same, so forward and adjoint
  operators must agree bit for bit;
* the Gut product over row records (cell, count and inline entries: two
  dependent loads per row) against the coil-pair kernel over the CSR
  (MLG_GUT_REC=0 / 1 forces either), in the masked adjoint: bit for bit.  Shapes: 256-point lines x 16 coils
(16-column bundles), 192-point radix-3 lines x 12 coils (24 columns: two
lines per bundle), 2-D 512-point lines (two load boxes of 256 rows), 8 coils
(two lines per bundle), and a bundle count that leaves the last CTAs with
fewer bundles than the others.  The device wait flag must stay clear."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
import monalisa_b200 as mb
from monalisa_b200 import traj
out = {}
for name, imDim, n, spokes, nread, nCh in (("c16", 3, 64, 600, 128, 16), ("c12", 3, 48, 500, 96, 12),
                                          ("c8", 3, 32, 300, 64, 8), ("r2d", 2, 256, 64, 512, 4)):
    N = 2 * n
    if imDim == 3:
        t = traj.bmTraj_fullRadial3_phyllotaxis_lineAssym2(nread, spokes, 1, N / nread)
        ve = traj.bmVolumeElement_full_radial3(t)
    else:
        t = traj.golden_angle_radial2(nread, spokes, N / nread)
        ve = np.ones(t.shape[1])
    Gu, Gut = mb.bmTraj2SparseMat(t, ve, [N] * imDim, [1] * imDim)
    rec = mb.SensaRecon(Gu, Gut, traj.coil_maps([n] * imDim, nCh, 4), [n] * imDim)
    rng = np.random.default_rng(9)
    x = torch.from_numpy((rng.standard_normal(n ** imDim) + 1j * rng.standard_normal(n ** imDim)).astype(np.complex64)).cuda()
    y = rec.plan.shanna(x)
    out[name + "_y"] = y.cpu().numpy()
    for mode in ("full_grid", "masked", "fused"):
        rec.plan.adjoint_mode = mode
        out[name + "_x_" + mode] = rec.plan.nakatsha(y).cpu().numpy()
    rec.plan.status()
    rec.plan.close()
np.savez(sys.argv[2], **out)
"""


def _run(tmp_path, tma, rec=1):
    path = str(tmp_path / f"out_tma{tma}_rec{rec}.npz")
    env = dict(os.environ, MLG_FFT_TMA=str(tma), MLG_GUT_REC=str(rec))
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, path], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.load(path)


def test_tma_passes_bit_identical_to_cp_async_passes(tmp_path):
    a, b = _run(tmp_path, 1), _run(tmp_path, 0)
    assert set(a.files) == set(b.files)
    for k in a.files:
        assert np.isfinite(a[k]).all(), k
        assert np.array_equal(a[k], b[k]), k


def test_gut_records_bit_identical_to_pair_kernel(tmp_path):
    a, b = _run(tmp_path, 1, 1), _run(tmp_path, 1, 0)
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k


def test_plan_variants_agree_and_the_tuner_picks_one():
    """The per-plan kernel variants (TMA / cp.async passes, CSR / record Gut
    rows, whole / chunk-masked forward grid stores) in one process: the same outputs bit for bit in every
    combination; the variant tuner times them and keeps a valid one."""
    import torch

    import monalisa_b200 as mb
    from monalisa_b200 import traj

    n, N, nCh = 48, 96, 12
    t = traj.bmTraj_fullRadial3_phyllotaxis_lineAssym2(96, 500, 1, 1.0)
    Gu, Gut = mb.bmTraj2SparseMat(t, traj.bmVolumeElement_full_radial3(t), [N] * 3, [1, 1, 1])
    rec = mb.SensaRecon(Gu, Gut, traj.coil_maps([n] * 3, nCh, 4), [n] * 3)
    plan = rec.plan
    plan.adjoint_mode = "masked"
    rng = np.random.default_rng(2)
    x = torch.from_numpy((rng.standard_normal(n ** 3) + 1j * rng.standard_normal(n ** 3)).astype(np.complex64)).cuda()
    outs = []
    assert plan.variant["fwd_masked_store"] == 1  # Gu and Gut of one trajectory: covered
    for bufs in (2, 3, 0):
        for recs in (0, 1):
            for masked_store in (1, 0):
                plan.variant = {"pass_buffers": bufs, "gut_records": recs, "fwd_masked_store": masked_store}
                y = plan.shanna(x)
                outs.append((y.cpu().numpy(), plan.nakatsha(y).cpu().numpy()))
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0]) and np.array_equal(o[1], outs[0][1])
    times = plan.autotune(2)
    assert {"passes_tma_2buf", "passes_tma_3buf", "passes_cp_async"} <= set(times)
    if plan.variant["pass_buffers"] >= 2:
        assert "fwd_full_store" in times
    if plan.adjoint_mode == "masked":
        assert {"gut_csr", "gut_records"} <= set(times)
    assert plan.variant["pass_buffers"] in (0, 2, 3) and plan.variant["gut_records"] in (0, 1)
    plan.status()
    plan.close()
