"""Mixed precision (FP16 matrix values, the 3-D transforms' intermediate in
scaled FP16 inside the CG steps, FP32 k-space vectors, sums and FFT arithmetic,
FP64 CG scalars) against the FP64 restatement of the same
discrete reconstruction, and the forward model against the FP64 direct
NUDFT.

Gates: the mixed CG-SENSE image within relative L2 1e-3 of the FP64
restatement (bmSensa.m with every product in double); the mixed forward
model's error against the direct NUDFT at 2048 samples no more than 1e-3
above the FP32 model's (that error is the gridding approximation itself).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def case():
    from monalisa_b200 import traj

    n, N, nCh = 24, 48, 8
    t = traj.bmTraj_fullRadial3_phyllotaxis_lineAssym2(48, 500, 1, 1.0)
    ve = traj.bmVolumeElement_full_radial3(t)
    n_u, N_u = np.array([n] * 3), np.array([N] * 3)
    C = traj.coil_maps(n_u, nCh, 6)
    x_true = traj.ellipsoid_phantom(n_u, 5, 7)
    G = oracle.traj2sparsemat(t, ve, N_u, [1, 1, 1], "gauss", 3, [0.61, 10])
    KFC = oracle.bmKF(C, N_u, n_u, [1, 1, 1], nCh, "gauss", 3, [0.61, 10])
    y = oracle.bmShanna(x_true, G["Gu"], KFC, n_u)
    rng = np.random.default_rng(8)
    y = (y + 1e-3 * np.abs(y).mean() * (rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape))
         ).astype(np.complex64)
    return dict(t=t, ve=ve, n_u=n_u, N_u=N_u, C=C, x_true=x_true, G=G, y=y, nCh=nCh)


def _recon(case, precision):
    import monalisa_b200 as mb

    Gu, Gut = mb.bmTraj2SparseMat(case["t"], case["ve"], case["N_u"], [1, 1, 1], "gauss", 3, [0.61, 10])
    r = mb.SensaRecon(Gu, Gut, case["C"], case["n_u"], precision=precision)
    return r, r.run_host(case["y"], case["ve"], nIter=1, nCGD=10)


def test_mixed_cg_sense_within_1e3_of_fp64(case):
    x64 = oracle.bmSensa(np.zeros(int(np.prod(case["n_u"]))), case["y"], case["ve"], case["C"], case["G"]["Gu"],
                         case["G"]["Gut"], case["n_u"], 10, dtype=np.complex128)
    r32, x32 = _recon(case, "fp32")
    rm, xm = _recon(case, "mixed")
    assert rm.plan.precision == "mixed" and rm.plan.adjoint_mode != "fused"
    assert rm.plan.half_intermediate  # 3-D, 8 coils, TMA passes: B in FP16 inside the CG steps
    rh, xh = _recon(case, "fp16_values")
    assert rh.plan.precision == "fp16_values"
    e32, em, eh = rel(x32, x64), rel(xm, x64), rel(xh, x64)
    assert e32 <= 1e-4, e32
    assert em <= 1e-3, em
    assert eh <= 1e-3, eh
    assert em > e32 and eh > e32  # the reduced-precision paths really run in lower precision


def test_mixed_fp16_intermediate_on_and_off(case):
    """The same mixed solve with the 3-D transforms' intermediate and the
    forward grid in scaled FP16 (TMA line passes) and in FP32 (cp.async
    passes, which cannot load FP16): both within 1e-3 of the FP64 restatement, and different from each
    other (the FP16 storage really runs); an FP32 plan reports it off."""
    x64 = oracle.bmSensa(np.zeros(int(np.prod(case["n_u"]))), case["y"], case["ve"], case["C"], case["G"]["Gu"],
                         case["G"]["Gut"], case["n_u"], 10, dtype=np.complex128)
    r32, _ = _recon(case, "fp32")
    assert not r32.plan.half_intermediate
    out = {}
    for buffers in (2, 0):
        import monalisa_b200 as mb

        Gu, Gut = mb.bmTraj2SparseMat(case["t"], case["ve"], case["N_u"], [1, 1, 1], "gauss", 3, [0.61, 10])
        r = mb.SensaRecon(Gu, Gut, case["C"], case["n_u"], precision="mixed")
        r.plan.variant = {"pass_buffers": buffers}
        assert r.plan.half_intermediate == (buffers == 2)
        assert r.plan.half_grid == (buffers == 2)  # 8 coils, 27-entry Gu rows: the grid in FP16 too
        out[buffers] = r.run_host(case["y"], case["ve"], nIter=1, nCGD=10)
    e_on, e_off = rel(out[2], x64), rel(out[0], x64)
    assert e_on <= 1e-3 and e_off <= 1e-3, (e_on, e_off)
    assert rel(out[2], out[0]) > 0, "FP16 intermediate had no effect"


def test_mixed_forward_model_vs_nudft(case):
    """Forward model error against the FP64 NUDFT at 2048 samples: FP32 and
    mixed (the plan's forward operator: FP16 matrix values; the CG steps'
    FP16 transform intermediate is covered by the image test above)."""
    import monalisa_b200 as mb
    import torch

    idx = np.random.default_rng(9).choice(case["t"].shape[1], 2048, replace=False)
    ref = oracle.nudft_fp64(case["x_true"], case["C"], case["t"][:, idx], case["n_u"], [1, 1, 1], case["N_u"])
    x = torch.from_numpy(case["x_true"]).cuda()
    errs = {}
    for prec in ("fp32", "mixed"):
        r, _ = _recon(case, prec)
        y = r.plan.shanna(x)
        errs[prec] = rel(y.cpu().numpy()[idx], ref)
    assert errs["fp32"] < 0.2  # the gridding approximation (Gaussian window, nWin 3)
    assert errs["mixed"] - errs["fp32"] <= 1e-3, errs
