"""The standalone C++ driver on the GPU: in file mode its reconstruction
(mlg_traj2sparsemat3 -> mlg_deapodization -> KFC / KFC_conj on the host ->
mlg_plan_create -> mlg_sensa) must equal the Python API's
(bmTraj2SparseMat -> SensaRecon.run_host) bit for bit on the same inputs --
a small c1-like 2-D golden-angle case with one coil and a 4-coil case with
coil maps; its synthetic workloads must run and reconstruct their phantom."""
import json
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "driver", "_bin", "monalisa_driver")


def _run(args):
    from monalisa_b200 import build

    build.build()
    r = subprocess.run([DRIVER] + args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("nCh,kernel,kp", [(1, "kaiser", [1.95, 10, 10]), (4, "gauss", [0.61, 10])])
def test_driver_matches_python_api_bit_for_bit(tmp_path, nCh, kernel, kp):
    import monalisa_b200 as mb
    from monalisa_b200 import traj as T

    n, N, nRead, nSpoke = 64, 128, 128, 60
    t = T.golden_angle_radial2(nRead, nSpoke, N / nRead)
    ve = T.bmVolumeElement_voronoi_full_radial2(T.bmTraj_fullRadial2_lineAssym2(nRead, nSpoke, N / nRead), nRead)
    rng = np.random.default_rng(31 + nCh)
    C = T.coil_maps([n, n], nCh, 7) if nCh > 1 else np.ones((n * n, 1), np.complex64)
    y = (rng.standard_normal((t.shape[1], nCh)) + 1j * rng.standard_normal((t.shape[1], nCh))).astype(np.complex64)
    files = {}
    for name, arr in (("t", np.asarray(t, np.float64)), ("ve", np.asarray(ve, np.float64)), ("C", C), ("y", y)):
        files[name] = str(tmp_path / f"{name}.npy")
        np.save(files[name], arr)
    out = str(tmp_path / "x.npy")
    info = _run(["--traj", files["t"], "--ve", files["ve"], "--kspace", files["y"], "--coils_file", files["C"],
                 "--N", f"{N},{N}", "--n", f"{n},{n}", "--dK", "1,1", "--kernel", kernel, "--nWin", "3",
                 "--kernelParam", ",".join(map(str, kp)), "--nIter", "1", "--nCGD", "20", "--out", out])
    x_drv = np.load(out)
    Gu, Gut = mb.bmTraj2SparseMat(t, ve, [N, N], [1, 1], kernel, 3, kp)
    rec = mb.SensaRecon(Gu, Gut, C, [n, n])
    hist = []
    x_py = rec.run_host(y, ve, nIter=1, nCGD=20, residual=hist)
    rec.plan.close()
    assert x_drv.shape == x_py.shape
    assert np.array_equal(x_drv, x_py)
    assert info["residual"][0] == hist[0]


@pytest.mark.parametrize("kind,extra", [("radial2d", ["--n", "64", "--spokes", "96", "--samples", "128"]),
                                        ("koosh3d", ["--n", "24", "--spokes", "600", "--samples", "48",
                                                     "--coils", "4"])])
def test_driver_synthetic_workloads(kind, extra):
    info = _run(["--synthetic", kind, "--nCGD", "15", "--repeat", "2"] + extra)
    assert np.isfinite(info["residual"]).all() and info["recon_ms"] > 0
    assert info["rel_err_vs_phantom"] < 0.5, info
