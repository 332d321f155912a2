"""Setup computations on the device: the deapodisation (bmK.m:6-156) must
equal the host computation bit for bit (same FP64 passes and summation
order, round-to-nearest operations), and the radial volume elements
(bmVolumeElement_full_radial3.m, bmVolumeElement_voronoi_full_radial2.m)
must match the restatement in monalisa_b200.traj within 1e-12 relative (FP64
on both sides; the means and the dot products are summed in other orders)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N_u,kernel,nWin,kp", [([64], "gauss", 3, [0.61, 10]),
                                                ([48, 40], "gauss", 3, [0.61, 10]),
                                                ([32, 24, 40], "gauss", 3, [0.61, 10]),
                                                ([40, 40], "kaiser", 3, [1.95, 10, 10]),
                                                ([24, 32, 16], "kaiser", 5, [2.5, 12, 8])])
def test_device_deapodization_is_bit_identical(N_u, kernel, nWin, kp):
    from monalisa_b200 import operators

    host = operators.bmK(N_u, np.ones(len(N_u)), 1, kernel, nWin, kp)[:, 0]
    dev = operators.bmK_dev(N_u, np.ones(len(N_u)), kernel, nWin, kp).cpu().numpy()
    assert np.array_equal(host, dev)


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_device_volume_elements_3d_match():
    from monalisa_b200 import traj

    for nRead, nSpoke in ((64, 300), (128, 1000)):
        t = traj.bmTraj_fullRadial3_phyllotaxis_lineAssym2(nRead, nSpoke, 1, 1.0)
        ref = traj.bmVolumeElement_full_radial3(t)
        dev = traj.bmVolumeElement_radial_dev(t).cpu().numpy()
        assert _rel(dev, ref) <= 1e-12
        assert np.all(np.abs(dev - ref) <= 1e-10 * np.abs(ref) + 1e-300)


def test_device_volume_elements_2d_match():
    from monalisa_b200 import traj

    cases = [(traj.bmTraj_fullRadial2_lineAssym2(64, 40, 1.0), 64), (traj.golden_angle_radial2(96, 55, 1.0), 96)]
    for t, N in cases:
        ref = traj.bmVolumeElement_voronoi_full_radial2(t, N)
        dev = traj.bmVolumeElement_radial_dev(t, N).cpu().numpy()
        assert _rel(dev, ref) <= 1e-12
        assert np.all(np.abs(dev - ref) <= 1e-10 * np.abs(ref) + 1e-300)


def test_device_volume_elements_reject_bad_shapes():
    import torch

    from monalisa_b200 import _native as NN
    from monalisa_b200._native import MonalisaError

    t = torch.zeros((3, 100), dtype=torch.float64, device="cuda")
    v = torch.empty(100, dtype=torch.float64, device="cuda")
    with pytest.raises(MonalisaError):
        NN.call("mlg_volume_element_radial_dev", 3, 100, 48, NN.tptr(t), NN.tptr(v), NN.stream_ptr())
    with pytest.raises(MonalisaError):
        NN.call("mlg_volume_element_radial_dev", 1, 100, 50, NN.tptr(t), NN.tptr(v), NN.stream_ptr())
