"""Mitosius ingest into the temporal-TV path: frame bins written as a
mitosius (MAT v5), loaded, their Gu / Gut built on the device and solved,
give exactly the reconstruction of the same bins passed in memory.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_mitosius_ingest_equals_in_memory(tmp_path):
    import monalisa_b200 as mb
    from monalisa_b200 import mitosius, traj

    rng = np.random.default_rng(11)
    N, n, nCh, nFr = 32, 16, 2, 3
    N_u, n_u = np.array([N, N]), np.array([n, n])
    C = traj.coil_maps(n_u, nCh, 4)
    KFC = oracle.bmKF(C, N_u, n_u, [1, 1], nCh, "gauss", 3, [0.61, 10])
    t_all = traj.golden_angle_radial2(N, 20 * nFr, 1.0)
    ts, ves, ys = [], [], []
    for f in range(nFr):
        t = t_all[:, f * 20 * N:(f + 1) * 20 * N]
        v = np.asarray(traj.bmVolumeElement_voronoi_full_radial2(t, N), np.float32)
        g = oracle.traj2sparsemat(t, v, N_u, [1, 1], "gauss", 3, [0.61, 10])
        y = oracle.bmShanna(traj.ellipsoid_phantom(n_u, 3, 30 + f), g["Gu"], KFC, n_u)
        y = (y + 1e-3 * np.abs(y).mean() * rng.standard_normal(y.shape)).astype(np.complex64)
        ts.append(t)
        ves.append(v)
        ys.append(y)
    d = str(tmp_path / "bins")
    mitosius.bmMitosius_create(d, ys, ts, ves)
    chain, y2, ve2 = mitosius.frame_bin_chain(d, C, n_u, N_u, [1, 1])
    args = (0.02, 0.2, 3, 3, 10.0)
    x_m = chain.run_host(y2, ve2, None, *args)
    chain.close()
    mats = [mb.bmTraj2SparseMat(t, v, N_u, [1, 1]) for t, v in zip(ts, ves)]
    direct = mb.TevaMorphosiaChain([m[0] for m in mats], [m[1] for m in mats], C, n_u, [1, 1])
    x_d = direct.run_host(ys, ves, None, *args)
    direct.close()
    for f in range(nFr):
        assert np.array_equal(x_m[f], x_d[f])
    assert np.linalg.norm(x_m[0]) > 0
