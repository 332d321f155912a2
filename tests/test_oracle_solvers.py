"""Consistency of the oracle's solver restatements (CPU).

With one frame the temporal sparsifier is F x = x - x = 0, so
bmTevaMorphosia_chain's x-update is CG-SENSE and the two restatements
(bmTevaMorphosia_chain.m, bmSensa.m) must give the same image, bit for bit;
its data term must equal bmSensa's monitoring residual.
"""
import numpy as np

import oracle


def test_tevamorphosia_one_frame_is_sensa():
    rng = np.random.default_rng(11)
    N_u, n_u, nCh, nPt = np.array([16, 16]), np.array([8, 8]), 2, 600
    t = rng.uniform(-8, 8, (2, nPt))
    ve = rng.uniform(0.5, 1.5, nPt).astype(np.float32)
    G = oracle.traj2sparsemat(t, ve, N_u, [1, 1], "gauss", 3, [0.61, 10])
    C = (rng.standard_normal((64, nCh)) + 1j * rng.standard_normal((64, nCh))).astype(np.complex64)
    y = (rng.standard_normal((nPt, nCh)) + 1j * rng.standard_normal((nPt, nCh))).astype(np.complex64)
    x0 = np.zeros(64, np.complex64)
    hs, ht = [], []
    xs = oracle.bmSensa(x0, y, ve, C, G["Gu"], G["Gut"], n_u, 4, ve_max=1.2, nIter=2, history=hs)
    xt = oracle.bmTevaMorphosia_chain([x0], [y], [ve], C, [G["Gu"]], [G["Gut"]], n_u, 0.01, 0.1, 4, 1.2, 2,
                                      history=ht)
    assert np.array_equal(xs, xt[0])
    assert [h[1] for h in ht] == hs
    assert all(h[2] == 0.0 for h in ht)


def test_back_gradient_transpose_is_its_adjoint():
    """bmBackGradientT is the adjoint of bmBackGradient on fields whose first
    slice along each axis is zero (the only fields bmSteva feeds it: z - u -
    grad x keeps those slices at 0)."""
    rng = np.random.default_rng(12)
    for n_u, dX in (([6, 5, 4], [0.5, 0.25, 2.0]), ([7, 9], [1.0, 0.125])):
        nu = int(np.prod(n_u))
        x = (rng.standard_normal(nu) + 1j * rng.standard_normal(nu)).astype(np.complex64)
        g = oracle.back_gradient((rng.standard_normal(nu) + 1j * rng.standard_normal(nu)).astype(np.complex64),
                                 n_u, [1.0] * len(n_u))  # zero first slices
        lhs = np.vdot(oracle.back_gradient(x, n_u, dX).astype(np.complex128), g.astype(np.complex128))
        rhs = np.vdot(x.astype(np.complex128), oracle.back_gradient_T(g, n_u, dX).astype(np.complex128))
        assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_steva_reduces_the_residual():
    rng = np.random.default_rng(13)
    N_u, n_u, nCh, nPt = np.array([16, 16]), np.array([8, 8]), 2, 700
    t = rng.uniform(-8, 8, (2, nPt))
    ve = rng.uniform(0.5, 1.5, nPt).astype(np.float32)
    G = oracle.traj2sparsemat(t, ve, N_u, [1, 1], "gauss", 3, [0.61, 10])
    C = (rng.standard_normal((64, nCh)) + 1j * rng.standard_normal((64, nCh))).astype(np.complex64)
    y = (rng.standard_normal((nPt, nCh)) + 1j * rng.standard_normal((nPt, nCh))).astype(np.complex64)
    h = []
    x = oracle.bmSteva(np.zeros(64, np.complex64), y, ve, C, G["Gu"], G["Gut"], n_u, 1e-3, 1e-2, 4, None, 3,
                       history=h)
    assert x.shape == (64,) and np.isfinite(x).all()
    assert h[-1][0] < float(np.sum(np.abs(y) ** 2 * ve[:, None]))
