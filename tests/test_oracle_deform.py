"""Deformation-field matrices (bmImDeformField2SparseMat.m with the weights
of bmImDeformField2sparseMat_ind_weight.m) restated in the oracle, pinned
by known answers: a zero field is the identity, an integer displacement a
(cyclic with torus_flag) shift, a half-pixel displacement splits a pixel
evenly over its two neighbours; Gut is Gu's transpose and Gn's rows sum to
one.  The reference has no tests or fixtures for these matrices and MATLAB
is not installed, so these identities are the pin.  The temporal chain with
identity deformation matrices equals the chain without them, bit for bit.
"""
import numpy as np
import pytest

import oracle


def dense(G):
    return G.to_scipy().toarray().astype(np.float64)


@pytest.mark.parametrize("N_u", [[7], [5, 4], [4, 3, 5]])
@pytest.mark.parametrize("torus", [False, True])
def test_zero_field_is_identity(N_u, torus):
    nPt = int(np.prod(N_u))
    out = oracle.deform2sparsemat(np.zeros((len(N_u), nPt)), N_u, torus_flag=torus)
    assert np.array_equal(dense(out["Gu"]), np.eye(nPt))
    assert np.array_equal(dense(out["Gut"]), np.eye(nPt))


def _shift_index(N_u, shift, wrap):
    """Target pixel of every pixel under an integer shift (-1: outside)."""
    coords = np.stack(np.meshgrid(*[np.arange(n) for n in N_u], indexing="ij"))
    coords = coords.reshape(len(N_u), -1, order="F") + np.asarray(shift)[:, None]
    inside = np.all((coords >= 0) & (coords < np.asarray(N_u)[:, None]), axis=0)
    coords = np.mod(coords, np.asarray(N_u)[:, None])
    lin = np.ravel_multi_index(tuple(coords), N_u, order="F")
    return np.where(inside | wrap, lin, -1)


@pytest.mark.parametrize("torus", [False, True])
def test_integer_shift(torus):
    N_u, shift = [5, 4], [1, -2]
    nPt = 20
    v = np.repeat(np.asarray(shift, np.float64)[:, None], nPt, axis=1)
    G = dense(oracle.deform2sparsemat(v, N_u, torus_flag=torus)["Gu"])
    tgt = _shift_index(N_u, shift, torus)
    want = np.zeros((nPt, nPt))
    for p, q in enumerate(tgt):
        if q >= 0:
            want[p, q] = 1.0
    assert np.array_equal(G, want)


def test_half_pixel_shift_splits_evenly():
    N = 6
    G = dense(oracle.deform2sparsemat(np.full((1, N), 0.5), [N])["Gu"])
    for p in range(N - 1):  # t = p + 1.5 between pixels p and p + 1
        assert G[p, p] == np.float32(0.5) and G[p, p + 1] == np.float32(0.5)
    assert not G[N - 1].any()  # t = N + 0.5 leaves the image


def test_transpose_gn_and_adjoint():
    rng = np.random.default_rng(4)
    N_u = [9, 7]
    nPt = 63
    v = 1.3 * rng.standard_normal((2, nPt))
    Dn = rng.uniform(0.5, 2.0, nPt)
    out = oracle.deform2sparsemat(v, N_u, Dn=Dn, want=("Gn", "Gu", "Gut"))
    Gu, Gut, Gn = dense(out["Gu"]), dense(out["Gut"]), dense(out["Gn"])
    assert np.array_equal(Gut, Gu.T)
    rs = Gu.sum(axis=1)
    assert np.allclose(rs[rs != 0], 1.0, atol=1e-6)
    gs = Gn.sum(axis=1)
    assert np.allclose(gs[gs != 0], 1.0, atol=1e-6)
    # same stored entries, transposed (values differ: weighted by Dn and
    # normalised per cell; tiny bump weights can round to an FP32 zero in one
    # and not in the other)
    ent = lambda G: {(int(r), int(c)) for r, c in zip(*G.to_scipy().tocoo().coords)}
    assert ent(out["Gn"]) == {(c, r) for r, c in ent(out["Gu"])}
    x, y = rng.standard_normal(nPt), rng.standard_normal(nPt)
    assert abs(np.dot(Gu @ x, y) - np.dot(x, Gut @ y)) <= 1e-12 * np.abs(Gu).sum() * np.abs(x).max() * np.abs(y).max()


def test_chain_identity_deformation_is_no_deformation():
    from monalisa_b200 import traj

    rng = np.random.default_rng(2)
    N_u, n_u, nCh, nFr = np.array([16, 16]), np.array([8, 8]), 2, 2
    C = traj.coil_maps(n_u, nCh, 3)
    KFC = oracle.bmKF(C, N_u, n_u, [1, 1], nCh, "gauss", 3, [0.61, 10])
    t_all = traj.golden_angle_radial2(16, 24, 1.0)
    G, y, ve = [], [], []
    for f in range(nFr):
        t = t_all[:, f * 12 * 16:(f + 1) * 12 * 16]
        v = traj.bmVolumeElement_voronoi_full_radial2(t, 16)
        g = oracle.traj2sparsemat(t, v, N_u, [1, 1], "gauss", 3, [0.61, 10])
        xt = traj.ellipsoid_phantom(n_u, 3, 10 + f)
        G.append(g)
        y.append(oracle.bmShanna(xt, g["Gu"], KFC, n_u).astype(np.complex64))
        ve.append(np.asarray(v, np.float32))
    eye = oracle.deform2sparsemat(np.zeros((2, 64)), n_u)
    x0 = [(0.1 * rng.standard_normal(64)).astype(np.complex64) for _ in range(nFr)]
    args = (x0, y, ve, C, [g["Gu"] for g in G], [g["Gut"] for g in G], n_u, 0.02, 0.2, 2, 10.0, 2)
    h0, h1 = [], []
    a = oracle.bmTevaMorphosia_chain(*args, history=h0)
    b = oracle.bmTevaMorphosia_chain(*args, history=h1, Tu=[eye["Gu"]] * nFr, Tut=[eye["Gut"]] * nFr)
    for f in range(nFr):
        assert np.array_equal(a[f], b[f])
    assert h0 == h1
