"""Generates the golden fixtures in this directory.

The Monalisa reference ships no tests, fixtures or golden vectors, so the
fixtures are produced by running the reference's own C++ MEX kernels,
compiled unmodified from the reference tree against the project's MEX-API
shim (``make -C oracle ref``), on small seeded inputs.  Run from the repo
root (needs the reference tree, so it runs only where it is mounted):

    make -C oracle ref port && python tests/golden/make_golden.py

Each ``.npz`` stores the inputs exactly as passed to the MEX gateway and the
gateway's outputs.  Matrices come from the numpy restatement of
bmTraj2SparseMat (oracle/oracle.py); the kernels consuming them are the
reference's.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402


def _traj2(nSpoke, nRead, N, rng, jitter=0.0):
    ang = np.arange(nSpoke) * np.pi / ((1 + 5 ** 0.5) / 2)
    r = (np.arange(nRead) - nRead // 2) * (N / 2) / (nRead // 2)
    t = np.stack([np.outer(r, np.cos(ang)).ravel(order="F"), np.outer(r, np.sin(ang)).ravel(order="F")])
    return t + jitter * rng.standard_normal(t.shape)


def leight(rng, imDim, N, nCh, nPt, nWin, sigma, name):
    t = rng.uniform(1.0, N + 0.999, size=(imDim, nPt)).astype(np.float32)
    # a few points on exact nodes, on the border and outside the window range
    t[:, 0] = 1.0
    t[:, 1] = float(N)
    t[:, 2] = N / 2 + 0.5
    aR = rng.standard_normal((nCh, nPt)).astype(np.float32)
    aI = rng.standard_normal((nCh, nPt)).astype(np.float32)
    Dn = rng.uniform(0.1, 2.0, size=(1, nPt)).astype(np.float32)
    m = oracle.ref_mex(f"bmGridder_n2u_leight{imDim}_mex")
    args_t = [t[i][None, :] for i in range(imDim)]
    Ns = [np.int32(N)] * imDim
    if imDim == 1:
        # the reference gateway reads prhs[4] as Dn and prhs[9..11] as nWin
        # and kernel parameters (bmGridder_n2u_leight1_mex.cpp:54-67)
        args = [aR, aI, args_t[0], None, Dn, np.int32(nCh), np.int32(nPt), Ns[0], None,
                np.int32(nWin), np.float32(sigma), np.float32(10)]
    else:
        args = [aR, aI, *args_t, Dn, np.int32(nCh), np.int32(nPt), *Ns, np.int32(nWin),
                np.float32(sigma), np.float32(10)]
    bR, bI = m(*args, nlhs=2)
    np.savez_compressed(os.path.join(HERE, name), t=t, aR=aR, aI=aI, Dn=Dn, N=N, nCh=nCh, nPt=nPt,
                        nWin=nWin, sigma=np.float32(sigma), imDim=imDim, bR=bR, bI=bI)


def n2u(rng, name):
    N_u = np.array([16, 16])
    t = _traj2(12, 16, 16, rng, 0.3)
    nPt = t.shape[1]
    Dn = rng.uniform(0.5, 1.5, nPt)
    keep, w, nJump, nNb = oracle.gridder_n2u_weights(t, Dn, N_u, [1, 1], "kaiser", 3, [1.95, 10, 10])
    nCh = 3
    aR = rng.standard_normal((nCh, int(keep.sum()))).astype(np.float32)
    aI = rng.standard_normal((nCh, int(keep.sum()))).astype(np.float32)
    m = oracle.ref_mex("bmGridder_n2u_mex")
    bR, bI = m(aR, aI, w[None, :], nJump[None, :], np.int32(nCh), np.int32(nNb), np.int32(aR.shape[1]),
               np.int32(N_u.prod()), nlhs=2)
    np.savez_compressed(os.path.join(HERE, name), aR=aR, aI=aI, w=w, nJump=nJump, nCh=nCh, nNb=nNb,
                        nPt=aR.shape[1], Nu_tot=int(N_u.prod()), bR=bR, bI=bI)


def spmv(rng, name):
    N_u = np.array([16, 16])
    t = _traj2(10, 24, 16, rng, 0.2)
    nPt = t.shape[1]
    ve = rng.uniform(0.5, 1.5, nPt)
    G = oracle.traj2sparsemat(t, ve, N_u, [1, 1], "gauss", 3, [0.61, 10])
    Gu, Gut = G["Gu"], G["Gut"]
    nVec = 3
    v_u = (rng.standard_normal((Gu.r_size, nVec)) + 1j * rng.standard_normal((Gu.r_size, nVec))).astype(np.complex64)
    v_t = (rng.standard_normal((Gut.r_size, nVec)) + 1j * rng.standard_normal((Gut.r_size, nVec))).astype(np.complex64)
    out = {}
    for tag, Gm, v in (("u", Gu, v_u), ("t", Gut, v_t)):
        lj = Gm.l_jump if Gm.l_jump.size else None
        flag = np.int32(1 if lj is not None else 0)
        common = (np.int32(Gm.r_size), Gm.r_jump[None, :], Gm.r_nJump[None, :], Gm.m_val[None, :],
                  np.int32(Gm.l_size), None if lj is None else lj[None, :], np.int32(Gm.l_nJump), flag)
        for kern in ("bmSparseMat_cC_oBlock_omp_mex", "bmSparseMat_cC_oBlock_mex"):
            wR, wI = oracle.ref_mex(kern)(*common, np.ascontiguousarray(v.real), np.ascontiguousarray(v.imag),
                                          np.int32(nVec), nlhs=2)
            out[f"{tag}_{kern}"] = wR + 1j * wI
        # row layout, complex via separate imaginary storage
        vr = np.ascontiguousarray(v.T)
        w = oracle.ref_mex("bmSparseMat_cR_oBlock_mex")(*common, vr, np.int32(nVec), nlhs=1)
        out[f"{tag}_bmSparseMat_cR_oBlock_mex"] = w
        # real column layout
        wr = oracle.ref_mex("bmSparseMat_rC_oBlock_mex")(*common, np.ascontiguousarray(v.real), np.int32(nVec), nlhs=1)
        out[f"{tag}_bmSparseMat_rC_oBlock_mex"] = wr
        for f in ("r_size", "r_jump", "r_nJump", "m_val", "l_size", "l_jump", "l_nJump"):
            out[f"{tag}_G_{f}"] = np.asarray(getattr(Gm, f))
    idx, chk = oracle.ref_mex("bmSparseMat_r_nJump2index_mex")(np.int32(Gu.l_size), Gu.r_nJump[None, :],
                                                               np.int64(Gu.r_nJump.sum()), nlhs=2)
    out["r_nJump2index"] = idx
    np.savez_compressed(os.path.join(HERE, name), v_u=v_u, v_t=v_t, t=t, ve=ve, **out)


def operators(rng, name):
    """Shanna / Nakatsha / CG-SENSE on a small 2D case, with the reference's
    cC_oBlock_omp SpMV inside the restated MATLAB operators."""
    n_u = np.array([16, 16])
    N_u = np.array([32, 32])
    t = _traj2(24, 32, 32, rng)
    nPt = t.shape[1]
    ve = rng.uniform(0.5, 1.5, nPt)
    G = oracle.traj2sparsemat(t, ve, N_u, [1, 1], "kaiser", 3, [1.95, 10, 10])
    nCh = 2
    C = (rng.standard_normal((n_u.prod(), nCh)) + 1j * rng.standard_normal((n_u.prod(), nCh))).astype(np.complex64)
    KFC = oracle.bmKF(C, N_u, n_u, [1, 1], nCh, "kaiser", 3, [1.95, 10, 10])
    KFC_conj = oracle.bmKF_conj(np.conj(C), N_u, n_u, [1, 1], nCh, "kaiser", 3, [1.95, 10, 10])
    x = (rng.standard_normal(n_u.prod()) + 1j * rng.standard_normal(n_u.prod())).astype(np.complex64)
    y = (rng.standard_normal((nPt, nCh)) + 1j * rng.standard_normal((nPt, nCh))).astype(np.complex64)
    spm = oracle.SpMV("reference")
    yS = oracle.bmShanna(x, G["Gu"], KFC, n_u, spm)
    xN = oracle.bmNakatsha(y, G["Gut"], KFC_conj, True, n_u, spm)
    hist = []
    xs = oracle.bmSensa(np.zeros(n_u.prod(), np.complex64), y, ve, C, G["Gu"], G["Gut"], n_u, 5, 10.0, 1,
                        spm, history=hist)
    np.savez_compressed(os.path.join(HERE, name), t=t, ve=ve, C=C, KFC=KFC, KFC_conj=KFC_conj, x=x, y=y,
                        shanna=yS, nakatsha=xN, sensa=xs, sensa_residual=np.array(hist), n_u=n_u, N_u=N_u)


def main():
    if not oracle.ref_available():
        sys.exit("oracle/_ref not built: run `make -C oracle ref port` first")
    rng = np.random.default_rng(20231)
    leight(rng, 1, 24, 2, 40, 3, 0.61, "leight1_gauss.npz")
    leight(rng, 2, 16, 2, 60, 3, 0.61, "leight2_gauss.npz")
    leight(rng, 2, 16, 3, 60, 4, 0.5, "leight2_even.npz")
    leight(rng, 3, 8, 3, 50, 3, 0.61, "leight3_gauss.npz")
    n2u(rng, "n2u_kaiser.npz")
    spmv(rng, "spmv.npz")
    operators(rng, "operators2d.npz")
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
