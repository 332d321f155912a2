"""Input generators: radial trajectories, volume elements, coil
sensitivities and phantoms (seeded, synthetic).

Trajectories:
  bmTraj_fullRadial2_lineAssym2        src/traj2/bmTraj_fullRadial2_lineAssym2.m:10-21
  bmTraj_fullRadial3_phyllotaxis_lineAssym2
                                       src/traj3/bmTraj_fullRadial3_phyllotaxis_lineAssym2.m:45-56
  bmPhyllotaxisAngle3                  src/traj3/bmPhyllotaxisAngle3.m:24-52
  golden_angle_radial2: 2-D radial with golden-angle spoke order (radii as
                        in bmTraj_fullRadial2_lineAssym2)
Volume elements:
  bmVolumeElement1                     src/geom1/bmVolumeElement1.m
  bmVolumeElement_full_radial3         src/geom3/bmVolumeElement_full_radial3.m:42-49
  bmVolumeElement_voronoi_full_radial2 src/geom2/bmVolumeElement_voronoi_full_radial2.m:55-73
Coil maps: degree <= 2 Legendre tensor basis with seeded N(0,1) complex
coefficients and magnitude rescaling, after
src/coilSense/simu/bcaNeith_coilSensitivitySimulation2.m:11-79 (2-D there,
extended to 3-D here).
"""
from __future__ import annotations

import numpy as np

GOLDEN = (1 + 5 ** 0.5) / 2


def bmTraj_fullRadial2_lineAssym2(N, nSeg, dK_n):
    """Equal-angle 2-D radial lines: t [2, N*nSeg]."""
    kMax = N * dK_n / 2
    phi = np.linspace(0, 2 * np.pi, nSeg + 1)[:-1]
    r = (np.arange(N) - N // 2) * kMax / (N // 2)
    t = np.zeros((N, nSeg, 2))
    t[:, :, 0] = np.outer(r, np.cos(phi))
    t[:, :, 1] = np.outer(r, np.sin(phi))
    return t.reshape(N * nSeg, 2, order="F").T.copy()


def golden_angle_radial2(N, nSeg, dK_n):
    """2-D radial, spoke k at angle k*180deg/golden ratio (full diameter
    spokes), radii (-N/2 .. N/2-1) * kMax/(N/2): t [2, N*nSeg]."""
    kMax = N * dK_n / 2
    phi = np.arange(nSeg) * np.pi / GOLDEN
    r = (np.arange(N) - N // 2) * kMax / (N // 2)
    x = np.outer(r, np.cos(phi))
    y = np.outer(r, np.sin(phi))
    return np.stack([x.ravel(order="F"), y.ravel(order="F")])


def bmPhyllotaxisAngle3(nseg, nshot, flagSelfNav=False, counter_start=1):
    """Spiral phyllotaxis angles (theta, phi) [nseg*nshot]."""
    golden_angle = 2 * np.pi - 2 * np.pi / GOLDEN
    nseg_tot = nseg * nshot
    nseg_pure = nseg_tot - nshot if flagSelfNav else nseg_tot
    q = np.pi / (2 * np.sqrt(nseg_pure))
    phi = np.zeros(nseg_tot)
    theta = np.zeros(nseg_tot)
    counter = counter_start
    for i in range(nseg):
        for j in range(nshot):
            idx = i + j * nseg
            if flagSelfNav and i == 0:
                continue
            phi[idx] = np.mod(counter * golden_angle, 2 * np.pi)
            theta[idx] = q * np.sqrt(counter)
            counter += 1
    return theta, phi


def bmTraj_fullRadial3_phyllotaxis_lineAssym2(N, nSeg, nShot, dK_n, flagSelfNav=False, counter_start=1,
                                              q_segments=None):
    """3-D koosh-ball lines through the centre: t [3, N*nSeg*nShot]."""
    if N % 2:
        raise ValueError("N_n must be even")
    theta, phi = bmPhyllotaxisAngle3(nSeg, nShot, flagSelfNav, counter_start)
    if q_segments is not None:  # spread a subset over the angular range of q_segments lines
        q = np.pi / (2 * np.sqrt(q_segments))
        theta = q * np.sqrt(np.arange(counter_start, counter_start + nSeg * nShot))
    r = np.arange(-0.5, 0.5 - 1 / N + 1e-12, 1 / N)[:N]
    x = np.outer(r, np.cos(phi) * np.sin(theta))
    y = np.outer(r, np.sin(phi) * np.sin(theta))
    z = np.outer(r, np.cos(theta))
    return np.stack([x.ravel(order="F"), y.ravel(order="F"), z.ravel(order="F")]) * N * dK_n


def bmVolumeElement1(x):
    """1-D Voronoi lengths of each column, ordered by the first column."""
    x = np.asarray(x, np.float64)
    if x.ndim == 1:
        x = x[:, None]
    perm = np.argsort(x[:, 0], kind="stable")
    inv = np.argsort(perm, kind="stable")
    s = x[perm]
    mid = (s[1:] + s[:-1]) / 2
    mid = np.concatenate([s[:1] - (mid[:1] - s[:1]), mid, s[-1:] + (s[-1:] - mid[-1:])])
    return (mid[1:] - mid[:-1])[inv]


def _line_direction(t):
    """bmTraj_lineDirection: mean unit direction of each line [imDim, nLine]."""
    imDim, N, nLine = t.shape
    e = t - t[:, :1, :]
    e = e[:, int(np.ceil(N / 2)) - 1:, :]
    nrm = np.sqrt(np.sum(e ** 2, axis=0, keepdims=True))
    with np.errstate(invalid="ignore", divide="ignore"):
        e = e / nrm
    return np.nanmean(e, axis=1)


def bmVolumeElement_full_radial3(t):
    """Volume elements of 3-D full radial lines (lines of N points)."""
    raise_if = np.asarray(t).shape[0] != 3
    if raise_if:
        raise ValueError("The trajectory must be 3Dim. ")
    return _ve_full_radial(t, 3)


def bmVolumeElement_voronoi_full_radial2(t, N=None):
    """Volume elements of 2-D full radial lines (angular Voronoi)."""
    return _ve_full_radial(t, 2, N)


def _ve_full_radial(t, imDim, N=None):
    t = np.asarray(t, np.float64)
    nPt = t.shape[1]
    if N is None:
        # points per line: first return to the line start direction
        N = _points_per_line(t)
    nLine = nPt // N
    tl = t.reshape(imDim, N, nLine, order="F")
    e = _line_direction(tl)
    dr = np.stack([tl[:, :, i].T @ e[:, i] for i in range(nLine)], 1)  # [N, nLine]
    dr = bmVolumeElement1(dr)
    if imDim == 3:
        ds = 4 * np.pi * np.sum(tl ** 2, axis=0) / (2 * nLine)
        v = dr.ravel(order="F") * ds.ravel(order="F")
        dr0 = np.mean(dr[N // 2, :]) / 2
        v0 = (4 / 3) * np.pi * dr0 ** 3 / (2 * nLine)
    else:
        ee = np.concatenate([e, -e], axis=1)
        ang = np.angle(ee[0] + 1j * ee[1])
        perm = np.argsort(ang, kind="stable")
        inv = np.argsort(perm, kind="stable")
        a = ang[perm]
        cut = (np.pi - a[-1]) + (a[0] + np.pi)
        vor = np.zeros_like(a)
        vor[1:-1] = (a[2:] - a[:-2]) / 2
        vor[0] = (a[1] - a[0]) / 2 + cut / 2
        vor[-1] = (a[-1] - a[-2]) / 2 + cut / 2
        vor = vor[inv][:nLine]
        ds = np.sqrt(np.sum(tl ** 2, axis=0)) * vor[None, :]
        v = dr.ravel(order="F") * ds.ravel(order="F")
        dr0 = np.mean(dr[N // 2, :]) / 2
        v0 = np.pi * dr0 ** 2 / (2 * nLine)
    v[N // 2::N] = v0
    return v


def bmVolumeElement_radial_dev(t, N=None):
    """Volume elements of a full radial trajectory computed on the device
    (mlg_volume_element_radial_dev): 3-D as bmVolumeElement_full_radial3,
    2-D as bmVolumeElement_voronoi_full_radial2.  t [imDim, nPt] (host or
    CUDA); returns a CUDA float64 tensor [nPt]."""
    import torch

    from . import _native as NN

    tt = torch.as_tensor(np.asarray(t, np.float64) if not torch.is_tensor(t) else t, dtype=torch.float64)
    tt = tt.to("cuda").contiguous()
    imDim, nPt = int(tt.shape[0]), int(tt.shape[1])
    if N is None:
        N = _points_per_line(tt.cpu().numpy())
    v = torch.empty(nPt, dtype=torch.float64, device="cuda")
    NN.call("mlg_volume_element_radial_dev", imDim, nPt, int(N), NN.tptr(tt), NN.tptr(v), NN.stream_ptr())
    return v


def _points_per_line(t):
    r = np.sqrt(np.sum(t ** 2, axis=0))
    # lines are symmetric around the centre: the first zero-radius sample is at N/2
    z = np.nonzero(r < 1e-9)[0]
    if z.size == 0:
        raise ValueError("cannot infer the line length; pass N")
    return int(2 * z[0])


def coil_maps(n_u, nCh, seed):
    """Smooth random complex sensitivities [prod(n_u), nCh] (complex64)."""
    rng = np.random.default_rng(seed)
    n_u = [int(v) for v in np.ravel(n_u)]
    d = len(n_u)
    axes = [np.linspace(-0.5, 0.5, n) for n in n_u]
    # Legendre polynomials of degree 0..2 along each axis: the tensor basis
    # P_k0(x) P_k1(y) P_k2(z) is evaluated separably
    P1 = [np.stack([np.ones_like(a), a, 0.5 * (3 * a ** 2 - 1)], 1) for a in axes]  # [n_d, 3]
    sub = "xyz"[:d]
    expr = "".join("ijk"[:d]) + "," + ",".join(f"{sub[k]}{'ijk'[k]}" for k in range(d)) + "->" + sub
    out = np.zeros((int(np.prod(n_u)), nCh), np.complex64)

    def field_of(coef):  # coefficients in the order of the basis index (k0, k1, k2), last fastest
        return np.einsum(expr, coef.reshape((3,) * d), *P1, optimize=True).ravel(order="F")

    for c in range(nCh):
        m = field_of(rng.standard_normal(3 ** d)) + 1j * field_of(rng.standard_normal(3 ** d))
        mag = np.abs(m)
        mag = mag * (1 / (mag.max() - mag.min()))
        out[:, c] = (mag * np.exp(1j * np.angle(m))).astype(np.complex64)
    return out


def ellipsoid_phantom(n_u, n_ellipsoids, seed):
    """Sum of random ellipsoids with complex amplitudes, [prod(n_u)] complex64."""
    rng = np.random.default_rng(seed)
    n_u = [int(v) for v in np.ravel(n_u)]
    grids = np.meshgrid(*[np.linspace(-1, 1, n) for n in n_u], indexing="ij")
    img = np.zeros(grids[0].shape, np.complex128)
    for _ in range(n_ellipsoids):
        c = rng.uniform(-0.5, 0.5, len(n_u))
        ax = rng.uniform(0.1, 0.5, len(n_u))
        amp = rng.uniform(0.2, 1.0) * np.exp(1j * rng.uniform(0, 2 * np.pi))
        r2 = sum(((g - ci) / ai) ** 2 for g, ci, ai in zip(grids, c, ax))
        img[r2 <= 1] += amp
    return img.ravel(order="F").astype(np.complex64)
