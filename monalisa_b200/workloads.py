"""Seeded synthetic workloads with the shapes of the benchmark
configurations (no public dataset is involved; the reference's example data
is not available).

koosh3d: 3-D koosh-ball radial (spiral-phyllotaxis spoke directions),
  128^3 image, 256^3 grid (oversampling 2), 4096 spokes x 256 samples,
  16 coils with smooth random complex sensitivities, k-space simulated from a
  random ellipsoid phantom by the forward operator, CG-SENSE 30 iterations,
  Gaussian window nWin = 3, (sigma, K_max) = (0.61, 10).
radial2d: 2-D golden-angle radial, 256^2 image, 512^2 grid, 256 spokes x 512
  samples, Kaiser-Bessel width 3, 1 coil, i.i.d. Gaussian complex64 k-space.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import traj as T


@dataclass
class Workload:
    name: str
    imDim: int
    n_u: np.ndarray
    N_u: np.ndarray
    dK_u: np.ndarray
    nCh: int
    nCGD: int
    kernelType: str
    nWin: int
    kernelParam: list
    t: np.ndarray = None
    ve: np.ndarray = None
    C: np.ndarray = None
    x_true: np.ndarray = None
    y: np.ndarray = None  # host k-space [nPt, nCh] when not simulated on the device
    info: dict = field(default_factory=dict)

    @property
    def nPt(self) -> int:
        return int(self.t.shape[1])


def koosh3d(n=128, oversampling=2, nSpoke=4096, nRead=256, nCh=16, nCGD=30, seed=2) -> Workload:
    N = n * oversampling
    w = Workload("koosh3d", 3, np.array([n] * 3), np.array([N] * 3), np.ones(3), nCh, nCGD, "gauss", 3, [0.61, 10])
    # the reference generator with N = nRead points per line covering +-N/2 grid units
    w.t = T.bmTraj_fullRadial3_phyllotaxis_lineAssym2(nRead, nSpoke, 1, N / nRead)
    w.ve = T.bmVolumeElement_full_radial3(w.t)
    w.C = T.coil_maps(w.n_u, nCh, seed)
    w.x_true = T.ellipsoid_phantom(w.n_u, 10, seed + 100)
    w.info = dict(image=f"{n}^3", grid=f"{N}^3", spokes=nSpoke, samples_per_spoke=nRead, coils=nCh,
                  kernel="gauss nWin=3 sigma=0.61", iterations=nCGD, seed=seed)
    return w


def radial2d(n=256, oversampling=2, nSpoke=256, nRead=512, nCh=1, nCGD=20, seed=1) -> Workload:
    N = n * oversampling
    w = Workload("radial2d", 2, np.array([n] * 2), np.array([N] * 2), np.ones(2), nCh, nCGD, "kaiser", 3,
                 [1.95, 10, 10])
    w.t = T.golden_angle_radial2(nRead, nSpoke, N / nRead)
    w.ve = T.bmVolumeElement_voronoi_full_radial2(T.bmTraj_fullRadial2_lineAssym2(nRead, nSpoke, N / nRead), nRead)
    rng = np.random.default_rng(seed)
    w.C = np.ones((int(np.prod(w.n_u)), nCh), np.complex64)
    w.y = (rng.standard_normal((w.t.shape[1], nCh)) + 1j * rng.standard_normal((w.t.shape[1], nCh))).astype(np.complex64)
    w.info = dict(image=f"{n}^2", grid=f"{N}^2", spokes=nSpoke, samples_per_spoke=nRead, coils=nCh,
                  kernel="kaiser nWin=3 tau=1.95 alpha=10", iterations=nCGD, seed=seed)
    return w


@dataclass
class BinnedWorkload:
    """Frame bins of one temporal reconstruction: per-bin trajectories t[f],
    volume elements ve[f] and phantoms x_true[f]; one coil set C."""
    name: str
    n_u: np.ndarray
    N_u: np.ndarray
    dK_u: np.ndarray
    nCh: int
    kernelType: str
    nWin: int
    kernelParam: list
    delta: float
    rho: float
    nIter: int
    nCGD: int
    t: list = field(default_factory=list)
    ve: list = field(default_factory=list)
    x_true: list = field(default_factory=list)
    C: np.ndarray = None
    info: dict = field(default_factory=dict)

    @property
    def nFr(self) -> int:
        return len(self.t)

    @property
    def nPt(self) -> list:
        return [int(t.shape[1]) for t in self.t]


def koosh3d_bins(n=96, oversampling=2, nFr=20, spokes=(200, 1500), nRead=256, nCh=12, nIter=30, nCGD=5,
                 seed=3) -> BinnedWorkload:
    """3-D koosh-ball frame bins: bin f takes rng.integers(200, 1501) spokes,
    the next run of one spiral-phyllotaxis sequence (continuing its counter,
    directions spread over the whole sequence's angular range), 256 samples
    per spoke; 96^3 image, 192^3 grid, 12 coils; temporal-TV ADMM with
    delta = 0.01, rho = 10 delta, 30 iterations of 5 CG steps.  The phantom's
    ellipsoids drift and pulse from bin to bin."""
    N = n * oversampling
    rng = np.random.default_rng(seed)
    counts = rng.integers(spokes[0], spokes[1] + 1, nFr)
    total = int(counts.sum())
    w = BinnedWorkload("koosh3d_bins", np.array([n] * 3), np.array([N] * 3), np.ones(3), nCh, "gauss", 3, [0.61, 10],
                       0.01, 0.1, nIter, nCGD)
    w.C = T.coil_maps(w.n_u, nCh, seed)
    base = T.ellipsoid_phantom(w.n_u, 10, seed + 100)
    counter = 1
    for f, ns in enumerate(counts):
        t = T.bmTraj_fullRadial3_phyllotaxis_lineAssym2(nRead, int(ns), 1, N / nRead, counter_start=counter,
                                                        q_segments=total)
        counter += int(ns)
        w.t.append(t)
        w.ve.append(T.bmVolumeElement_full_radial3(t))
        phase = 2 * np.pi * f / nFr
        w.x_true.append((base * (1 + 0.2 * np.sin(phase))
                         + 0.3 * T.ellipsoid_phantom(w.n_u, 1, seed + 200 + f)).astype(np.complex64))
    w.info = dict(image=f"{n}^3", grid=f"{N}^3", bins=nFr, spokes_per_bin=[int(c) for c in counts],
                  samples_per_spoke=nRead, coils=nCh, kernel="gauss nWin=3 sigma=0.61", admm_iterations=nIter,
                  cg_steps=nCGD, delta=0.01, rho=0.1, seed=seed)
    return w


# request mix for serving: 60 % 2-D golden-angle radial (256^2 image, 512^2
# grid, 128-512 spokes x 512 samples), 40 % 3-D koosh ball (96^3 or 128^3
# image, 1000-4096 spokes x 256 samples), 8-16 coils, CG-SENSE with 20 CG
# steps, Poisson arrivals.  A fixed set of protocol templates (trajectory,
# volume elements, coil maps, phantom) stands for the scanner protocols the
# requests come from; each template is one trajectory key.
SERVING_TEMPLATES_2D = ((128, 8), (256, 12), (512, 16))               # spokes, coils
SERVING_TEMPLATES_3D = ((96, 1024, 8), (128, 2048, 12), (128, 4096, 16))  # n, spokes, coils


def serving_templates(seed=5, scale=1.0):
    """The protocol templates of the serving mix; ``scale`` < 1 shrinks the
    spoke counts (tests)."""
    out = []
    for k, (ns, nCh) in enumerate(SERVING_TEMPLATES_2D):
        ns = max(8, int(ns * scale))
        n, N = 256, 512
        t = T.golden_angle_radial2(512, ns, N / 512)
        ve = T.bmVolumeElement_voronoi_full_radial2(T.bmTraj_fullRadial2_lineAssym2(512, ns, N / 512), 512)
        out.append(dict(key=("2d", k), imDim=2, t=t, ve=ve, N_u=np.array([N, N]), n_u=np.array([n, n]),
                        C=T.coil_maps([n, n], nCh, seed + k), x_true=T.ellipsoid_phantom([n, n], 6, seed + 10 + k)))
    for k, (n, ns, nCh) in enumerate(SERVING_TEMPLATES_3D):
        ns = max(16, int(ns * scale))
        N = 2 * n
        t = T.bmTraj_fullRadial3_phyllotaxis_lineAssym2(256, ns, 1, N / 256)
        out.append(dict(key=("3d", k), imDim=3, t=t, ve=T.bmVolumeElement_full_radial3(t), N_u=np.array([N] * 3),
                        n_u=np.array([n] * 3), C=T.coil_maps([n] * 3, nCh, seed + 20 + k),
                        x_true=T.ellipsoid_phantom([n] * 3, 8, seed + 30 + k)))
    return out


def serving_schedule(n_requests, rate, seed=5):
    """Poisson arrival offsets (seconds) and template indices: 60 % drawn from
    the 2-D templates, 40 % from the 3-D ones."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    is3d = rng.random(n_requests) < 0.4
    n2, n3 = len(SERVING_TEMPLATES_2D), len(SERVING_TEMPLATES_3D)
    tmpl = np.where(is3d, n2 + rng.integers(0, n3, n_requests), rng.integers(0, n2, n_requests))
    return arrivals, tmpl
