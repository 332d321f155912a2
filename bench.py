#!/usr/bin/env python
"""Benchmark: CG-SENSE reconstructions per second on one B200 per rank.

Workload (one "step" = one reconstruction): 3-D koosh-ball radial, 128^3
image on a 256^3 grid (oversampling 2), 4096 spokes x 256 samples, 16 coils,
CG-SENSE with 30 CG updates (bmSensa with one outer iteration and nCGD = 30:
32 forward and 30 adjoint operator applications).  Inputs are seeded
synthetic data with these shapes; the k-space data are simulated from an
ellipsoid phantom by the forward operator.

Every rank runs its own reconstruction (replicas: one recon does not span
GPUs), so `value` = (ranks x steps) / max-over-ranks time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

The reference arm times the reference's CPU path on the host cores: its own
C++ sparse-matrix kernel (compiled from source into oracle/_ref; the plain-C
restatement when that is absent) inside the numpy/scipy restatement of the
MATLAB operators.  Each step is a bounded sample (one forward + one adjoint
operator application on 8 of the 16 coils, about 12 s on 16 cores),
extrapolated to a full reconstruction; `--ref-sample full` times whole
reconstructions instead (about 12 minutes each), which validates the
extrapolation.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "recons/sec & p50/p99 latency vs plain GPU at ≤1e-3 rel err; gridding HBM GB/s"
UNIT = "recons/s"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []
        self._p = None
        self._t = None

    def start(self):
        try:
            self._p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                        "-lms", "200", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                       stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._p = None

    def _read(self):
        for line in self._p.stdout:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self._p is not None:
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except Exception:
                self._p.kill()
        if self._t is not None:
            self._t.join(timeout=2)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# profile order of mlg_plan_profile: forward x/y/z passes, Gu, the Gut product
# (all rows, non-empty rows, or only the long rows, by adjoint strategy),
# inverse z pass (reading the grid, the occupancy-masked grid, or gathering
# the Gut rows itself), inverse y, inverse x (fused coil sum)
STAGES = ["fwd_x", "fwd_y", "fwd_z", "gu", "gut", "inv_z", "inv_y", "inv_x"]


def algorithmic_bytes(w, Gu, Gut, nCh, adjoint, masked_store=False):
    """Bytes each stage must move at least, for one operator application
    (forward passes read the non-zero part only and write what the next pass
    needs; the inverse passes keep only the cropped lines).  The Gut / inverse
    z split depends on the adjoint strategy the plan runs; with masked
    forward stores the forward z pass must write only the cells Gu reads."""
    nnz = Gu.nnz
    nPt = Gu.l_size
    N0, N1, N2 = (int(v) for v in w.N_u)
    n0, n1, n2 = (int(v) for v in w.n_u)
    Nu, nu = N0 * N1 * N2, n0 * n1 * n2
    A = N0 * n1 * n2 * nCh * 8
    B = N0 * N1 * n2 * nCh * 8
    G = Nu * nCh * 8
    touched, n_long = Gut.row_stats()
    T = touched * nCh * 8  # the non-empty grid cells
    ysrc = nnz * 8 + nPt * nCh * 8 + 4 * nPt  # entries, k-space rows, their weights once
    if adjoint == "masked":
        gut, inv_z = ysrc + 12 * touched + T, T + Nu // 8 + B
    elif adjoint == "fused":
        gut, inv_z = n_long * nCh * 8, ysrc + 4 * (Nu + 1) + B
    else:
        gut, inv_z = ysrc + 4 * (Nu + 1) + G, G + B
    return {
        "fwd_x": nu * 8 + nu * nCh * 8 + A, "fwd_y": A + B, "fwd_z": B + (T if masked_store else G),
        "gu": nnz * 8 + 4 * (nPt + 1) + T + nPt * nCh * 8,
        "gut": gut, "inv_z": inv_z, "inv_y": B + A, "inv_x": A + nu * nCh * 8 + nu * 8,
    }


class PlainGpuSensa:
    """The comparison arm the metric names ("vs plain GPU"): CG-SENSE with
    the reference's operators moved to the GPU as stock library calls and
    nothing fused -- x .* KFC, zero-fill, fftshift(fftn(ifftshift)) by
    torch.fft (cuFFT), Gu / Gut as cuSPARSE CSR products of the real
    matrices with [cells, 2 nCh] float views, crop, .* KFC_conj, coil sum,
    and bmSensa.m's CG loop with single-precision dot products and a host
    check of the stopping test each step.  Not part of the library."""

    def __init__(self, w, Gu, Gut, KFC, KFCc, dev, dtype=None):
        import warnings

        import torch

        warnings.filterwarnings("ignore", message=".*[Ss]parse.*")
        self.t = torch
        self.dev = dev
        # complex64 (the plain arm) or complex128: the same discrete
        # reconstruction with every product in double (FP32 inputs promoted)
        self.dtype = dtype or torch.complex64
        rdt = torch.float64 if self.dtype == torch.complex128 else torch.float32
        self.n = [int(v) for v in w.n_u]
        self.N = [int(v) for v in w.N_u]
        self.nCh = int(w.nCh)

        def csr(D):
            indptr, indices, data = D.download().to_csr()
            return torch.sparse_csr_tensor(torch.from_numpy(indptr.astype(np.int32)).to(dev),
                                           torch.from_numpy(indices).to(dev), torch.from_numpy(data).to(dev, rdt),
                                           size=(D.l_size, D.r_size))

        self.Gu, self.Gut = csr(Gu), csr(Gut)
        nu = int(np.prod(self.n))
        self.KFC = torch.from_numpy(np.ascontiguousarray(np.asarray(KFC, np.complex64).reshape(nu, -1, order="F").T)).to(dev, self.dtype)
        self.KFCc = torch.from_numpy(np.ascontiguousarray(np.asarray(KFCc, np.complex64).reshape(nu, -1, order="F").T)).to(dev, self.dtype)
        self.dims = tuple(range(1, 1 + len(self.n)))
        self.box = tuple(slice(N // 2 - n // 2, N // 2 - n // 2 + n) for N, n in zip(self.N[::-1], self.n[::-1]))

    def M(self, x):
        t, C = self.t, self.nCh
        v = (self.KFC * x[None, :]).reshape(C, *self.n[::-1])
        g = t.zeros((C, *self.N[::-1]), dtype=self.dtype, device=self.dev)
        g[(slice(None),) + self.box] = v
        g = t.fft.fftshift(t.fft.fftn(t.fft.ifftshift(g, dim=self.dims), dim=self.dims), dim=self.dims)
        g = t.view_as_real(g.reshape(C, -1).T.contiguous()).reshape(-1, 2 * C)
        return t.view_as_complex(t.sparse.mm(self.Gu, g).reshape(-1, C, 2).contiguous())

    def MH(self, y, HY, scale):
        t, C = self.t, self.nCh
        yr = t.view_as_real((HY[:, None] * y).contiguous()).reshape(-1, 2 * C)
        g = t.view_as_complex(t.sparse.mm(self.Gut, yr).reshape(-1, C, 2).contiguous())
        g = g.T.reshape(C, *self.N[::-1])
        g = t.fft.fftshift(t.fft.ifftn(t.fft.ifftshift(g, dim=self.dims), dim=self.dims), dim=self.dims)
        v = g[(slice(None),) + self.box].reshape(C, -1)
        return scale * (self.KFCc * v).sum(0)

    def sensa(self, y, ve, HX, nCGD):
        t = self.t
        eps = 10 * float(np.finfo(np.float32).eps)
        y = y.to(self.dtype)
        HY = t.minimum(ve, ve.max()).to(self.KFC.real.dtype)
        x = t.zeros(int(np.prod(self.n)), dtype=self.dtype, device=self.dev)
        invHX = float(np.float32(1) / np.float32(HX))
        res = y - self.M(x)
        dagM = self.MH(res, HY, invHX)
        sq = HX * float(t.vdot(dagM, dagM).real)
        p = dagM
        for i in range(1, nCGD + 1):
            if sq < eps:
                break
            Mp = self.M(p)
            a = sq / float(t.vdot(Mp.reshape(-1), (HY[:, None] * Mp).reshape(-1)).real)
            x = x + a * p
            if i == nCGD:
                break
            res = res - a * Mp
            dagM = self.MH(res, HY, invHX)
            sqn = HX * float(t.vdot(dagM, dagM).real)
            p = dagM + (sqn / sq) * p
            sq = sqn
        r = y - self.M(x)  # monitoring (bmSensa.m:82-83)
        float(t.vdot(r.reshape(-1), (HY[:, None] * r).reshape(-1)).real)
        return x


def nudft_fp64(x, C, t, n_u, dK_u, N_u, dev):
    """FP64 direct NUDFT of an image on the device: y_j = sum_r C(r) x(r)
    exp(-2 pi i k_j . r) / prod(N_u) / prod(dK_u), pixel r of index i at
    (i - n_u/2) / (dK_u N_u), k_j = t[:, j] in physical units -- what the
    gridded forward operator approximates (no window, no deapodisation)."""
    import torch

    n_u = [int(v) for v in n_u]
    N_u = np.asarray(N_u, np.float64)
    dK_u = np.asarray(dK_u, np.float64)
    dX = 1.0 / (dK_u * N_u)
    nPix = int(np.prod(n_u))
    idx = torch.arange(nPix, device=dev)
    r, stride = [], 1
    for d, n in enumerate(n_u):
        r.append(((idx // stride) % n - n // 2).to(torch.float64) * float(dX[d]))
        stride *= n
    r = torch.stack(r, 0)  # [imDim, nPix]
    Cx = torch.as_tensor(np.asarray(C, np.complex64), device=dev).to(torch.complex128) * \
        torch.as_tensor(np.asarray(x, np.complex64), device=dev).to(torch.complex128)[:, None]
    tt = torch.as_tensor(np.asarray(t, np.float64), device=dev)  # [imDim, nS]
    out = torch.zeros((tt.shape[1], Cx.shape[1]), dtype=torch.complex128, device=dev)
    for p0 in range(0, nPix, 65536):
        ph = torch.exp(torch.complex(torch.zeros((), dtype=torch.float64, device=dev),
                                     -2 * np.pi * (tt.T @ r[:, p0:p0 + 65536])))
        out += ph @ Cx[p0:p0 + 65536]
    return out * (1.0 / float(np.prod(N_u)) / float(np.prod(dK_u)))


def run_gpu(args):
    import torch

    from monalisa_b200 import replicas

    ws, rank, local = replicas.world()
    torch.cuda.set_device(local)
    replicas.init("nccl", timeout_s=600)
    import monalisa_b200 as mb
    from monalisa_b200 import _native as N
    from monalisa_b200.workloads import koosh3d

    t0 = time.time()
    w = koosh3d()
    Gu, Gut = mb.bmTraj2SparseMat(w.t, w.ve, w.N_u, w.dK_u, w.kernelType, w.nWin, w.kernelParam)
    rec = mb.SensaRecon(Gu, Gut, w.C, w.n_u, autotune=args.adjoint == "auto")
    if args.adjoint != "auto":  # fixed strategy (profiling: launch timing under a profiler misleads the tuner)
        rec.plan.adjoint_mode = args.adjoint
    dev = torch.device("cuda", local)
    x_true = torch.from_numpy(w.x_true).to(dev)
    y = rec.plan.shanna(x_true)
    gen = torch.Generator(device=dev).manual_seed(1234)
    noise = torch.randn(y.shape, dtype=torch.complex64, device=dev, generator=gen)
    y += noise * (y.abs().mean() * 1e-3)
    ve = torch.from_numpy(np.ascontiguousarray(w.ve, np.float32)).to(dev)
    nu = int(np.prod(w.n_u))
    x = torch.zeros(nu, dtype=torch.complex64, device=dev)
    torch.cuda.synchronize()
    setup_s = time.time() - t0

    def step():
        x.zero_()
        rec.run_dev(y, ve, x, nIter=1, nCGD=w.nCGD)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # accuracy of the reconstruction against the phantom (reported, not gated)
    err = float((x - x_true).norm() / x_true.norm())

    clocks = ClockSampler(local)
    clocks.start()
    l0 = N.launch_count()
    stream = torch.cuda.current_stream()
    replicas.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    replicas.barrier()
    launches = N.launch_count() - l0
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms = replicas.max_over_ranks(ms, device=dev)
    value = replicas.throughput(ws, args.steps, ms / 1e3)

    # end to end through the C ABI with host buffers (pinned), copies inside
    ypin = torch.empty((w.nPt, w.nCh), dtype=torch.complex64, pin_memory=True)
    ypin.copy_(y)
    yR = np.ascontiguousarray(ypin.numpy().real.T)
    yI = np.ascontiguousarray(ypin.numpy().imag.T)
    yR_p = torch.empty(yR.shape, dtype=torch.float32, pin_memory=True).numpy()
    yI_p = torch.empty(yI.shape, dtype=torch.float32, pin_memory=True).numpy()
    yR_p[...] = yR
    yI_p[...] = yI
    ve_h = torch.empty(w.nPt, dtype=torch.float32, pin_memory=True).numpy()
    ve_h[...] = w.ve
    xR = torch.empty(nu, dtype=torch.float32, pin_memory=True).numpy()
    xI = torch.empty(nu, dtype=torch.float32, pin_memory=True).numpy()
    res = np.zeros(1)

    def e2e_step():
        xR[...] = 0
        xI[...] = 0
        N.call("mlg_sensa", rec.plan.handle, N.fptr(yR_p), N.fptr(yI_p), N.fptr(ve_h), 0.0, 1, w.nCGD, N.fptr(xR),
               N.fptr(xI), N.dptr(res))

    e2e_step()
    replicas.barrier()
    ta = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = replicas.max_over_ranks(time.perf_counter() - ta, device=dev)
    e2e = {"value": replicas.throughput(ws, args.steps, e2e_s), "unit": UNIT, "h2d_bytes_per_step": int(yR_p.nbytes + yI_p.nbytes +
                                                                                     ve_h.nbytes + xR.nbytes +
                                                                                     xI.nbytes),
           "d2h_bytes_per_step": int(xR.nbytes + xI.nbytes + res.nbytes)}

    # per-stage live timing of the operator kernels (CUDA events on the
    # plan's stream) -> roofline of the dominant kernel of this library
    st = np.zeros(len(STAGES))
    N.call("mlg_plan_profile", rec.plan.handle, 5, N.dptr(st))
    B = algorithmic_bytes(w, Gu, Gut, w.nCh, rec.plan.adjoint_mode,
                          masked_store=bool(rec.plan.variant["fwd_masked_store"]))
    peak, peak_kind = _peaks()
    stages = {}
    for i, nm in enumerate(STAGES):
        gbs = B[nm] / (st[i] * 1e-3) / 1e9 if st[i] > 0 else 0.0
        stages[nm] = {"ms": round(float(st[i]), 4), "algorithmic_bytes": int(B[nm]), "GBps": round(gbs, 1),
                      "frac": round(gbs / peak, 4)}
    dom = max(STAGES, key=lambda k: stages[k]["ms"])
    traffic_file = os.path.join(ROOT, "profiles", "traffic.json")
    traffic = None
    if os.path.exists(traffic_file):
        with open(traffic_file) as f:
            traffic = json.load(f).get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": stages[dom]["GBps"], "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": stages[dom]["frac"], "traffic": traffic,
                "stages": stages}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, _to_oracle(w, Gu), _to_oracle(w, Gut), y.cpu().numpy())

    # the same reconstruction by the plain GPU arm (stock cuFFT / cuSPARSE
    # calls, nothing fused), one warm-up run and one timed run, and the
    # relative difference of the two reconstructions
    plain = None
    if not args.no_plain:
        HX = np.float32(1)
        for d in range(3):
            HX = np.float32(HX * np.float32(np.float32(1) / np.float32(w.dK_u[d]) / np.float32(w.N_u[d])))
        pg = PlainGpuSensa(w, Gu, Gut, rec.KFC, rec.KFC_conj, dev)
        pg.sensa(y, ve, float(HX), w.nCGD)
        torch.cuda.synchronize()
        e0.record(stream)
        xp = pg.sensa(y, ve, float(HX), w.nCGD)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_plain = e0.elapsed_time(e1)
        step()
        torch.cuda.synchronize()
        plain = {"recons_per_s": round(1000.0 / ms_plain, 4), "ms_per_recon": round(ms_plain, 2),
                 "speedup": round(ms_plain / (ms / args.steps), 2),
                 "rel_diff": float((x - xp).norm() / xp.norm()),
                 "arm": "torch.fft (cuFFT) + torch.sparse CSR (cuSPARSE), FP32 CG scalars, same inputs"}
        del pg, xp

    # the other configurations of the benchmark, each timed with CUDA events
    extra = {}
    adjoint_c2 = rec.plan.adjoint_mode
    variant_c2 = rec.plan.variant  # the headline plan closes before the JSON line
    if not args.no_extra:
        x_fp32 = x.clone()
        ref64 = _c4_references(w, Gu, Gut, rec, y, ve, x_fp32, dev)
        extra["c4_mixed_precision"] = {
            "fp32": {"rel_err_vs_fp64": ref64["fp32_vs_fp64"], "nudft_rel_err": ref64["nudft_fp32"]},
            **{p: _mixed(w, Gu, Gut, y, ve, x_fp32, ms / args.steps, plain, stream, ref64, p)
               for p in ("mixed", "fp16_values")},
            "fp64_reference": ref64["about"]}
        rec.plan.close()
        extra["c1_radial2d"] = _c1(stream)
        from monalisa_b200.workloads import radial2d

        extra["gridding_leight"] = {
            "c2": _gridder(w, stream, "3D koosh 4096x256 samples, 16 coils -> 256^3 grid, Gauss nWin 3"),
            "c1": _gridder(radial2d(), stream, "2D radial 256x512 samples, 1 coil -> 512^2 grid, nWin 3 "
                                               "(inside L2)")}
        extra["c3_frame_bins"] = _c3(stream)
        if rank == 0:
            extra["c5_serving"] = _c5()

    out = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 (fp32 data, fp64 CG scalars)",
        "data": "synthetic (seeded koosh-ball trajectory, random coil maps, ellipsoid phantom)",
        "config": _config(w, ws),
        "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
        "recon_rel_err_vs_phantom": round(err, 5), "setup_s": round(setup_s, 2),
        "autotune": {"adjoint": adjoint_c2, "variant": variant_c2,
                     "ms": {k: round(v, 4) for k, v in (rec.tuning or {}).items()}},
        "vs_plain_gpu": plain,
        **extra,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    rec.plan.close()
    replicas.shutdown()


def _event_ms(fn, reps, stream):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _event_ms_median(fn, reps, stream):
    """Median of `reps` separately timed calls (CUDA events on `stream`): for
    the plain-GPU arms, whose host-side stopping test each CG step makes a
    single run sensitive to host scheduling."""
    import torch

    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return float(np.median(out))


def _HX(w):
    """HX = prod((1/dK_u)/N_u) in single precision (bmSensa.m:26-27)."""
    HX = np.float32(1)
    for d in range(len(w.N_u)):
        HX = np.float32(HX * np.float32(np.float32(1) / np.float32(w.dK_u[d]) / np.float32(w.N_u[d])))
    return float(HX)


def _c4_references(w, Gu, Gut, rec, y, ve, x_fp32, dev):
    """c4's references at full size: (i) the FP64 restatement of the same
    discrete reconstruction (bmSensa.m with every product in double: the
    FP32 matrices, KFC and data promoted to FP64, torch.fft / torch.sparse
    in complex128 on the device), and (iii) the FP64 direct NUDFT of the
    phantom at 2048 seeded samples, against which each precision's forward
    model is compared (the gridding approximation itself)."""
    import torch

    pg = PlainGpuSensa(w, Gu, Gut, rec.KFC, rec.KFC_conj, dev, dtype=torch.complex128)
    x64 = pg.sensa(y, ve, _HX(w), w.nCGD)
    del pg
    torch.cuda.empty_cache()
    idx = np.sort(np.random.default_rng(2048).choice(w.nPt, 2048, replace=False))
    nud = nudft_fp64(w.x_true, w.C, w.t[:, idx], w.n_u, w.dK_u, w.N_u, dev)
    xt = torch.from_numpy(w.x_true).to(dev)
    idx_d = torch.from_numpy(idx).to(dev)

    def nudft_err(plan):
        yy = plan.shanna(xt)[idx_d].to(torch.complex128)
        return float((yy - nud).norm() / nud.norm())

    rel64 = lambda xx: float((xx.to(torch.complex128) - x64).norm() / x64.norm())
    return {"x64": x64, "rel64": rel64, "nudft_err": nudft_err, "fp32_vs_fp64": rel64(x_fp32),
            "nudft_fp32": nudft_err(rec.plan),
            "about": "(i) FP64 restatement: bmSensa with FP32 inputs promoted to complex128, torch.fft/torch.sparse "
                     "on the device, 30 CG; (iii) FP64 direct NUDFT of the phantom at 2048 seeded samples vs each "
                     "precision's forward operator (FP16 values; the CG steps' FP16 transform intermediate is "
                     "covered by (i))"}


def _mixed(w, Gu, Gut, y, ve, x_fp32, ms_fp32, plain, stream, ref64, precision="mixed"):
    """c4: the c2 reconstruction in reduced precision: 'mixed' (FP16 matrix
    values, the 3-D transforms' intermediate stored in scaled FP16 inside
    the CG steps, FP32 k-space vectors and sums, FP64 scalars) or
    'fp16_values' (FP16 matrix values only).  Errors: against the FP64
    restatement (gate 1e-3), the FP32 reconstruction, and the change of the
    forward model's error against the FP64 NUDFT (at most 1e-3)."""
    import torch

    import monalisa_b200 as mb

    rec = mb.SensaRecon(Gu, Gut, w.C, w.n_u, precision=precision, autotune=True)
    x = torch.zeros_like(x_fp32)

    def step():
        x.zero_()
        rec.run_dev(y, ve, x, nIter=1, nCGD=w.nCGD)

    for _ in range(2):
        step()
    ms = _event_ms(step, 3, stream)
    out = {"workload": f"c2 inputs (3D koosh 128^3/256^3, 16 coils, 30 CG), precision {precision}",
           "recons_per_s": round(1000.0 / ms, 4), "ms_per_recon": round(ms, 2),
           "speedup_vs_fp32": round(ms_fp32 / ms, 3),
           "speedup_vs_plain_gpu": round(plain["ms_per_recon"] / ms, 2) if plain else None,
           "rel_diff_vs_fp32_recon": float((x - x_fp32).norm() / x_fp32.norm()),
           "rel_err_vs_fp64": ref64["rel64"](x),
           "nudft_rel_err": ref64["nudft_err"](rec.plan),
           "adjoint": rec.plan.adjoint_mode, "variant": rec.plan.variant,
           "half_intermediate": rec.plan.half_intermediate,
           "precision": {"mixed": "fp16 matrix values, 3-D transform intermediate (after forward y / adjoint z "
                                  "pass) in fp16 x 2^k inside the CG steps where half_intermediate, fp32 "
                                  "k-space vectors/sums/FFT arithmetic, fp64 CG scalars",
                         "fp16_values": "fp16 matrix values, fp32 k-space/sums/FFT, fp64 CG scalars"}[precision]}
    out["nudft_err_delta"] = out["nudft_rel_err"] - ref64["nudft_fp32"]
    out["gates"] = {"rel_err_vs_fp64 <= 1e-3": out["rel_err_vs_fp64"] <= 1e-3,
                    "nudft_err_delta <= 1e-3": out["nudft_err_delta"] <= 1e-3}
    rec.plan.close()
    return out


def _c1(stream):
    """c1: 2-D golden-angle radial CG-SENSE, 256^2 / 512^2, 1 coil, KB, 20 CG;
    beside it the plain-GPU arm and the reference CPU path (whole
    reconstructions: bmSensa with the reference's SpMV kernel, which runs
    2 x nCh = 2 OpenMP threads for one coil, as in the reference)."""
    import torch

    import monalisa_b200 as mb
    from monalisa_b200.workloads import radial2d

    w = radial2d()
    Gu, Gut = mb.bmTraj2SparseMat(w.t, w.ve, w.N_u, w.dK_u, w.kernelType, w.nWin, w.kernelParam)
    rec = mb.SensaRecon(Gu, Gut, w.C, w.n_u, autotune=True)
    y = torch.from_numpy(w.y).cuda()
    ve = torch.from_numpy(np.ascontiguousarray(w.ve, np.float32)).cuda()
    x = torch.zeros(int(np.prod(w.n_u)), dtype=torch.complex64, device="cuda")

    def step():
        x.zero_()
        rec.run_dev(y, ve, x, nIter=1, nCGD=w.nCGD)

    for _ in range(3):
        step()
    ms = _event_ms(step, 10, stream)
    adjoint = rec.plan.adjoint_mode
    pg = PlainGpuSensa(w, Gu, Gut, rec.KFC, rec.KFC_conj, torch.device("cuda"))
    HX = _HX(w)
    pg.sensa(y, ve, HX, w.nCGD)
    box = {}
    ms_plain = _event_ms_median(lambda: box.__setitem__("x", pg.sensa(y, ve, HX, w.nCGD)), 5, stream)
    step()
    torch.cuda.synchronize()
    plain = {"recons_per_s": round(1000.0 / ms_plain, 3), "ms_per_recon": round(ms_plain, 3),
             "speedup": round(ms_plain / ms, 2), "rel_diff": float((x - box["x"]).norm() / box["x"].norm())}
    del pg, box
    ref = ReferenceCpu(w, _to_oracle(w, Gu), _to_oracle(w, Gut), w.y, coils=w.nCh, kfc=(rec.KFC, rec.KFC_conj))
    ref.recon()  # warm-up
    t_cpu = statistics.median(ref.recon() for _ in range(3))
    x_cpu = np.asarray(ref.last_image).ravel()
    cpu = {"value": round(1.0 / t_cpu, 4), "unit": UNIT, "s_per_recon": round(t_cpu, 3), "cores": ref.cores,
           "kind": ref.kind, "sample": "whole reconstructions (median of 3): bmSensa restatement with the "
                                       "reference's bmSparseMat_cC_oBlock_omp_mex and scipy.fft",
           "rel_diff_vs_gpu": float(np.linalg.norm(x.cpu().numpy() - x_cpu) / np.linalg.norm(x_cpu))}
    rec.plan.close()
    return {"workload": "2D golden-angle radial 256^2 image, 512^2 grid, 256x512 samples, 1 coil, KB nWin 3, "
                        "20 CG iterations from x = 0 (working set inside L2)",
            "recons_per_s": round(1000.0 / ms, 3), "ms_per_recon": round(ms, 3), "adjoint": adjoint,
            "vs_plain_gpu": plain, "cpu_baseline": cpu, "speedup_vs_cpu": round(t_cpu * 1e3 / ms, 1)}


def _gridder(w, stream, label, reps=5):
    """The leight adjoint gridder (bmGridder_n2u_leight, §8 row a1) on a
    workload's samples: device buffers in and out (mlg_gridder_n2u_leight_dev),
    CUDA-event time per call, achieved GB/s of the algorithmic bytes
    nPt (4 d + 4) + nPt nCh 8 + prod(N_u) nCh 8 + prod(N_u) 4 (positions and
    Dn, split complex samples, split complex grid, weight sums)."""
    import torch

    from monalisa_b200 import _native as N
    from monalisa_b200.gridding import _leight_prepare

    rng = np.random.default_rng(7)
    data = (rng.standard_normal((w.nCh, w.t.shape[1])) + 1j * rng.standard_normal((w.nCh, w.t.shape[1]))).astype(
        np.complex64)
    aR, aI, tx, Dn, nCh, nPt, Ns = _leight_prepare(data, w.t, w.ve, w.N_u, w.dK_u)
    d = len(w.N_u)
    up = lambda a: torch.from_numpy(a).cuda() if a is not None else None
    dA, dI, dD = up(aR), up(aI), up(Dn)
    dT = [up(v) for v in tx]
    nu = int(np.prod(Ns))
    bR = torch.empty((nu, nCh), dtype=torch.float32, device="cuda")
    bI = torch.empty_like(bR)
    kp = np.ravel(w.kernelParam).astype(np.float64)

    def call():
        N.call("mlg_gridder_n2u_leight_dev", d, N.tptr(dA), N.tptr(dI), N.tptr(dT[0]), N.tptr(dT[1]), N.tptr(dT[2]),
               N.tptr(dD), nCh, nPt, Ns[0], Ns[1], Ns[2], int(w.nWin), float(kp[0]), float(kp[1]), N.tptr(bR),
               N.tptr(bI), N.stream_ptr())

    for _ in range(3):
        call()
    ms = _event_ms(call, reps, stream)
    B = nPt * (4 * d + 4) + nPt * nCh * 8 + nu * nCh * 8 + nu * 4
    peak, kind = _peaks()
    gbs = B / (ms * 1e-3) / 1e9
    return {"workload": label, "ms": round(ms, 4), "algorithmic_bytes": int(B), "GBps": round(gbs, 1),
            "frac": round(gbs / peak, 4), "peak": peak, "peak_kind": kind}


def _c3(stream):
    """c3: temporal-TV ADMM over 20 koosh frame bins (96^3 / 192^3, 12 coils,
    30 ADMM x 5 CG)."""
    import torch

    import monalisa_b200 as mb
    from monalisa_b200.workloads import koosh3d_bins

    w = koosh3d_bins()
    mats = [mb.bmTraj2SparseMat(t, v, w.N_u, w.dK_u, w.kernelType, w.nWin, w.kernelParam) for t, v in zip(w.t, w.ve)]
    chain = mb.TevaMorphosiaChain([m[0] for m in mats], [m[1] for m in mats], w.C, w.n_u, autotune=True)
    gen = torch.Generator(device="cuda").manual_seed(33)
    ys = []
    for f in range(w.nFr):
        yy = chain.plans[f].shanna(torch.from_numpy(w.x_true[f]).cuda())
        yy += torch.randn(yy.shape, dtype=torch.complex64, device="cuda", generator=gen) * (yy.abs().mean() * 1e-3)
        ys.append(yy)
    y = torch.cat(ys)
    ve = torch.from_numpy(np.concatenate(w.ve).astype(np.float32)).cuda()
    nu = int(np.prod(w.n_u))
    x, z, u = [torch.zeros((w.nFr, nu), dtype=torch.complex64, device="cuda") for _ in range(3)]
    chain.run_dev(y, ve, x, z, u, w.delta, w.rho, 1, w.nCGD, 10.0)  # warm-up (captures the CG step)
    hist = []

    def recon():
        x.zero_()
        hist.clear()
        chain.run_dev(y, ve, x, z, u, w.delta, w.rho, w.nIter, w.nCGD, 10.0, history=hist)

    ms = _event_ms(recon, 1, stream)
    chain.close()
    ops = w.nFr * (w.nIter * (w.nCGD + 1) + 1), w.nFr * w.nIter * w.nCGD
    per_bin = (w.nIter * (w.nCGD + 1) + 1, w.nIter * w.nCGD)
    # plain-GPU operators (stock cuFFT / cuSPARSE per bin, nothing fused):
    # every bin's forward and adjoint timed once, extrapolated to the
    # reconstruction's operator count (the ADMM vector work is not counted)
    from monalisa_b200.workloads import Workload

    KFC = mb.bmKF(w.C, w.N_u, w.n_u, w.dK_u, w.nCh, w.kernelType, w.nWin, w.kernelParam)
    KFCc = mb.bmKF_conj(np.conj(w.C), w.N_u, w.n_u, w.dK_u, w.nCh, w.kernelType, w.nWin, w.kernelParam)
    wb = Workload("bin", 3, w.n_u, w.N_u, w.dK_u, w.nCh, w.nCGD, w.kernelType, w.nWin, w.kernelParam)
    ve_all = np.concatenate(w.ve).astype(np.float32)
    offs = np.concatenate([[0], np.cumsum(w.nPt)])
    HX = _HX(wb)
    fwd_ms = bwd_ms = 0.0
    for f in range(w.nFr):
        pg = PlainGpuSensa(wb, mats[f][0], mats[f][1], KFC, KFCc, torch.device("cuda"))
        xf = torch.from_numpy(w.x_true[f]).cuda()
        hy = torch.from_numpy(np.minimum(ve_all[offs[f]:offs[f + 1]], np.float32(10.0))).cuda()
        pg.M(xf)
        pg.MH(ys[f], hy, 1.0 / HX)
        fwd_ms += _event_ms(lambda: pg.M(xf), 2, stream)
        bwd_ms += _event_ms(lambda: pg.MH(ys[f], hy, 1.0 / HX), 2, stream)
        del pg
    plain_ms = per_bin[0] * fwd_ms + per_bin[1] * bwd_ms
    # reference CPU path: one forward + one adjoint on 8 of the 12 coils for
    # the bins with the fewest and the most samples, a line in the sample
    # count through the two, summed over the bins and their operator counts
    order = np.argsort(w.nPt)
    pts, cost = [], []
    ref = None
    for f in (int(order[0]), int(order[-1])):
        wf = Workload("bin", 3, w.n_u, w.N_u, w.dK_u, w.nCh, w.nCGD, w.kernelType, w.nWin, w.kernelParam)
        wf.t, wf.ve, wf.C, wf.x_true = w.t[f], w.ve[f], w.C, w.x_true[f]
        ref = ReferenceCpu(wf, _to_oracle(wf, mats[f][0]), _to_oracle(wf, mats[f][1]), ys[f].cpu().numpy(), coils=8,
                           kfc=(KFC, KFCc))
        fwd, adj = ref.sample()
        sc = w.nCh / ref.coils
        pts.append(w.nPt[f])
        cost.append((fwd * sc, adj * sc))
    slope = [(cost[1][k] - cost[0][k]) / max(pts[1] - pts[0], 1) for k in range(2)]
    cpu_s = sum(per_bin[k] * (cost[0][k] + slope[k] * (n - pts[0])) for n in w.nPt for k in range(2))
    return {"workload": "20 koosh frame bins (200-1500 spokes x 256), 96^3 image, 192^3 grid, 12 coils, "
                        "temporal-TV ADMM 30 x 5 CG",
            "recons_per_s": round(1000.0 / ms, 4), "s_per_recon": round(ms / 1000.0, 3),
            "ms_per_admm_iteration": round(ms / w.nIter, 2), "shanna_nakatsha_per_recon": list(ops),
            "objective_first_last": [hist[0][0], hist[-1][0]], "samples": int(sum(w.nPt)),
            "vs_plain_gpu": {"s_per_recon": round(plain_ms / 1e3, 3), "speedup": round(plain_ms / ms, 2),
                             "arm": "torch.fft + torch.sparse CSR operators per bin, each bin's forward and "
                                    "adjoint timed once and multiplied by the operator counts (ADMM vector work "
                                    "not counted)"},
            "cpu_baseline": {"s_per_recon": round(cpu_s, 1), "value": round(1.0 / cpu_s, 6), "unit": UNIT,
                             "cores": ref.cores, "kind": ref.kind,
                             "sample": f"1 forward + 1 adjoint on 8 of 12 coils for the bins of {pts[0]} and "
                                       f"{pts[1]} samples (x1.5 coils), linear in the sample count, summed over "
                                       f"the 20 bins x {per_bin[0]} forward + {per_bin[1]} adjoint applications"},
            "speedup_vs_cpu": round(cpu_s * 1e3 / ms, 1)}


def _c5():
    """c5: the serving mix (60 % 2-D, 40 % 3-D, 8-16 coils, 20 CG), Poisson
    arrivals, continuous admission on one GPU: 2000 requests at the
    configuration's 50 requests/s and 1000 at 20 requests/s (below the GPU's
    capacity for this mix, so latency there is mostly service time).  Beside
    them, serial per-request latencies of the plain-GPU arm (whole
    reconstructions with stock cuFFT / cuSPARSE calls) and of the reference
    CPU path (one forward + one adjoint on up to 8 coils, extrapolated to 22
    forward + 20 adjoint applications on all coils), averaged over the mix."""
    import torch

    import monalisa_b200 as mb
    from monalisa_b200 import serving
    from monalisa_b200.workloads import Workload, serving_schedule, serving_templates

    templates = serving_templates()
    for k, tp in enumerate(templates):
        tp["y"] = serving.simulate_data(tp, seed=k)
    server = serving.ReconServer(workers=4)
    serving.run_poisson(server, templates, np.zeros(len(templates)), np.arange(len(templates)))
    runs = {}
    for rate, n in ((50.0, 2000), (20.0, 1000)):
        arrivals, tmpl = serving_schedule(n, rate)
        reqs = serving.run_poisson(server, templates, arrivals, tmpl)
        runs[f"{rate:g}_req_per_s"] = {"offered_rate": rate, **{k: (round(v, 2) if isinstance(v, float) else v)
                                                                 for k, v in serving.latency_stats(reqs).items()}}
    server.close()
    # serial latency per template: plain GPU and reference CPU
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream()
    plain_ms, cpu_s = [], []
    ref = None
    for k, tp in enumerate(templates):
        nCh = tp["C"].shape[1]
        kt, kp = ("kaiser", [1.95, 10, 10]) if tp["imDim"] == 2 else ("gauss", [0.61, 10])
        wt = Workload(f"t{k}", tp["imDim"], tp["n_u"], tp["N_u"], np.ones(tp["imDim"]), nCh, 20, kt, 3, kp)
        wt.t, wt.ve, wt.C, wt.x_true = tp["t"], tp["ve"], tp["C"], tp["x_true"]
        Gu, Gut = mb.bmTraj2SparseMat(wt.t, wt.ve, wt.N_u, wt.dK_u, kt, 3, kp)
        KFC = mb.bmKF(wt.C, wt.N_u, wt.n_u, wt.dK_u, nCh, kt, 3, kp)
        KFCc = mb.bmKF_conj(np.conj(wt.C), wt.N_u, wt.n_u, wt.dK_u, nCh, kt, 3, kp)
        pg = PlainGpuSensa(wt, Gu, Gut, KFC, KFCc, dev)
        yd = torch.from_numpy(np.asarray(tp["y"], np.complex64)).to(dev)
        ved = torch.from_numpy(np.asarray(wt.ve, np.float32)).to(dev)
        pg.sensa(yd, ved, _HX(wt), 20)
        plain_ms.append(_event_ms(lambda: pg.sensa(yd, ved, _HX(wt), 20), 1, stream))
        del pg
        ref = ReferenceCpu(wt, _to_oracle(wt, Gu), _to_oracle(wt, Gut), tp["y"], coils=8, kfc=(KFC, KFCc))
        fwd, adj = ref.sample()
        cpu_s.append(ref.recon_s(fwd, adj))
    _, tmpl = serving_schedule(2000, 50.0)
    mix = np.bincount(tmpl, minlength=len(templates)) / len(tmpl)
    mean_plain = float(np.dot(mix, plain_ms))
    mean_cpu = float(np.dot(mix, cpu_s))
    return {"workload": "Poisson arrivals: 60% 2D 256^2/512^2 (128-512 spokes x 512), 40% 3D 96^3-128^3 "
                        "(1024-4096 spokes x 256), 8-16 coils, CG-SENSE 20, 4 workers, admission by free HBM",
            **runs,
            "plain_gpu_serial": {"mean_ms_per_request": round(mean_plain, 1),
                                 "recons_per_s": round(1e3 / mean_plain, 2),
                                 "per_template_ms": [round(v, 1) for v in plain_ms]},
            "cpu_serial": {"mean_s_per_request": round(mean_cpu, 2), "recons_per_s": round(1.0 / mean_cpu, 4),
                           "per_template_s": [round(v, 2) for v in cpu_s], "cores": ref.cores, "kind": ref.kind,
                           "sample": "per template: 1 forward + 1 adjoint on up to 8 coils, extrapolated to 22 "
                                     "forward + 20 adjoint on all coils; averaged over the request mix"}}


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    return oracle


def _to_oracle(w, D):
    """A device matrix as the oracle's jump-format matrix (input transfer)."""
    oracle = _oracle()
    b = D.download()
    return oracle.SparseMat(r_size=b.r_size, l_size=b.l_size, r_nJump=b.r_nJump, m_val=b.m_val, r_jump=b.r_jump,
                            l_jump=b.l_jump, l_nJump=b.l_nJump, N_u=w.N_u, d_u=w.dK_u, kernel_type=w.kernelType,
                            nWin=w.nWin, kernelParam=np.array(w.kernelParam))


class ReferenceCpu:
    """The reference CPU path on a workload's inputs: the reference's own
    bmSparseMat_cC_oBlock_omp_mex (compiled from source into oracle/_ref;
    the C restatement when that is absent) inside the numpy/scipy
    restatement of bmShanna_MATLAB / bmNakatsha_MATLAB, scipy.fft with all
    host threads.  A bounded sample (`sample`) is one forward and one
    adjoint operator application on `coils` of the coils -- the operators are
    per coil, and 8 coils already give the reference kernel's OpenMP loop
    (2 x coils iterations) 16 threads -- extrapolated to one reconstruction of
    (nCGD + 2) forward and nCGD adjoint applications on all coils; `recon`
    times a whole reconstruction (bmSensa with its CG BLAS-1).  KFC /
    KFC_conj may be given (set-up, not timed)."""

    def __init__(self, w, gu, gut, y, coils=8, kfc=None):
        oracle = _oracle()
        self.o = oracle
        self.w, self.gu, self.gut = w, gu, gut
        self.kind = "reference" if oracle.ref_available() else "port"
        self.cores = os.cpu_count() or 1
        os.environ.setdefault("OMP_NUM_THREADS", str(self.cores))
        self.coils = min(coils, w.nCh)
        C = np.asarray(w.C, np.complex64)[:, :self.coils]
        if kfc is not None:
            self.KFC = np.ascontiguousarray(np.asarray(kfc[0])[:, :self.coils])
            self.KFCc = np.ascontiguousarray(np.asarray(kfc[1])[:, :self.coils])
        else:
            self.KFC = oracle.bmKF(C, w.N_u, w.n_u, w.dK_u, self.coils, w.kernelType, w.nWin, w.kernelParam)
            self.KFCc = oracle.bmKF_conj(np.conj(C), w.N_u, w.n_u, w.dK_u, self.coils, w.kernelType, w.nWin,
                                         w.kernelParam)
        self.y = np.ascontiguousarray(np.asarray(y, np.complex64)[:, :self.coils])
        self.yfull = np.asarray(y, np.complex64)
        self.spm = oracle.SpMV(self.kind)
        self.last_image = None

    def sample(self):
        """Seconds of one forward and one adjoint application on the sample coils."""
        o, w = self.o, self.w
        x = w.x_true if w.x_true is not None else np.ones(int(np.prod(w.n_u)), np.complex64)
        t0 = time.perf_counter()
        o.bmShanna(x, self.gu, self.KFC, w.n_u, self.spm, workers=self.cores)
        t1 = time.perf_counter()
        o.bmNakatsha(self.y, self.gut, self.KFCc, True, w.n_u, self.spm, workers=self.cores)
        t2 = time.perf_counter()
        return t1 - t0, t2 - t1

    def recon_s(self, fwd, adj):
        w = self.w
        return ((w.nCGD + 2) * fwd + w.nCGD * adj) * (w.nCh / self.coils)

    def describe(self, fwd, adj):
        w = self.w
        spmv = ("reference bmSparseMat_cC_oBlock_omp_mex compiled from source" if self.kind == "reference"
                else "C restatement")
        return (f"1 forward ({fwd:.2f} s) + 1 adjoint ({adj:.2f} s) operator application on {self.coils} of "
                f"{w.nCh} coils at full size, extrapolated x{w.nCh / self.coils:g} coils to {w.nCGD + 2} forward + "
                f"{w.nCGD} adjoint applications per recon; SpMV = {spmv}, FFT = scipy.fft (workers={self.cores})")

    def recon(self):
        """Seconds of one whole reconstruction (all coils, nCGD CG updates)."""
        o, w = self.o, self.w
        t0 = time.perf_counter()
        self.last_image = o.bmSensa(np.zeros(int(np.prod(w.n_u)), np.complex64), self.yfull, w.ve, w.C, self.gu,
                                    self.gut, w.n_u, w.nCGD, spmv=self.spm, workers=self.cores)
        return time.perf_counter() - t0


def cpu_baseline(w, gu, gut, y):
    """The reference CPU path on one bounded sample, for the GPU arm's line."""
    ref = ReferenceCpu(w, gu, gut, y)
    fwd, adj = ref.sample()
    return {"value": round(1.0 / ref.recon_s(fwd, adj), 6), "unit": UNIT, "cores": ref.cores, "kind": ref.kind,
            "sample": ref.describe(fwd, adj)}


def run_reference(args):
    from monalisa_b200 import replicas

    ws, rank, local = replicas.world()
    if rank != 0:
        return
    from monalisa_b200.workloads import koosh3d

    oracle = _oracle()
    w = koosh3d()
    G = oracle.traj2sparsemat(w.t, w.ve, w.N_u, w.dK_u, w.kernelType, w.nWin, w.kernelParam)
    rng = np.random.default_rng(5)
    y = (rng.standard_normal((w.nPt, w.nCh)) + 1j * rng.standard_normal((w.nPt, w.nCh))).astype(np.complex64)
    ref = ReferenceCpu(w, G["Gu"], G["Gut"], y)
    step_s, recons = [], []
    desc = ""
    for i in range(args.warmup + args.steps):
        if args.ref_sample == "full":
            dt = ref.recon()
            rs, desc = dt, f"one whole reconstruction ({w.nCGD} CG updates, all {w.nCh} coils) per step"
        else:
            fwd, adj = ref.sample()
            dt, rs, desc = fwd + adj, ref.recon_s(fwd, adj), ref.describe(fwd, adj)
        if i >= args.warmup:
            step_s.append(dt)
            recons.append(rs)
    value = round(1.0 / statistics.median(recons), 6)
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(1e3 * statistics.mean(step_s), 1),
           "step": ("a bounded sample per step: " if args.ref_sample != "full" else "") + desc,
           "recon_s_median": round(statistics.median(recons), 2), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
           "config": _config(w, ws),
           "cpu_baseline": {"value": value, "unit": UNIT, "kind": ref.kind, "cores": ref.cores, "sample": desc},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def _config(w, ws):
    """The config of the headline line; the same dict in both arms."""
    return {"workload": "3D koosh-ball CG-SENSE: 128^3 image, 256^3 grid, 4096x256 samples, 16 coils, "
                        "30 CG iterations", "parallelism": f"replicas x{ws}",
            "l2": "working set (2.1 GB grid) larger than L2 each step", **w.info}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-sample", default="sample", choices=["sample", "full"],
                    help="reference arm: a bounded operator sample per step (default) or a whole reconstruction")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-GPU comparison arm")
    ap.add_argument("--no-extra", action="store_true", help="skip the c1 / c3 / c4 / c5 configurations")
    ap.add_argument("--adjoint", default="auto", choices=["auto", "masked", "fused", "full_grid"],
                    help="adjoint strategy of the headline plan (auto: autotuned)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
