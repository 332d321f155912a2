"""Serving reconstructions: continuous admission of CG-SENSE requests on one
GPU.

A request carries its trajectory, volume elements, coil maps and k-space
data (the inputs of bmSensa, src/fourier123/solver_function/imDim/
nonCartesian/bmSensa.m:6-96).  ``ReconServer`` keeps a queue and a pool of
worker threads, each issuing its reconstructions on a CUDA stream of its own
(the library's calls release the interpreter lock, so reconstructions of
different requests overlap on the GPU).  A queued request starts as soon as
a worker is free and its estimated device footprint fits into the free HBM
minus a reserve; a request that does not fit waits while smaller ones behind
it may start (no head-of-line blocking).  Device matrices are cached per
trajectory key (least recently used first out), so repeated protocols skip
the matrix build.

Every reconstruction is deterministic (fixed-order sums, no atomics on the
CG path), so a request's image does not depend on what else runs beside it.
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class ReconRequest:
    """One CG-SENSE reconstruction.  t [imDim, nPt] physical units, ve
    [nPt], C [prod(n_u), nCh], y [nPt, nCh] complex64."""
    t: np.ndarray
    ve: np.ndarray
    C: np.ndarray
    y: np.ndarray
    N_u: np.ndarray
    n_u: np.ndarray
    dK_u: np.ndarray = None
    nCGD: int = 20
    kernelType: str = "gauss"
    nWin: int = 3
    kernelParam: tuple = (0.61, 10)
    traj_key: object = None      # requests with the same key share device matrices
    coil_key: object = None      # with traj_key: requests with both keys equal reuse a solver plan
    precision: str = "fp32"
    rid: int = 0
    # filled in by the server
    x: np.ndarray = None
    error: str = None
    t_submit: float = 0.0
    t_start: float = 0.0
    t_done: float = 0.0
    done: threading.Event = field(default_factory=threading.Event, repr=False)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit

    def device_bytes(self) -> int:
        """Estimated device footprint of this request's reconstruction:
        matrices (entries of Gu, Gut and their sign-folded copies), the grid
        and FFT buffers, KFC / KFC_conj and the solver's work vectors."""
        imDim = int(np.ravel(self.N_u).size)
        N = int(np.prod(self.N_u))
        n = int(np.prod(self.n_u))
        nPt = int(np.asarray(self.t).shape[-1])
        nCh = int(np.asarray(self.C).reshape(n, -1).shape[1])
        nnz = nPt * int(self.nWin) ** imDim
        mats = nnz * (4 + 4 + 4) * 2 + 4 * (nPt + N)
        grid = N * nCh * 8 * 2  # grid + the larger pass buffer
        kfc = n * nCh * 8 * 2
        work = 2 * n * 8 + 2 * nPt * nCh * 8 + nPt * 4
        return int(1.2 * (mats + grid + kfc + work))


class Scheduler:
    """The admission core, independent of the GPU: ``free_bytes()`` reports
    the device memory available, ``execute(req)`` runs one request.  Workers
    take the first queued request that fits into free memory minus the
    reserve and the footprints of the requests still running."""

    def __init__(self, execute, free_bytes, workers=4, reserve_bytes=4 << 30):
        self._execute = execute
        self._free = free_bytes
        self._reserve = int(reserve_bytes)
        self._queue = collections.deque()
        self._cv = threading.Condition()
        self._inflight = 0          # bytes admitted and not yet finished
        self._stop = False
        self.order = []             # request ids in start order
        self._threads = [threading.Thread(target=self._loop, args=(i,), daemon=True) for i in range(workers)]
        for th in self._threads:
            th.start()

    def submit(self, req: ReconRequest) -> ReconRequest:
        req.t_submit = time.perf_counter()
        with self._cv:
            self._queue.append(req)
            self._cv.notify_all()
        return req

    def _take(self):
        """First queued request that fits (called with the lock held)."""
        budget = self._free() - self._reserve - self._inflight
        for i, r in enumerate(self._queue):
            need = r.device_bytes()
            if need <= budget or (self._inflight == 0 and i == 0):  # an idle device always takes the head
                del self._queue[i]
                self._inflight += need
                return r, need
        return None, 0

    def _loop(self, worker):
        while True:
            with self._cv:
                while True:
                    if self._stop and not self._queue:
                        return
                    req, need = self._take() if self._queue else (None, 0)
                    if req is not None:
                        self.order.append(req.rid)
                        break
                    self._cv.wait(timeout=0.05)
            req.t_start = time.perf_counter()
            try:
                req.x = self._execute(req, worker)
            except Exception as e:  # reported on the request, the server keeps going
                req.error = f"{type(e).__name__}: {e}"
            req.t_done = time.perf_counter()
            with self._cv:
                self._inflight -= need
                self._cv.notify_all()
            req.done.set()

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for th in self._threads:
            th.join()


class ReconServer:
    """CG-SENSE requests on one GPU with continuous admission (see the module
    docstring).  ``workers`` reconstructions run at a time at most, each on a
    CUDA stream of its own; ``reserve_gb`` of device memory stays free;
    ``cache`` device matrix pairs are kept per trajectory key."""

    def __init__(self, device=0, workers=4, reserve_gb=8.0, cache=16):
        import torch

        self.torch = torch
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        self._streams = [torch.cuda.Stream(device=self.device) for _ in range(workers)]
        self._cache = collections.OrderedDict()
        self._cache_cap = int(cache)
        self._cache_lock = threading.Lock()
        self._plan_lock = threading.Lock()
        self._plans = collections.OrderedDict()
        self._reserve = int(reserve_gb * (1 << 30))
        self._sched = Scheduler(self._run, self._free_bytes, workers, int(reserve_gb * (1 << 30)))

    def _free_bytes(self):
        free, _ = self.torch.cuda.mem_get_info(self.device)
        return free

    def _matrices(self, req):
        import monalisa_b200 as mb

        key = req.traj_key
        if key is not None:
            with self._cache_lock:
                if key in self._cache:
                    self._cache.move_to_end(key)
                    return self._cache[key]
        dK = np.ones(np.ravel(req.N_u).size) if req.dK_u is None else req.dK_u
        mats = mb.bmTraj2SparseMat(req.t, req.ve, req.N_u, dK, req.kernelType, req.nWin, req.kernelParam)
        if key is not None:
            with self._cache_lock:
                self._cache[key] = mats
                while len(self._cache) > self._cache_cap:
                    self._cache.popitem(last=False)
        return mats

    def _run(self, req, worker):
        import monalisa_b200 as mb

        torch = self.torch
        torch.cuda.set_device(self.device)
        with torch.cuda.stream(self._streams[worker]):
            pkey = (req.traj_key, req.coil_key, req.precision) if req.traj_key is not None and \
                req.coil_key is not None else None
            rec = self._checkout(pkey)
            if rec is None:
                Gu, Gut = self._matrices(req)
                self._make_room(req.device_bytes())
                # plans over one cached matrix pair build that pair's occupancy
                # tables on first use: plan creation is serialised, solves are not
                with self._plan_lock:
                    rec = mb.SensaRecon(Gu, Gut, req.C, req.n_u, req.dK_u, precision=req.precision)
            keep = False
            try:
                y = torch.from_numpy(np.ascontiguousarray(req.y, np.complex64)).to(self.device, non_blocking=True)
                ve = torch.from_numpy(np.ascontiguousarray(np.ravel(req.ve), np.float32)).to(self.device)
                x = torch.zeros(int(np.prod(req.n_u)), dtype=torch.complex64, device=self.device)
                rec.run_dev(y, ve, x, nIter=1, nCGD=req.nCGD)
                out = x.cpu().numpy()
                keep = pkey is not None
            finally:
                if keep:
                    self._checkin(pkey, rec)
                else:
                    rec.plan.close()
        return out

    # idle solver plans per (trajectory, coil maps, precision): a plan is used
    # by one request at a time (checked out), returned afterwards, and the
    # least recently returned idle plans go when memory is short
    def _checkout(self, pkey):
        if pkey is None:
            return None
        with self._cache_lock:
            pool = self._plans.get(pkey)
            if pool:
                self._plans.move_to_end(pkey)
                return pool.pop()
        return None

    def _checkin(self, pkey, rec):
        with self._cache_lock:
            self._plans.setdefault(pkey, []).append(rec)
            self._plans.move_to_end(pkey)

    def _make_room(self, need):
        """Closes idle cached plans, least recently used first, until `need`
        bytes fit above the reserve."""
        while self._free_bytes() - self._reserve < need:
            with self._cache_lock:
                victim = None
                for k in self._plans:
                    if self._plans[k]:
                        victim = self._plans[k].pop(0)
                        break
            if victim is None:
                return
            victim.plan.close()

    def submit(self, req: ReconRequest) -> ReconRequest:
        return self._sched.submit(req)

    @property
    def start_order(self):
        return list(self._sched.order)

    def close(self):
        self._sched.close()
        with self._cache_lock:
            plans = [r for pool in self._plans.values() for r in pool]
            self._plans.clear()
        for r in plans:
            r.plan.close()


def latency_stats(reqs):
    """p50 / p99 / mean latency (seconds) and throughput of finished requests."""
    lat = np.array([r.latency for r in reqs if r.error is None])
    span = max(r.t_done for r in reqs) - min(r.t_submit for r in reqs)
    return {"n": int(lat.size), "errors": sum(r.error is not None for r in reqs),
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "recons_per_s": float(lat.size / span)}


def simulate_data(template, seed=0, noise=1e-3):
    """k-space data of a template: the forward operator applied to its
    phantom on the GPU, plus complex Gaussian noise."""
    import torch

    import monalisa_b200 as mb

    Gu, Gut = mb.bmTraj2SparseMat(template["t"], template["ve"], template["N_u"], np.ones(template["imDim"]))
    rec = mb.SensaRecon(Gu, Gut, template["C"], template["n_u"])
    y = rec.plan.shanna(torch.from_numpy(template["x_true"]).cuda())
    gen = torch.Generator(device=y.device).manual_seed(seed)
    y += torch.randn(y.shape, dtype=torch.complex64, device=y.device, generator=gen) * (y.abs().mean() * noise)
    out = y.cpu().numpy()
    rec.plan.close()
    return out


def run_poisson(server, templates, arrivals, tmpl, nCGD=20, reuse_plans=True):
    """Submits one request per arrival time (seconds from now) built from
    templates[tmpl[i]] (its y must be set), waits for all, returns the
    requests.  reuse_plans: a template's requests share trajectory and coil
    keys (one session), so solver plans are reused."""
    t0 = time.perf_counter()
    reqs = []
    for i, (a, k) in enumerate(zip(arrivals, tmpl)):
        tp = templates[int(k)]
        delay = t0 + float(a) - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        reqs.append(server.submit(ReconRequest(t=tp["t"], ve=tp["ve"], C=tp["C"], y=tp["y"], N_u=tp["N_u"],
                                               n_u=tp["n_u"], nCGD=nCGD, traj_key=tp["key"],
                                               coil_key=tp["key"] if reuse_plans else None, rid=i)))
    for r in reqs:
        r.done.wait()
    return reqs


def main(argv=None):
    """python -m monalisa_b200.serving [--requests N] [--rate R] [--workers W]:
    the serving mix on one GPU; prints one JSON line of latency statistics."""
    import argparse
    import json

    from .workloads import serving_schedule, serving_templates

    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=100)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--no-plan-reuse", action="store_true", help="build every request's plan afresh")
    args = ap.parse_args(argv)
    templates = serving_templates(scale=args.scale)
    for k, tp in enumerate(templates):
        tp["y"] = simulate_data(tp, seed=k)
    arrivals, tmpl = serving_schedule(args.requests, args.rate)
    server = ReconServer(workers=args.workers)
    reuse = not args.no_plan_reuse
    # warm-up: one request per protocol (first launches, matrix and plan caches)
    run_poisson(server, templates, np.zeros(len(templates)), np.arange(len(templates)), reuse_plans=reuse)
    reqs = run_poisson(server, templates, arrivals, tmpl, reuse_plans=reuse)
    server.close()
    print(json.dumps({"requests": args.requests, "rate": args.rate, "workers": args.workers, "plan_reuse": reuse,
                      **latency_stats(reqs)}))


if __name__ == "__main__":
    main()
