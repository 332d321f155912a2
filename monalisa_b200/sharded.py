"""Frame bins of one temporal-TV reconstruction, or the coils of one
CG-SENSE reconstruction, sharded over ranks.

Frame bins:

bmTevaMorphosia_chain (src/fourier123/solver_function/imDim_morphosia/
nonCartesian/bmTevaMorphosia_chain.m:6-195) couples its frames in two ways
only: the circular temporal difference F x_i = x_i - x_{i-1} (private_F,
:262-269) with its adjoint F* z_i = (1/HX)(HZ z_i - HZ z_{i+1})
(private_dagF, :282-289), and the CG scalars, which are sums over all
frames (:126-163, with bmEuclideProd).  Everything else -- the forward and
adjoint operators of each frame, the prox and the z/u updates -- is per
frame.  So each rank holds a contiguous run of frames; an application of F
needs the last frame of the previous rank and one of F* the first frame of
the next rank (one boundary image each, exchanged around the ring), and
every CG step all-reduces its FP64 partial sums.  With one rank this is the
single-GPU reconstruction.

The per-frame operators come from an engine: ``PlanEngine`` runs them with
this library's NUFFT plans on the rank's GPU (collectives over NCCL); any
object with the same methods works (the tests run the restatement on CPU
tensors over gloo).  Images are complex64 torch tensors [prod(n_u)], k-space
[nPt_i, nCh].  Deformation fields (Tu/Tut) are not supported here; the
single-GPU chain (solvers.TevaMorphosiaChain) has them.

Coils (bmSensa, src/fourier123/solver_function/imDim/nonCartesian/
bmSensa.m:6-96): the forward model of each coil is independent, and coils
meet only in the coil sum of the adjoint (bmNakatsha_MATLAB.m:55) and in the
k-space norms of the CG steps (bmSensa.m:59, :83).  Each rank holds a run of
coils (its k-space columns and coil maps); an adjoint is the rank's partial
coil sum followed by one all-reduce of a prod(n_u) complex64 image, and each
k-space norm one all-reduce of an FP64 scalar.  The image-space quantities
(x, p, the adjoint residual and its norm, bmSensa.m:45, :73) are then the
same on every rank, so the CG recurrences run redundantly without further
exchange.
"""
from __future__ import annotations

import numpy as np


def shard_frames(cost, world: int):
    """Contiguous runs of frames, one per rank, balancing `cost` (one value
    per frame, e.g. a + b * nPt): rank r gets frames [bounds[r], bounds[r+1])."""
    cost = np.asarray(cost, np.float64)
    nFr = cost.size
    if world < 1 or world > nFr:
        raise ValueError(f"{nFr} frames cannot be split over {world} ranks")
    csum = np.concatenate([[0.0], np.cumsum(cost)])
    bounds = [0]
    for r in range(1, world):
        target = csum[-1] * r / world
        b = int(np.argmin(np.abs(csum - target)))
        b = min(max(b, bounds[-1] + 1), nFr - (world - r))  # every rank keeps >= 1 frame
        bounds.append(b)
    bounds.append(nFr)
    return bounds


class PlanEngine:
    """Per-frame operators of the local frames on this rank's GPU: NUFFT
    plans that share one grid (NufftPlan.sharing), HY = min(ve, ve_max)."""

    def __init__(self, Gu, Gut, C, n_u, dK_u=None):
        import torch

        from .solvers import SensaRecon

        from .operators import NufftPlan

        base = SensaRecon(Gu[0], Gut[0], C, n_u, dK_u)
        self._base = base
        self.plans = [base.plan] + [NufftPlan.sharing(base.plan, Gu[i], Gut[i]) for i in range(1, len(Gu))]
        self.n_u = base.n_u
        self.nCh = base.nCh
        self.dev = torch.device("cuda", torch.cuda.current_device())
        # HX = prod((1/dK_u)/N_u) in single precision (bmTevaMorphosia_chain.m:33-34)
        dX = (np.float32(1) / base.dK_u.astype(np.float32)) / base.N_u.astype(np.float32)
        self.HX = float(np.float32(np.prod(dX)))

    def M(self, i, x):
        return self.plans[i].shanna(x)

    def MH(self, i, r, HY, scale):
        return self.plans[i].nakatsha(r, HY, scale)

    def close(self):
        for p in self.plans[1:]:
            p.close()
        self._base.plan.close()


class ShardedTevaMorphosia:
    """bmTevaMorphosia_chain over the frames [lo, hi) of `nFr` held by this
    rank ('normal' and 'adapt' regularisation modes, z and u initialised as
    in :75-81).  `group` is a torch.distributed process group (None: one
    process, no collectives)."""

    def __init__(self, engine, lo: int, hi: int, nFr: int, group=None):
        self.e = engine
        self.lo, self.hi, self.nFr = lo, hi, nFr
        self.group = group
        if group is not None:
            import torch.distributed as dist

            self.dist = dist
            self.rank = dist.get_rank(group)
            self.world = dist.get_world_size(group)
        else:
            self.dist, self.rank, self.world = None, 0, 1

    # ---- collectives ------------------------------------------------------------
    def _allreduce(self, vals):
        import torch

        t = torch.tensor(vals, dtype=torch.float64, device=self._dev)
        if self.dist is not None:  # a group of one rank still runs the collective
            self.dist.all_reduce(t, group=self.group)
        return [float(v) for v in t.cpu()]

    def _ring(self, send, to_next: bool):
        """Sends `send` to the next rank (to_next) or the previous one and
        returns the image received from the other side (ring order)."""
        import torch

        if self.world == 1:
            return send
        nxt, prv = (self.rank + 1) % self.world, (self.rank - 1) % self.world
        dst, src = (nxt, prv) if to_next else (prv, nxt)
        gdst = self.dist.get_global_rank(self.group, dst) if self.group is not None else dst
        gsrc = self.dist.get_global_rank(self.group, src) if self.group is not None else src
        sbuf = torch.view_as_real(send.contiguous()).contiguous()
        rbuf = torch.empty_like(sbuf)
        ops = [self.dist.P2POp(self.dist.isend, sbuf, gdst, self.group),
               self.dist.P2POp(self.dist.irecv, rbuf, gsrc, self.group)]
        for req in self.dist.batch_isend_irecv(ops):
            req.wait()
        return torch.view_as_complex(rbuf)

    # ---- operators over the local frames ---------------------------------------
    def F(self, x):
        """F x_i = x_i - x_{i-1} (circular over all frames)."""
        prev = self._ring(x[-1], to_next=True)  # the previous rank's last frame
        return [x[k] - (x[k - 1] if k > 0 else prev) for k in range(len(x))]

    def dagF(self, z):
        """F* z_i = (1/HX)(HZ z_i - HZ z_{i+1})."""
        nxt = self._ring(z[0], to_next=False)  # the next rank's first frame
        hz, inv = self.HZ, 1.0 / self.HX
        n = len(z)
        return [inv * (hz * z[k] - hz * (z[k + 1] if k + 1 < n else nxt)) for k in range(n)]

    @staticmethod
    def _dot(v, h=None):
        vr, vi = v.real.double(), v.imag.double()
        s = vr * vr + vi * vi
        if h is not None:
            s = s * h.double()[:, None] if s.dim() == 2 else s * h.double()
        return float(s.sum())

    def run(self, y, ve, x, delta, rho, nIter, nCGD, ve_max, regul_mode="normal", history=None):
        """y, ve: lists over the local frames ([nPt_i, nCh], [nPt_i]); x: list
        of local initial images (updated in place).  Returns x."""
        import torch

        e = self.e
        L = self.hi - self.lo
        if not (len(y) == len(ve) == len(x) == L):
            raise ValueError("y, ve and x need one entry per local frame")
        self._dev = x[0].device
        myEps = 10 * float(np.finfo(np.float32).eps)
        self.HX = e.HX
        self.HZ = float(np.float32(e.HX))
        HX, HZ = self.HX, self.HZ
        HY = [torch.clamp(v.to(torch.float32), max=float(np.float32(ve_max))) for v in ve]
        invHX = 1.0 / HX
        M = lambda v: [e.M(k, v[k]) for k in range(L)]
        dagM = lambda r: [e.MH(k, r[k], HY[k], invHX) for k in range(L)]
        dl = np.full(nIter, np.float32(abs(delta)), np.float32) if np.isscalar(delta) else \
            np.linspace(abs(delta[0]), abs(delta[1]), nIter).astype(np.float32)
        rl = np.full(nIter, np.float32(abs(rho)), np.float32) if np.isscalar(rho) else \
            np.linspace(abs(rho[0]), abs(rho[1]), nIter).astype(np.float32)
        z = self.F(x)
        u = [torch.zeros_like(v) for v in x]

        def dafi_regul(xx):  # private_dafi_regul (:211-224)
            Mx = M(xx)
            prev = self._ring(xx[-1], to_next=True)
            reg = 0.0
            for k in range(L):
                tr = (xx[k - 1] if k > 0 else prev) - xx[k]
                reg += HZ * float(tr.real.double().abs().sum() + tr.imag.double().abs().sum())
            d, r = self._allreduce([sum(self._dot(y[k] - Mx[k], HY[k]) for k in range(L)), reg])
            return d, r

        dafi, regul = dafi_regul(x) if regul_mode == "adapt" else (None, None)
        for c in range(nIter):
            dlt, r = float(dl[c]), float(rl[c])
            if regul_mode == "adapt":
                dlt = float(np.float32(dlt * regul / dafi))
                r = float(np.float32(r * dlt))
            rf = float(np.float32(r))
            Mx = M(x)
            res_y = [y[k] - Mx[k] for k in range(L)]
            Fx = self.F(x)
            res_z = [(z[k] - u[k]) - Fx[k] for k in range(L)]
            dMy, dFz = dagM(res_y), self.dagF(res_z)
            dA = [dMy[k] + rf * dFz[k] for k in range(L)]
            p = dA
            sq_next = HX * self._allreduce([sum(self._dot(v) for v in dA)])[0]
            for j in range(1, nCGD + 1):
                res_y_c, res_z_c, sq_c, p_c = res_y, res_z, sq_next, p
                if sq_c < myEps:
                    break
                Mp, Fp = M(p_c), self.F(p_c)
                sM, sF = self._allreduce([sum(self._dot(Mp[k], HY[k]) for k in range(L)),
                                          sum(self._dot(v) for v in Fp)])
                a = sq_c / (sM + sF * (r * HZ))
                af = float(np.float32(a))
                x = [x[k] + af * p_c[k] for k in range(L)]
                if j == nCGD:
                    break
                res_y = [res_y_c[k] - af * Mp[k] for k in range(L)]
                res_z = [res_z_c[k] - af * Fp[k] for k in range(L)]
                dMy, dFz = dagM(res_y), self.dagF(res_z)
                dA = [dMy[k] + rf * dFz[k] for k in range(L)]
                sq_next = HX * self._allreduce([sum(self._dot(v) for v in dA)])[0]
                bf = float(np.float32(sq_next / sq_c))
                p = [dA[k] + bf * p_c[k] for k in range(L)]
            Fx = self.F(x)
            Fxu = [u[k] + Fx[k] for k in range(L)]
            thr = float(np.float32(dlt / r))
            z = [_prox_one_norm(v, thr) for v in Fxu]
            u = [Fxu[k] - z[k] for k in range(L)]
            if history is not None or regul_mode == "adapt":
                dafi, regul = dafi_regul(x)
                if history is not None:
                    history.append((0.5 * dafi + 0.5 * dlt * regul, dafi, regul))
        return x


def _prox_one_norm(v, s):
    """bmProx_oneNorm.m:6-35: soft threshold of the real and imaginary parts
    separately."""
    import torch

    re = torch.sign(v.real) * torch.clamp(v.real.abs() - s, min=0)
    im = torch.sign(v.imag) * torch.clamp(v.imag.abs() - s, min=0)
    return torch.complex(re, im)


def shard_coils(nCh: int, world: int):
    """Contiguous runs of coils, one per rank: rank r gets coils
    [bounds[r], bounds[r+1]).  Runs are whole coil pairs where every rank can
    have one (the coil-pair kernels and the Gut row records want even coil
    counts); an odd last coil goes to the last rank."""
    if world < 1 or world > nCh:
        raise ValueError(f"{nCh} coils cannot be split over {world} ranks")
    unit = 2 if nCh >= 2 * world else 1
    units, spare = divmod(nCh, unit)
    q, rem = divmod(units, world)
    sizes = [(q + (1 if r < rem else 0)) * unit for r in range(world)]
    sizes[-1] += spare
    bounds = [0]
    for s in sizes:
        bounds.append(bounds[-1] + s)
    return bounds


class CoilPlanEngine:
    """The operators of the coils [lo, hi) on this rank's GPU: a NUFFT plan
    whose KFC / KFC_conj hold those coils only.  Gu / Gut may be device
    matrices shared by several engines on one GPU (a plan keeps what it
    derives from them, e.g. Gut's row records, to itself)."""

    def __init__(self, Gu, Gut, C, n_u, lo: int, hi: int, dK_u=None):
        from .solvers import SensaRecon

        nu = int(np.prod(np.ravel(n_u)))
        C = np.asarray(C, np.complex64).reshape(nu, -1, order="F")
        if not (0 <= lo < hi <= C.shape[1]):
            raise ValueError(f"coils [{lo}, {hi}) outside the {C.shape[1]} coil maps")
        self._recon = SensaRecon(Gu, Gut, np.ascontiguousarray(C[:, lo:hi]), n_u, dK_u)
        self.plan = self._recon.plan
        self.lo, self.hi = lo, hi
        r = self._recon
        # HX = prod((1/dK_u)/N_u) in single precision (bmSensa.m:26-27)
        dX = (np.float32(1) / r.dK_u.astype(np.float32)) / r.N_u.astype(np.float32)
        self.HX = float(np.prod(dX.astype(np.float32)))

    def M(self, x):
        return self.plan.shanna(x)

    def MH(self, r, HY, scale):
        return self.plan.nakatsha(r, HY, scale)

    def close(self):
        self.plan.close()


class CoilShardedSensa:
    """bmSensa.m:6-96 over the coils held by this rank.  `engines` are this
    rank's coil groups in coil order (one or more; each has M(x) -> k-space
    [nPt, nCh_g], MH(r, HY, scale) -> scale * its partial coil sum of the
    adjoint of HY .* r, and HX); `group` is a torch.distributed process group
    (None: one process, no collectives).  Several groups on one rank are
    summed in order before the all-reduce."""

    def __init__(self, engines, group=None):
        self.engines = list(engines)
        if not self.engines:
            raise ValueError("at least one coil group per rank")
        self.HX = self.engines[0].HX
        self.group = group
        if group is not None:
            import torch.distributed as dist

            self.dist = dist
        else:
            self.dist = None

    def _allreduce(self, vals, dev):
        import torch

        t = torch.tensor(vals, dtype=torch.float64, device=dev)
        if self.dist is not None:
            self.dist.all_reduce(t, group=self.group)
        return [float(v) for v in t.cpu()]

    def _coil_sum(self, parts):
        """Partial coil sums of this rank's groups, then one all-reduce of the
        image (the coil sum of bmNakatsha_MATLAB.m:55 across ranks)."""
        import torch

        img = parts[0]
        for q in parts[1:]:
            img = img + q
        if self.dist is not None:
            buf = torch.view_as_real(img.contiguous()).contiguous()
            self.dist.all_reduce(buf, group=self.group)
            img = torch.view_as_complex(buf)
        return img

    @staticmethod
    def _dot(v, h=None):
        vr, vi = v.real.double(), v.imag.double()
        s = vr * vr + vi * vi
        if h is not None:
            s = s * (h.double()[:, None] if s.dim() == 2 else h.double())
        return float(s.sum())

    def run(self, y, ve, x, nIter=1, nCGD=20, ve_max=None, history=None):
        """y: list over this rank's coil groups of k-space [nPt, nCh_g]; ve
        [nPt] float32; x [prod(n_u)] initial image, the same on every rank.
        Returns the image (the same on every rank).  ``history`` receives the
        monitored residual ||y - M x||^2_HY of each outer iteration
        (bmSensa.m:82-84), summed over all coils."""
        import torch

        E = self.engines
        if len(y) != len(E):
            raise ValueError("y needs one k-space block per coil group")
        dev = x.device
        myEps = 10 * float(np.finfo(np.float32).eps)
        HX = self.HX
        if ve_max is None:
            ve_max = float(ve.max())  # bmSensa.m:29-31 (the same ve on every rank)
        HY = torch.clamp(ve.to(torch.float32), max=float(np.float32(ve_max)))  # bmSensa.m:32
        invHX = 1.0 / HX
        M = lambda v: [e.M(v) for e in E]
        dagM = lambda r: self._coil_sum([e.MH(r[g], HY, invHX) for g, e in enumerate(E)])
        kdot = lambda v: self._allreduce([sum(self._dot(b, HY) for b in v)], dev)[0]
        for _ in range(nIter):
            Mx = M(x)
            res = [y[g] - Mx[g] for g in range(len(E))]  # bmSensa.m:43
            g_img = dagM(res)  # :44
            sq_next = HX * self._dot(g_img)  # :45
            p = g_img
            for i in range(1, nCGD + 1):
                res_c, sq_c, p_c = res, sq_next, p
                if sq_c < myEps:  # :54-56
                    break
                Mp = M(p_c)
                a = sq_c / kdot(Mp)  # :58-61
                af = float(np.float32(a))
                x = x + af * p_c  # :63
                if i == nCGD:
                    break
                res = [res_c[g] - af * Mp[g] for g in range(len(E))]  # :71
                g_img = dagM(res)  # :72
                sq_next = HX * self._dot(g_img)  # :73
                bf = float(np.float32(sq_next / sq_c))  # :75
                p = g_img + bf * p_c  # :77
            Mx = M(x)
            R = kdot([y[g] - Mx[g] for g in range(len(E))])  # :82-83
            if history is not None:
                history.append(R)
        return x
