"""Continuous-batching maximum-likelihood serving on one GPU, and a replica
router over the GPUs of a node.

No counterpart in the reference (its driver stops at the factor,
hicma_parsec/testing_dpotrf.c:830-903).  Each request is one Gaussian
log-likelihood evaluation: generate the covariance of its point set in TLR
form, factor it, return log det, the solve A^{-1} y and the log-likelihood.

Requests are admitted as they arrive when a slot (a context: one stream pair
and one workspace) is free and their HBM footprint fits in the budget; admitted
requests run concurrently, so their kernels overlap on the device.  Every
request runs the same deterministic kernels on its own context, so its result
does not depend on what else is in flight.

A request whose near-diagonal tiles are not compressible within its maxrank
(generation INFO = -1, STARSH_gen.jdf:169-171) is handled by widening the dense
band to cover those tiles (band regeneration, band_regenerate.jdf:124-143)
before the optional band auto-tuning (band_size_auto_tuning.jdf:201-318).
"""
from __future__ import annotations

import math
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import tlr


@dataclass
class MLERequest:
    rid: int
    kind: int            # tlr.KIND_* of a point kernel (statistics or electrodynamics)
    n: int
    nb: int
    beta: float          # length scale
    sigma: float         # variance
    noise: float         # nugget
    acc: float           # accuracy e
    seed: int            # point placement and right-hand side
    arrival: float = 0.0  # seconds after the stream start
    maxrank: int = 0      # 0: min(NB/2 - 1, 200)
    autoband: bool = True

    @property
    def ndim(self) -> int:
        return tlr.KIND_NDIM[self.kind]

    def rhs(self) -> np.ndarray:
        return np.random.default_rng(self.seed + 7919).standard_normal(self.n)

    def cap(self) -> int:
        return self.maxrank or min(self.nb // 2 - 1, 200)


@dataclass
class MLEResult:
    rid: int
    n: int
    logdet: float = float("nan")
    loglik: float = float("nan")
    x: np.ndarray | None = None
    band: int = 1
    status: int = 0
    error: str = ""
    overflow: int = 0
    t_admit: float = 0.0
    t_done: float = 0.0
    latency: float = 0.0
    device: int = -1
    gpu_s: dict = field(default_factory=dict)


def sample_requests(count: int, seed: int = 0, rate: float = 2.0, n_min: int = 10000, n_max: int = 200000,
                    tiles=(1000, 1350, 1800, 2000, 2700)) -> list[MLERequest]:
    """Request stream of the serving benchmark: dimension 2D or 3D; N log-uniform
    in [n_min, n_max] rounded to the tile size; kernel sqexp or exp (3D);
    length scale U[0.03, 0.3]; variance U[0.5, 2]; nugget log-U[1e-6, 1e-2];
    e in {1e-6, 1e-8, 1e-9}; Poisson arrivals at `rate` requests/s."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        ndim = int(rng.integers(2, 4))
        kind = tlr.KIND_SQEXP_2D if ndim == 2 else (tlr.KIND_SQEXP_3D if rng.random() < 0.5 else tlr.KIND_EXP_3D)
        nb = int(rng.choice(tiles))
        n = int(math.exp(rng.uniform(math.log(n_min), math.log(n_max))))
        n = max(nb * 2, int(round(n / nb)) * nb)
        out.append(MLERequest(rid=i, kind=kind, n=n, nb=nb, beta=float(rng.uniform(0.03, 0.3)),
                              sigma=float(rng.uniform(0.5, 2.0)),
                              noise=float(math.exp(rng.uniform(math.log(1e-6), math.log(1e-2)))),
                              acc=float(rng.choice([1e-6, 1e-8, 1e-9])), seed=int(rng.integers(0, 2**31)),
                              arrival=t))
    return out


def footprint_bytes(req: MLERequest, band_guess: int = 3) -> int:
    """Device bytes a request holds: dense band, fixed-capacity low-rank slots
    and the diagonal inverses (memory model of testing_dpotrf.c:598-599 with
    the slot capacity in place of the average rank)."""
    nt = req.n // req.nb
    nb = req.nb
    b = min(band_guess, nt)
    slots = (nt - 1) * nt // 2
    return 8 * (nt * b * nb * nb + slots * 2 * nb * req.cap() + nt * nb * nb)


def solve_request(ctx: tlr.Context, req: MLERequest) -> MLEResult:
    """Generate, factor and evaluate one request on `ctx` (blocking)."""
    res = MLEResult(rid=req.rid, n=req.n)
    prob = tlr.Problem(kind=req.kind, beta=req.beta, sigma=req.sigma, noise=req.noise, seed=req.seed)
    A = None
    try:
        t0 = time.perf_counter()
        A = tlr.TLRMatrix(ctx, req.n, req.nb, req.cap(), 1)
        info = A.generate(prob, req.acc, req.cap())
        nt = req.n // req.nb
        G = A.rank_map()
        band = 1
        if info != 0:
            # tiles rejected by the rank rule become dense: widen the band over them
            rej = A.rejected_tiles()
            band = max(2, max(m - n for m, n in rej) + 1)
        if req.autoband and info == 0:
            b = tlr.parsec_band_size_auto_tuning(G, nt, req.nb)
            band = max(band, b)
        if band > 1:
            A.band_regenerate(prob, min(band, nt))
        t1 = time.perf_counter()
        info = A.potrf(req.acc, req.cap())
        t2 = time.perf_counter()
        if info != 0:
            res.status = info
            res.error = f"not positive definite (info {info})"
            return res
        y = req.rhs()
        ll, ld, x = A.loglik(y)
        t3 = time.perf_counter()
        st = A.stats()
        res.logdet, res.loglik, res.x, res.band = ld, ll, x, A.band_size
        res.overflow = int(st[2])
        res.gpu_s = {"generate": t1 - t0, "factor": t2 - t1, "solve": t3 - t2}
    except tlr.TLRError as e:
        res.status = e.code
        res.error = str(e)
    finally:
        if A is not None:
            A.close()
    return res


class ReplicaRouter:
    """Routes a request stream over the GPUs of one node as replicas: every
    request runs whole on one GPU and no data crosses between GPUs.

    Each GPU has `slots` contexts and an HBM budget.  A request is admitted to
    the healthy GPU that has a free slot and the most budget left after taking
    the request's footprint (ties go to the lower device index).  A request
    larger than a GPU's whole budget is admitted only to an idle GPU and runs
    there alone.  A solve that fails at the CUDA level (status ERR_CUDA, or an
    exception out of the solve) marks its GPU failed: the GPU takes no further
    requests, its contexts are not reused, and the request is routed once more
    to another healthy GPU.  When no healthy GPU is left, the remaining
    requests complete with status ERR_CUDA.  A GPU whose contexts cannot be
    created at start-up is marked failed the same way (the reason is kept in
    ``init_errors``); the router starts if at least one GPU does.

    `make_context(device)`, `solve(ctx, req)` and `footprint(req)` default to
    the library's context, :func:`solve_request` and :func:`footprint_bytes`.
    """

    def __init__(self, devices=(0,), slots: int = 4, hbm_budgets=None, workspace_bytes: int = 2 << 30,
                 make_context=None, solve=None, footprint=None):
        self.devices = list(devices)
        self.slots = slots
        self.workspace_bytes = workspace_bytes
        self._solve = solve or solve_request
        self._footprint = footprint or footprint_bytes
        make_context = make_context or (lambda d: tlr.Context(d, workspace_bytes))
        if hbm_budgets is None:
            import torch
            hbm_budgets = []
            for d in self.devices:
                free, _ = torch.cuda.mem_get_info(d)
                hbm_budgets.append(int(0.8 * free) - slots * workspace_bytes)
        self.hbm_budgets = [int(b) for b in hbm_budgets]
        if len(self.hbm_budgets) != len(self.devices):
            raise ValueError("one HBM budget per device")
        self.failed: set = set()        # indices into devices
        self.init_errors: dict = {}     # device index -> why its contexts could not be created
        self._ctxs = {}
        for i, d in enumerate(self.devices):
            made = []
            try:
                for _ in range(slots):
                    made.append(make_context(d))
            except Exception as e:      # a GPU that cannot start serves nothing; the others go on
                for ctx in made:
                    try:
                        ctx.close()
                    except Exception:
                        pass
                made = []
                self.failed.add(i)
                self.init_errors[i] = f"{type(e).__name__}: {e}"
            self._ctxs[i] = made
        if len(self.failed) == len(self.devices):
            raise RuntimeError(f"no GPU could be initialised: {self.init_errors}")

    def close(self):
        for ctxs in self._ctxs.values():
            for c in ctxs:
                try:
                    c.close()
                except Exception:       # a failed GPU may refuse; the others still close
                    pass
        self._ctxs = {}

    def _choose(self, fp: int, free, budget, exclude) -> int | None:
        best = None
        for i in range(len(self.devices)):
            if i in self.failed or i in exclude or not free[i]:
                continue
            full = self.hbm_budgets[i]
            if fp > budget[i] and budget[i] < full:
                continue
            room = budget[i] - fp
            if best is None or room > best[0]:
                best = (room, i)
        return None if best is None else best[1]

    def run(self, requests: list[MLERequest], realtime: bool = True) -> list[MLEResult]:
        """Serve `requests` (sorted by arrival).  With realtime=False all
        requests are available at t=0 (saturation).  Returns results in
        request order with admission and completion times, latency and the
        device each ran on."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        results: dict[int, MLEResult] = {}
        free = {i: list(self._ctxs.get(i, [])) for i in range(len(self.devices))}
        budget = list(self.hbm_budgets)
        cv = threading.Condition()
        t0 = time.perf_counter()
        admit_time: dict[int, float] = {}
        threads: list[threading.Thread] = []

        def no_device_result(req):
            r = MLEResult(rid=req.rid, n=req.n, status=tlr.ERR_CUDA, error="no healthy GPU left")
            r.t_done = time.perf_counter() - t0
            r.latency = r.t_done - (req.arrival if realtime else 0.0)
            return r

        def admit(req, exclude):
            """Block until a GPU takes `req`; returns (device index, ctx, fp) or None."""
            fp = self._footprint(req)
            with cv:
                while True:
                    healthy = [i for i in range(len(self.devices)) if i not in self.failed and i not in exclude]
                    if not healthy:
                        return None
                    i = self._choose(fp, free, budget, exclude)
                    if i is not None:
                        budget[i] -= fp
                        return i, free[i].pop(), fp
                    cv.wait()

        def worker(req, i, ctx, fp, tried):
            try:
                r = self._solve(ctx, req)
                device_fault = r.status == tlr.ERR_CUDA
            except Exception as e:          # a failing solve must not take the router down
                r = MLEResult(rid=req.rid, n=req.n, status=tlr.ERR_CUDA, error=f"{type(e).__name__}: {e}")
                device_fault = True
            with cv:
                budget[i] += fp
                if device_fault:
                    self.failed.add(i)
                    free[i] = []
                else:
                    free[i].append(ctx)
                cv.notify_all()
            if device_fault and len(tried) < 2:
                nxt = admit(req, exclude=set(tried))
                if nxt is not None:
                    j, ctx2, fp2 = nxt
                    worker(req, j, ctx2, fp2, tried + [j])
                    return
                r.error += "; no other healthy GPU to retry on"
            r.device = self.devices[i]
            r.t_admit = admit_time[req.rid]
            r.t_done = time.perf_counter() - t0
            r.latency = r.t_done - (req.arrival if realtime else 0.0)
            with cv:
                results[req.rid] = r
                cv.notify_all()

        for req in reqs:
            if realtime:
                wait = req.arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
            got = admit(req, exclude=set())
            if got is None:
                with cv:
                    results[req.rid] = no_device_result(req)
                continue
            i, ctx, fp = got
            admit_time[req.rid] = time.perf_counter() - t0
            th = threading.Thread(target=worker, args=(req, i, ctx, fp, [i]), daemon=True)
            th.start()
            threads.append(th)
        for th in threads:
            th.join()
        return [results[r.rid] for r in requests]


class MLEServer(ReplicaRouter):
    """Admission-controlled concurrent request loop on one GPU."""

    def __init__(self, device: int = 0, slots: int = 4, hbm_budget: int | None = None,
                 workspace_bytes: int = 2 << 30, **kw):
        super().__init__(devices=[device], slots=slots,
                         hbm_budgets=None if hbm_budget is None else [hbm_budget],
                         workspace_bytes=workspace_bytes, **kw)
        self.device = device
        self.hbm_budget = self.hbm_budgets[0]


def summarize(results: list[MLEResult], makespan: float) -> dict:
    ok = [r for r in results if r.status == 0]
    lat = sorted(r.latency for r in ok)

    def pct(p):
        if not lat:
            return None
        return lat[min(len(lat) - 1, int(math.ceil(p / 100.0 * len(lat))) - 1)]

    return {"requests": len(results), "ok": len(ok), "solves_per_s": len(ok) / makespan if makespan > 0 else None,
            "p50_s": pct(50), "p99_s": pct(99), "makespan_s": makespan,
            "overflowed": sum(1 for r in ok if r.overflow)}
