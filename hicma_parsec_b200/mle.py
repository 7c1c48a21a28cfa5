"""Maximum-likelihood fit of covariance parameters on one GPU.

No counterpart in the reference (its driver stops at the factor,
hicma_parsec/testing_dpotrf.c:830-903).  It is the consumer the log-likelihood
path exists for: for a fixed point set and observation vector y, find the
length scale beta, the variance sigma and the nugget that maximise

    l(theta) = -1/2 (y^T Sigma(theta)^-1 y + log det Sigma(theta) + N log 2 pi)

with a gradient-free simplex search (Nelder and Mead, 1965) over the logarithms
of the three parameters, so that every candidate stays positive.  Each
evaluation generates Sigma(theta) in TLR form on the device, factors it and
returns the log-likelihood; the points are generated once from the seed, so
every evaluation sees the same point set.  A candidate whose factorization
fails (not positive definite at this accuracy) counts as -inf.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import tlr


def nelder_mead(f, x0, step, max_evals: int = 60, xtol: float = 1e-4, ftol: float = 1e-8):
    """Minimise f from x0 with the standard coefficients (reflection 1,
    expansion 2, contraction 1/2, shrink 1/2).  Deterministic: ties keep the
    earlier vertex.  Returns (x_best, f_best, evaluations)."""
    x0 = np.asarray(x0, dtype=float)
    n = x0.size
    simplex = [x0.copy()]
    for i in range(n):
        v = x0.copy()
        v[i] += step[i] if np.ndim(step) else step
        simplex.append(v)
    values = [f(v) for v in simplex]
    evals = len(values)
    while evals < max_evals:
        order = sorted(range(n + 1), key=lambda i: (values[i], i))
        simplex = [simplex[i] for i in order]
        values = [values[i] for i in order]
        spread_x = max(np.max(np.abs(v - simplex[0])) for v in simplex[1:])
        if spread_x <= xtol and abs(values[-1] - values[0]) <= ftol * (1.0 + abs(values[0])):
            break
        centroid = np.mean(simplex[:-1], axis=0)
        xr = centroid + (centroid - simplex[-1])
        fr = f(xr); evals += 1
        if fr < values[0]:
            xe = centroid + 2.0 * (centroid - simplex[-1])
            fe = f(xe); evals += 1
            simplex[-1], values[-1] = (xe, fe) if fe < fr else (xr, fr)
        elif fr < values[-2]:
            simplex[-1], values[-1] = xr, fr
        else:
            outside = fr < values[-1]
            xc = centroid + 0.5 * ((xr if outside else simplex[-1]) - centroid)
            fc = f(xc); evals += 1
            if fc < (fr if outside else values[-1]):
                simplex[-1], values[-1] = xc, fc
            else:
                for i in range(1, n + 1):
                    simplex[i] = simplex[0] + 0.5 * (simplex[i] - simplex[0])
                    values[i] = f(simplex[i]); evals += 1
    best = min(range(n + 1), key=lambda i: (values[i], i))
    return simplex[best], values[best], evals


@dataclass
class MLEFit:
    beta: float
    sigma: float
    noise: float
    loglik: float
    evaluations: int
    history: list = field(default_factory=list)   # (beta, sigma, noise, loglik) per evaluation


def device_loglik(ctx: "tlr.Context", kind: int, n: int, nb: int, y: np.ndarray, acc: float,
                  maxrank: int, seed: int = 0, autoband: bool = True):
    """Return the evaluator l(beta, sigma, noise) for one point set (seed) and y:
    generate, optionally widen the band, factor, log-likelihood; -inf when the
    approximate matrix is not positive definite."""
    nt = n // nb

    def evaluate(beta: float, sigma: float, noise: float) -> float:
        prob = tlr.Problem(kind=kind, beta=beta, sigma=sigma, noise=noise, seed=seed)
        A = tlr.TLRMatrix(ctx, n, nb, maxrank, 1)
        try:
            info = A.generate(prob, acc, maxrank)
            band = 1
            if info != 0:
                band = max(2, max(m - k for m, k in A.rejected_tiles()) + 1)
            elif autoband:
                band = tlr.parsec_band_size_auto_tuning(A.rank_map(), nt, nb)
            if band > 1:
                A.band_regenerate(prob, min(band, nt))
            if A.potrf(acc, maxrank) != 0:
                return -math.inf
            ll, _, _ = A.loglik(y)
            return ll
        finally:
            A.close()

    return evaluate


def fit_mle(evaluate, theta0, max_evals: int = 40, step: float = 0.5) -> MLEFit:
    """Maximise evaluate(beta, sigma, noise) from theta0 = (beta, sigma, noise)
    by a simplex search over (log beta, log sigma, log noise)."""
    hist = []

    def objective(x):
        beta, sigma, noise = (float(math.exp(v)) for v in x)
        ll = evaluate(beta, sigma, noise)
        hist.append((beta, sigma, noise, ll))
        return -ll if math.isfinite(ll) else math.inf

    x0 = np.log(np.asarray(theta0, dtype=float))
    x, fx, evals = nelder_mead(objective, x0, step, max_evals=max_evals)
    beta, sigma, noise = (float(math.exp(v)) for v in x)
    return MLEFit(beta=beta, sigma=sigma, noise=noise, loglik=-fx, evaluations=evals, history=hist)
