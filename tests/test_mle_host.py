"""Host logic of the maximum-likelihood fit (no GPU): the simplex search and the
parameter handling, with the device evaluation replaced by known functions."""
import math

import numpy as np

from hicma_parsec_b200 import mle
from oracle import tlr_oracle as O


def test_nelder_mead_quadratic():
    f = lambda x: (x[0] - 1.0) ** 2 + 3.0 * (x[1] + 2.0) ** 2 + 0.5 * (x[2] - 0.25) ** 2
    x, fx, evals = mle.nelder_mead(f, [0.0, 0.0, 0.0], 0.5, max_evals=400, xtol=1e-7, ftol=1e-14)
    assert np.allclose(x, [1.0, -2.0, 0.25], atol=1e-3) and fx < 1e-6 and evals <= 400


def test_fit_recovers_known_maximum_and_skips_failures():
    target = np.log([0.12, 1.3, 2e-3])

    def evaluate(beta, sigma, noise):
        if noise < 1e-6:
            return -math.inf                      # a candidate whose factorization failed
        d = np.log([beta, sigma, noise]) - target
        return 100.0 - float(d @ d)

    fit = mle.fit_mle(evaluate, (0.1, 1.0, 1e-3), max_evals=300)
    assert abs(math.log(fit.beta / 0.12)) < 0.02
    assert abs(math.log(fit.sigma / 1.3)) < 0.02
    assert abs(math.log(fit.noise / 2e-3)) < 0.02
    assert fit.loglik > 99.99 and len(fit.history) == fit.evaluations


def test_fit_improves_a_gaussian_likelihood():
    # exact log-likelihood of a small 2D sqexp field (dense, CPU) in place of the device path
    n = 300
    true = O.Problem(kind=2, beta=0.15, sigma=1.0, noise=1e-2)
    pts = O.gen_points(n, 2)
    y = np.linalg.cholesky(O.dense_matrix(true, pts)) @ np.random.default_rng(3).standard_normal(n)

    def evaluate(beta, sigma, noise):
        S = O.dense_matrix(O.Problem(kind=2, beta=beta, sigma=sigma, noise=noise), pts)
        try:
            L = np.linalg.cholesky(S)
        except np.linalg.LinAlgError:
            return -math.inf
        z = np.linalg.solve(L, y)
        return -0.5 * (z @ z + 2.0 * np.log(np.diag(L)).sum() + n * math.log(2 * math.pi))

    start = (0.05, 0.5, 5e-2)
    fit = mle.fit_mle(evaluate, start, max_evals=60)
    assert fit.loglik > evaluate(*start) + 1.0
    assert fit.loglik >= max(h[3] for h in fit.history) - 1e-9
