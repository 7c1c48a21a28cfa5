"""The device evaluator of the maximum-likelihood fit on the reference's test
size (N=2700, tile 270): its log-likelihood matches the dense FP64 value of
the oracle, and a short simplex search improves a poor starting point."""
import math

import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu

N, NB, TOL, MAXRANK = 2700, 270, 1e-8, 130


def test_device_loglik_and_fit(ctx):
    from hicma_parsec_b200 import mle
    true = dict(beta=0.1, sigma=1.0, noise=1e-2)
    pts = O.gen_points(N, 2)
    S = O.dense_matrix(O.Problem(kind=2, **true), pts)
    L = np.linalg.cholesky(S)
    y = L @ np.random.default_rng(11).standard_normal(N)
    z = np.linalg.solve(L, y)
    ll_dense = -0.5 * (z @ z + 2.0 * np.log(np.diag(L)).sum() + N * math.log(2 * math.pi))
    evaluate = mle.device_loglik(ctx, 2, N, NB, y, TOL, MAXRANK)
    ll = evaluate(**true)
    assert abs(ll - ll_dense) <= 1e-6 * abs(ll_dense), (ll, ll_dense)
    start = (0.05, 0.6, 5e-2)
    fit = mle.fit_mle(evaluate, start, max_evals=10)
    assert fit.loglik > evaluate(*start)
