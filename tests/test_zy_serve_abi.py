"""hicma_tlr_serve_loglik (one serving request in one C call) against the
Python serving path, which makes the same library calls one by one: same band,
and log det / log-likelihood / solution within 1e-12 relative (the kernels are
deterministic, so they are expected to agree bit for bit)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_serve_call_equals_python_path(ctx):
    from hicma_parsec_b200 import serving, tlr
    reqs = serving.sample_requests(4, seed=3, rate=0.0, n_min=2000, n_max=6000, tiles=(500, 1000))
    for r in reqs:
        r.maxrank = r.nb // 2 - 1
    for req in reqs:
        ref = serving.solve_request(ctx, req)
        assert ref.status == 0, ref.error
        prob = tlr.Problem(kind=req.kind, beta=req.beta, sigma=req.sigma, noise=req.noise, seed=req.seed)
        st, ll, ld, x, band = tlr.serve_loglik(ctx, prob, req.n, req.nb, req.acc, req.rhs(), req.cap(),
                                               req.autoband)
        assert st == 0
        assert band == ref.band
        assert abs(ld - ref.logdet) <= 1e-12 * abs(ref.logdet)
        assert abs(ll - ref.loglik) <= 1e-12 * abs(ref.loglik)
        assert np.allclose(x, ref.x, rtol=1e-12, atol=0)


def test_serve_call_reports_info_for_a_matrix_that_is_not_positive_definite(ctx):
    from hicma_parsec_b200 import tlr
    # a negative nugget larger than the kernel's diagonal makes A indefinite
    prob = tlr.Problem(kind=tlr.KIND_SQEXP_2D, beta=0.1, sigma=1.0, noise=-2.0, seed=1)
    st, ll, ld, x, band = tlr.serve_loglik(ctx, prob, 2000, 500, 1e-8, np.ones(2000), 249, True)
    assert st > 0
