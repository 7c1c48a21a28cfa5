"""Scaled twins of the full-size workloads, fully dense-checked on the device:
the same kernel, tile size, accuracy and maxrank as the N=270,000 2D and
N=108,000 3D workloads at N=27,000 (10 x 10 tiles), where an N x N matrix
fits.  Bars: ||A - L L^T||_F / ||A||_F <= 10 e against the exact covariance
(the reference's check_dpotrf2, testing_dpotrf.c:111-180, with the 10 e bar),
and the matrix-free probe estimate that the full-size runs report within a
factor 2 of that dense residual."""
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TWINS = {
    "2D sqexp, maxrank 150": dict(kind=2, maxrank=150, autoband=False),
    "3D exp, maxrank 1350, auto band": dict(kind=4, maxrank=1350, autoband=True),
}


@pytest.mark.parametrize("name", sorted(TWINS))
def test_scaled_twin_dense_check(name):
    from hicma_parsec_b200 import tlr
    cfg = TWINS[name]
    n, nb, acc = 27000, 2700, 1e-8
    ctx = tlr.Context(0, 16 << 30)
    A = None
    try:
        prob = tlr.Problem(kind=cfg["kind"], noise=1e-4, beta=0.1, sigma=1.0, seed=0)
        A = tlr.TLRMatrix(ctx, n, nb, cfg["maxrank"], 1)
        assert A.generate(prob, acc, cfg["maxrank"]) == 0
        if cfg["autoband"]:
            b = tlr.parsec_band_size_auto_tuning(A.rank_map(), n // nb, nb)
            if b > 1:
                A.band_regenerate(prob, b)
        assert A.potrf(acc, cfg["maxrank"]) == 0
        res, _ = A.check(prob)
        assert res <= 10 * acc, res
        est = A.check_probe(prob, 16, 0)
        assert 0.5 * res <= est <= 2.0 * res, (res, est)
    finally:
        if A is not None:
            A.close()
        ctx.close()
