"""Property tests (hypothesis) of the oracle's building blocks and of the
library's host-side generators, over random shapes, ranks and seeds:

* recompression C_new = [Cu, Au] [Cv, -Y]^T: U has orthonormal columns, every
  discarded singular value is below acc (spectral error < acc, Frobenius
  error <= acc sqrt(K - r)), the rank is capped at maxrank with the overflow
  flag, and the Householder and shifted-CholeskyQR3 V sides agree;
* points: the library's generator equals the oracle's bit for bit for every
  point kind, size and seed;
* band auto-tuning: the library equals the oracle on random rank maps."""
import numpy as np
import pytest
from hypothesis import HealthCheck, assume, given, settings
from hypothesis import strategies as st

from oracle import tlr_oracle as O

SETTINGS = settings(max_examples=25, deadline=None, suppress_health_check=[HealthCheck.too_slow])


def _orth(rng, n, k):
    if k == 0:
        return np.zeros((n, 0))
    q, _ = np.linalg.qr(rng.standard_normal((n, k)))
    return q


@SETTINGS
@given(nb=st.integers(8, 96), rc=st.integers(0, 12), ra=st.integers(0, 12), seed=st.integers(0, 2**31 - 1),
       decay=st.floats(0.05, 0.9), acc_exp=st.integers(-12, -3))
def test_recompress_invariants(nb, rc, ra, seed, decay, acc_exp):
    rng = np.random.default_rng(seed)
    rc, ra = min(rc, nb // 2), min(ra, nb // 2)
    Cu = _orth(rng, nb, rc)
    Cv = rng.standard_normal((nb, rc)) * decay ** np.arange(rc)
    Au = _orth(rng, nb, ra)
    Y = rng.standard_normal((nb, ra)) * decay ** np.arange(ra)
    acc = 10.0 ** acc_exp
    K = rc + ra
    U, V, r, ov = O.recompress(Cu, Cv, Au, Y, acc, maxrank=nb)
    assert not ov and 0 <= r <= K and U.shape == (nb, r) and V.shape == (nb, r)
    if r:
        assert np.allclose(U.T @ U, np.eye(r), atol=1e-12)
    E = (Cu @ Cv.T - Au @ Y.T) - U @ V.T
    sv = np.linalg.svd(Cu @ Cv.T - Au @ Y.T, compute_uv=False)
    scale = max(1.0, sv[0] if sv.size else 0.0)
    assert np.linalg.norm(E, 2) <= acc + 1e-13 * scale
    assert np.linalg.norm(E) <= acc * np.sqrt(max(K - r, 0)) + 1e-12 * scale
    assert r == int(np.count_nonzero(sv[:K] >= acc)) or abs(sv[min(r, K - 1)] - acc) <= 1e-12 * scale
    U2, V2, r2, _ = O.recompress(Cu, Cv, Au, Y, acc, maxrank=nb, v_side="scholqr3")
    assert r2 == r
    if r:
        assert np.linalg.norm(U2 @ V2.T - U @ V.T, 2) <= 1e-9 * scale
    if r > 1:
        _, _, r3, ov3 = O.recompress(Cu, Cv, Au, Y, acc, maxrank=r - 1)
        assert r3 == r - 1 and ov3


@SETTINGS
@given(kind=st.sampled_from([1, 2, 3, 4, 5]), n=st.integers(1, 3000), seed=st.integers(0, 2**63 - 1))
def test_points_library_equals_oracle(kind, n, seed):
    from hicma_parsec_b200 import tlr
    P = tlr.points(tlr.Problem(kind=kind, seed=seed), n)
    np.testing.assert_array_equal(P, O.gen_points(n, O.KIND_NDIM[kind], seed).T)


@SETTINGS
@given(nt=st.integers(2, 30), nb=st.integers(2, 4000), seed=st.integers(0, 2**31 - 1), band=st.integers(1, 3))
def test_band_autotune_and_stats_library_equal_oracle(nt, nb, seed, band):
    from hicma_parsec_b200 import tlr
    rng = np.random.default_rng(seed)
    G = rng.integers(0, max(1, nb // 2), size=nt * nt).astype(np.int32)
    assert tlr.parsec_band_size_auto_tuning(G, nt, nb) == O.band_autotune(G, nt, nb)
    if band < nt:
        mn, mx, av = tlr.HICMA_get_stat2(G, nt, band)
        omn, omx, oav = O.rank_stat(G, nt, band)
        assert (mn, mx) == (omn, omx) and av == pytest.approx(oav, rel=1e-15)


@settings(max_examples=12, deadline=None, suppress_health_check=[HealthCheck.too_slow, HealthCheck.filter_too_much])
@given(kind=st.sampled_from([2, 3, 4]), nt=st.integers(2, 6), nb=st.sampled_from([48, 64, 96]),
       beta=st.floats(0.01, 0.1), noise_exp=st.integers(-4, -1), band=st.integers(1, 3),
       tol_exp=st.integers(-10, -6), seed=st.integers(0, 1000))
def test_tlr_factorization_meets_the_check(kind, nt, nb, beta, noise_exp, band, tol_exp, seed):
    """Whenever generation accepts every tile, the oracle's TLR Cholesky meets
    the reference's check at 10 e and its log det matches the dense one."""
    n, tol = nt * nb, 10.0 ** tol_exp
    band = min(band, nt)
    prob = O.Problem(kind=kind, beta=beta, noise=10.0 ** noise_exp, seed=seed)
    pts = O.gen_points(n, O.KIND_NDIM[kind], seed)
    T, info = O.generate(prob, n, nb, tol, nb // 2 - 1, band, pts)
    assume(info == 0)                            # else a tile needs rank >= NB/2: rejected by the rule
    st_ = O.tlr_potrf(T, tol)
    assert st_.info == 0
    A = O.dense_matrix(prob, pts)
    assert O.check_dpotrf2(O.uncompress(T), A) <= 10 * tol
    ld = 2.0 * np.sum(np.log(np.diag(np.linalg.cholesky(A))))
    assert abs(O.logdet(T) - ld) <= 1e-6 * abs(ld)
