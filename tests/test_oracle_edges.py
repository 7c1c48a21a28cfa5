"""Edge cases of the CPU oracle (the restated reference algorithm) at sizes that
finish in seconds: band > 1, one tile, rank-0 inputs, fixed rank, the maxrank
cap, the generation rejection rule, and solve / log-likelihood against dense."""
import math

import numpy as np
import pytest

from oracle import tlr_oracle as O

N, NB = 540, 54


@pytest.fixture(scope="module")
def setup():
    prob = O.Problem(kind=2, beta=0.02, noise=1e-2)     # short length scale: tiles compress at N=540
    pts = O.gen_points(N, 2)
    return prob, pts, O.dense_matrix(prob, pts)


@pytest.mark.parametrize("band", [1, 2, 3])
def test_band_factorization_meets_checks(setup, band):
    prob, pts, A = setup
    T, info = O.generate(prob, N, NB, 1e-9, NB // 2 - 1, band, pts)
    assert info == 0
    assert all(T.is_dense(m, n) for (m, n) in T.dense)
    st = O.tlr_potrf(T, 1e-9)
    assert st.info == 0
    L = O.uncompress(T)
    assert O.check_dpotrf2(L, A) <= 10 * 1e-9
    ld_dense = 2.0 * np.log(np.diag(np.linalg.cholesky(A))).sum()
    assert abs(O.logdet(T) - ld_dense) <= 1e-8 * abs(ld_dense)


def test_single_tile_is_dense_cholesky(setup):
    prob, pts, _ = setup
    T, info = O.generate(prob, NB, NB, 1e-9, 20, 1, pts[:NB])
    assert info == 0 and list(T.dense) == [(0, 0)] and not T.U
    A0 = T.dense[(0, 0)].copy()
    assert O.tlr_potrf(T, 1e-9).info == 0
    assert np.allclose(T.dense[(0, 0)], np.linalg.cholesky(A0))


def test_solve_and_loglik_match_dense(setup):
    prob, pts, A = setup
    T, _ = O.generate(prob, N, NB, 1e-10, NB // 2 - 1, 1, pts)
    assert O.tlr_potrf(T, 1e-10).info == 0
    y = np.random.default_rng(5).standard_normal(N)
    ll, ld, x = O.loglik(T, y)
    xd = np.linalg.solve(A, y)
    assert np.linalg.norm(x - xd) <= 1e-6 * np.linalg.norm(xd)
    lld = -0.5 * (y @ xd + np.linalg.slogdet(A)[1] + N * math.log(2 * math.pi))
    assert abs(ll - lld) <= 1e-8 * abs(lld)
    Y = np.stack([y, 2 * y], axis=1)          # several right-hand sides at once
    X = O.solve(T, Y)
    assert np.allclose(X[:, 1], 2 * X[:, 0])


def test_recompress_rank_zero_inputs():
    rng = np.random.default_rng(0)
    nb = 40
    U, V, r, ov = O.recompress(np.zeros((nb, 0)), np.zeros((nb, 0)), np.zeros((nb, 0)), np.zeros((nb, 0)), 1e-8, 10)
    assert r == 0 and U.shape == (nb, 0) and not ov
    Au, _ = np.linalg.qr(rng.standard_normal((nb, 3)))
    Y = rng.standard_normal((nb, 3))
    U, V, r, _ = O.recompress(np.zeros((nb, 0)), np.zeros((nb, 0)), Au, Y, 1e-12, 10)
    assert r == 3 and np.allclose(U @ V.T, -Au @ Y.T)


def test_recompress_fixed_rank_and_cap():
    rng = np.random.default_rng(1)
    nb = 60
    Cu, _ = np.linalg.qr(rng.standard_normal((nb, 8)))
    Cv = rng.standard_normal((nb, 8))
    Au, _ = np.linalg.qr(rng.standard_normal((nb, 8)))
    Y = rng.standard_normal((nb, 8))
    _, _, r, ov = O.recompress(Cu, Cv, Au, Y, 1e-12, 30, fixed_rank=5)
    assert r == 5 and not ov
    _, _, r, ov = O.recompress(Cu, Cv, Au, Y, 1e-12, 6)        # full rank 16 > maxrank 6
    assert r == 6 and ov


def test_generation_rejects_tiles_that_do_not_compress():
    # at beta = 0.03 the first sub-diagonal tiles need rank >= NB/2 and are rejected
    # (info -1, rank 0 stored); a band of 2 keeps them dense and generation succeeds
    prob = O.Problem(kind=2, beta=0.03, noise=1e-2)
    pts = O.gen_points(N, 2)
    T, info = O.generate(prob, N, NB, 1e-9, NB // 2 - 1, 1, pts)
    assert info == -1
    assert any(T.rank(m, n) == 0 and m - n == 1 for (m, n) in T.U)
    T2, info2 = O.generate(prob, N, NB, 1e-9, NB // 2 - 1, 2, pts)
    assert info2 == 0 and T2.is_dense(1, 0)
    O.band_regenerate(T, prob, pts, 2)
    for key in T2.U:
        assert np.allclose(T.U[key] @ T.V[key].T, T2.U[key] @ T2.V[key].T)


@pytest.mark.parametrize("kind,k", [(1, 50.0), (5, 5.0)])
def test_electrodynamics_kinds(kind, k):
    """-D 1 / -D 5: sin(k r)/r with add_diag (default N) on the diagonal.  The
    kernel is positive semi-definite in 2D and 3D, so the matrix is SPD with
    smallest eigenvalue about N - k; the TLR factor meets the reference check."""
    n, nb = 2700, 270
    prob = O.Problem(kind=kind, wave_k=k)
    pts = O.gen_points(n, O.KIND_NDIM[kind])
    A = O.dense_matrix(prob, pts)
    assert np.all(np.diag(A) == n) and np.allclose(A, A.T)
    off = A[1, 0]
    r = float(np.sqrt(np.sum((pts[1] - pts[0]) ** 2)))
    assert off == np.sin(k * r) / r
    assert np.linalg.eigvalsh(A)[0] >= n - k - 1e-6 * n
    T, info = O.generate(prob, n, nb, 1e-8, 130, 1, pts)
    assert info == 0
    assert O.tlr_potrf(T, 1e-8).info == 0
    assert O.check_dpotrf2(O.uncompress(T), A) <= 1e-8
    assert O.dense_matrix(O.Problem(kind=kind, wave_k=k, add_diag=7.0), pts)[3, 3] == 7.0


def test_gaussian_counter_generator():
    """The counter generator shared with the device sketches: u2 of entry i is
    the uniform of counter 2i + 1, and the sample moments are those of N(0, 1)."""
    g = O.gaussian_counter(123, 300, 200)
    assert g.shape == (300, 200)
    assert abs(g.mean()) < 0.01 and abs(g.var() - 1.0) < 0.02
    u = O.uniform01(123, np.array([1, 3]))
    assert np.all((u >= 0.0) & (u < 1.0))
    assert np.array_equal(O.gaussian_counter(123, 300, 200), g)
    assert not np.array_equal(O.gaussian_counter(124, 300, 200), g)


def test_randtlr_equal_ranks_and_factor():
    """-D 0: orthonormal per-block bases, every off-band tile with spectrum
    0.5^k, hence one rank everywhere (27 at e = 1e-8), and a factor that meets
    the reference check."""
    n, nb = 2700, 270
    prob = O.Problem(kind=O.KIND_RANDTLR)
    B = O.problem_points(prob, n, nb)
    K = 64
    assert B.shape == (n, 2 * K)
    for m in (0, 7):
        Q = B[m * nb:(m + 1) * nb, :K]
        assert np.allclose(Q.T @ Q, np.eye(K), atol=1e-13)
        assert np.allclose(B[m * nb:(m + 1) * nb, K:], Q * 0.5 ** np.arange(K))
    s = np.linalg.svd(O.cov_block(prob, B, 5 * nb, nb, 2 * nb, nb), compute_uv=False)
    assert np.allclose(s[:30], 0.5 ** np.arange(30), rtol=1e-12, atol=1e-15)
    A = O.dense_matrix(prob, B)
    assert np.all((np.diag(A) > n) & (np.diag(A) < n + 1.0))       # add_diag defaults to N
    T, info = O.generate(prob, n, nb, 1e-8, 130, 1, B)
    assert info == 0
    assert {T.rank(m, c) for (m, c) in T.U} == {27}
    assert O.tlr_potrf(T, 1e-8).info == 0
    assert O.check_dpotrf2(O.uncompress(T), A) <= 1e-8
    small = O.problem_points(prob, 120, 40)                         # K = min(NB, 64) = 40
    assert small.shape == (120, 80)


def test_scholqr3_v_side_keeps_ranks_and_accuracy():
    """Shifted CholeskyQR3 for R_V (Gram products and triangular multiplies, the
    tensor-core-friendly candidate for the device's V-side QR) gives the same
    final ranks, residual and log det as Householder on the reference's case."""
    prob = O.Problem(kind=2, noise=1e-4)
    pts = O.gen_points(2700, 2)
    T0, info = O.generate(prob, 2700, 270, 1e-8, 130, 1, pts)
    assert info == 0
    Th, Tc = T0.copy(), T0.copy()
    assert O.tlr_potrf(Th, 1e-8).info == 0
    assert O.tlr_potrf(Tc, 1e-8, v_side="scholqr3").info == 0
    Gh, Gc = Th.rank_array(), Tc.rank_array()
    assert np.array_equal(Gh, Gc)
    A = O.dense_matrix(prob, pts)
    rh, rc = O.check_dpotrf2(O.uncompress(Th), A), O.check_dpotrf2(O.uncompress(Tc), A)
    assert rc <= 10 * 1e-8 and abs(rc - rh) <= 0.01 * rh
    assert abs(O.logdet(Tc) - O.logdet(Th)) <= 1e-12 * abs(O.logdet(Th))
    # R factor itself: R^T R = V^T V and upper triangular, also for dependent columns
    rng = np.random.default_rng(2)
    V = rng.standard_normal((300, 40)) @ np.diag(10.0 ** -np.arange(40) * 0.25)
    V[:, 39] = V[:, 3]                                      # an exactly dependent column
    R = O.r_factor_scholqr3(V)
    assert np.allclose(np.tril(R, -1), 0.0)
    assert np.linalg.norm(R.T @ R - V.T @ V) <= 1e-12 * np.linalg.norm(V.T @ V)


def test_scholqr3_both_sides_keeps_ranks_and_accuracy():
    """The device's form for stacked ranks up to 48: shifted CholeskyQR3 on both
    sides of every recompression ([Cu, Au] = Q_U R_U with Q_U formed, no
    Gram-Schmidt projection; R_V only on the V side) gives the Householder
    oracle's final ranks, residual and log det on the reference's case, and
    Q_U is orthonormal to working precision even with dependent columns."""
    prob = O.Problem(kind=2, noise=1e-4)
    pts = O.gen_points(2700, 2)
    T0, info = O.generate(prob, 2700, 270, 1e-8, 130, 1, pts)
    assert info == 0
    Th, Tc = T0.copy(), T0.copy()
    assert O.tlr_potrf(Th, 1e-8).info == 0
    assert O.tlr_potrf(Tc, 1e-8, v_side="scholqr3", u_side="scholqr3").info == 0
    assert np.array_equal(Th.rank_array(), Tc.rank_array())
    A = O.dense_matrix(prob, pts)
    rh, rc = O.check_dpotrf2(O.uncompress(Th), A), O.check_dpotrf2(O.uncompress(Tc), A)
    assert rc <= 10 * 1e-8 and abs(rc - rh) <= 0.01 * rh
    assert abs(O.logdet(Tc) - O.logdet(Th)) <= 1e-12 * abs(O.logdet(Th))
    for (m, n), U in Tc.U.items():
        r = U.shape[1]
        if r:
            assert np.linalg.norm(U.T @ U - np.eye(r)) <= 1e-12
    rng = np.random.default_rng(3)
    Q0, _ = np.linalg.qr(rng.standard_normal((500, 20)))
    V = np.hstack([Q0, Q0[:, :5] @ rng.standard_normal((5, 8)) + 1e-13 * rng.standard_normal((500, 8))])
    Q, R = O.qr_scholqr3(V)
    assert np.allclose(np.tril(R, -1), 0.0)
    assert np.linalg.norm(Q @ R - V) <= 1e-13 * np.linalg.norm(V)


def test_rcholqr_both_sides_keeps_ranks_and_accuracy():
    """The device's form for stacks up to 64 columns: randomized CholeskyQR on
    both sides of every recompression gives the Householder oracle's final
    ranks, residual and log det on the reference's case, with Q_U orthonormal
    to working precision and one pass over the rows per QR."""
    import scipy.linalg as sla
    prob = O.Problem(kind=2, noise=1e-4)
    pts = O.gen_points(2700, 2)
    T0, info = O.generate(prob, 2700, 270, 1e-8, 130, 1, pts)
    assert info == 0
    Th, Tc = T0.copy(), T0.copy()
    assert O.tlr_potrf(Th, 1e-8).info == 0
    passes = []
    orig = O.qr_rcholqr

    def counted(X):
        out = orig(X)
        passes.append(out[3])
        return out

    O.qr_rcholqr = counted
    try:
        assert O.tlr_potrf(Tc, 1e-8, v_side="rcholqr", u_side="rcholqr").info == 0
    finally:
        O.qr_rcholqr = orig
    assert passes and max(passes) == 1
    assert np.array_equal(Th.rank_array(), Tc.rank_array())
    A = O.dense_matrix(prob, pts)
    rh, rc = O.check_dpotrf2(O.uncompress(Th), A), O.check_dpotrf2(O.uncompress(Tc), A)
    assert rc <= 10 * 1e-8 and abs(rc - rh) <= 0.01 * rh
    assert abs(O.logdet(Tc) - O.logdet(Th)) <= 1e-12 * abs(O.logdet(Th))
    for (m, n), U in Tc.U.items():
        r = U.shape[1]
        if r:
            assert np.linalg.norm(U.T @ U - np.eye(r)) <= 1e-12
    # the factors themselves
    rng = np.random.default_rng(4)
    X = rng.standard_normal((2700, 60)) @ np.diag(10.0 ** (-0.2 * np.arange(60)))
    Y, Rc, R, p = O.qr_rcholqr(X)
    Q = sla.solve_triangular(Rc, Y.T, trans="T", lower=False).T
    assert p == 1 and np.allclose(np.tril(R, -1), 0.0)
    assert np.linalg.norm(Q @ R - X) <= 1e-14 * np.linalg.norm(X)
    assert np.linalg.norm(Q.T @ Q - np.eye(60)) <= 1e-13


def _rcholqr_q(X):
    import scipy.linalg as sla
    Y, Rc, R, p = O.qr_rcholqr(X)
    return sla.solve_triangular(Rc, Y.T, trans="T", lower=False).T, R, p


def sketch_null_column(m, i):
    """A unit column whose sketch is exactly zero: rows i and i + 256 share a
    bucket, with entries that cancel under the sketch's signs."""
    s = O.sketch_signs(m)
    c = np.zeros(m)
    c[i], c[i + O.RCQ_ROWS] = s[i], -s[i + O.RCQ_ROWS]
    return c / np.sqrt(2.0)


@pytest.mark.parametrize("case", ["sketch_null", "zero_and_dependent", "all_zero", "scaled", "short", "near_dependent"])
def test_rcholqr_adversarial_inputs(case):
    """Randomized CholeskyQR on inputs built against it: a column the sketch
    cannot see (the repeat rule must fire and restore orthogonality), zero and
    exactly dependent columns (no repeat; Q R = X), an all-zero matrix (R = 0,
    everything finite), column scales 1e-150..1e100, fewer rows than sketch
    rows, and nearly dependent blocks."""
    rng = np.random.default_rng(5)
    m = 100 if case == "short" else 2700
    Q0, _ = np.linalg.qr(rng.standard_normal((m, 20)))
    if case == "sketch_null":
        c = sketch_null_column(m, 5)
        Q0 = Q0 - np.outer(c, c @ Q0)
        X = np.hstack([Q0, c[:, None]])
    elif case == "zero_and_dependent":
        X = np.hstack([Q0, np.zeros((m, 3)), 2.0 * Q0[:, :4]])
    elif case == "all_zero":
        X = np.zeros((m, 12))
    elif case == "scaled":
        X = rng.standard_normal((m, 30)) * 10.0 ** np.linspace(-150, 100, 30)
    elif case == "short":
        X = rng.standard_normal((m, 40))
    else:
        X = np.hstack([Q0, Q0[:, :5] @ rng.standard_normal((5, 8)) + 1e-13 * rng.standard_normal((m, 8))])
    Q, R, p = _rcholqr_q(X)
    K = X.shape[1]
    assert np.isfinite(Q).all() and np.isfinite(R).all()
    assert np.allclose(np.tril(R, -1), 0.0)
    assert p == (2 if case == "sketch_null" else 1)
    if case == "all_zero":
        assert not R.any()
        return
    assert np.linalg.norm(Q @ R - X) <= 1e-14 * np.linalg.norm(X)
    if case in ("sketch_null", "scaled", "short", "near_dependent"):
        assert np.linalg.norm(Q.T @ Q - np.eye(K)) <= 1e-13
    else:
        # the live columns stay orthonormal; the null directions of X carry R(j, j) ~ 0
        live = np.abs(np.diag(R)) > 1e-6 * np.abs(np.diag(R)).max()
        Ql = Q[:, live]
        assert np.linalg.norm(Ql.T @ Ql - np.eye(Ql.shape[1])) <= 1e-13


def test_sketch_signs_pinned():
    """The sketch's row signs (lowbias32 hash, low bit) for rows 0..15, pinned so
    that the restatement and the device's hash cannot drift apart unnoticed."""
    # computed independently by a C program (uint32 arithmetic)
    assert O.sketch_signs(16).tolist() == [1.0, 1.0, -1.0, -1.0, -1.0, 1.0, -1.0, 1.0,
                                           1.0, -1.0, -1.0, -1.0, 1.0, -1.0, 1.0, -1.0]


@pytest.mark.parametrize("band", [1, 2])
def test_dag_oracle_matches_sequential_oracle(band):
    """The task-graph run on host threads (the timed CPU baseline) computes the
    same factorization as the sequential oracle: same ranks, same op counts,
    factors equal up to BLAS rounding."""
    prob = O.Problem(kind=2, noise=1e-4)
    n, nb = 2700, 270
    pts = O.gen_points(n, 2)
    T, info = O.generate(prob, n, nb, 1e-8, 130, band, pts)
    assert info == 0
    T2 = T.copy()
    st1 = O.tlr_potrf(T, 1e-8)
    st2 = O.tlr_potrf_dag(T2, 1e-8, threads=4)
    assert st1.info == 0 and st2.info == 0
    assert np.array_equal(T.rank_array(), T2.rank_array())
    assert np.array_equal(st1.tileopcounters, st2.tileopcounters)
    assert np.array_equal(st1.rank_min, st2.rank_min) and np.array_equal(st1.rank_max, st2.rank_max)
    L1, L2 = O.uncompress(T), O.uncompress(T2)
    assert np.linalg.norm(L1 - L2) <= 1e-10 * np.linalg.norm(L1)
