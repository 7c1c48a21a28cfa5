"""Kernel-level parity of the CUDA library against the CPU oracle / numpy.

Each test calls the C ABI (include/hicma_tlr.h) on device buffers owned by
torch and compares with the oracle's restatement of the same reference step.
Tolerances are stated per test (FP64 throughout).
"""
import math

import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(a: np.ndarray):
    """Column-major device copy of a 2-D array: torch shape (cols, rows)."""
    a = np.asarray(a, dtype=np.float64)
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def host(t, rows=None):
    a = t.detach().cpu().numpy().T
    return a if rows is None else a[:rows]


def stream():
    return torch.cuda.current_stream().cuda_stream


def test_cov_tiles_match_oracle(ctx):
    from hicma_parsec_b200 import tlr
    for kind, n, nb, tiles in [(2, 2700, 270, [(0, 0), (3, 1), (9, 0)]), (4, 1000, 250, [(1, 1), (3, 0)]),
                               (3, 1331, 121, [(10, 2), (5, 5)])]:
        prob = tlr.Problem(kind=kind, noise=1e-4, beta=0.1)
        P = tlr.points(prob, n)
        dP = torch.from_numpy(P).cuda()
        pts = P.T.copy()
        oprob = O.Problem(kind=kind, noise=1e-4, beta=0.1)
        for (m, c) in tiles:
            out = torch.zeros((nb, nb), dtype=torch.float64, device="cuda")
            rc = tlr.load_library().hicma_tlr_k_cov(tlr.CProblem(kind, 0.1, 0.5, 1e-4, 1.0, 0), dP.data_ptr(), n,
                                                   m * nb, nb, c * nb, nb, out.data_ptr(), nb, stream())
            assert rc == 0, tlr.last_error()
            ref = O.cov_block(oprob, pts, m * nb, nb, c * nb, nb)
            got = host(out)
            # exp() of CUDA vs the host libm: at most a few ulps apart
            assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)) < 1e-14


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (64, 64, 16), (65, 130, 17), (270, 33, 270),
                                   (1000, 70, 1000), (129, 257, 0)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_dgemm_dmma(m, n, k, ta, tb):
    from hicma_parsec_b200 import tlr
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    rng = np.random.default_rng(m * 1000 + n * 10 + k + ta * 3 + tb)
    A = rng.standard_normal((k, m) if ta else (m, k))
    B = rng.standard_normal((n, k) if tb else (k, n))
    C = rng.standard_normal((m, n))
    alpha, beta = -1.25, 0.5
    dA, dB, dC = dev(A), dev(B), dev(C)
    lda, ldb = A.shape[0], B.shape[0]
    pa = dA.data_ptr() if dA.numel() else dC.data_ptr()
    pb = dB.data_ptr() if dB.numel() else dC.data_ptr()
    rc = tlr.load_library().hicma_tlr_k_dgemm(ta, tb, m, n, k, alpha, pa, max(lda, 1), pb,
                                             max(ldb, 1), beta, dC.data_ptr(), m, stream())
    assert rc == 0
    ref = alpha * ((A.T if ta else A) @ (B.T if tb else B)) + beta * C
    scale = (np.abs(A).max() * np.abs(B).max() * max(k, 1)) if k else 1.0
    # FP64 with k-term accumulation: |error| <= k * eps * |A||B|
    assert np.max(np.abs(host(dC) - ref)) <= 4 * max(k, 1) * 2.3e-16 * scale + 1e-15


@pytest.mark.parametrize("n", [64, 270, 1000, 2700])
def test_potrf_tile_and_inverse(ctx, n):
    from hicma_parsec_b200 import tlr
    pts = O.gen_points(n, 2, 3)
    A = O.cov_block(O.Problem(kind=2, noise=1e-2), pts, 0, n, 0, n)
    dA = dev(A)
    dL = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = tlr.load_library().hicma_tlr_k_potrf(ctx.h, n, dA.data_ptr(), n, dL.data_ptr(), info.data_ptr(), 0)
    assert rc == 0, tlr.last_error()
    assert int(info.item()) == 0
    L = np.tril(host(dA))
    Lref = np.linalg.cholesky(A)
    # backward stable Cholesky: ||L L^T - A|| / ||A|| ~ n eps
    assert np.linalg.norm(L @ L.T - A) / np.linalg.norm(A) < 1e-13
    assert np.max(np.abs(L - Lref)) < 1e-8 * np.max(np.abs(Lref))
    Li = host(dL)
    assert np.allclose(np.triu(Li, 1), 0.0)
    assert np.linalg.norm(Li @ L - np.eye(n)) < 1e-9 * n


def test_potrf_reports_info(ctx):
    from hicma_parsec_b200 import tlr
    n = 200
    pts = O.gen_points(n, 2, 5)
    A = O.cov_block(O.Problem(kind=2, noise=1e-2), pts, 0, n, 0, n)
    A[150, 150] = -5.0          # leading minor 151 is not positive definite
    dA = dev(A)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = tlr.load_library().hicma_tlr_k_potrf(ctx.h, n, dA.data_ptr(), n, None, info.data_ptr(), 1000)
    assert rc == 0
    _, iinfo = O.potrf_tile(A)
    assert iinfo == 151
    assert int(info.item()) == 1000 + 151


def _c1_tiles(noise=1e-4):
    prob = O.Problem(kind=2, noise=noise)
    pts = O.gen_points(2700, 2)
    T, info = O.generate(prob, 2700, 270, 1e-8, 130, 1, pts)
    assert info == 0
    return T, prob, pts


def _slot(U, V, cap):
    nb, r = U.shape
    u = np.zeros((nb, cap)); v = np.zeros((nb, cap))
    u[:, :r] = U; v[:, :r] = V
    return dev(u), dev(v)


@pytest.mark.parametrize("case", ["lr", "dense_b", "rank0_c"])
def test_lr_update_matches_oracle(ctx, case):
    """One potrf_dgemm(m, n, k) low-rank-C task: HCORE_dgemm_qr_svd(+b_dense)."""
    from hicma_parsec_b200 import tlr
    import ctypes as C
    T, prob, pts = _c1_tiles()
    m, n, k = 7, 4, 2
    Au, Av = T.U[(m, k)], T.V[(m, k)]
    cap = 130
    if case == "dense_b":
        B = O.cov_block(prob, pts, n * 270, 270, k * 270, 270)
        Y = B @ Av
    else:
        Bu, Bv = T.U[(n, k)], T.V[(n, k)]
        Y = Bu @ (Bv.T @ Av)
    if case == "rank0_c":
        Cu, Cv = np.zeros((270, 0)), np.zeros((270, 0))
    else:
        Cu, Cv = T.U[(m, n)], T.V[(m, n)]
    Uref, Vref, rref, _ = O.recompress(Cu, Cv, Au, Y, 1e-8, cap)
    dAu, dAv = _slot(Au, Av, cap)
    dCu, dCv = _slot(Cu, Cv, cap)
    rc = C.c_int(Cu.shape[1])
    torch.cuda.synchronize()
    if case == "dense_b":
        dB = dev(B)
        code = tlr.load_library().hicma_tlr_k_lr_update(ctx.h, 270, dAu.data_ptr(), dAv.data_ptr(), Au.shape[1],
                                                       dB.data_ptr(), None, 0, dCu.data_ptr(), dCv.data_ptr(),
                                                       C.byref(rc), 1e-8, cap, 0)
    else:
        dBu, dBv = _slot(Bu, Bv, cap)
        code = tlr.load_library().hicma_tlr_k_lr_update(ctx.h, 270, dAu.data_ptr(), dAv.data_ptr(), Au.shape[1],
                                                       dBu.data_ptr(), dBv.data_ptr(), Bu.shape[1], dCu.data_ptr(),
                                                       dCv.data_ptr(), C.byref(rc), 1e-8, cap, 0)
    assert code == 0, tlr.last_error()
    r = rc.value
    assert abs(r - rref) <= 1, (r, rref)
    U, V = host(dCu)[:, :r], host(dCv)[:, :r]
    exact = Cu @ Cv.T - Au @ Y.T
    # absolute truncation at acc = 1e-8 per singular value: error <= sqrt(K) * acc
    err = np.linalg.norm(U @ V.T - exact, 2)
    assert err <= 3e-8, err
    assert np.linalg.norm(U.T @ U - np.eye(r)) < 1e-12   # U keeps orthonormal columns


@pytest.mark.parametrize("case", ["sketch_null", "zero_column", "near_dependent"])
def test_lr_update_cholqr_adversarial(ctx, case):
    """Recompressions whose stacks (18 columns: the randomized CholeskyQR path)
    are built against it: a column of Cu that the sketch cannot see (rows 3 and
    259 share a bucket and cancel under its signs, so the repeat rule has to
    fire), a zero column in Cu, and an update lying within 1e-12 of span(Cu).
    Rank within 1 of the Householder oracle, U V^T within the truncation bound
    of the exact product, U orthonormal to 1e-12."""
    from hicma_parsec_b200 import tlr
    import ctypes as C
    nb, cap = 270, 64
    rng = np.random.default_rng(11)
    Q0, _ = np.linalg.qr(rng.standard_normal((nb, 12)))
    if case == "sketch_null":
        s = O.sketch_signs(nb)
        c = np.zeros(nb)
        c[3], c[3 + O.RCQ_ROWS] = s[3], -s[3 + O.RCQ_ROWS]
        c /= np.sqrt(2.0)
        Q1, _ = np.linalg.qr(Q0[:, :11] - np.outer(c, c @ Q0[:, :11]))
        Cu = np.hstack([Q1, c[:, None]])
    elif case == "zero_column":
        Cu = np.hstack([Q0[:, :11], np.zeros((nb, 1))])
    else:
        Cu = Q0
    Cv = rng.standard_normal((nb, 12)) * 10.0 ** -np.linspace(0, 6, 12)
    if case == "near_dependent":
        Au, _ = np.linalg.qr(Q0[:, :4] @ rng.standard_normal((4, 6)) + 1e-12 * rng.standard_normal((nb, 6)))
    else:
        Au, _ = np.linalg.qr(rng.standard_normal((nb, 6)))
    Av = 1e-2 * rng.standard_normal((nb, 6))
    Bu, _ = np.linalg.qr(rng.standard_normal((nb, 6)))
    Bv = rng.standard_normal((nb, 6))
    Y = Bu @ (Bv.T @ Av)
    _, _, rref, _ = O.recompress(Cu, Cv, Au, Y, 1e-8, cap)
    dAu, dAv = _slot(Au, Av, cap)
    dBu, dBv = _slot(Bu, Bv, cap)
    dCu, dCv = _slot(Cu, Cv, cap)
    rc = C.c_int(Cu.shape[1])
    torch.cuda.synchronize()
    code = tlr.load_library().hicma_tlr_k_lr_update(ctx.h, nb, dAu.data_ptr(), dAv.data_ptr(), 6, dBu.data_ptr(),
                                                   dBv.data_ptr(), 6, dCu.data_ptr(), dCv.data_ptr(), C.byref(rc),
                                                   1e-8, cap, 0)
    assert code == 0, tlr.last_error()
    r = rc.value
    assert abs(r - rref) <= 1, (r, rref)
    U, V = host(dCu)[:, :r], host(dCv)[:, :r]
    assert np.isfinite(U).all() and np.isfinite(V).all()
    exact = Cu @ Cv.T - Au @ Y.T
    # absolute truncation at acc = 1e-8 per singular value: error <= sqrt(K) * acc
    assert np.linalg.norm(U @ V.T - exact, 2) <= math.sqrt(18) * 1e-8
    assert np.linalg.norm(U.T @ U - np.eye(r)) < 1e-12


def test_compress_matches_oracle(ctx):
    from hicma_parsec_b200 import tlr
    import ctypes as C
    prob = O.Problem(kind=2, noise=1e-4)
    pts = O.gen_points(2700, 2)
    for (m, n) in [(1, 0), (5, 2), (9, 0)]:
        A = O.cov_block(prob, pts, m * 270, 270, n * 270, 270)
        _, _, rref = O.compress_tile(A, 1e-8, 130)
        dA = dev(A)
        dU = torch.zeros((130, 270), dtype=torch.float64, device="cuda")
        dV = torch.zeros((130, 270), dtype=torch.float64, device="cuda")
        r = C.c_int()
        torch.cuda.synchronize()
        code = tlr.load_library().hicma_tlr_k_compress(ctx.h, 270, dA.data_ptr(), dU.data_ptr(), dV.data_ptr(),
                                                      130, 1e-8, C.byref(r))
        assert code == 0, tlr.last_error()
        assert abs(r.value - rref) <= 2, (m, n, r.value, rref)
        U, V = host(dU)[:, :r.value], host(dV)[:, :r.value]
        assert np.linalg.norm(U @ V.T - A) <= 3e-8 * np.linalg.norm(A)
