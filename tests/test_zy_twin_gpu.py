"""Twins of the full-size workloads, fully checked at N = 27,000 (10 x 10
tiles of 2700), where an N x N matrix fits on the device and the CPU oracle
can replay the factorization: the leading 10 x 10 tiles of the N = 270,000 2D
squared-exponential, the N = 108,000 3D exponential and the N = 216,000 3D
squared-exponential matrices (the first 27,000 of their Morton-ordered
points), so every tile is one of the full-size matrix's own tiles, with its
kernel, tile size, accuracy and maxrank; the twin's Cholesky factor is the
leading block of the full factor.

Bars, per twin:
- ||A - L L^T||_F / ||A||_F <= 10 e against the exact covariance (the
  reference's check_dpotrf2, testing_dpotrf.c:111-180, with the 10 e bar), and
  the matrix-free probe estimate the full-size runs report within a factor 2
  of that dense residual;
- log-determinant against the dense FP64 Cholesky of the exact covariance
  (cuSOLVER through torch, used here as the oracle only): relative error
  within the bound stated per twin below;
- per-tile final ranks within +/-2 of the oracle's TLR Cholesky
  (oracle.tlr_potrf) replayed on the CPU from the same generated tiles, where
  the oracle finishes in a test's time (maxrank <= 500).

Log-determinant bound.  With the nugget 1e-4 of these workloads the
factorization's own truncation error dominates the log-determinant: the CPU
oracle of the reference algorithm is at 9e-9 on the reference's 2700 case at
e = 1e-8 and its error grows with the number of truncated tiles.  Each twin
states the bound it meets at e = 1e-8 and the accuracy at which it meets the
1e-8 bar (measured on a B200 and recorded beside the full-size results).
"""
import ctypes

import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N, NB = 27000, 2700

# kind 2: 2D sqexp, kind 4: 3D exp, kind 3: 3D sqexp; n_full: the workload
# whose leading tiles the twin takes.  logdet_e8: the log-determinant bound met
# at e = 1e-8, and e_strict (when set): the accuracy at which the twin meets the
# 1e-8 bar.  Measured on a B200: 2D 1.15e-6 at e = 1e-8, 1.1e-8 at 1e-9, 1.0e-10
# at 1e-10; 3D exponential below 1e-15 at every e; 3D squared exponential
# 1.55e-7 at 1e-8, 1.0e-9 at 1e-9.  The oracle replaying the same tiles has the
# same error to the digits shown: it is the truncation error of the algorithm.
TWINS = {
    "2D sqexp, maxrank 150": dict(kind=2, n_full=270000, maxrank=150, autoband=False, oracle_ranks=True,
                                  logdet_e8=1.5e-6, e_strict=1e-10),
    "3D exp, maxrank 1350, auto band": dict(kind=4, n_full=108000, maxrank=1350, autoband=True,
                                            oracle_ranks=False, logdet_e8=1e-8, e_strict=None),
    "3D sqexp, maxrank 500, auto band": dict(kind=3, n_full=216000, maxrank=500, autoband=True,
                                             oracle_ranks=True, logdet_e8=2e-7, e_strict=1e-9),
}


def twin_points(tlr, prob, cfg):
    """The first N Morton-ordered points of the full-size workload."""
    return np.ascontiguousarray(tlr.points(prob, cfg["n_full"])[:, :N])


def _dense_logdet(tlr, prob, n, points):
    """2 sum log diag chol(A) of the exact covariance at the given points,
    built on the device by the library's covariance kernel and factored by
    cuSOLVER."""
    lib = tlr.load_library()
    pts = torch.from_numpy(np.ascontiguousarray(points)).cuda()
    A = torch.empty((n, n), dtype=torch.float64, device="cuda")   # row-major view = column-major A^T = A
    cp = prob.c()
    torch.cuda.synchronize()
    rc = lib.hicma_tlr_k_cov(ctypes.byref(cp), ctypes.c_void_p(pts.data_ptr()), n, 0, n, 0, n,
                             ctypes.c_void_p(A.data_ptr()), n, None)
    assert rc == 0, tlr.last_error()
    torch.cuda.synchronize()
    L = torch.linalg.cholesky(A)
    ld = float(2.0 * torch.log(torch.diagonal(L)).sum().item())
    del A, L, pts
    torch.cuda.empty_cache()
    return ld


def _snapshot(A, nt, band, maxrank):
    """The generated tiles as an oracle matrix (same input for the replay)."""
    T = O.TLRMatrix(A.n, A.nb, band, maxrank)
    for m in range(nt):
        for n in range(m + 1):
            t = A.tile(m, n)
            if m - n < band:
                T.dense[(m, n)] = np.array(t)
            else:
                T.U[(m, n)], T.V[(m, n)] = np.array(t[0]), np.array(t[1])
    return T


def _factor(tlr, ctx, prob, cfg, acc, want_snapshot, pts):
    A = tlr.TLRMatrix(ctx, N, NB, cfg["maxrank"], 1)
    assert A.generate(prob, acc, cfg["maxrank"], pts=pts) == 0
    if cfg["autoband"]:
        b = tlr.parsec_band_size_auto_tuning(A.rank_map(), N // NB, NB)
        if b > 1:
            A.band_regenerate(prob, b)
    T = _snapshot(A, N // NB, A.band_size, cfg["maxrank"]) if want_snapshot else None
    assert A.potrf(acc, cfg["maxrank"]) == 0
    return A, T


@pytest.mark.parametrize("name", sorted(TWINS))
def test_scaled_twin(name):
    from hicma_parsec_b200 import tlr
    cfg = TWINS[name]
    acc = 1e-8
    prob = tlr.Problem(kind=cfg["kind"], noise=1e-4, beta=0.1, sigma=1.0, seed=0)
    pts = twin_points(tlr, prob, cfg)
    ld_dense = _dense_logdet(tlr, prob, N, pts)
    ctx = tlr.Context(0, 16 << 30)
    A = None
    try:
        A, T = _factor(tlr, ctx, prob, cfg, acc, cfg["oracle_ranks"], pts)
        res, _ = A.check(prob)
        assert res <= 10 * acc, res
        est = A.check_probe(prob, 16, 0)
        assert 0.5 * res <= est <= 2.0 * res, (res, est)
        ld = A.logdet()
        err = abs(ld - ld_dense) / abs(ld_dense)
        assert err <= cfg["logdet_e8"], (err, cfg["logdet_e8"])
        if T is not None:
            G = A.rank_map()
            O.tlr_potrf(T, acc)
            Gref = T.rank_array()
            off = Gref >= 0
            assert np.array_equal(G >= 0, off)
            assert np.max(np.abs(G[off] - Gref[off])) <= 2, np.max(np.abs(G[off] - Gref[off]))
            # the device factor's log-determinant is the oracle's on the same tiles
            assert abs(ld - O.logdet(T)) <= 1e-9 * abs(ld_dense)
        A.close()
        A = None
        if cfg["e_strict"]:
            # the accuracy at which the log-determinant meets the 1e-8 bar
            A, _ = _factor(tlr, ctx, prob, cfg, cfg["e_strict"], False, pts)
            err = abs(A.logdet() - ld_dense) / abs(ld_dense)
            assert err <= 1e-8, (err, cfg["e_strict"])
    finally:
        if A is not None:
            A.close()
        ctx.close()
