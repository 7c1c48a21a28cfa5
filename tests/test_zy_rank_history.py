"""Rank history (the reference's dcRank record: initial / minimum / maximum /
final rank per off-band tile, HiCMA_dpotrf_L_2flow.jdf:353-361,683-691,1101-1106)
and the critical-path op count (op_path, :201,303-313,443-462) of the GPU
factorization against the oracle on ``-N 2700 -t 270 -e 1e-8 -u 130 -D 2``.
Initial and final ranks within +/-2 of the oracle's (randomized range finder
against exact SVD, the bar of the other rank parity tests), minimum and maximum
within +/-3; op counts within 2%."""
import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N, NB, TOL, MAXRANK = 2700, 270, 1e-8, 130


def test_rank_history_and_path_ops_match_oracle(ctx):
    from hicma_parsec_b200 import tlr
    prob = tlr.Problem(kind=2, noise=0.1)
    A = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 1)
    try:
        with pytest.raises(tlr.TLRError):
            A.rank_history()                      # before any factorization
        assert A.generate(prob, TOL, MAXRANK) == 0
        assert A.potrf(TOL) == 0
        h = A.rank_history()
        st = A.stats()
        T, _ = O.generate(O.Problem(kind=2, noise=0.1), N, NB, TOL, MAXRANK, 1, O.gen_points(N, 2))
        ost = O.tlr_potrf(T, TOL)
        low = ost.rank_init >= 0
        assert np.array_equal(h["initial"] >= 0, low)
        assert np.max(np.abs(h["initial"][low] - ost.rank_init[low])) <= 2
        # the extremes run over every intermediate update, where the two runs'
        # rank differences can add up over a few panels: one more rank of slack
        for key, ref in (("minimum", ost.rank_min), ("maximum", ost.rank_max)):
            assert np.max(np.abs(h[key][low] - ref[low])) <= 3, key
        G = A.rank_map().reshape(N // NB, N // NB).T
        assert np.array_equal(h["final"][low], G[low])
        assert np.all(h["minimum"][low] <= h["final"][low]) and np.all(h["final"][low] <= h["maximum"][low])
        assert abs(st[10] - ost.op_path) <= 0.02 * ost.op_path
        assert 0 < st[10] < st[1]
    finally:
        A.close()


def test_reference_signature_fills_rank_record(ctx):
    """hicma_tlr_dpotrf_L_rank takes HiCMA_dpotrf_L's full parameter list, the
    Rank descriptor included (hicma_parsec.h:38-56): its 4-int record per tile
    (initial, minimum, maximum, final at [(n*NT + m)*4 + q]) equals the rank
    history of the same factorization, and Ar its final rank map."""
    import ctypes as C
    from hicma_parsec_b200 import tlr
    nt = N // NB
    A = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 1)
    try:
        assert A.generate(tlr.Problem(kind=2, noise=0.1), TOL, MAXRANK) == 0
        la, two = C.c_int(-1), C.c_int(0)
        cpt = np.zeros(6, dtype=np.float64)
        Ar = np.zeros(nt * nt, dtype=np.int32)
        rank = np.full(4 * nt * nt, -7, dtype=np.int32)
        info = A.lib.hicma_tlr_dpotrf_L_rank(ctx.h, tlr.LOWER, A.h, Ar.ctypes.data_as(C.c_void_p),
                                             rank.ctypes.data_as(C.c_void_p), TOL, 0, MAXRANK, C.byref(la), 1,
                                             NB, MAXRANK, 0, C.byref(two), None, None,
                                             cpt.ctypes.data_as(C.c_void_p), 0)
        assert info == 0, tlr.last_error()
        h = A.rank_history()                     # NT x NT arrays indexed [m, n]
        R = rank.reshape(nt, nt, 4)              # [n, m, q]
        for q, key in enumerate(("initial", "minimum", "maximum", "final")):
            assert np.array_equal(R[:, :, q].T, h[key]), key
        low = h["initial"] >= 0
        assert low.any()
        assert np.array_equal(h["final"][low], Ar.reshape(nt, nt).T[low])
    finally:
        A.close()
