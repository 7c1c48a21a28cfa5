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
