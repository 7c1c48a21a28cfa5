"""Asynchronous factorization (HiCMA_dpotrf_L_2flow_New / _Destruct,
hicma_parsec/hicma_parsec_internal.h:295-315, as hicma_tlr_dpotrf_L_start /
_wait): the result equals the synchronous call's (bit for bit expected;
bar 1e-12 relative on log det), a second start while one is in flight and a
wait without a start are state errors, and an argument error raised on the
background thread reaches the caller with its message."""
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N, NB, TOL, MAXRANK = 2700, 270, 1e-8, 130


def test_start_wait_equals_sync(ctx):
    from hicma_parsec_b200 import tlr
    prob = tlr.Problem(kind=2, noise=0.1)
    A = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 1)
    B = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 1)
    try:
        assert A.generate(prob, TOL, MAXRANK) == 0 and B.generate(prob, TOL, MAXRANK) == 0
        A.potrf_start(TOL)
        with pytest.raises(tlr.TLRError) as e:
            B.potrf_start(TOL)
        assert e.value.code == tlr.ERR_STATE
        assert A.potrf_wait() == 0
        with pytest.raises(tlr.TLRError) as e:
            A.potrf_wait()
        assert e.value.code == tlr.ERR_STATE
        assert B.potrf(TOL) == 0
        assert abs(A.logdet() - B.logdet()) <= 1e-12 * abs(B.logdet())
        # maxrank above NB/2 is refused inside the background call
        C = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 1)
        try:
            assert C.generate(prob, TOL, MAXRANK) == 0
            C.potrf_start(TOL, maxrank=NB // 2 + 1)
            with pytest.raises(tlr.TLRError) as e:
                C.potrf_wait()
            assert e.value.code == tlr.ERR_ARG
            assert "maxrank" in str(e.value)
        finally:
            C.close()
    finally:
        A.close()
        B.close()
