"""Whole-matrix host transfer in the reference's packed layout and per-class
profiling.  The store holds every band tile (row m, n = m-band+1..m) and then
the packed [U, V] of every off-band tile (row m, n = 0..m-band; V at offset
NB*rank, HiCMA_dpotrf_L_2flow.jdf:386,518-519): checked tile by tile against
hicma_tlr_tile_get; a store written into a fresh descriptor factors to the same
log det (same data, same kernels: bar 1e-12 relative); a rank above the slot
capacity is refused.  Profiling counts launches and device time per class."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N, NB, TOL, MAXRANK, BAND = 2700, 270, 1e-8, 130, 2


def test_store_layout_round_trip_and_profiling(ctx):
    from hicma_parsec_b200 import tlr
    nt = N // NB
    prob = tlr.Problem(kind=2, noise=0.1)
    A = tlr.TLRMatrix(ctx, N, NB, MAXRANK, BAND)
    B = tlr.TLRMatrix(ctx, N, NB, MAXRANK, BAND)
    try:
        assert A.generate(prob, TOL, MAXRANK) == 0
        nbytes = A.store_bytes()
        buf = np.empty(nbytes // 8)
        ranks = np.empty(nt * nt, dtype=np.int32)
        A.store_get(buf.ctypes.data, ranks)
        p = 0
        for m in range(nt):
            for n in range(max(0, m - BAND + 1), m + 1):
                tile = buf[p:p + NB * NB].reshape(NB, NB, order="F")
                assert np.array_equal(tile, A.tile(m, n)), (m, n)
                assert ranks[n * nt + m] == -1
                p += NB * NB
        for m in range(BAND, nt):
            for n in range(0, m - BAND + 1):
                r = int(ranks[n * nt + m])
                U, V = A.tile(m, n)
                assert U.shape[1] == r
                assert np.array_equal(buf[p:p + NB * r].reshape(NB, r, order="F"), U)
                assert np.array_equal(buf[p + NB * r:p + 2 * NB * r].reshape(NB, r, order="F"), V)
                p += 2 * NB * r
        assert p * 8 == nbytes
        B.store_set(buf.ctypes.data, ranks)
        assert np.array_equal(B.rank_map(), A.rank_map())
        bad = ranks.copy()
        bad[1 * nt + 5] = MAXRANK + 1               # tile (5, 1) is off the band
        with pytest.raises(tlr.TLRError) as e:
            B.store_set(buf.ctypes.data, bad)
        assert e.value.code == tlr.ERR_ARG
        B.store_set(buf.ctypes.data, ranks)
        ctx.prof_enable(True)
        try:
            assert A.potrf(TOL) == 0
            prof = ctx.prof_read()
        finally:
            ctx.prof_enable(False)
        assert B.potrf(TOL) == 0
        assert abs(A.logdet() - B.logdet()) <= 1e-12 * abs(B.logdet())
        assert prof["potrf"]["launches"] >= nt and prof["potrf"]["seconds"] > 0
        assert prof["qr"]["launches"] > 0 and prof["core_svd"]["launches"] > 0
        assert prof["gemm_trsm"]["launches"] > 0 and prof["gemm_trsm"]["flops"] > 0
        assert all(v["seconds"] >= 0 for v in prof.values())
    finally:
        A.close()
        B.close()


def test_copy_adopts_a_widened_band(ctx):
    """hicma_tlr_desc_copy onto a descriptor created like the source: a band the
    source widened after generation is adopted (the driver's copy for
    check_diff after band auto-tuning); a different creation band is refused."""
    from hicma_parsec_b200 import tlr
    prob = tlr.Problem(kind=2, noise=0.1)
    A = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 1)
    B = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 1)
    C = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 2)
    try:
        assert A.generate(prob, TOL, MAXRANK) == 0
        A.band_regenerate(prob, 3)
        B.copy_from(A)
        assert B.band_size == 3
        assert np.array_equal(B.rank_map(), A.rank_map())
        assert np.array_equal(B.tile(5, 3), A.tile(5, 3))
        with pytest.raises(tlr.TLRError) as e:
            C.copy_from(A)
        assert e.value.code == tlr.ERR_ARG
        assert A.potrf(TOL) == 0 and B.potrf(TOL) == 0
        assert abs(A.logdet() - B.logdet()) <= 1e-12 * abs(A.logdet())
    finally:
        A.close()
        B.close()
        C.close()


def test_store_stream_copies_each_final_column(ctx):
    """hicma_tlr_store_stream: the factorization copies every tile column into a
    page-locked host buffer as the column becomes final (column layout: band
    tiles, then the packed [U, V] of the off-band tiles with their final ranks),
    checked tile by tile against the factored descriptor; stats[15] is the byte
    count.  A buffer too small for the factor stops the copy-out (stats[15] = -1)
    and leaves the factor itself unchanged; the arming lasts one factorization."""
    from hicma_parsec_b200 import tlr
    nt = N // NB
    prob = tlr.Problem(kind=2, noise=0.1)
    A = tlr.TLRMatrix(ctx, N, NB, MAXRANK, BAND)
    B = tlr.TLRMatrix(ctx, N, NB, MAXRANK, BAND)
    try:
        assert A.generate(prob, TOL, MAXRANK) == 0
        B.copy_from(A)
        cap = (nt * BAND * NB * NB + nt * nt * NB * MAXRANK) * 8
        buf = torch.empty(cap // 8, dtype=torch.float64, pin_memory=True)
        A.store_stream(buf.data_ptr(), cap)
        assert A.potrf(TOL) == 0
        written = int(A.stats()[15])
        assert written > 0
        host = buf.numpy()
        p = 0
        for n in range(nt):
            for m in range(n, nt):
                t = A.tile(m, n)
                if m - n < BAND:
                    assert np.array_equal(host[p:p + NB * NB].reshape(NB, NB, order="F"), t), (m, n)
                    p += NB * NB
                else:
                    U, V = t
                    r = U.shape[1]
                    assert np.array_equal(host[p:p + NB * r].reshape(NB, r, order="F"), U), (m, n)
                    assert np.array_equal(host[p + NB * r:p + 2 * NB * r].reshape(NB, r, order="F"), V), (m, n)
                    p += 2 * NB * r
        assert p * 8 == written
        # too small: the copy-out stops, the factor does not change; no arming afterwards
        B.store_stream(buf.data_ptr(), 8 * NB * NB)
        assert B.potrf(TOL) == 0
        assert B.stats()[15] == -1
        assert abs(A.logdet() - B.logdet()) <= 1e-12 * abs(A.logdet())
    finally:
        A.close()
        B.close()
