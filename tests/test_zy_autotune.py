"""Autotuner on the GPU: the measured choices come from the candidate sets,
the medians are recorded, and a factorization with the tuned table (and with
the extreme settings: every rank-wide output on 128 x 32 tiles, the tile POTRF
on one CTA) gives the residual and log-determinant of the default table
(bars: residual <= 10 e against the dense oracle; log det within 1e-10
relative of the default run, whose GEMM tiling may round differently)."""
import math

import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N, NB, TOL, MAXRANK = 2700, 270, 1e-8, 130


def factor(ctx):
    from hicma_parsec_b200 import tlr
    A = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 1)
    try:
        assert A.generate(tlr.Problem(kind=2, noise=0.1), TOL, MAXRANK) == 0
        assert A.potrf(TOL) == 0
        return A.logdet(), A.uncompress()
    finally:
        A.close()


def test_autotune_choices_and_results():
    from hicma_parsec_b200 import tlr
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    ctx = tlr.Context(0, 1 << 30)
    try:
        assert ctx.tuning() == (32, 0)
        ld0, _ = factor(ctx)
        res = ctx.autotune(NB, MAXRANK, reps=3)
        assert res["gemm_narrow_n"] in (32, 48, 64, 96, 128)
        assert res["potrf_grid"] in (max(1, nsm // 2), nsm, 2 * nsm)
        assert all(math.isfinite(v) and v > 0 for v in res["potrf_ms"])
        for w, d in res["gemm_ms"].items():
            assert math.isfinite(d["128x32"]) and math.isfinite(d["64x64"])   # all widths <= maxrank
        assert ctx.tuning() == (res["gemm_narrow_n"], res["potrf_grid"])
        Aex = O.dense_matrix(O.Problem(kind=2, noise=0.1), O.gen_points(N, 2))
        for table in ((res["gemm_narrow_n"], res["potrf_grid"]), (4096, 1)):
            ctx.set_tuning(*table)
            ld, L = factor(ctx)
            assert abs(ld - ld0) <= 1e-10 * abs(ld0), table
            assert O.check_dpotrf2(L, Aex) <= 10 * TOL, table
        with pytest.raises(tlr.TLRError):
            ctx.set_tuning(-1, 0)
        with pytest.raises(tlr.TLRError):
            ctx.set_tuning(32, 17 * nsm)
    finally:
        ctx.close()
