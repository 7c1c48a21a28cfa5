"""Host-side logic of the serving loop (no GPU): request sampling follows the
stated distribution, footprints, percentiles."""
import math

import numpy as np

from hicma_parsec_b200 import serving, tlr


def test_request_distribution():
    reqs = serving.sample_requests(400, seed=1, rate=5.0)
    assert all(r.n % r.nb == 0 for r in reqs)
    assert all(10000 - 2700 <= r.n <= 200000 + 2700 for r in reqs)
    assert {r.kind for r in reqs} == {tlr.KIND_SQEXP_2D, tlr.KIND_SQEXP_3D, tlr.KIND_EXP_3D}
    assert all(0.03 <= r.beta <= 0.3 and 0.5 <= r.sigma <= 2.0 and 1e-6 <= r.noise <= 1e-2 for r in reqs)
    assert {r.acc for r in reqs} == {1e-6, 1e-8, 1e-9}
    gaps = np.diff([0.0] + [r.arrival for r in reqs])
    assert abs(gaps.mean() - 0.2) < 0.05           # Poisson, rate 5/s
    logn = np.log([r.n for r in reqs])
    assert abs(np.median(logn) - 0.5 * (math.log(1e4) + math.log(2e5))) < 0.4


def test_footprint_and_summary():
    r = serving.MLERequest(rid=0, kind=2, n=20000, nb=1000, beta=0.1, sigma=1, noise=1e-4, acc=1e-8, seed=0)
    nt = 20
    assert serving.footprint_bytes(r, band_guess=1) == 8 * (nt * 1000 * 1000 + nt * (nt - 1) // 2 * 2 * 1000 * 200
                                                             + nt * 1000 * 1000)
    res = [serving.MLEResult(rid=i, n=1, latency=float(i + 1)) for i in range(100)]
    s = serving.summarize(res, makespan=50.0)
    assert s["solves_per_s"] == 2.0 and s["p50_s"] == 50.0 and s["p99_s"] == 99.0
