"""The allocation-free tile Cholesky, hicma_tlr_k_potrf_noalloc.

Some callers cannot allocate device memory (a host framework that owns all
device buffers, or a latency-critical loop that must not trigger the
synchronisation an allocation can cause).  This entry point serves them with
scratch held in a fixed array inside the library.  The test calls it through
the C ABI twice in a row (different sizes, so the second call runs on the
scratch left behind by the first) and compares each result with the existing
allocating entry point, hicma_tlr_k_potrf, on the same input, using the
tolerances of the POTRF parity test.  It sits in a file of its own that pytest
collects last, and it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from oracle import tlr_oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)).cuda()


def _host(t):
    return t.detach().cpu().numpy().T


def _spd(n, seed):
    pts = O.gen_points(n, 2, seed)
    return O.cov_block(O.Problem(kind=2, noise=1e-2), pts, 0, n, 0, n)


def test_noalloc_potrf_matches_allocating_entry(ctx):
    from hicma_parsec_b200 import tlr
    lib = tlr.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    for call, n in enumerate((2700, 1000)):
        A = _spd(n, 11 + call)
        # existing entry point (context workspace)
        dA1 = _dev(A)
        dL1 = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        info1 = torch.zeros(1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert lib.hicma_tlr_k_potrf(ctx.h, n, dA1.data_ptr(), n, dL1.data_ptr(), info1.data_ptr(), 0) == 0, \
            tlr.last_error()
        # allocation-free entry point on the caller's stream; L^-1 buffer starts non-zero on purpose
        dA2 = _dev(A)
        dL2 = torch.full((n, n), 7.0, dtype=torch.float64, device="cuda")
        info2 = torch.zeros(1, dtype=torch.int32, device="cuda")
        rc = lib.hicma_tlr_k_potrf_noalloc(n, dA2.data_ptr(), n, dL2.data_ptr(), info2.data_ptr(), 0, stream)
        assert rc == 0, tlr.last_error()
        torch.cuda.synchronize()
        assert int(info1.item()) == 0 and int(info2.item()) == 0
        L1, L2 = np.tril(_host(dA1)), np.tril(_host(dA2))
        Li1, Li2 = _host(dL1), _host(dL2)
        np.testing.assert_allclose(L2, L1, rtol=0, atol=1e-8 * np.max(np.abs(L1)))
        np.testing.assert_allclose(Li2, Li1, rtol=0, atol=1e-9 * np.max(np.abs(Li1)))
        assert np.allclose(np.triu(Li2, 1), 0.0)
        assert np.linalg.norm(L2 @ L2.T - A) / np.linalg.norm(A) < 1e-13
        assert np.linalg.norm(Li2 @ L2 - np.eye(n)) < 1e-9 * n


def test_noalloc_potrf_without_inverse_and_not_spd(ctx):
    """With no L^-1 buffer the scratch array holds each diagonal-block inverse
    that the panel product reads; a tile that is not positive definite reports
    the same info (info_offset + first failing column) as the allocating entry."""
    from hicma_parsec_b200 import tlr
    lib = tlr.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    n = 1500
    A = _spd(n, 5)
    dA1, dA2 = _dev(A), _dev(A)
    info1 = torch.zeros(1, dtype=torch.int32, device="cuda")
    info2 = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert lib.hicma_tlr_k_potrf(ctx.h, n, dA1.data_ptr(), n, None, info1.data_ptr(), 0) == 0, tlr.last_error()
    assert lib.hicma_tlr_k_potrf_noalloc(n, dA2.data_ptr(), n, None, info2.data_ptr(), 0, stream) == 0, \
        tlr.last_error()
    torch.cuda.synchronize()
    assert int(info1.item()) == 0 and int(info2.item()) == 0
    L1, L2 = np.tril(_host(dA1)), np.tril(_host(dA2))
    np.testing.assert_allclose(L2, L1, rtol=0, atol=1e-8 * np.max(np.abs(L1)))
    assert np.linalg.norm(L2 @ L2.T - A) / np.linalg.norm(A) < 1e-13
    # not positive definite from column 700 on (its diagonal entry made negative)
    B = A.copy()
    B[700, 700] = -1.0
    offset = 5 * 2700
    dB1, dB2 = _dev(B), _dev(B)
    info1.zero_()
    info2.zero_()
    torch.cuda.synchronize()
    assert lib.hicma_tlr_k_potrf(ctx.h, n, dB1.data_ptr(), n, None, info1.data_ptr(), offset) == 0, tlr.last_error()
    assert lib.hicma_tlr_k_potrf_noalloc(n, dB2.data_ptr(), n, None, info2.data_ptr(), offset, stream) == 0, \
        tlr.last_error()
    torch.cuda.synchronize()
    assert int(info1.item()) == offset + 701
    assert int(info2.item()) == int(info1.item())


def test_noalloc_potrf_rejects_oversize():
    from hicma_parsec_b200 import tlr
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    lib = tlr.load_library()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.hicma_tlr_k_potrf_noalloc(4097, buf.data_ptr(), 4097, None, info.data_ptr(), 0, None)
    assert rc == tlr.ERR_ARG
    assert "4096" in tlr.last_error()
