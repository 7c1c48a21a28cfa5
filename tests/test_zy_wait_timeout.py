"""Failure detection on the GPU without a fault: the tile POTRF task queue's
bounded dependency wait is made to run out (a counter that nothing sets), the
call returns HICMA_TLR_ERR_TIMEOUT, the other waiting CTAs leave on the abort
flag instead of running out their own (longer) limits, and the CUDA context
stays usable (a GEMM afterwards is exact to FP64 rounding)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def probe(lib, p0, p1, nblocks):
    ms = C.c_double(-1.0)
    rc = lib.hicma_tlr_k_wait_probe(p0, p1, nblocks, C.byref(ms), None)
    return rc, ms.value


def test_bounded_wait_reports_timeout_and_context_survives(ctx):
    from hicma_parsec_b200 import tlr
    lib = tlr.load_library()
    rc, ms1 = probe(lib, 1 << 18, 1 << 18, 1)
    assert rc == tlr.ERR_TIMEOUT
    assert "gave up" in tlr.last_error()
    assert 0.0 < ms1 < 5000.0
    # three more CTAs with 8x the limit: they leave when CTA 0 raises the abort flag
    rc, ms4 = probe(lib, 1 << 18, 1 << 21, 4)
    assert rc == tlr.ERR_TIMEOUT
    assert ms4 < 3.0 * ms1 + 5.0, (ms1, ms4)
    # arguments outside the bounds are refused before any launch
    assert probe(lib, 0, 1, 1)[0] == tlr.ERR_ARG
    assert probe(lib, 1, 1 << 27, 1)[0] == tlr.ERR_ARG
    # the context and the device still work
    rng = np.random.default_rng(0)
    A = rng.standard_normal((64, 48))
    B = rng.standard_normal((48, 40))
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    dC = torch.zeros((40, 64), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert lib.hicma_tlr_k_dgemm(0, 0, 64, 40, 48, 1.0, dA.data_ptr(), 64, dB.data_ptr(), 48, 0.0,
                                 dC.data_ptr(), 64, s) == 0
    assert np.allclose(dC.cpu().numpy().T, A @ B, rtol=1e-13, atol=1e-13)
