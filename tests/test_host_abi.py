"""The C-ABI library loads on a machine without a GPU, exports every entry
point declared in include/hicma_tlr.h, and its host-only functions (point
placement, band auto-tuning, rank statistics) agree with the oracle bit for
bit.  No device work is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import tlr_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hicma_tlr.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hicma_tlr_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from hicma_parsec_b200 import tlr
    return tlr.load_library()


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_library_is_sm100a(lib):
    from hicma_parsec_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)
    assert os.path.exists(build.LIB)


@pytest.mark.parametrize("kind,n", [(2, 2700), (2, 10000), (3, 1000), (4, 4913), (3, 999), (1, 2700), (5, 1000)])
def test_points_bit_identical(kind, n):
    from hicma_parsec_b200 import tlr
    P = tlr.points(tlr.Problem(kind=kind, seed=0), n)
    Q = O.gen_points(n, O.KIND_NDIM[kind], 0)
    np.testing.assert_array_equal(P, Q.T)


def test_band_autotune_matches_oracle():
    from hicma_parsec_b200 import tlr
    rng = np.random.default_rng(11)
    for _ in range(100):
        nt, nb = int(rng.integers(3, 25)), int(rng.integers(50, 3000))
        G = rng.integers(0, nb // 2, size=nt * nt).astype(np.int32)
        assert tlr.parsec_band_size_auto_tuning(G, nt, nb) == O.band_autotune(G, nt, nb)


def test_rank_stat_matches_oracle():
    from hicma_parsec_b200 import tlr
    rng = np.random.default_rng(5)
    for band in (1, 2, 4):
        G = rng.integers(0, 100, size=144).astype(np.int32)
        mn, mx, av = tlr.HICMA_get_stat2(G, 12, band)
        omn, omx, oav = O.rank_stat(G, 12, band)
        assert (mn, mx) == (omn, omx) and av == pytest.approx(oav, rel=1e-15)


def test_argument_errors_without_gpu(lib):
    from hicma_parsec_b200 import tlr
    with pytest.raises(tlr.TLRError):
        tlr.points(tlr.Problem(kind=9), 10)
    G = np.zeros(4, np.int32)
    assert lib.hicma_tlr_band_autotune(None, 2, 10, 0) == tlr.ERR_ARG
    # serve_loglik validates its arguments before any device work
    y = np.zeros(10)
    d = ctypes.c_double()
    prob = tlr.Problem().c()
    assert lib.hicma_tlr_serve_loglik(None, ctypes.byref(prob), 10, 5, 1e-8, 0, 1,
                                      y.ctypes.data_as(ctypes.c_void_p), ctypes.byref(d), ctypes.byref(d),
                                      None, None) == tlr.ERR_ARG
    # the autotuner and its table need a context
    t = np.zeros(2, np.int32)
    assert lib.hicma_tlr_autotune(None, 270, 130, 3, t.ctypes.data_as(ctypes.c_void_p), None) == tlr.ERR_ARG
    assert lib.hicma_tlr_tuning_get(None, t.ctypes.data_as(ctypes.c_void_p)) == tlr.ERR_ARG
    assert lib.hicma_tlr_tuning_set(None, t.ctypes.data_as(ctypes.c_void_p)) == tlr.ERR_ARG
    # the reference-signature factorization (with the Rank record) refuses a
    # null context before any device work and leaves Rank untouched
    rank = np.full(16, 7, np.int32)
    assert lib.hicma_tlr_dpotrf_L_rank(None, tlr.LOWER, None, None, rank.ctypes.data_as(ctypes.c_void_p), 1e-8, 0,
                                       130, None, 1, 0, 130, 0, None, None, None, None, 0) == tlr.ERR_ARG
    assert np.all(rank == 7)
    # the wait probe refuses out-of-range limits before touching the device
    assert lib.hicma_tlr_k_wait_probe(0, 1, 1, None, None) == tlr.ERR_ARG
    assert lib.hicma_tlr_k_wait_probe(1, 1, 65, None, None) == tlr.ERR_ARG


@pytest.mark.parametrize("kind,radius", [(0, 0.0), (6, 0.5), (7, 0.0), (8, 0.5)])
def test_kinds_without_points_are_argument_errors(lib, kind, radius):
    """randtlr (-D 0) has no points (its bases are built on the device by the
    generator); md-3d-virus (-D 6) takes its points from a mesh file
    (hicma_tlr_points_mesh); md-3d-cube (-D 7) needs a positive RBF radius;
    kind 8 does not exist.  The C library answers hicma_tlr_points with an
    argument error for each."""
    import ctypes as C
    from hicma_parsec_b200 import tlr
    buf = np.zeros(30)
    prob = tlr.CProblem(kind, 0.1, 0.5, 0.1, 1.0, 0, 50.0, 0.0, 0, radius, 1, 1, -1.0)
    assert lib.hicma_tlr_points(C.byref(prob), 10, buf.ctypes.data_as(C.c_void_p)) == tlr.ERR_ARG


def test_problem_struct_layout_matches_header(tmp_path):
    """The ctypes mirror of hicma_tlr_problem has the C header's size and field
    offsets (checked with the host C compiler)."""
    import shutil
    import subprocess
    from hicma_parsec_b200 import tlr
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    fields = [name for name, _ in tlr.CProblem._fields_]
    src = tmp_path / "layout.c"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    body = "".join(f'    printf("{f} %zu\\n", offsetof(hicma_tlr_problem, {f}));\n' for f in fields)
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "hicma_tlr.h"\nint main(void) {\n'
                   '    printf("size %zu\\n", sizeof(hicma_tlr_problem));\n' + body + "    return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", inc, str(src), "-o", str(exe)], check=True, capture_output=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                        text=True).stdout.splitlines())
    assert int(out["size"]) == ctypes.sizeof(tlr.CProblem)
    for f in fields:
        assert int(out[f]) == getattr(tlr.CProblem, f).offset, f


def test_rank_stat_and_autotune_edges():
    """Empty low-rank parts (band >= NT) and the smallest grids, against the
    oracle: the reference's INT_MAX / 0 / NaN statistics and its band loop,
    which returns NT when no band beats the TLR cost."""
    from hicma_parsec_b200 import tlr
    G = np.full(9, 5, dtype=np.int32)
    mn, mx, av = tlr.HICMA_get_stat2(G, 3, 3)
    omn, omx, oav = O.rank_stat(G, 3, 3)
    assert (mn, mx) == (omn, omx) == (2**31 - 1, 0) and np.isnan(av) and np.isnan(oav)
    for nt in (1, 2, 3):
        for nb in (2, 270, 2700):
            for r in (0, 1, nb // 2):
                G = np.full(nt * nt, r, dtype=np.int32)
                assert tlr.parsec_band_size_auto_tuning(G, nt, nb) == O.band_autotune(G, nt, nb), (nt, nb, r)
