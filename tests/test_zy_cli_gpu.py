"""The command-line driver on the GPU, run the way the reference's two CTest
entries run its driver (hicma_parsec/CMakeLists.txt:59-62: ``testing_dpotrf_tlr
-N 2700 -t 270 -e 1e-8 -u 130 -D 2 -v --check``, as ``dpotrf-2flow`` and as
``dpotrf-3flow`` with ``-E 0 -Z 1``): pass/fail is the return code, which ORs
info != 0 and the two checks against the dense factorization
(testing_dpotrf.c:800-803,851-853,891-893).  The R-LO record and the
--print-rank maps are read back with the log parser."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ARGS = ["-N", "2700", "-t", "270", "-e", "1e-8", "-u", "130", "-D", "2", "-v", "--check"]


def run_cli(*extra):
    from hicma_parsec_b200 import build
    r = subprocess.run([build.CLI, *ARGS, *extra], capture_output=True, text=True, timeout=300)
    return r


@pytest.mark.parametrize("name,extra,two_flow", [("dpotrf-2flow", ["-W", "1"], 1),
                                                 ("dpotrf-3flow", ["-E", "0", "-Z", "1"], 0)])
def test_reference_ctest_cases(name, extra, two_flow):
    from hicma_parsec_b200 import ranklog
    r = run_cli(*extra)
    assert r.returncode == 0, (name, r.stdout[-3000:], r.stderr[-2000:])
    assert "Factorization is CORRECT" in r.stdout and "SAME matrices" in r.stdout
    log = ranklog.parse_log(r.stdout)
    assert len(log.records) == 1
    rec = log.records[0]
    assert (rec["N"], rec["NB"], rec["maxrank"], rec["kind"], rec["problem"]) == (2700, 270, 130, 2, "st-2d-sqexp")
    assert rec["two_flow"] == two_flow
    assert rec["total_numop"] > 0 and 0 < rec["total_path"] < rec["total_numop"]
    assert rec["total_band"] + rec["total_offband"] == pytest.approx(rec["total_numop"], rel=1e-5)   # %le: 7 digits
    assert 0 <= rec["fminrk"] <= rec["favgrk"] <= rec["fmaxrk"] <= 130


def test_print_rank_maps():
    from hicma_parsec_b200 import ranklog
    r = run_cli("-E", "0", "--print-rank")
    assert r.returncode == 0, r.stderr[-2000:]
    log = ranklog.parse_log(r.stdout)
    nt = 10
    init, final = log.map("initial"), log.map("final")
    assert init.shape == (nt, nt) and final.shape == (nt, nt)
    low = np.tril(np.ones((nt, nt), bool), -1)
    assert np.all(init[~low] == -1) and np.all(final[~low] == -1)
    for title in ranklog.HISTORY_TITLES:
        assert log.map(title).shape == (nt, nt)
    assert np.array_equal(log.map("Final Rank")[low], final[low])
    assert np.array_equal(log.map("Initial Rank")[low], init[low])
    mn, mx = log.map("Minimum Rank"), log.map("Maximum Rank")
    assert np.all(mn[low] <= final[low]) and np.all(final[low] <= mx[low])
    assert np.array_equal(log.map("Difference Rank, max - min"), mx - mn)
