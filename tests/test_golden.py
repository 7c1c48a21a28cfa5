"""Golden vectors made from the reference's own code: hicma_parsec/op_counts.h
compiled unchanged (oracle/Makefile, tests/golden/make_op_counts.py) and run
over a grid of sizes (config tile sizes and ranks, edge values, arguments that
wrap around 64 bits).  Both restatements, the CPU oracle's and the library's
(hicma_tlr_op_counts, which the factorization counters and the band
auto-tuning use), must give the same unsigned values, bit for bit."""
import json
import os

import pytest

from oracle import tlr_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "op_counts.json")


@pytest.fixture(scope="module")
def rows():
    with open(GOLDEN) as f:
        g = json.load(f)
    assert g["fields"] == ["op", "a", "b", "c", "d", "r"]
    assert len(g["rows"]) > 1000
    return g["rows"]


def test_oracle_matches_reference_op_counts(rows):
    bad = [r for r in rows if O.op_counts(r[0], r[1], r[2], r[3], r[4]) != r[5]]
    assert not bad, bad[:5]


def test_library_matches_reference_op_counts(rows):
    from hicma_parsec_b200 import tlr
    lib = tlr.load_library()
    bad = [r for r in rows if lib.hicma_tlr_op_counts(r[0].encode(), r[1], r[2], r[3], r[4]) != r[5]]
    assert not bad, bad[:5]


def test_fixture_covers_every_operation_and_wraparound(rows):
    assert {r[0] for r in rows} == set("qctmsor")
    assert any(r[0] == "q" and r[2] == 1 << 21 for r in rows)    # 2 n^3 wraps to 0


def test_dense_equivalent_flops_match_reference():
    """FLOPS_DPOTRF of hicma_parsec/flops.h (the driver's dense-equivalent
    GFLOP/s column) against the oracle's restatement, bit for bit."""
    with open(GOLDEN) as f:
        g = json.load(f)
    assert len(g["flops_dpotrf"]) >= 10
    for n, ref in g["flops_dpotrf"]:
        assert O.flops_dpotrf(n) == ref, n
