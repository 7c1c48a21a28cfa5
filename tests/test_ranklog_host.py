"""Rank-map / R-LO log tooling (CPU): the record parser against the field
order of hicma_parsec/testing_dpotrf.c:1028-1059, the rank-map blocks of
testing_dpotrf.c:91-106 and rank_print.jdf:128-183 (round trip through the
formatters), and map differences, on maps from the oracle's factorization."""
import numpy as np
import pytest

from hicma_parsec_b200 import ranklog
from oracle import tlr_oracle as O

RLO_FMT = ("R-LO %d %d %d %d   %d %d   %d %d %d %d   %d %s %.1e %g %d %g   %d %d %d %d %d %d %d %d   "
           "%g %d %d   %g %d %d   %g %d %d   %f %f   %f %f %f %f    %f %f %f %f %f    "
           "%e %e %e %e %e %f %f %d  ")


def rlo_line(kind=2, extra=""):
    vals = (2700, 2700, 270, 270, 300, 300, 1, 1, 1, 1, kind, "st-2d-sqexp", 1e-8, 2700.0, 0, 50.0,
            0, 1, 1, 0, 1, 130, 130, 130, 18.2, 3, 44, 18.2, 3, 44, 21.5, 2, 57,
            0.5, 1.2, 0.25, 0.1, 0.1, 0.05, 1.5, 2.18, 0.01, 0.0, 0.0,
            7.9e12, 1.0e12, 6.9e12, 4.0e11, 7.5e12, 0.145, 0.053, 1)
    return RLO_FMT % vals + extra + 'GITHASH:N/A    "testing_dpotrf_tlr -N 2700 -t 270 "'


def test_rlo_record_fields():
    r = ranklog.parse_rlo(rlo_line())
    assert (r["N"], r["NB"], r["kind"], r["problem"]) == (2700, 270, 2, "st-2d-sqexp")
    assert r["tol"] == 1e-8 and r["maxrank"] == 130 and r["band_size"] == 1
    assert (r["fminrk"], r["fmaxrk"]) == (2, 57) and r["favgrk"] == pytest.approx(21.5)
    assert r["total_numop"] == pytest.approx(7.9e12) and r["total_path"] == pytest.approx(4.0e11)
    assert r["two_flow"] == 1 and r["githash"] == "GITHASH:N/A"
    assert r["command"] == "testing_dpotrf_tlr -N 2700 -t 270"


def test_rlo_record_with_rbf_fields():
    r = ranklog.parse_rlo(rlo_line(kind=6, extra="%d %d %d  %g %g " % (1, 3, 2, 0.5, 0.75)))
    assert (r["order"], r["numobj"], r["rbf_kernel"]) == (1, 3, 2)
    assert r["radius"] == 0.5 and r["density"] == 0.75 and r["githash"] == "GITHASH:N/A"
    with pytest.raises(ValueError):
        ranklog.parse_rlo("R-LO 1 2 3")


@pytest.fixture(scope="module")
def oracle_run():
    n, nb = 1080, 108
    prob = O.Problem(kind=2, beta=0.02, noise=1e-2)
    T, info = O.generate(prob, n, nb, 1e-8, 53, 1)
    assert info == 0
    G0 = T.rank_array().reshape(n // nb, n // nb).T.copy()       # [m, n]
    st = O.tlr_potrf(T, 1e-8)
    assert st.info == 0
    G1 = T.rank_array().reshape(n // nb, n // nb).T.copy()
    return G0, G1, st


def test_oracle_rank_history_invariants(oracle_run):
    G0, G1, st = oracle_run
    low = st.rank_init >= 0
    assert np.array_equal(st.rank_init[low], G0[low])
    assert np.all(st.rank_min[low] <= st.rank_init[low]) and np.all(st.rank_init[low] <= st.rank_max[low])
    assert np.all(st.rank_min[low] <= G1[low]) and np.all(G1[low] <= st.rank_max[low])
    assert np.all(st.rank_init[0, :] == -1)                        # no low-rank tiles in row 0
    assert np.any(st.rank_max[low] > st.rank_min[low])             # some ranks moved


def test_rank_maps_round_trip(oracle_run):
    G0, G1, st = oracle_run
    text = (ranklog.format_rank_tile("init_rank_tile", G0, 1) + "noise line\n" +
            ranklog.format_rank_history(st.rank_init, st.rank_min, st.rank_max, G1) +
            ranklog.format_rank_tile("rank_tile", G1, 1) + rlo_line() + "\n")
    log = ranklog.parse_log(text)
    nt = G0.shape[0]
    low = np.tril(np.ones((nt, nt), bool), -1)
    assert np.array_equal(log.map("initial")[low], G0[low])
    assert np.all(log.map("initial")[~low] == -1)
    assert np.array_equal(log.map("final")[low], G1[low])
    assert np.array_equal(log.map("Minimum Rank")[low], st.rank_min[low])
    assert np.all(log.map("Maximum Rank")[~low] == 0)
    assert np.array_equal(log.map("Difference Rank, max - min"), np.where(low, st.rank_max - st.rank_min, 0))
    assert len(log.records) == 1 and log.records[0]["N"] == 2700


def test_map_differences(oracle_run):
    G0, G1, _ = oracle_run
    d = ranklog.diff_maps(G1, G1.copy())
    assert d.differing == 0 and d.max_abs == 0 and not d.worst
    H = G1.copy()
    H[7, 2] += 3
    H[9, 8] -= 1
    d = ranklog.diff_maps(G1, H, tol=2)
    assert d.differing == 1 and d.max_abs == 3
    assert d.worst[0] == (7, 2, int(G1[7, 2]), int(G1[7, 2]) + 3)
    assert d.by_subdiagonal[5] == 3 and d.by_subdiagonal[1] == 1
    with pytest.raises(ValueError):
        ranklog.diff_maps(G1, G1[:3, :3])


def test_compare_logs_command(tmp_path, oracle_run):
    G0, G1, st = oracle_run
    a = ranklog.format_rank_tile("rank_tile", G1, 1) + rlo_line() + "\n"
    H = G1.copy()
    H[5, 0] += 4
    b = ranklog.format_rank_tile("rank_tile", H, 1) + rlo_line() + "\n"
    pa, pb = tmp_path / "a.log", tmp_path / "b.log"
    pa.write_text(a)
    pb.write_text(b)
    assert ranklog.main([str(pa), str(pa)]) == 0
    assert ranklog.main([str(pa), str(pb), "--tol", "4"]) == 0
    assert ranklog.main([str(pa), str(pb), "--tol", "3"]) == 1
    res = ranklog.compare_logs(ranklog.parse_log(a), ranklog.parse_log(b))
    assert res["same_problem"] and res["maps"]["final"].max_abs == 4


from hypothesis import given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402


@settings(max_examples=30, deadline=None)
@given(nt=st.integers(1, 14), band=st.integers(1, 4), seed=st.integers(0, 10**6))
def test_rank_map_blocks_round_trip(nt, band, seed):
    """Any rank map printed in the driver's formats parses back to itself."""
    rng = np.random.default_rng(seed)
    G = np.where(np.tril(np.ones((nt, nt), bool), -band), rng.integers(0, 999, (nt, nt)), -1)
    mn = np.where(G >= 0, np.maximum(G - rng.integers(0, 5, (nt, nt)), 0), -1)
    mx = np.where(G >= 0, G + rng.integers(0, 5, (nt, nt)), -1)
    text = (ranklog.format_rank_tile("init_rank_tile", G, band) + ranklog.format_rank_history(G, mn, mx, G) +
            ranklog.format_rank_tile("rank_tile", G, band))
    log = ranklog.parse_log(text)
    low = G >= 0
    assert np.array_equal(log.map("initial"), np.where(low, G, -1))
    assert np.array_equal(log.map("final"), np.where(low, G, -1))
    assert np.array_equal(log.map("Maximum Rank"), np.where(low, mx, 0))
    assert np.array_equal(log.map("Difference Rank, max - min"), np.where(low, mx - mn, 0))
    d = ranklog.diff_maps(log.map("final"), G, 0, band)
    assert d.differing == 0
