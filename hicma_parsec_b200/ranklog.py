"""Rank-map and R-LO record tooling for driver logs.

Reads the text that ``testing_dpotrf_tlr`` prints (and that the reference
driver prints in the same formats): the ``R-LO`` summary record
(hicma_parsec/testing_dpotrf.c:1028-1059), the rank-map blocks of
``tlr_rank_stat`` under PRINT_RANK (``init_rank_tile NT NT`` / ``rank_tile NT
NT``, testing_dpotrf.c:91-106) and the five maps of ``parsec_rank_print``
(Initial / Minimum / Maximum / Final / Difference Rank, rank_print.jdf:128-183).
Two logs of the same problem (two builds, two machines, this engine against
the reference) are compared map by map over the low-rank tiles.

    python -m hicma_parsec_b200.ranklog run_a.log run_b.log [--tol 2]
"""
from __future__ import annotations

import argparse
import re
import sys
from dataclasses import dataclass, field

import numpy as np

HISTORY_TITLES = ("Initial Rank", "Minimum Rank", "Maximum Rank", "Final Rank", "Difference Rank, max - min")

# R-LO fields in print order (testing_dpotrf.c:1029-1043); the RBF problems
# (-D 6, 7) add five fields before the git hash (:1044-1047).
RLO_FIELDS = (
    ("N", int), ("N_cols", int), ("NB", int), ("NB_cols", int), ("HNB", int), ("HNB_cols", int),
    ("nodes", int), ("P", int), ("Q", int), ("cores", int),
    ("kind", int), ("problem", str), ("tol", float), ("add_diag", float), ("fixedrk", int), ("wave_k", float),
    ("send_full_tile", int), ("band_size", int), ("lookahead", int), ("reserved", int), ("auto_band", int),
    ("maxrank", int), ("genmaxrank", int), ("compmaxrank", int),
    ("iavgrk_before", float), ("iminrk_before", int), ("imaxrk_before", int),
    ("iavgrk", float), ("iminrk", int), ("imaxrk", int),
    ("favgrk", float), ("fminrk", int), ("fmaxrk", int),
    ("memory_per_node", float), ("memory_per_node_max", float),
    ("time_critical_path", float), ("time_path_0", float), ("time_path_1", float), ("time_path_2", float),
    ("time_starsh", float), ("time_hicma", float), ("time_opt_band", float), ("time_regenerate", float),
    ("time_reserved", float),
    ("total_numop", float), ("total_band", float), ("total_offband", float), ("total_path", float),
    ("total_offpath", float), ("ratio_band", float), ("ratio_path", float), ("two_flow", int),
)
RBF_FIELDS = (("order", int), ("numobj", int), ("rbf_kernel", int), ("radius", float), ("density", float))


def _num(conv, tok: str):
    if conv is str:
        return tok
    if tok.lower() in ("nan", "-nan", "inf", "-inf"):
        return float(tok.replace("-nan", "nan"))
    return conv(float(tok)) if conv is int and ("." in tok or "e" in tok.lower()) else conv(tok)


def parse_rlo(line: str) -> dict:
    """Fields of one ``R-LO`` record; 'githash' and 'command' (the quoted argv)
    are added at the end."""
    if not line.startswith("R-LO "):
        raise ValueError("not an R-LO record")
    head, _, tail = line.partition('"')
    command = tail.rsplit('"', 1)[0].strip() if tail else ""
    toks = head.split()[1:]
    out = {}
    n = len(RLO_FIELDS)
    if len(toks) < n + 1:
        raise ValueError(f"R-LO record has {len(toks)} fields, expected at least {n + 1}")
    for (name, conv), tok in zip(RLO_FIELDS, toks):
        out[name] = _num(conv, tok)
    rest = toks[n:]
    if out["kind"] in (6, 7) and len(rest) >= len(RBF_FIELDS) + 1:
        for (name, conv), tok in zip(RBF_FIELDS, rest):
            out[name] = _num(conv, tok)
        rest = rest[len(RBF_FIELDS):]
    out["githash"] = rest[0] if rest else ""
    out["command"] = command
    return out


@dataclass
class RankLog:
    """What one log holds: R-LO records, the tlr_rank_stat maps in order of
    appearance (name, NT x NT array) and the rank-history maps by title."""
    records: list = field(default_factory=list)
    rank_tiles: list = field(default_factory=list)
    history: dict = field(default_factory=dict)

    def map(self, which: str) -> np.ndarray | None:
        """'initial' (first init_rank_tile), 'initial_band' (last
        init_rank_tile), 'final' (rank_tile), or a history title."""
        if which in self.history:
            return self.history[which]
        names = [n for n, _ in self.rank_tiles]
        if which == "initial" and "init_rank_tile" in names:
            return self.rank_tiles[names.index("init_rank_tile")][1]
        if which == "initial_band" and "init_rank_tile" in names:
            return [g for n, g in self.rank_tiles if n == "init_rank_tile"][-1]
        if which == "final" and "rank_tile" in names:
            return self.rank_tiles[names.index("rank_tile")][1]
        return None


_INT_ROW = re.compile(r"^\s*-?\d+(\s+-?\d+)*\s*$")


def parse_log(text: str) -> RankLog:
    out = RankLog()
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        ln = lines[i]
        m = re.match(r"^(init_rank_tile|rank_tile) (\d+) (\d+)\s*$", ln)
        if m:
            nt = int(m.group(2))
            rows = [[int(v) for v in lines[i + 1 + r].split()] for r in range(nt)]
            out.rank_tiles.append((m.group(1), np.array(rows, dtype=np.int64)))
            i += 1 + nt
            continue
        if ln.strip() in HISTORY_TITLES:
            title = ln.strip()
            rows = []
            j = i + 1
            while j < len(lines) and _INT_ROW.match(lines[j]):
                rows.append([int(v) for v in lines[j].split()])
                j += 1
            out.history[title] = np.array(rows, dtype=np.int64)
            i = j
            continue
        if ln.startswith("R-LO "):
            out.records.append(parse_rlo(ln))
        i += 1
    return out


def format_rank_tile(strid: str, G: np.ndarray, band_size: int) -> str:
    """The tlr_rank_stat block for an NT x NT map G[m, n] (-1 inside the band
    and above the diagonal), as the driver prints it."""
    nt = G.shape[0]
    rows = ["".join("%3d " % (G[i, j] if i - j >= band_size else -1) for j in range(nt)) for i in range(nt)]
    return f"{strid} {nt} {nt}\n" + "\n".join(rows) + "\n"


def format_rank_history(initial, minimum, maximum, final) -> str:
    """The five parsec_rank_print maps; tiles outside the low-rank part (-1 in
    `initial`) print 0."""
    low = np.asarray(initial) >= 0
    maps = [initial, minimum, maximum, final, np.asarray(maximum) - np.asarray(minimum)]
    out = []
    for title, M in zip(HISTORY_TITLES, maps):
        M = np.where(low, M, 0)
        out.append("\n" + title + "\n" + "".join("".join("%3d " % v for v in row) + "\n" for row in M) + "\n\n")
    return "".join(out)


@dataclass
class RankDiff:
    tiles: int
    differing: int              # |a - b| > tol
    max_abs: int
    mean_abs: float
    by_subdiagonal: dict        # m - n -> max |a - b|
    worst: list                 # (m, n, a, b), largest differences first


def diff_maps(a: np.ndarray, b: np.ndarray, tol: int = 0, band_size: int = 1, limit: int = 10) -> RankDiff:
    """Compare two NT x NT rank maps over the low-rank tiles (m - n >= band)."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        raise ValueError(f"maps differ in shape: {a.shape} vs {b.shape}")
    nt = a.shape[0]
    m, n = np.tril_indices(nt, -band_size)
    d = np.abs(a[m, n] - b[m, n])
    by = {}
    for s in np.unique(m - n):
        by[int(s)] = int(d[(m - n) == s].max())
    order = np.argsort(-d, kind="stable")[:limit]
    worst = [(int(m[i]), int(n[i]), int(a[m[i], n[i]]), int(b[m[i], n[i]])) for i in order if d[i] > 0]
    return RankDiff(tiles=int(d.size), differing=int(np.count_nonzero(d > tol)), max_abs=int(d.max()) if d.size else 0,
                    mean_abs=float(d.mean()) if d.size else 0.0, by_subdiagonal=by, worst=worst)


RECORD_KEYS = ("iminrk", "imaxrk", "iavgrk", "fminrk", "fmaxrk", "favgrk", "band_size", "total_numop", "total_path",
               "time_starsh", "time_hicma")


def compare_logs(a: RankLog, b: RankLog, tol: int = 0) -> dict:
    """Map-by-map differences plus the R-LO fields side by side."""
    out = {"maps": {}, "records": {}}
    band = a.records[0]["band_size"] if a.records else 1
    for which in ("initial", "initial_band", "final") + HISTORY_TITLES:
        ma, mb = a.map(which), b.map(which)
        if ma is None or mb is None:
            continue
        bs = 1 if which == "initial" else band
        out["maps"][which] = diff_maps(ma, mb, tol, bs)
    if a.records and b.records:
        ra, rb = a.records[0], b.records[0]
        for k in RECORD_KEYS:
            if k in ra and k in rb:
                out["records"][k] = (ra[k], rb[k])
        same = ("N", "NB", "kind", "tol", "maxrank")
        out["same_problem"] = all(ra.get(k) == rb.get(k) for k in same)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Compare the rank maps and R-LO records of two driver logs.")
    ap.add_argument("log_a")
    ap.add_argument("log_b")
    ap.add_argument("--tol", type=int, default=0, help="rank difference tolerated per tile")
    args = ap.parse_args(argv)
    with open(args.log_a) as f:
        a = parse_log(f.read())
    with open(args.log_b) as f:
        b = parse_log(f.read())
    res = compare_logs(a, b, args.tol)
    if "same_problem" in res and not res["same_problem"]:
        print("warning: the R-LO records describe different problems")
    for which, d in res["maps"].items():
        print(f"{which:28s} tiles {d.tiles:6d}  >tol {d.differing:6d}  max |d| {d.max_abs:4d}  "
              f"mean |d| {d.mean_abs:.3f}  worst {d.worst[:3]}")
    for k, (va, vb) in res["records"].items():
        print(f"{k:28s} {va!s:>14s} {vb!s:>14s}")
    bad = any(d.differing for d in res["maps"].values())
    return 1 if bad else 0


if __name__ == "__main__":
    sys.exit(main())
