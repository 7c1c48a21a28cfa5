"""Regenerates tests/golden/op_counts.json from the reference's own
hicma_parsec/op_counts.h and hicma_parsec/flops.h: builds
oracle/_ref/op_counts_golden with oracle/Makefile (the reference tree must be
present) and stores its output.

    python tests/golden/make_op_counts.py <reference root>

The reference root may also come from the HICMA_REFERENCE_ROOT environment
variable; there is no default.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main(ref: str) -> None:
    oracle = os.path.join(ROOT, "oracle")
    subprocess.run(["make", "-s", "-C", oracle, f"REF={ref}"], check=True)
    out = subprocess.run([os.path.join(oracle, "_ref", "op_counts_golden")], check=True, capture_output=True,
                         text=True).stdout
    recs = [json.loads(line) for line in out.splitlines() if line.strip()]
    rows = [r for r in recs if "op" in r]
    flops = [[r["flops_dpotrf"], r["r"]] for r in recs if "flops_dpotrf" in r]
    with open(os.path.join(HERE, "op_counts.json"), "w") as f:
        json.dump({"source": "hicma_parsec/op_counts.h and flops.h (reference tree, compiled unchanged)",
                   "fields": ["op", "a", "b", "c", "d", "r"],
                   "rows": [[r["op"], r["a"], r["b"], r["c"], r["d"], r["r"]] for r in rows],
                   "flops_dpotrf": flops}, f, separators=(",", ":"))
    print(f"{len(rows)} op_counts rows, {len(flops)} FLOPS_DPOTRF sizes")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HICMA_REFERENCE_ROOT", "")
    if not ref:
        sys.exit("usage: make_op_counts.py <reference root> (or set HICMA_REFERENCE_ROOT)")
    main(ref)
