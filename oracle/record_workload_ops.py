"""Record the op_counts total of a benchmark workload for `bench.py --impl reference`.

The reference arm times the oracle's task bodies on a bounded panel-0 sample and
scales the time by the workload's total op count (op_counts.h formulas summed
over every task of the factorization).  That total depends on the ranks the
factorization produces, so it is taken from a GPU run of the same workload:

    python bench.py --config c2 --no-e2e --no-cpu > run.json
    python oracle/record_workload_ops.py c2 run.json

writes {"c2": {"total_ops": ..., "source": ...}} into oracle/workload_ops.json.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "workload_ops.json")


def main():
    cfg, path = sys.argv[1], sys.argv[2]
    line = [l for l in open(path) if l.strip().startswith("{")][-1]
    rec = json.loads(line)
    data = json.load(open(FIXTURE)) if os.path.exists(FIXTURE) else {}
    data[cfg] = {"total_ops": float(rec["op_counts_flops"]),
                 "source": f"bench.py --config {cfg}: op_counts_flops of the GPU factorization",
                 "workload": rec["config"]["workload"]}
    with open(FIXTURE, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
