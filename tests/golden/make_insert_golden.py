"""Extract the reference's single-insert grid construction baselines into a compact fixture.

The reference pins graph construction with checked-in JSON baselines written by
diskann/src/graph/test/cases/grid_insert.rs: a lattice is inserted point by point into an
empty index (start point [size] * dim, max_degree 2 * dim, target degree max(2, 2 * dim - 2),
L_build 100, alpha 1.2), then searched with k = L = 10 for the all -1 and all `size` queries.
This script keeps the one-by-one cases (`insert_*_single/ibc_none.json`) and, per search, the
query, results, comparisons and hops.  Run it against a checkout of the reference:

    python tests/golden/make_insert_golden.py /path/to/reference
"""

import json
import os
import sys

CASES = "diskann/test/generated/graph/test/cases/grid_insert"


def main(ref_root: str) -> None:
    out = []
    root = os.path.join(ref_root, CASES)
    for case in sorted(os.listdir(root)):
        if not case.endswith("_single"):
            continue
        with open(os.path.join(root, case, "ibc_none.json")) as f:
            c = json.load(f)["payload"]
        out.append({
            "source": f"{CASES}/{case}/ibc_none.json",
            "grid_dims": c["grid_dims"],
            "grid_size": c["grid_size"],
            "num_inserted": c["num_inserted"],
            "searches": [{"query": s["query"], "results": s["results"],
                          "comparisons": s["comparisons"], "hops": s["hops"],
                          "num_results": s["num_results"]} for s in c["searches"]],
        })
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "grid_insert.json")
    with open(dst, "w") as f:
        json.dump(out, f)
    print(f"wrote {len(out)} single-insert cases to {dst}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_insert_golden.py <path to a checkout of the reference>")
    main(sys.argv[1])
