"""Extract the reference's grid-search and flat-kNN regression baselines into compact fixtures.

The reference pins its greedy beam search with checked-in JSON baselines produced by
``diskann/src/graph/test/cases/grid_search.rs:86-218`` (exact result ids and distances,
comparison and hop counts for Knn(k=10, L=10, beam 1/2/4) on 1-D, 3-D and 4-D lattices) and
its brute-force search with ``diskann/src/flat/test/cases/flat_knn_search.rs``.

This script reads those files from a checkout of the reference and keeps only the fields the
tests compare.  Run it from the repository root:

    python tests/golden/make_golden.py /path/to/reference

It writes ``tests/golden/grid_search.json``, ``tests/golden/flat_knn_search.json``,
``tests/golden/range_search.json`` (range_search.rs's baselines with the Range parameters of
each case) and ``tests/golden/paged_search.json`` (paged_search.rs's pages).
"""

import json
import os
import sys

GRID_DIR = "diskann/test/generated/graph/test/cases/grid_search"
RANGE_DIR = "diskann/test/generated/graph/test/cases/range_search"
# Range parameters of each case (diskann/src/graph/test/cases/range_search.rs): 3-D grid of
# size 5, default query, beam width 1; (max_returned or None, initial_slack, range_slack).
RANGE_CASES = {
    "basic_range_search.json": (None, 1.0, 1.0),
    "inner_radius_filtering.json": (None, 1.0, 1.0),
    "two_round_search.json": (None, 1.0, 1.0),
    "max_results_respected_means_no_second_round.json": (4, 1.0, 1.0),
    "max_results_respected_and_second_round_triggered.json": (5, 1.0, 1.0),
}
PAGED_DIR = "diskann/test/generated/graph/test/cases/paged_search"
PAGED_FILES = ["basic_paged_search.json", "single_page.json", "small_page_size.json"]
FLAT_DIR = "diskann/test/generated/flat/test/cases/flat_knn_search"
GRID_FILES = ["search_1_100.json", "search_3_5.json", "search_4_4.json"]
FLAT_FILES = ["search_1_100.json", "search_2_5.json", "search_3_4.json"]


def main(ref_root: str) -> None:
    out_dir = os.path.dirname(os.path.abspath(__file__))

    grid = []
    for name in GRID_FILES:
        with open(os.path.join(ref_root, GRID_DIR, name)) as f:
            doc = json.load(f)
        for case in doc["payload"]:
            grid.append(
                {
                    "source": f"{GRID_DIR}/{name}",
                    "grid_dims": case["grid_dims"],
                    "grid_size": case["grid_size"],
                    "beam_width": case["beam_width"],
                    "k": 10,
                    "l": 10,
                    "query": case["query"],
                    "results": case["results"],
                    "comparisons": case["comparisons"],
                    "hops": case["hops"],
                    "num_results": case["num_results"],
                }
            )
    with open(os.path.join(out_dir, "grid_search.json"), "w") as f:
        json.dump(grid, f, indent=1)

    flat = []
    for name in FLAT_FILES:
        with open(os.path.join(ref_root, FLAT_DIR, name)) as f:
            doc = json.load(f)
        for case in doc["payload"]:
            flat.append(
                {
                    "source": f"{FLAT_DIR}/{name}",
                    "grid_dims": case["grid_dims"],
                    "grid_size": case["grid_size"],
                    "k": case["k"],
                    "query": case["query"],
                    "ground_truth": case["ground_truth"],
                    "result_count": case["result_count"],
                }
            )
    with open(os.path.join(out_dir, "flat_knn_search.json"), "w") as f:
        json.dump(flat, f, indent=1)

    rng = []
    for name, (max_returned, initial_slack, range_slack) in RANGE_CASES.items():
        with open(os.path.join(ref_root, RANGE_DIR, name)) as f:
            c = json.load(f)["payload"]
        rng.append(
            {
                "source": f"{RANGE_DIR}/{name}",
                "grid_dims": 3,
                "grid_size": c["grid_size"],
                "query": c["query"],
                "radius": c["radius"],
                "inner_radius": c["inner_radius"],
                "starting_l": c["starting_l"],
                "max_returned": max_returned,
                "initial_slack": initial_slack,
                "range_slack": range_slack,
                "results": c["results"],
                "comparisons": c["comparisons"],
                "hops": c["hops"],
                "result_count": c["result_count"],
                "second_round": c["range_search_second_round"],
            }
        )
    with open(os.path.join(out_dir, "range_search.json"), "w") as f:
        json.dump(rng, f, indent=1)
    paged = []
    for name in PAGED_FILES:
        with open(os.path.join(ref_root, PAGED_DIR, name)) as f:
            c = json.load(f)["payload"]
        paged.append(
            {
                "source": f"{PAGED_DIR}/{name}",
                "grid_dims": c["dims"],
                "grid_size": c["grid_size"],
                "query": c["query"],
                "search_l": c["search_l"],
                "page_size": c["page_size"],
                "pages": c["pages"],
                "total_results": c["total_results"],
            }
        )
    with open(os.path.join(out_dir, "paged_search.json"), "w") as f:
        json.dump(paged, f)
    print(f"wrote {len(grid)} grid, {len(flat)} flat, {len(rng)} range and {len(paged)} paged "
          f"cases to {out_dir}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to a checkout of the reference>")
    main(sys.argv[1])
