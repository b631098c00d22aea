"""Generate tests/golden/kats.json from the reference's own literal tests.

Run where the kiddo sources are available:
    python tests/golden/make_golden.py /path/to/kiddo
The reference is Rust and cannot be built here, so its known-answer tests are
read as text: the literal inputs and asserted outputs are extracted (or, for
the short ones, transcribed with the file:line they come from) into a JSON
fixture that the oracle and the GPU engine are both checked against.
"""
from __future__ import annotations

import json
import os
import re
import sys


def issue_258_points(src: str):
    """src/kd_tree/query/within.rs: fn issue_258_test_data()."""
    body = src[src.index("fn issue_258_test_data()"):]
    body = body[:body.index("]\n    }")]
    pairs = re.findall(r"\[\s*([0-9.eE+-]+)\s*,\s*([0-9.eE+-]+)\s*\]", body)
    return [[float(a), float(b)] for a, b in pairs]


def donnelly_cases(src: str):
    """src/stem_strategy/donnelly/core.rs tests: the rstest cases of
    donnelly_core_get_child_idx_produces_correct_values (path -> stem index) and
    donnelly_core_get_both_child_idxs_produces_correct_values (path -> both
    children), all for DonnellyCore::<3>."""
    paths, children = [], []
    for block in src.split("#[rstest]")[1:]:
        m = re.search(r"fn (\w+)\(", block)
        if not m:
            continue
        name = m.group(1)
        head = block[:m.start()]
        if name == "donnelly_core_get_child_idx_produces_correct_values":
            for v, e in re.findall(r"#\[case\(vec!\[([a-z, ]*)\],\s*(\d+)\)\]", head):
                path = [x.strip() == "true" for x in v.split(",") if x.strip()]
                paths.append({"bh": 3, "path": path, "stem_idx": int(e)})
        elif name == "donnelly_core_get_both_child_idxs_produces_correct_values":
            for v, l, r in re.findall(
                    r"#\[case\(vec!\[([a-z, ]*)\],\s*\((\d+),\s*(\d+)\)\)\]", head):
                path = [x.strip() == "true" for x in v.split(",") if x.strip()]
                children.append({"bh": 3, "path": path, "children": [int(l), int(r)]})
    return paths, children


def main(ref_root: str):
    within_rs = open(os.path.join(ref_root, "src/kd_tree/query/within.rs")).read()
    p258 = issue_258_points(within_rs)
    assert len(p258) >= 20, len(p258)
    q = p258[4]
    r2 = 36.0
    expected_258 = []
    for i, p in enumerate(p258):
        d = (q[0] - p[0]) ** 2 + (q[1] - p[1]) ** 2
        if d <= r2:
            expected_258.append(i)

    kats = [
        {   # src/lib.rs:120-151 and README.md:110-135
            "name": "lib_rs_readme_diagonal", "dtype": "f64",
            "points": [[0, 0], [1, 1], [2, 2], [3, 3]], "items": None,
            "checks": [
                {"family": "nearest_one", "query": [0, 0], "expect_items": [0],
                 "expect_dists": [0.0]},
                {"family": "nearest_n", "k": 3, "query": [0, 0], "expect_items": [0, 1, 2],
                 "expect_dists": [0.0, 2.0, 8.0]},
            ]},
        {   # src/kd_tree/query/within.rs:115-141
            "name": "within_exclusive_boundaries", "dtype": "f64",
            "points": [[0.0, 0.0], [1.0, 0.0], [2.0, 0.0], [0.5, 0.0]], "items": None,
            "checks": [
                {"family": "within", "radius": 1.0, "query": [0, 0], "expect_items": [0, 3, 1]},
                {"family": "within", "radius": 1.0, "exclusive": True, "query": [0, 0],
                 "expect_items": [0, 3]},
            ]},
        {   # src/kd_tree/query/builder.rs:2346-2373 (create_scratch doc example)
            "name": "create_scratch_first_items", "dtype": "f64",
            "points": [[0.0, 0.0], [1.0, 1.0], [0.2, 0.1]], "items": [10, 11, 12],
            "checks": [
                {"family": "nearest_n", "k": 2, "query": q_, "expect_first_item": it}
                for q_, it in (([0.1, 0.1], 12), ([0.9, 0.9], 11), ([0.25, 0.15], 12))
            ]},
        {   # README.md:150-174 (periodic boundary example)
            "name": "readme_periodic", "dtype": "f64",
            "points": [[0.05, 0.50], [0.95, 0.50], [0.40, 0.40]], "items": None,
            "box": [1.0, 1.0],
            "checks": [
                {"family": "periodic_nearest_one", "query": [0.99, 0.50], "expect_items": [1]},
                {"family": "periodic_nearest_n", "k": 2, "radius": 0.10, "query": [0.99, 0.50],
                 "expect_len": 2},
            ]},
        {   # src/kd_tree/mod.rs:1129-1151
            "name": "new_from_entries_preserves_explicit_items", "dtype": "f32",
            "points": [[0.0, 0.0], [5.0, 5.0], [10.0, 10.0]], "items": [42, 7, 99],
            "checks": [
                {"family": "nearest_one", "query": [5.1, 4.9], "expect_items": [7]},
            ]},
        {   # src/kd_tree/query/within.rs:333-389 (issue 258 regression)
            "name": "issue_258_within", "dtype": "f64", "points": p258, "items": None,
            "checks": [
                {"family": "within", "radius": r2, "query": q, "expect_item_set": expected_258,
                 "expect_dist_is_manual_sq": True},
            ]},
    ]
    # src/kd_tree/query/within.rs:89,143-183 and nearest_n.rs:83-: tile-boundary
    # cases, points generated by the reference's own formula.
    for n in (1, 2, 4, 8, 32, 33, 47):
        pts = [[((i * 5) % 97) / 97.0, ((i * 13 + 1) % 97) / 97.0, ((i * 23 + 2) % 97) / 97.0]
               for i in range(n)]
        kats.append({
            "name": f"tile_boundary_{n}", "dtype": "f32", "points": pts, "items": None,
            "checks": [{"family": "within_brute", "metric": "manhattan", "radius": 0.35,
                        "query": [0.31, 0.47, 0.59]}]})
    core_rs = open(os.path.join(ref_root, "src/stem_strategy/donnelly/core.rs")).read()
    dpaths, dchildren = donnelly_cases(core_rs)
    assert len(dpaths) >= 40 and len(dchildren) >= 40, (len(dpaths), len(dchildren))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kats.json")
    with open(out, "w") as f:
        json.dump({"source": "kiddo v6.0.0-alpha.3 literal tests", "kats": kats,
                   "donnelly_paths": dpaths, "donnelly_children": dchildren}, f, indent=1)
    print(out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path to the kiddo source tree>")
    main(sys.argv[1])
