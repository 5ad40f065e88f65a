"""Writes tests/golden/known_answers.json: known-answer cases of the
reference's own tests for this path, transcribed with their inputs and the
values those tests assert (file:line of each source is kept in the case).

Scalar-aggregate cases of the reference are restated as GROUP BY over a
constant key (one group), which has the same per-group semantics.
Run: python tests/golden/make_golden.py
"""

from __future__ import annotations

import json
import math
from pathlib import Path

OUT = Path(__file__).resolve().parent / "known_answers.json"
NaN = "NaN"


def c(dtype, values, valid=None, scale=0):
    d = {"dtype": dtype, "values": values}
    if valid is not None:
        d["valid"] = valid
    if scale:
        d["scale"] = scale
    return d


def const_key(n):
    return c("i32", [0] * n)


groupby = []

# aggregate_nulls_e2e.rs:118-190 (+ :379-382 COUNT(*) includes NULL rows)
groupby.append({
    "name": "i32_with_nulls", "source": "tests/aggregate_nulls_e2e.rs:118-190,379-382",
    "columns": {"k": const_key(6), "v": c("i32", [10, 0, -5, 30, 0, 7], [1, 0, 1, 1, 0, 1])},
    "group_by": ["k"],
    "aggs": [["count", "v"], ["sum", "v"], ["min", "v"], ["max", "v"], ["avg", "v"], ["count_star", None]],
    "expected": {"keys": [[0]], "aggs": [[4], [42], [-5], [30], [10.5], [6]], "agg_valid": [[1]] * 6},
})
# aggregate_nulls_e2e.rs:193-240
groupby.append({
    "name": "i64_with_nulls", "source": "tests/aggregate_nulls_e2e.rs:193-240",
    "columns": {"k": const_key(5), "v": c("i64", [100, 0, 0, 50, 25], [1, 0, 0, 1, 1])},
    "group_by": ["k"],
    "aggs": [["count", "v"], ["sum", "v"], ["min", "v"], ["max", "v"], ["avg", "v"]],
    "expected": {"keys": [[0]], "aggs": [[3], [175], [25], [100], [175 / 3]], "agg_valid": [[1]] * 5},
})
# aggregate_nulls_e2e.rs:329-375
groupby.append({
    "name": "f64_with_nulls", "source": "tests/aggregate_nulls_e2e.rs:329-375",
    "columns": {"k": const_key(5), "v": c("f64", [10.0, 0.0, 20.0, 30.0, 0.0], [1, 0, 1, 1, 0])},
    "group_by": ["k"],
    "aggs": [["count", "v"], ["sum", "v"], ["min", "v"], ["max", "v"], ["avg", "v"]],
    "expected": {"keys": [[0]], "aggs": [[3], [60.0], [10.0], [30.0], [20.0]], "agg_valid": [[1]] * 5},
})
# aggregate_nulls_e2e.rs:392-420
groupby.append({
    "name": "i64_no_nulls", "source": "tests/aggregate_nulls_e2e.rs:392-420",
    "columns": {"k": const_key(5), "v": c("i64", [1, 2, 3, 4, 5])},
    "group_by": ["k"],
    "aggs": [["count", "v"], ["sum", "v"], ["min", "v"], ["max", "v"]],
    "expected": {"keys": [[0]], "aggs": [[5], [15], [1], [5]], "agg_valid": [[1]] * 4},
})
# aggregate_nulls_e2e.rs:438-470 (all NULL -> SUM/MIN/MAX NULL, COUNT 0)
groupby.append({
    "name": "all_null_i64", "source": "tests/aggregate_nulls_e2e.rs:438-470,515-560",
    "columns": {"k": const_key(3), "v": c("i64", [0, 0, 0], [0, 0, 0])},
    "group_by": ["k"],
    "aggs": [["count", "v"], ["sum", "v"], ["min", "v"], ["max", "v"]],
    "expected": {"keys": [[0]], "aggs": [[0], [0], [0], [0]], "agg_valid": [[1], [0], [0], [0]]},
})
groupby.append({
    "name": "all_null_f64", "source": "tests/aggregate_nulls_e2e.rs:455-470,526-535",
    "columns": {"k": const_key(3), "v": c("f64", [0.0, 0.0, 0.0], [0, 0, 0])},
    "group_by": ["k"],
    "aggs": [["count", "v"], ["min", "v"], ["max", "v"]],
    "expected": {"keys": [[0]], "aggs": [[0], [0.0], [0.0]], "agg_valid": [[1], [0], [0]]},
})
# aggregate_nulls_e2e.rs:472-500
groupby.append({
    "name": "nulls_at_boundaries", "source": "tests/aggregate_nulls_e2e.rs:472-500",
    "columns": {"k": const_key(5), "v": c("i64", [0, 7, 11, 13, 0], [0, 1, 1, 1, 0])},
    "group_by": ["k"],
    "aggs": [["count", "v"], ["sum", "v"], ["min", "v"], ["max", "v"]],
    "expected": {"keys": [[0]], "aggs": [[3], [31], [7], [13]], "agg_valid": [[1]] * 4},
})
# semantics_e2e.rs:321-356 two-key COUNT(v) skips NULLs
groupby.append({
    "name": "two_key_count_excludes_nulls", "source": "tests/semantics_e2e.rs:321-356",
    "columns": {"k1": c("i32", [i // 4 for i in range(8)]), "k2": c("i32", [(i // 2) % 2 for i in range(8)]),
                "v": c("i64", [i if i % 2 == 0 else 0 for i in range(8)], [1 if i % 2 == 0 else 0 for i in range(8)])},
    "group_by": ["k1", "k2"],
    "aggs": [["count", "v"]],
    "expected": {"keys": [[0, 0], [0, 1], [1, 0], [1, 1]], "aggs": [[1, 1, 1, 1]], "agg_valid": [[1, 1, 1, 1]]},
})
# semantics_e2e.rs:359-405 grouped float MIN/MAX with NaN (NaN is the largest)
groupby.append({
    "name": "float_min_max_nan", "source": "tests/semantics_e2e.rs:359-405",
    "columns": {"k": c("i32", [0, 0, 0, 1, 1]), "v": c("f64", [1.0, NaN, 2.0, -3.0, 0.5])},
    "group_by": ["k"],
    "aggs": [["min", "v"], ["max", "v"]],
    "expected": {"keys": [[0], [1]], "aggs": [[1.0, -3.0], [NaN, 0.5]], "agg_valid": [[1, 1], [1, 1]]},
})
# semantics_e2e.rs:409-430 all-NaN group
groupby.append({
    "name": "float_all_nan", "source": "tests/semantics_e2e.rs:409-430",
    "columns": {"k": c("i32", [0, 0, 0]), "v": c("f64", [NaN, NaN, NaN])},
    "group_by": ["k"],
    "aggs": [["min", "v"], ["max", "v"]],
    "expected": {"keys": [[0]], "aggs": [[NaN], [NaN]], "agg_valid": [[1], [1]]},
})
# semantics_e2e.rs:503-530 all-NULL key -> one NULL group
groupby.append({
    "name": "all_null_key_one_group", "source": "tests/semantics_e2e.rs:503-530",
    "columns": {"k": c("i32", [0] * 6, [0] * 6),
                "v": c("i64", [i if i % 2 == 0 else 0 for i in range(6)], [1 if i % 2 == 0 else 0 for i in range(6)])},
    "group_by": ["k"],
    "aggs": [["count_star", None], ["count", "v"]],
    "expected": {"keys": [[None]], "aggs": [[6], [3]], "agg_valid": [[1], [1]]},
})
# groupby_tier2_orchestrator.rs:726-760 hand vector, oracle = per-key HashMap sum
keys8 = [1, 2, 1, 3, 2, 1, 4, 3]
vals8 = [10.0, 20.0, 11.0, 30.0, 21.0, 12.0, 40.0, 31.0]
sums = {}
for k, v in zip(keys8, vals8):
    sums[k] = sums.get(k, 0.0) + v
groupby.append({
    "name": "tier2_hand_vector", "source": "src/exec/groupby_tier2_orchestrator.rs:726-760",
    "columns": {"k": c("i32", keys8), "v": c("f64", vals8)},
    "group_by": ["k"],
    "aggs": [["sum", "v"]],
    "expected": {"keys": [[k] for k in sorted(sums)], "aggs": [[sums[k] for k in sorted(sums)]],
                 "agg_valid": [[1] * len(sums)]},
})
# decimal_type_test.rs:322-362, 365-395 (SUM(Decimal128) widens to (38, s), skips NULLs)
groupby.append({
    "name": "decimal_sum_basic", "source": "tests/decimal_type_test.rs:322-362",
    "columns": {"k": const_key(5), "d": c("dec128", [123, -456, 789, 1, 10000], scale=2)},
    "group_by": ["k"],
    "aggs": [["sum", "d"]],
    "expected": {"keys": [[0]], "aggs": [[123 - 456 + 789 + 1 + 10000]], "agg_valid": [[1]]},
})
groupby.append({
    "name": "decimal_sum_skips_nulls", "source": "tests/decimal_type_test.rs:365-395",
    "columns": {"k": const_key(5), "d": c("dec128", [100, 0, -25, 0, 75], [1, 0, 1, 0, 1], scale=2)},
    "group_by": ["k"],
    "aggs": [["sum", "d"]],
    "expected": {"keys": [[0]], "aggs": [[150]], "agg_valid": [[1]]},
})
big = 10 ** 38 - 1
groupby.append({
    "name": "decimal_sum_overflow", "source": "tests/decimal_type_test.rs:397-430",
    "columns": {"k": const_key(2), "d": c("dec128", [str(big), str(big)])},
    "group_by": ["k"],
    "aggs": [["sum", "d"]],
    "expected": {"error": "overflow", "message_contains": ["overflow", "Decimal128"]},
})

# Join: gpu_join_e2e.rs:66-140 (4096 unique build keys, 8192 probe keys i % 8192)
join = [{
    "name": "inner_join_int32_basic", "source": "tests/gpu_join_e2e.rs:27-28,66-140",
    "build": c("i32", list(range(4096))), "probe": c("i32", [i % 8192 for i in range(8192)]),
    "expected": {"n_pairs": 4096, "pairs": "probe_row -> build_row == probe_key for probe_key < 4096"},
}, {
    "name": "inner_join_int64_basic", "source": "tests/gpu_join_e2e.rs:142-200",
    "build": c("i64", list(range(4096))), "probe": c("i64", [i % 8192 for i in range(8192)]),
    "expected": {"n_pairs": 4096, "pairs": "probe_row -> build_row == probe_key for probe_key < 4096"},
}, {
    "name": "all_null_keys_no_rows", "source": "tests/semantics_e2e.rs:533-575",
    "build": c("i32", [0] * 4, [0] * 4), "probe": c("i32", [0] * 4, [0] * 4),
    "expected": {"n_pairs": 0},
}]

# Sort key transform unit tests: gpu_sort.rs:3810-3935
sort_keys = [{
    "name": "f32_asc_orders_floats", "source": "src/exec/gpu_sort.rs:3810-3840", "dtype": "f32",
    "values": ["-inf", -1e30, -1.5, 0.0, 1.5, 1e30, "inf"], "property": "strictly_increasing",
}, {
    "name": "f32_neg_zero_equals_pos_zero", "source": "src/exec/gpu_sort.rs:3842-3851", "dtype": "f32",
    "values": [-0.0, 0.0], "property": "all_equal",
}, {
    "name": "f32_nan_canonical_and_last", "source": "src/exec/gpu_sort.rs:3858-3877", "dtype": "f32",
    "bits": [0x7FC00000, 0xFFC00000, 0x7F800001, 0xFFC0DEAD], "property": "all_equal_and_above_inf",
}, {
    "name": "f32_desc_reverses", "source": "src/exec/gpu_sort.rs:3882-3890", "dtype": "f32", "descending": True,
    "values": [-2.0, -0.5, 0.0, 0.5, 2.0], "property": "strictly_decreasing",
}, {
    "name": "f64_asc_orders_floats", "source": "src/exec/gpu_sort.rs:3895-3925", "dtype": "f64",
    "values": ["-inf", -1e300, -3.25, 0.0, 3.25, 1e300, "inf"], "property": "strictly_increasing",
}]

# ORDER BY e2e: sort_e2e.rs:55-160 (shuffle_deterministic fixtures; output equals sorted(input))
sort = [
    {"name": "order_by_int32_asc", "source": "tests/sort_e2e.rs:55-90", "dtype": "i32", "n": 16384,
     "gen": "shuffle_iota", "seed": 0xDEADBEEF, "descending": False},
    {"name": "order_by_int32_desc", "source": "tests/sort_e2e.rs:92-126", "dtype": "i32", "n": 16384,
     "gen": "shuffle_iota", "seed": 0xFEEDFACE, "descending": True},
    {"name": "order_by_int64_asc_non_pow2", "source": "tests/sort_e2e.rs:128-160", "dtype": "i64", "n": 20000,
     "gen": "mul7919_mod_shuffle", "seed": 0xC001CAFE, "descending": False},
    {"name": "order_by_float64_asc", "source": "tests/sort_e2e.rs:162-190", "dtype": "f64", "n": 17000,
     "gen": "sin_golden", "descending": False},
]


groupby_wide = []
# groupby_wide.rs:1404-1436 (two_int64_keys_sum_count_avg): three (a, b) tuples, output sorted by (a, b)
_rows = [(1, 10, 100), (2, 10, 7), (1, 20, 50), (1, 10, 200), (2, 10, 8), (2, 10, 9)]
groupby_wide.append({
    "name": "two_int64_keys_sum_count_avg", "source": "src/exec/groupby_wide.rs:1404-1436",
    "columns": {"a": c("i64", [r[0] for r in _rows]), "b": c("i64", [r[1] for r in _rows]),
                "v": c("i64", [r[2] for r in _rows])},
    "group_by": ["a", "b"], "aggs": [["sum", "v"], ["count", "v"], ["avg", "v"]],
    "expected": {"k0": [1, 1, 2], "k1": [10, 20, 10], "aggs": [[300, 50, 24], [2, 1, 3], [150.0, 50.0, 8.0]]},
})
# groupby_wide.rs:1438-1471 (deterministic_ordering): a in 0..20, b in 0..5, v = a * 100 + b, one row
# per (a, b); the test asserts 100 groups in (a, b) order, so each group's SUM and AVG are its v.
_rows = [(a, b, a * 100 + b) for a in range(20) for b in range(5)]
groupby_wide.append({
    "name": "deterministic_ordering", "source": "src/exec/groupby_wide.rs:1438-1471",
    "columns": {"a": c("i64", [r[0] for r in _rows]), "b": c("i64", [r[1] for r in _rows]),
                "v": c("i64", [r[2] for r in _rows])},
    "group_by": ["a", "b"], "aggs": [["sum", "v"], ["count", "v"], ["avg", "v"]],
    "expected": {"k0": [r[0] for r in _rows], "k1": [r[1] for r in _rows],
                 "aggs": [[r[2] for r in _rows], [1] * len(_rows), [float(r[2]) for r in _rows]]},
})

def main():
    doc = {"about": "known answers transcribed from the reference's tests for this path",
           "groupby": groupby, "groupby_wide": groupby_wide, "join": join, "sort_keys": sort_keys, "sort": sort}
    OUT.write_text(json.dumps(doc, indent=1, default=lambda x: None) + "\n")
    print(f"wrote {OUT} ({len(groupby)} groupby, {len(groupby_wide)} wide groupby, {len(join)} join, {len(sort_keys)} sort-key, {len(sort)} sort)")


if __name__ == "__main__":
    assert not math.isnan(1.0)
    main()
