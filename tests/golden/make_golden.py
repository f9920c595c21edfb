"""Generates tests/golden/reference_cases.json from the reference's own tests.

Run in a checkout that has the reference tree (default ../reference or the
path given as argv[1]); the GPU box only reads the committed JSON.

* test/sql/sirius-compat.test and test/sql/tpch-sirius.test are
  DuckDB sqllogictest files: every `statement ok/error` and `query` record is
  copied verbatim with its expected rows.
* tests/extension.rs holds Rust integration tests: the setup SQL
  (`execute_batch`) and the `gpu_processing` query text are extracted from
  the source; the expected values are the ones its assertions state, listed
  below with their line numbers.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

OUT = Path(__file__).with_name("reference_cases.json")

# Expected results of tests/extension.rs (test name -> rows, and how the test
# compares them). `ordered` means the test checks row order; `tol` is the
# absolute tolerance its assertions use (0 = exact).
EXTENSION_EXPECTED = {
    # :62-92
    "generic_plan_executes_filter_on_pinned_table": {"rows": [[3], [4], [5]], "ordered": False, "tol": 0},
    # :96-128
    "generic_plan_executes_projection_with_filter": {"rows": [[2, 20], [3, 30]], "ordered": False, "tol": 0},
    # :132-162
    "generic_plan_executes_multi_predicate_filter": {"rows": [[2, 20], [3, 30], [4, 40]], "ordered": False,
                                                     "tol": 0},
    # :166-195
    "generic_plan_executes_order_by_desc_with_limit": {"rows": [[5], [4], [3]], "ordered": True, "tol": 0},
    # :199-236
    "generic_plan_filters_by_string_and_date": {"rows": [[3], [4]], "ordered": False, "tol": 0},
    # :240-276
    "generic_plan_executes_ungrouped_aggregate": {"rows": [[140, 4, 20, 50]], "ordered": True, "tol": 0},
    # :280-317
    "generic_plan_executes_two_table_join": {"rows": [[10, 100], [11, 200]], "ordered": False, "tol": 0},
    # :321-357 (tolerance 0.1)
    "generic_plan_evaluates_compound_expression": {"rows": [[50.0], [95.0], [180.0]], "ordered": False,
                                                   "tol": 0.1},
    # :361-389 (tolerance 1.0)
    "generic_plan_evaluates_ungrouped_agg_with_expression": {"rows": [[325.0]], "ordered": True, "tol": 1.0},
    # :391-472: first two columns checked, tolerance 0.1 / 1.0
    "generic_plan_executes_q3_three_table_join_with_grouped_agg": {
        "rows": [[100, 1400.0], [102, 240.0]], "ordered": True, "tol": 1.0, "columns": 2},
    # :476-525
    "generic_plan_executes_simple_three_table_grouped_aggregate": {"rows": [[1, 450.0], [2, 200.0]],
                                                                   "ordered": True, "tol": 0},
    # :606-659 (revenue 275 / 170 by key)
    "single_table_gpu_query_hot_cache_is_visible": {"rows": [[1, 275.0], [2, 170.0]], "ordered": True,
                                                    "tol": 1.0},
    # :661-698
    "generic_plan_executes_grouped_aggregate": {"rows": [["A", 90], ["B", 60]], "ordered": True, "tol": 0.1},
    # :723-777
    "generic_plan_executes_grouped_mixed_aggregates": {
        "rows": [[90, "A", 3, 10, 50, 30.0], [60, "B", 2, 20, 40, 30.0]], "ordered": True, "tol": 0},
    # :781-825
    "gpu_grouped_aggregate_single_integer_key": {"rows": [[1, 275.0], [2, 170.0], [3, 255.0]], "ordered": True,
                                                 "tol": 1.0},
    # :829-871
    "gpu_grouped_aggregate_single_integer_key_two_sums": {
        "rows": [[1, 300.0, 275.0], [2, 200.0, 170.0], [3, 300.0, 255.0]], "ordered": True, "tol": 1e-9},
    # :875-928
    "gpu_grouped_aggregate_composite_key_multi_state": {
        "rows": [[1, 10, 2, 140.0, 40.0, 100.0, 70.0], [1, 20, 2, 80.0, 30.0, 50.0, 40.0],
                 [2, 10, 2, 100.0, 20.0, 80.0, 50.0]], "ordered": True, "tol": 1e-9},
    # :930-970 (revenue 275 / 170)
    "generic_plan_executes_grouped_aggregate_with_expression": {"rows": [[1, 275.0], [2, 170.0]],
                                                                "ordered": True, "tol": 1.0},
    # :974-1015
    "generic_plan_executes_two_table_grouped_aggregate": {"rows": [[10, 450.0], [20, 200.0]], "ordered": True,
                                                          "tol": 0},
    # :1052-1093
    "gpu_processing_preserves_qualified_duplicate_column_bindings": {"rows": [[1, 100], [2, 200]],
                                                                     "ordered": True, "tol": 0},
    # :1095-1138: LEFT JOIN is outside the offloaded subset (DuckDB fallback)
    "gpu_processing_falls_back_for_outer_join_queries": {"unsupported": True},
    # :1018-1050: the table is never registered (DuckDB fallback)
    "gpu_processing_falls_back_for_unpinned_tables": {"unsupported": True},
}


def rust_strings(src: str) -> list[str]:
    """String literals of a Rust source fragment, escapes resolved."""
    out, i = [], 0
    while True:
        i = src.find('"', i)
        if i < 0:
            return out
        j, s = i + 1, []
        while j < len(src):
            ch = src[j]
            if ch == "\\":
                nxt = src[j + 1]
                if nxt == "\n":  # line continuation: drop newline and leading whitespace
                    j += 2
                    while j < len(src) and src[j] in " \t":
                        j += 1
                    continue
                s.append({"n": "\n", "t": "\t", '"': '"', "\\": "\\"}.get(nxt, nxt))
                j += 2
                continue
            if ch == '"':
                break
            s.append(ch)
            j += 1
        out.append("".join(s))
        i = j + 1


def extension_cases(path: Path) -> list[dict]:
    text = path.read_text()
    cases = []
    for m in re.finditer(r"#\[test\]\s*fn (\w+)\(\)\s*\{", text):
        name = m.group(1)
        if name not in EXTENSION_EXPECTED:
            continue
        start = m.end()
        nxt = text.find("#[test]", start)
        body = text[start: nxt if nxt > 0 else len(text)]
        line = text[: m.start()].count("\n") + 1
        setup, query = [], None
        for call in re.finditer(r"\.(execute_batch|prepare)\(\s*", body):
            lit = rust_strings(body[call.end(): call.end() + 4000])[0]
            if call.group(1) == "execute_batch":
                setup.append(lit)
            elif "gpu_processing" in lit and query is None:
                query = lit
        if query is None:
            sql_var = re.search(r'let sql = "', body)
            if sql_var:
                query = rust_strings(body[sql_var.end() - 1:])[0]
        case = {"name": name, "source": f"tests/extension.rs:{line}", "setup": setup, "query": query}
        case.update(EXTENSION_EXPECTED[name])
        cases.append(case)
    return cases


def sqllogic_records(path: Path) -> list[dict]:
    lines = path.read_text().splitlines()
    recs, i = [], 0
    while i < len(lines):
        ln = lines[i].strip()
        if not ln or ln.startswith("#"):
            i += 1
            continue
        head_line = i + 1
        if ln.startswith("statement ok") or ln.startswith("statement error"):
            kind = "ok" if ln.startswith("statement ok") else "error"
            expect = ln[len("statement error"):].strip() if kind == "error" else ""
            i += 1
            sql = []
            while i < len(lines) and lines[i].strip():
                sql.append(lines[i])
                i += 1
            recs.append({"kind": "statement", "status": kind, "error": expect, "sql": "\n".join(sql),
                         "source": f"{path.name}:{head_line}"})
            continue
        if ln.startswith("query"):
            parts = ln.split()
            types, sort = parts[1], (parts[2] if len(parts) > 2 else "nosort")
            i += 1
            sql = []
            while i < len(lines) and lines[i].strip() != "----":
                sql.append(lines[i])
                i += 1
            i += 1
            rows = []
            while i < len(lines) and lines[i].strip():
                rows.append(lines[i].strip())
                i += 1
            recs.append({"kind": "query", "types": types, "sort": sort, "sql": "\n".join(sql), "rows": rows,
                         "source": f"{path.name}:{head_line}"})
            continue
        i += 1
    return recs


def main():
    ref = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parents[3] / "reference"
    data = {
        "extension": extension_cases(ref / "tests" / "extension.rs"),
        "sqllogic": {p.name: sqllogic_records(p) for p in sorted((ref / "test" / "sql").glob("*.test"))},
    }
    OUT.write_text(json.dumps(data, indent=1) + "\n")
    print(f"wrote {OUT} ({len(data['extension'])} extension cases, "
          f"{sum(len(v) for v in data['sqllogic'].values())} sqllogic records)")


if __name__ == "__main__":
    main()
