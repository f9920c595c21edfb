"""The reference's own test cases, run on the GPU through the C ABI.

tests/golden/reference_cases.json holds the SQL and expected results of the
reference's tests/extension.rs and test/sql/*.test (see make_golden.py).
The sqllogictest files never pin a table in the reference (every query
there ran through DuckDB's CPU fallback); here each table is registered with
gpu_register_table after it is created, so the same expected rows check the
GPU path.
"""
import datetime as dt
import decimal
import json
from pathlib import Path

import pytest

from mettle_b200 import MettleError
from mettle_b200 import _lib as L

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_cases.json").read_text())
EXT = {c["name"]: c for c in GOLDEN["extension"]}


def _cmp(a, b, tol):
    if isinstance(b, str) or isinstance(a, str):
        return str(a) == str(b)
    if isinstance(a, decimal.Decimal):
        a = float(a)
    return abs(float(a) - float(b)) <= tol


def _rows_match(got, want, ordered, tol, columns=None):
    if columns:
        got = [r[:columns] for r in got]
    if len(got) != len(want):
        return False
    if not ordered:
        key = lambda r: tuple(str(x) for x in r)
        got, want = sorted(got, key=key), sorted(want, key=key)
    return all(len(g) == len(w) and all(_cmp(x, y, tol) for x, y in zip(g, w)) for g, w in zip(got, want))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(EXT))
def test_extension_case(conn, name):
    case = EXT[name]
    for s in case["setup"]:
        conn.execute(s)
    if case.get("unsupported"):
        # The reference runs these on DuckDB's CPU path (duckdb_cpu_fallback):
        # outside the offloaded subset, or a table that was never pinned.
        with pytest.raises(MettleError) as e:
            conn.execute(case["query"])
        assert e.value.code == L.UNSUPPORTED
        return
    rows = conn.execute(case["query"]).fetchall()
    assert _rows_match(rows, case["rows"], case["ordered"], case["tol"], case.get("columns")), rows
    assert conn.last_execution_mode() == "cuda_generic_plan"


def render(v):
    """DuckDB sqllogictest rendering (test/run_sql_tests.py:251-268)."""
    if v is None:
        return "NULL"
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        r = f"{v:.6f}".rstrip("0")
        return r + "0" if r.endswith(".") else (r or "0.0")
    if isinstance(v, decimal.Decimal):
        return format(v.normalize(), "f")
    return str(v)


# Records outside the offloaded subset (the reference sends them to DuckDB too).
OUTSIDE_SUBSET = ("WITH filtered AS",)


@pytest.mark.gpu
@pytest.mark.parametrize("fname", sorted(GOLDEN["sqllogic"]))
def test_sqllogic_file(conn, fname):
    checked = 0
    for rec in GOLDEN["sqllogic"][fname]:
        sql = rec["sql"]
        if rec["kind"] == "statement":
            if rec["status"] == "error":
                with pytest.raises(MettleError) as e:
                    conn.execute(sql)
                assert rec["error"] in str(e.value), (rec["source"], str(e.value))
                continue
            conn.execute(sql)
            if conn.ctx and any(w in sql.upper() for w in ("CREATE TABLE", "INSERT INTO", "GPU_BUFFER_INIT")):
                for t in list(conn.tables):
                    conn.gpu_register_table(t)
            continue
        if any(m in sql for m in OUTSIDE_SUBSET):
            with pytest.raises(MettleError) as e:
                conn.execute(sql)
            assert e.value.code == L.UNSUPPORTED
            continue
        rows = conn.execute(sql).fetchall()
        got = [" ".join(render(v) for v in r) for r in rows]
        want = list(rec["rows"])
        assert len(rows[0]) if rows else True
        if rec["sort"] == "rowsort":
            got.sort()
            want.sort()
        assert got == want, (rec["source"], got, want)
        checked += 1
    assert checked >= 5
