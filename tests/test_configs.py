"""Parity of the GPU path with the CPU oracle on the benchmark workloads
through the C ABI. Integer, DECIMAL, DATE and
TIMESTAMP results must be bit-exact; FLOAT aggregates within 1e-6 relative
of an extended-precision sum."""
import numpy as np
import pytest

import oracle as orc
from mettle_b200 import MettleError
from mettle_b200 import _lib as L
from mettle_b200 import workloads as W

FLOAT_RTOL = 1e-6


def init(conn, cache="8 GB", processing="8 GB"):
    conn.execute(f"CALL gpu_buffer_init('{cache}', '{processing}')")


# ------------------------------------------------------------------ config 1
@pytest.mark.gpu
@pytest.mark.parametrize("n", [0, 1, 1000, 1_000_000])
def test_c1_plain_small_query(conn, oracle_lib, n):
    init(conn)
    d = W.numbers(n)
    conn.create_table("numbers", {"value": (L.T_INTEGER, d["value"])})
    conn.gpu_register_table("numbers")
    r = conn.gpu_processing(W.C1_SQL)
    rows = orc.filter_rows([(d["value"], ">", 500000)])
    rows = orc.sort_rows(d["value"], rows)
    want_v = orc.gather(d["value"], rows)
    want_s = orc.gather(d["value"], rows, "*", 10)
    assert r.names == ["value", "scaled"]
    assert np.array_equal(r.columns[0], want_v)
    assert np.array_equal(r.columns[1], want_s)


# ------------------------------------------------------------------ config 2
def scan_expect(d, col, op, lit_value):
    rows = orc.filter_rows([(d[col], op, lit_value)])
    return {
        "a": orc.gather(d["a"], rows), "b5": orc.gather(d["b"], rows, "+", 5),
        "c10": orc.gather(d["c"], rows, "*", np.float32(10)), "d": orc.gather(d["d"], rows),
        "e": orc.gather(d["e"], rows),
    }


def literal_value(col, sel):
    if col == "a":
        return int(sel * 2**31)
    if col == "b":
        return int(-(2**62) + sel * 2**63)
    if col == "c":
        return float(sel)
    if col == "d":
        return W.DAY0 + int(sel * W.SPAN_DAYS)
    us = int(sel * W.SPAN_DAYS * 86_400_000_000)
    return W.DAY0 * 86_400_000_000 + (us // 1_000_000) * 1_000_000


@pytest.fixture(scope="module")
def scan_conn(built_lib):
    from mettle_b200 import Connection
    c = Connection()
    init(c)
    d = W.scan(2_000_000)
    c.create_table("t", {"a": (L.T_INTEGER, d["a"]), "b": (L.T_BIGINT, d["b"]), "c": (L.T_FLOAT, d["c"]),
                         "d": (L.T_DATE, d["d"]), "e": (L.T_TIMESTAMP, d["e"])})
    c.gpu_register_table("t", upload=True)
    yield c, d
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("col", ["a", "b", "c", "d", "e"])
@pytest.mark.parametrize("op", ["=", "<", "<=", ">", ">="])
@pytest.mark.parametrize("sel", [0.01, 0.1, 0.5])
def test_c2_filter_projection(scan_conn, col, op, sel):
    conn, d = scan_conn
    s = sel if op in ("<", "<=") else 1.0 - sel
    if op == "=":
        # equality: a value that occurs in the column
        v = d[col][12345]
        if col in ("a", "b"):
            lit = str(int(v))
        elif col == "c":
            # a DOUBLE literal (scientific notation) equal to the FLOAT value; a
            # plain decimal literal is a DECIMAL, cast as (float)digits / (float)10^scale
            lit = f"{float(v):.17e}"
        elif col == "d":
            lit = f"DATE '{W.day_to_iso(int(v))}'"
        else:
            import datetime as dt
            t = dt.datetime(1970, 1, 1) + dt.timedelta(microseconds=int(v))
            lit = f"TIMESTAMP '{t.strftime('%Y-%m-%d %H:%M:%S.%f')}'"
        value = v.item()
    else:
        lit = W.scan_literal(col, s)
        value = literal_value(col, s)
    sql = f"SELECT a, b + 5 AS b5, c * 10 AS c10, d, e FROM t WHERE {col} {op} {lit}"
    r = conn.gpu_processing(sql)
    want = scan_expect(d, col, op, value)
    assert r.rows == len(want["a"])
    for i, name in enumerate(["a", "b5", "c10", "d", "e"]):
        assert np.array_equal(r.columns[i], want[name]), (sql, name)


@pytest.mark.gpu
def test_c2_multi_predicate_and_empty(scan_conn):
    conn, d = scan_conn
    r = conn.gpu_processing("SELECT a, d FROM t WHERE a < 1000000000 AND d >= DATE '1995-01-01' AND c < 0.25")
    rows = orc.filter_rows([(d["a"], "<", 1_000_000_000), (d["d"], ">=", W.day_to_iso and
                            (np.datetime64('1995-01-01') - np.datetime64('1970-01-01')).astype(int)),
                            (d["c"], "<", 0.25)])
    assert np.array_equal(r.columns[0], d["a"][rows])
    r = conn.gpu_processing("SELECT a FROM t WHERE a < 0")
    assert r.rows == 0


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 255, 256, 257, 100_003])
def test_scan_row_ids_and_gather_edges(conn, n):
    """The scan's late gather (survivor masks per 256-row tile, expanded into
    row ids, outputs gathered at them) at sizes around a tile, with every row,
    no row and the first half selected; each output type and constant
    arithmetic compared with numpy in row order."""
    init(conn, "1 GB", "1 GB")
    r = np.random.default_rng(n)
    d = {"a": np.arange(n, dtype=np.int32), "b": r.integers(-2**40, 2**40, n).astype(np.int64),
         "c": r.random(n, dtype=np.float32), "e": r.integers(0, 2**50, n).astype(np.int64)}
    conn.create_table("t", {"a": (L.T_INTEGER, d["a"]), "b": (L.T_BIGINT, d["b"]), "c": (L.T_FLOAT, d["c"]),
                            "e": (L.T_TIMESTAMP, d["e"])})
    conn.gpu_register_table("t")
    for where, m in (("a >= 0", d["a"] >= 0), ("a < 0", d["a"] < 0), (f"a < {n // 2}", d["a"] < n // 2)):
        res = conn.gpu_processing(f"SELECT a, b - 7 AS b7, c * 3 AS c3, e, a * 2 AS a2 FROM t WHERE {where}")
        assert res.rows == int(m.sum()), where
        assert np.array_equal(res.columns[0], d["a"][m])
        assert np.array_equal(res.columns[1], d["b"][m] - 7)
        assert np.array_equal(res.columns[2], (d["c"][m] * np.float32(3)).astype(np.float32))
        assert np.array_equal(res.columns[3], d["e"][m])
        assert np.array_equal(res.columns[4], d["a"][m] * 2)


@pytest.mark.gpu
def test_c2_full_size(conn):
    """The measured scan at its full size: 10^8 rows, half of them selected,
    every output column compared in row order with the oracle's gathers."""
    init(conn, "8 GB", "8 GB")
    d = W.scan(100_000_000)
    conn.create_table("t", {"a": (L.T_INTEGER, d["a"]), "b": (L.T_BIGINT, d["b"]), "c": (L.T_FLOAT, d["c"]),
                            "d": (L.T_DATE, d["d"]), "e": (L.T_TIMESTAMP, d["e"])})
    conn.gpu_register_table("t", upload=True)
    r = conn.gpu_processing(W.scan_sql("a", "<", 0.5))
    want = scan_expect(d, "a", "<", literal_value("a", 0.5))
    assert r.rows == len(want["a"]) and abs(r.rows - 50_000_000) < 100_000
    for i, name in enumerate(["a", "b5", "c10", "d", "e"]):
        assert np.array_equal(r.columns[i], want[name]), name


# ------------------------------------------------------------------ config 3
@pytest.mark.gpu
@pytest.mark.parametrize("groups,dist", [(1000, "uniform"), (1000, "zipf"), (100_000, "uniform"),
                                         (100_000, "zipf"), (1_500_000, "uniform")])
def test_c3_groupby_topk(conn, groups, dist):
    init(conn)
    d = W.groupby(n=3_000_000, groups=groups, dist=dist, seed_salt=groups)
    conn.create_table("t", {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]), "f": (L.T_FLOAT, d["f"])})
    conn.gpu_register_table("t")
    r = conn.gpu_processing(W.C3_SQL)
    want = orc.groupby_c3(d["k"], d["v"], d["f"], limit=100)
    rows = r.fetchall()
    assert len(rows) == len(want["k"])
    for i, row in enumerate(rows):
        k, sum_v, cnt, min_v, max_v, avg_v, sum_f, min_f, max_f, avg_f = row
        assert k == want["k"][i]
        assert sum_v == want["sum_v"][i]
        assert cnt == want["cnt"][i] and min_v == want["min_v"][i] and max_v == want["max_v"][i]
        assert avg_v == want["avg_v"][i]  # exact: DuckDB's extended-precision quotient
        assert abs(sum_f - want["sum_f"][i]) <= FLOAT_RTOL * abs(want["sum_f"][i])
        assert np.float32(min_f) == want["min_f"][i] and np.float32(max_f) == want["max_f"][i]
        assert abs(avg_f - want["avg_f"][i]) <= FLOAT_RTOL * abs(want["avg_f"][i])


@pytest.mark.gpu
def test_c3_all_groups_exact(conn):
    init(conn)
    d = W.groupby(n=500_000, groups=5000, dist="zipf", seed_salt=9)
    conn.create_table("t", {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]), "f": (L.T_FLOAT, d["f"])})
    conn.gpu_register_table("t")
    r = conn.gpu_processing("SELECT k, SUM(v), COUNT(*), MIN(v), MAX(v) FROM t GROUP BY k ORDER BY k")
    want = orc.groupby_c3(d["k"], d["v"], d["f"], limit=-1)
    assert r.rows == want["groups"]
    assert np.array_equal(r.columns[0], want["k"])
    assert [int(x[0]) for x in r.columns[1]] == [int(s) for s in want["sum_v"]]
    assert np.array_equal(r.columns[2], want["cnt"])
    assert np.array_equal(r.columns[3], want["min_v"]) and np.array_equal(r.columns[4], want["max_v"])


def _step_names(conn, sql):
    """Names of the device steps a prepared statement runs."""
    st = conn.prepare(sql)
    try:
        st.set_profiling(True)
        st.launch()
        st.fetch()
        return [n for n, _ in st.step_times()]
    finally:
        st.close()


def _check_c3_all_groups(res, want):
    """Every group of the config-3 aggregate (ordered by k) against the oracle:
    integers and AVG(BIGINT) exact, FLOAT sums and averages within 1e-6."""
    assert res.rows == want["groups"] == len(want["k"])
    k, sv, cnt, mnv, mxv, avg, sf, mnf, mxf, avgf = res.columns
    assert np.array_equal(k, want["k"])
    assert np.array_equal(sv[:, 0].view(np.uint64), want["sum_lo"])
    assert np.array_equal(sv[:, 1], want["sum_hi"])
    assert np.array_equal(cnt, want["cnt"])
    assert np.array_equal(mnv, want["min_v"]) and np.array_equal(mxv, want["max_v"])
    assert np.array_equal(avg, want["avg_v"])  # DuckDB's extended-precision quotient
    assert np.all(np.abs(sf - want["sum_f"]) <= FLOAT_RTOL * np.abs(want["sum_f"]))
    assert np.array_equal(mnf, want["min_f"]) and np.array_equal(mxf, want["max_f"])
    assert np.all(np.abs(avgf - want["avg_f"]) <= FLOAT_RTOL * np.abs(want["avg_f"]))


C3_ALL_GROUPS_SQL = ("SELECT k, SUM(v), COUNT(*), MIN(v), MAX(v), AVG(v), SUM(f), MIN(f), MAX(f), AVG(f) "
                     "FROM t GROUP BY k ORDER BY k")


@pytest.mark.gpu
@pytest.mark.parametrize("groups,dist", [(10, "uniform"), (100, "zipf"), (1000, "uniform"), (1000, "zipf")])
def test_c3_few_groups_one_pass_all_groups(conn, tmp_path, monkeypatch, groups, dist):
    """Few groups: one pass over the columns into per-CTA shared-memory tables
    (the plan's agg_few step; chosen through the autotuner's table above 16
    groups), with a warp's rows of one group combined before they update;
    every group on all ten aggregates against the oracle."""
    g = max(1, (groups - 1).bit_length())  # size classes: log2, rounded up
    path = tmp_path / "tune.txt"
    path.write_text(f"agg_one_key/g{g}/n23 1 0\n")  # 6*10^6 rows: class 2^23
    monkeypatch.setenv("METTLE_TUNE_FILE", str(path))
    init(conn)
    d = W.groupby(n=6_000_000, groups=groups, dist=dist, seed_salt=groups + 5)
    conn.create_table("t", {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]), "f": (L.T_FLOAT, d["f"])})
    conn.gpu_register_table("t", upload=True)
    assert any(s.startswith("agg_few") for s in _step_names(conn, C3_ALL_GROUPS_SQL))
    want = orc.groupby_c3(d["k"], d["v"], d["f"], limit=-1)
    _check_c3_all_groups(conn.gpu_processing(C3_ALL_GROUPS_SQL), want)
    r = conn.gpu_processing(W.C3_SQL)
    top = orc.groupby_c3(d["k"], d["v"], d["f"], limit=100)
    assert np.array_equal(r.columns[0], top["k"]) and np.array_equal(r.columns[5], top["avg_v"])


@pytest.mark.gpu
def test_few_groups_edge_keys_and_wide_sums(conn, tmp_path, monkeypatch):
    """The one-pass path with the empty-slot sentinel key and both int64
    extremes as keys (the sentinel's rows update the global table directly)
    and sums that need 128 bits (no combining)."""
    path = tmp_path / "tune.txt"
    path.write_text("agg_one_key/g6/n22 1 0\n")  # 53 groups over 3*10^6 rows
    monkeypatch.setenv("METTLE_TUNE_FILE", str(path))
    init(conn)
    r = np.random.default_rng(77)
    n = 3_000_000
    k = r.integers(0, 50, n).astype(np.int64) * 1_000_003
    k[::7] = -1
    k[::11] = np.iinfo(np.int64).min
    k[::13] = np.iinfo(np.int64).max
    v = r.integers(2**61, 2**62, n).astype(np.int64)  # sums beyond int64
    conn.create_table("t", {"k": (L.T_BIGINT, k), "v": (L.T_BIGINT, v)})
    conn.gpu_register_table("t")
    sql = "SELECT k, COUNT(*), SUM(v), MIN(v), MAX(v) FROM t GROUP BY k ORDER BY k"
    assert any(s.startswith("agg_few") for s in _step_names(conn, sql))
    res = conn.gpu_processing(sql)
    want = _grouped(k, {"v": v.astype(object)})
    rows = res.fetchall()
    assert [x[0] for x in rows] == want["k"].tolist()
    assert [x[1] for x in rows] == want["cnt"].tolist()
    assert [int(x[2]) for x in rows] == [int(s) for s in want["v_sum"]]
    assert [x[3] for x in rows] == [int(s) for s in want["v_min"]]
    assert [x[4] for x in rows] == [int(s) for s in want["v_max"]]


@pytest.mark.gpu
@pytest.mark.parametrize("groups,dist", [(1, "uniform"), (3, "zipf"), (12, "uniform")])
def test_fewest_groups_thread_private_states(conn, groups, dist):
    """The fewest groups: every thread keeps its own states of every group
    and the threads' states are combined at the end. All ten aggregates of
    every group against the oracle."""
    init(conn)
    d = W.groupby(n=5_000_000, groups=groups, dist=dist, seed_salt=groups + 11)
    conn.create_table("t", {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]), "f": (L.T_FLOAT, d["f"])})
    conn.gpu_register_table("t", upload=True)
    assert any(s.startswith("agg_few") for s in _step_names(conn, C3_ALL_GROUPS_SQL))
    want = orc.groupby_c3(d["k"], d["v"], d["f"], limit=-1)
    _check_c3_all_groups(conn.gpu_processing(C3_ALL_GROUPS_SQL), want)
    r = conn.gpu_processing(W.C3_SQL)
    top = orc.groupby_c3(d["k"], d["v"], d["f"], limit=100)
    assert np.array_equal(r.columns[0], top["k"]) and np.array_equal(r.columns[5], top["avg_v"])


@pytest.mark.gpu
def test_fewest_groups_edge_keys_and_wide_sums(conn):
    """Five groups whose keys are the empty-slot sentinel (-1; its rows
    update the global table directly) and both int64 extremes, with sums
    that need 128 bits."""
    init(conn)
    r = np.random.default_rng(5)
    n = 2_000_000
    keys = np.array([-1, np.iinfo(np.int64).min, np.iinfo(np.int64).max, 0, 42], dtype=np.int64)
    k = keys[r.integers(0, 5, n)]
    v = r.integers(2**61, 2**62, n).astype(np.int64)
    conn.create_table("w", {"k": (L.T_BIGINT, k), "v": (L.T_BIGINT, v)})
    conn.gpu_register_table("w")
    sql = "SELECT k, COUNT(*), SUM(v), MIN(v), MAX(v) FROM w GROUP BY k ORDER BY k"
    assert any(s.startswith("agg_few") for s in _step_names(conn, sql))
    rows = conn.gpu_processing(sql).fetchall()
    want = _grouped(k, {"v": v.astype(object)})
    assert [x[0] for x in rows] == want["k"].tolist()
    assert [x[1] for x in rows] == want["cnt"].tolist()
    assert [int(x[2]) for x in rows] == [int(s) for s in want["v_sum"]]
    assert [x[3] for x in rows] == [int(s) for s in want["v_min"]]
    assert [x[4] for x in rows] == [int(s) for s in want["v_max"]]


@pytest.mark.gpu
@pytest.mark.parametrize("n,groups,dist", [(20_000_000, 4_000_000, "uniform"), (40_000_000, 8_000_000, "zipf")])
def test_c3_many_partitions_all_groups(conn, n, groups, dist):
    """Millions of groups: the partitioned aggregation at thousands of
    partitions (the scan over the partition totals covers several entries per
    thread, and partitions hold more groups than a CTA's shared-memory table,
    so records also reach the global table directly), uniform and Zipf.
    Every group is compared on all ten aggregates, and the plan must have
    taken the partitioned steps."""
    init(conn, "16 GB", "16 GB")
    d = W.groupby(n=n, groups=groups, dist=dist, seed_salt=3)
    conn.create_table("t", {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]), "f": (L.T_FLOAT, d["f"])})
    conn.gpu_register_table("t", upload=True)
    steps = _step_names(conn, C3_ALL_GROUPS_SQL)
    assert "part_agg" in steps and "part_scan" in steps, steps
    want = orc.groupby_c3(d["k"], d["v"], d["f"], limit=-1)
    _check_c3_all_groups(conn.gpu_processing(C3_ALL_GROUPS_SQL), want)
    # and the headline form: top-100 by SUM(v) with the key as the tie-break
    r = conn.gpu_processing(W.C3_SQL)
    top = orc.groupby_c3(d["k"], d["v"], d["f"], limit=100)
    assert np.array_equal(r.columns[0], top["k"]) and np.array_equal(r.columns[2], top["cnt"])
    assert np.array_equal(r.columns[5], top["avg_v"])


@pytest.mark.gpu
def test_c3_highest_cardinality_all_groups(conn):
    """About four rows per group over 1.5*10^7 groups (the headline
    cardinality's rows per group): more groups than one level of partitions
    keeps within shared-memory tables."""
    init(conn, "16 GB", "16 GB")
    d = W.groupby(n=60_000_000, groups=15_000_000, dist="uniform", seed_salt=4)
    conn.create_table("t", {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]), "f": (L.T_FLOAT, d["f"])})
    conn.gpu_register_table("t", upload=True)
    want = orc.groupby_c3(d["k"], d["v"], d["f"], limit=-1)
    _check_c3_all_groups(conn.gpu_processing(C3_ALL_GROUPS_SQL), want)


def _grouped(keys, cols):
    """Per distinct key (ascending): COUNT and, per column, SUM / MIN / MAX / SUM(|x|)."""
    o = np.argsort(keys, kind="stable")
    ks = keys[o]
    starts = np.flatnonzero(np.r_[True, ks[1:] != ks[:-1]])
    out = {"k": ks[starts], "cnt": np.diff(np.r_[starts, len(ks)])}
    for name, c in cols.items():
        cs = c[o]
        out[name + "_sum"] = np.add.reduceat(cs, starts)
        out[name + "_min"] = np.minimum.reduceat(cs, starts)
        out[name + "_max"] = np.maximum.reduceat(cs, starts)
        out[name + "_abs"] = np.add.reduceat(np.abs(cs), starts)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("groups", [3000, 40_000])
def test_group_by_many_groups_edge_keys(conn, groups):
    """Group counts past the shared-memory table take the partitioned
    aggregation; keys include the empty-slot sentinel (-1) and both int64
    extremes, rows pass a filter, and a DOUBLE column feeds SUM/MIN/MAX."""
    init(conn)
    r = np.random.default_rng(groups)
    n = 1_000_000
    k = r.integers(-(groups // 2), groups // 2, n).astype(np.int64)
    k[::97] = -1
    k[::1009] = np.iinfo(np.int64).min
    k[::1013] = np.iinfo(np.int64).max
    v = r.integers(-10**12, 10**12, n).astype(np.int64)
    x = r.standard_normal(n)
    conn.create_table("t", {"k": (L.T_BIGINT, k), "v": (L.T_BIGINT, v), "x": (L.T_DOUBLE, x)})
    conn.gpu_register_table("t")
    res = conn.gpu_processing("SELECT k, COUNT(*), SUM(v), MIN(v), MAX(v), SUM(x), MIN(x), MAX(x) FROM t "
                              "WHERE v > -500000000000 GROUP BY k ORDER BY k")
    m = v > -500_000_000_000
    want = _grouped(k[m], {"v": v[m], "x": x[m]})
    rows = res.fetchall()
    assert len(rows) == len(want["k"])
    got = list(zip(*rows))
    assert np.array_equal(np.array(got[0], np.int64), want["k"])
    assert np.array_equal(np.array(got[1], np.int64), want["cnt"])
    assert [int(s) for s in got[2]] == [int(s) for s in want["v_sum"]]
    assert np.array_equal(np.array(got[3], np.int64), want["v_min"])
    assert np.array_equal(np.array(got[4], np.int64), want["v_max"])
    assert np.all(np.abs(np.array(got[5]) - want["x_sum"]) <= 1e-12 * want["x_abs"] + 1e-300)
    assert np.array_equal(np.array(got[6]), want["x_min"]) and np.array_equal(np.array(got[7]), want["x_max"])


@pytest.mark.gpu
@pytest.mark.parametrize("groups,dist", [(12, "uniform"), (100, "uniform"), (20_000, "zipf"), (300_000, "zipf")])
def test_group_by_repeated_keys_in_a_warp(conn, groups, dist):
    """Few groups, or a skewed key, put several records of one key in the
    same warp of the per-partition aggregation, which combines them before
    updating; every group must still see every row."""
    init(conn)
    r = np.random.default_rng(groups)
    n = 2_000_000
    if dist == "zipf":
        k = (r.zipf(1.1, n) % groups).astype(np.int64) * 104729 - 7
    else:
        k = r.integers(0, groups, n).astype(np.int64) * 104729 - 7
    v = r.integers(-10**9, 10**9, n).astype(np.int64)
    x = r.standard_normal(n)
    conn.create_table("t", {"k": (L.T_BIGINT, k), "v": (L.T_BIGINT, v), "x": (L.T_DOUBLE, x)})
    conn.gpu_register_table("t")
    res = conn.gpu_processing("SELECT k, COUNT(*), SUM(v), MIN(v), MAX(v), SUM(x), MIN(x), MAX(x) FROM t "
                              "GROUP BY k ORDER BY k")
    want = _grouped(k, {"v": v, "x": x})
    rows = res.fetchall()
    assert len(rows) == len(want["k"])
    got = list(zip(*rows))
    assert np.array_equal(np.array(got[0], np.int64), want["k"])
    assert np.array_equal(np.array(got[1], np.int64), want["cnt"])
    assert [int(s) for s in got[2]] == [int(s) for s in want["v_sum"]]
    assert np.array_equal(np.array(got[3], np.int64), want["v_min"])
    assert np.array_equal(np.array(got[4], np.int64), want["v_max"])
    assert np.all(np.abs(np.array(got[5]) - want["x_sum"]) <= 1e-12 * want["x_abs"] + 1e-300)
    assert np.array_equal(np.array(got[6]), want["x_min"]) and np.array_equal(np.array(got[7]), want["x_max"])


@pytest.mark.gpu
def test_group_by_probed_column_many_groups(conn):
    """A one-key aggregate whose key and input come through a join: the
    partition passes read the probed table's columns by row id."""
    init(conn)
    r = np.random.default_rng(31)
    n_ord, n_item = 200_000, 1_500_000
    o_id = r.permutation(n_ord).astype(np.int32)
    o_cust = r.integers(0, 30_000, n_ord).astype(np.int64)
    i_order = r.integers(0, n_ord + 50_000, n_item).astype(np.int32)  # some match no order
    i_val = r.integers(-1000, 100_000, n_item).astype(np.int64)
    conn.create_table("orders", {"o_id": (L.T_INTEGER, o_id), "o_cust": (L.T_BIGINT, o_cust)})
    conn.create_table("items", {"i_order": (L.T_INTEGER, i_order), "i_val": (L.T_BIGINT, i_val)})
    conn.gpu_register_table("orders")
    conn.gpu_register_table("items")
    res = conn.gpu_processing("SELECT o_cust, COUNT(*), SUM(i_val), MAX(i_val) FROM orders, items "
                              "WHERE i_order = o_id AND i_val > 0 GROUP BY o_cust ORDER BY o_cust")
    cust_of = np.full(n_ord + 50_000, -1, np.int64)
    cust_of[o_id] = o_cust
    c = cust_of[i_order]
    m = (c >= 0) & (i_val > 0)
    want = _grouped(c[m], {"v": i_val[m]})
    rows = res.fetchall()
    assert len(rows) == len(want["k"])
    got = list(zip(*rows))
    assert np.array_equal(np.array(got[0], np.int64), want["k"])
    assert np.array_equal(np.array(got[1], np.int64), want["cnt"])
    assert [int(s) for s in got[2]] == [int(s) for s in want["v_sum"]]
    assert np.array_equal(np.array(got[3], np.int64), want["v_max"])


@pytest.mark.gpu
@pytest.mark.parametrize("sql_aggs,cols", [
    ("COUNT(*)", ()),                                          # records hold the key alone
    ("COUNT(*), SUM(a)", "a"),                                 # key and one input
    ("COUNT(*), SUM(a), SUM(b), SUM(c)", "abc"),               # key, three inputs
    ("COUNT(*), SUM(a), SUM(b), SUM(c), SUM(d), SUM(e)", "abcde"),  # more inputs than a record holds
])
def test_group_by_many_groups_record_shapes(conn, sql_aggs, cols):
    init(conn)
    r = np.random.default_rng(7)
    n = 600_000
    k = r.integers(0, 50_000, n).astype(np.int64) * 7919
    data = {"k": (L.T_BIGINT, k)}
    vals = {c: r.integers(-1000, 1000, n).astype(np.int64) for c in "abcde"}
    for c in "abcde":
        data[c] = (L.T_BIGINT, vals[c])
    conn.create_table("t", data)
    conn.gpu_register_table("t")
    res = conn.gpu_processing(f"SELECT k, {sql_aggs} FROM t GROUP BY k ORDER BY k")
    want = _grouped(k, {c: vals[c] for c in cols})
    rows = res.fetchall()
    assert len(rows) == len(want["k"])
    got = list(zip(*rows))
    assert np.array_equal(np.array(got[0], np.int64), want["k"])
    assert np.array_equal(np.array(got[1], np.int64), want["cnt"])
    for i, c in enumerate(cols):
        assert [int(s) for s in got[2 + i]] == [int(s) for s in want[c + "_sum"]]


# ------------------------------------------------------------------ config 4
def q3_check(conn, t, limit=10):
    r = conn.gpu_processing(W.q3_sql(t.date, limit=limit))
    want = orc.q3(t, segment_code=1, limit=limit)
    rows = r.fetchall()
    assert len(rows) == len(want["key"])
    for i, (k, rev, date, prio) in enumerate(rows):
        assert k == want["key"][i]
        assert int(rev.scaleb(4)) == want["revenue"][i]  # DECIMAL(38,4), exact
        assert (date - __import__("datetime").date(1970, 1, 1)).days == want["date"][i]
        assert prio == want["prio"][i]
    return r


@pytest.mark.gpu
@pytest.mark.parametrize("scale", [0.001, 0.01])
def test_c4_pipeline_small(conn, scale):
    init(conn)
    t = W.q3(n_cust=int(1_500_000 * scale), n_ord=int(15_000_000 * scale), seed_salt=int(scale * 1000))
    W.register_q3(conn, t)
    q3_check(conn, t, limit=10)
    q3_check(conn, t, limit=1000)


@pytest.mark.gpu
def test_c4_pipeline_full_size(conn):
    init(conn, "16 GB", "16 GB")
    t = W.q3()
    W.register_q3(conn, t, upload=True)
    q3_check(conn, t, limit=10)


@pytest.mark.gpu
def test_prepared_statement_replays(conn):
    init(conn)
    t = W.q3(n_cust=15000, n_ord=150000, seed_salt=3)
    W.register_q3(conn, t)
    st = conn.prepare(W.q3_sql(t.date))
    assert st.kernel_count() >= 3
    outs = []
    for _ in range(3):
        st.launch()
        outs.append(st.fetch().fetchall())
    assert outs[0] == outs[1] == outs[2]
    assert outs[0] == conn.gpu_processing(W.q3_sql(t.date)).fetchall()
    st.close()


# ------------------------------------------------------------------ errors
@pytest.mark.gpu
def test_integer_overflow_is_an_error(conn):
    init(conn)
    conn.create_table("n", {"x": (L.T_INTEGER, np.array([1, 2, 2_000_000_000], np.int32))})
    conn.gpu_register_table("n")
    with pytest.raises(MettleError) as e:
        conn.gpu_processing("SELECT x * 10 FROM n")
    assert e.value.code == L.OVERFLOW
    assert conn.gpu_processing("SELECT x * 10 FROM n WHERE x < 10").fetchall() == [(10,), (20,)]


@pytest.mark.gpu
def test_unsupported_shapes(conn):
    init(conn)
    conn.create_table("n", {"x": (L.T_INTEGER, np.arange(10, dtype=np.int32))})
    conn.gpu_register_table("n")
    for sql in ["SELECT x FROM n WHERE x > 1 OR x < 0", "SELECT DISTINCT x FROM n",
                "SELECT x FROM n WHERE x IN (1, 2)", "WITH a AS (SELECT x FROM n) SELECT x FROM a",
                "SELECT x FROM missing_table"]:
        with pytest.raises(MettleError) as e:
            conn.gpu_processing(sql)
        assert e.value.code == L.UNSUPPORTED, sql


@pytest.mark.gpu
def test_budget_exceeded(conn):
    conn.execute("CALL gpu_buffer_init('64 KB', '64 KB', pinned_memory_size = '64 MB')")
    conn.create_table("big", {"x": (L.T_BIGINT, np.arange(100_000, dtype=np.int64))})
    conn.gpu_register_table("big")
    with pytest.raises(MettleError) as e:
        conn.gpu_processing("SELECT x FROM big WHERE x > 5")
    assert e.value.code == L.BUDGET_EXCEEDED
