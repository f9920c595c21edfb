"""The autotuner (mtl_autotune): it measures CTAs per SM, the rows a warp
takes per step and the hash load factor for a query's steps, keeps the
fastest per device in a file, and every query compiled afterwards uses them.
Launch shapes and capacities change speed only: results must stay exact
under any of them, including the extreme ones written into the table here."""
import re

import pytest

import oracle as orc
from mettle_b200 import Connection
from mettle_b200 import workloads as W


def _q3_rows(res):
    return [(r[0], int(r[1].scaleb(4)), r[3]) for r in res.fetchall()]


def _want(t):
    w = orc.q3(t, segment_code=1, limit=10)
    return list(zip(w["key"].tolist(), w["revenue"], w["prio"].tolist()))


@pytest.mark.gpu
@pytest.mark.parametrize("keys", ["dense", "sparse32"])
def test_autotune_writes_a_table_that_later_queries_use(tmp_path, monkeypatch, built_lib, keys):
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("METTLE_TUNE_FILE", str(path))
    t = W.q3(n_cust=30_000, n_ord=300_000, seed_salt=2, keys=keys)
    sql = W.q3_sql(t.date)
    with Connection() as conn:
        conn.execute("CALL gpu_buffer_init('4 GB', '4 GB')")
        W.register_q3(conn, t)
        report = conn.autotune(sql, reps=2)
        assert "ctas_per_sm" in report and str(path) in report
        if keys == "sparse32":
            assert "chose load factor" in report
        assert _q3_rows(conn.gpu_processing(sql)) == _want(t)
    lines = path.read_text().splitlines()
    assert any(line.startswith("pipeline:") for line in lines)
    # the most extreme shapes and the smallest load factor, by hand: a new
    # context reads them and the result stays exact
    forced = []
    for line in lines:
        key, a, b = line.split()
        if key.startswith("pipeline:"):
            forced.append(f"{key} 1 1024")  # one CTA per SM, 1024 rows per warp step
        else:
            forced.append(f"{key} 1.5 0")
    path.write_text("\n".join(forced) + "\n")
    with Connection() as conn:
        conn.execute("CALL gpu_buffer_init('4 GB', '4 GB')")
        W.register_q3(conn, t)
        st = conn.prepare(sql)
        for _ in range(2):
            st.launch()
            assert _q3_rows(st.fetch()) == _want(t)
        st.close()


@pytest.mark.gpu
def test_autotuned_shapes_keep_group_by_and_scan_exact(tmp_path, monkeypatch, built_lib):
    import numpy as np
    from mettle_b200 import _lib as L
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("METTLE_TUNE_FILE", str(path))
    d = W.groupby(n=2_000_000, groups=300, dist="zipf", seed_salt=8)
    with Connection() as conn:
        conn.execute("CALL gpu_buffer_init('2 GB', '2 GB')")
        conn.create_table("t", {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]), "f": (L.T_FLOAT, d["f"])})
        conn.gpu_register_table("t")
        report = conn.autotune(W.C3_SQL, reps=1)
        # few groups: the one-pass and the partitioned aggregation are both measured
        assert "one-key aggregate" in report
    for rows in (512, 1024):
        text = path.read_text()
        path.write_text(re.sub(r"^(pipeline:\S+) \S+ \S+$", rf"\1 1 {rows}", text, flags=re.M))
        with Connection() as conn:
            conn.execute("CALL gpu_buffer_init('2 GB', '2 GB')")
            conn.create_table("t", {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]),
                                    "f": (L.T_FLOAT, d["f"])})
            conn.gpu_register_table("t")
            r = conn.gpu_processing(W.C3_SQL)
            want = orc.groupby_c3(d["k"], d["v"], d["f"], limit=100)
            assert np.array_equal(r.columns[0], want["k"]) and np.array_equal(r.columns[2], want["cnt"])


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["two_pass", "lookback_cta_tiles", "lookback_warp_tiles"])
def test_materialize_strategies_keep_row_order(tmp_path, monkeypatch, built_lib, variant):
    """Order-preserving compaction in two passes (count, scan, write: the
    default), or in one pass with a decoupled look-back over 1024-row CTA
    tiles or 256-row warp tiles (each warp with its own look-back), chosen
    through the autotuner's table: the same rows in the same order,
    bit-exact against the oracle."""
    import numpy as np
    from mettle_b200 import _lib as L
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("METTLE_TUNE_FILE", str(path))
    lines = []
    if variant != "two_pass":
        lines.append("materialize_strategy/n22 1 0")  # 3*10^6 rows: size class 2^22
    if variant == "lookback_warp_tiles":
        # the scan streams a, b and c (16 bytes per row)
        lines.append("pipeline:materialize/n22/s16/p0/a0 2 256")
    path.write_text("".join(x + "\n" for x in lines))
    d = W.scan(3_000_000, seed_salt=4)
    sql = W.scan_sql("a", "<", 0.5)
    with Connection() as conn:
        conn.execute("CALL gpu_buffer_init('2 GB', '2 GB')")
        conn.create_table("t", {"a": (L.T_INTEGER, d["a"]), "b": (L.T_BIGINT, d["b"]), "c": (L.T_FLOAT, d["c"]),
                                "d": (L.T_DATE, d["d"]), "e": (L.T_TIMESTAMP, d["e"])})
        conn.gpu_register_table("t")
        st = conn.prepare(sql)
        st.set_profiling(True)
        st.launch()
        st.fetch()
        names = [n for n, _ in st.step_times()]
        st.close()
        if variant == "two_pass":
            assert "mat_scan" in names, names
        else:
            assert any(n.startswith("pipeline:materialize") for n in names), names
        r = conn.gpu_processing(sql)
        rows = orc.filter_rows([(d["a"], "<", int(0.5 * 2**31))])
        assert np.array_equal(r.columns[0], orc.gather(d["a"], rows))
        assert np.array_equal(r.columns[1], orc.gather(d["b"], rows, "+", 5))
        assert np.array_equal(r.columns[2], orc.gather(d["c"], rows, "*", np.float32(10)))
        assert np.array_equal(r.columns[4], orc.gather(d["e"], rows))


@pytest.mark.gpu
def test_autotune_measures_both_compactions(tmp_path, monkeypatch, built_lib):
    from mettle_b200 import _lib as L
    monkeypatch.setenv("METTLE_TUNE_FILE", str(tmp_path / "tune.txt"))
    d = W.scan(2_000_000, seed_salt=6)
    with Connection() as conn:
        conn.execute("CALL gpu_buffer_init('2 GB', '2 GB')")
        conn.create_table("t", {"a": (L.T_INTEGER, d["a"]), "b": (L.T_BIGINT, d["b"]), "c": (L.T_FLOAT, d["c"]),
                                "d": (L.T_DATE, d["d"]), "e": (L.T_TIMESTAMP, d["e"])})
        conn.gpu_register_table("t")
        report = conn.autotune(W.scan_sql("d", ">=", 0.1), reps=1)
        assert "compaction in one pass" in report and "compaction in two passes" in report
