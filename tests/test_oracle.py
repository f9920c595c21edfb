"""The CPU oracle pinned against the reference's golden vectors and against
independent numpy/Python restatements (no GPU needed)."""
import datetime as dt
import json
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

from mettle_b200 import workloads as W

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_cases.json").read_text())


def days(s):
    return (dt.date.fromisoformat(s) - dt.date(1970, 1, 1)).days


def q3_tables(customers, orders, lineitems, date):
    """Small config-4 tables; money given in whole units is converted to cents."""
    seg = W.SEGMENTS
    cust = {"c_custkey": np.array([c[0] for c in customers], np.int32),
            "c_mktsegment": np.array([seg.index(c[1]) if c[1] in seg else 99 for c in customers], np.int32)}
    ords = {"o_orderkey": np.array([o[0] for o in orders], np.int32),
            "o_custkey": np.array([o[1] for o in orders], np.int32),
            "o_orderdate": np.array([days(o[2]) for o in orders], np.int32),
            "o_shippriority": np.array([o[3] for o in orders], np.int32)}
    li = {"l_orderkey": np.array([x[0] for x in lineitems], np.int32),
          "l_extendedprice": np.array([round(x[1] * 100) for x in lineitems], np.int64),
          "l_discount": np.array([round(x[2] * 100) for x in lineitems], np.int64),
          "l_shipdate": np.array([days(x[3]) for x in lineitems], np.int32)}
    return W.Q3Tables(cust, ords, li, days(date))


SIRIUS_CUSTOMER = [(1, "HOUSEHOLD"), (2, "AUTOMOBILE"), (3, "HOUSEHOLD")]
SIRIUS_ORDERS = [(101, 1, "1995-03-01", 1), (102, 2, "1995-03-01", 2), (103, 3, "1995-04-01", 3),
                 (104, 3, "1995-03-10", 2)]
SIRIUS_LINEITEM = [(101, 100.0, 0.10, "1995-04-01"), (101, 50.0, 0.00, "1995-04-03"),
                   (102, 80.0, 0.20, "1995-04-01"), (103, 70.0, 0.00, "1995-04-10"),
                   (104, 40.0, 0.25, "1995-02-01"), (104, 30.0, 0.10, "1995-04-10")]


def test_golden_records_present():
    recs = GOLDEN["sqllogic"]["tpch-sirius.test"]
    assert any("101 140.0 1995-03-01 1" in r.get("rows", []) for r in recs)


def test_oracle_q3_sirius_golden(oracle_lib):
    # test/sql/tpch-sirius.test:1-54 -> 101 140.0 1995-03-01 1 / 104 27.0 1995-03-10 2
    t = q3_tables(SIRIUS_CUSTOMER, SIRIUS_ORDERS, SIRIUS_LINEITEM, "1995-03-25")
    r = oracle_lib.q3(t, segment_code=W.SEGMENTS.index("HOUSEHOLD"), limit=10)
    assert list(r["key"]) == [101, 104]
    assert r["revenue"] == [1400000, 270000]  # scale 4: 140.0000, 27.0000
    assert [W.day_to_iso(d) for d in r["date"]] == ["1995-03-01", "1995-03-10"]
    assert list(r["prio"]) == [1, 2]


def test_oracle_q3_strict_boundaries(oracle_lib):
    # test/sql/tpch-sirius.test:55-87: orderdate = D and shipdate = D rows are excluded
    orders = SIRIUS_ORDERS + [(105, 1, "1995-03-25", 4), (106, 1, "1995-03-24", 5)]
    lineitem = SIRIUS_LINEITEM + [(105, 500.0, 0.00, "1995-03-26"), (106, 60.0, 0.00, "1995-03-25")]
    t = q3_tables(SIRIUS_CUSTOMER, orders, lineitem, "1995-03-25")
    r = oracle_lib.q3(t, segment_code=W.SEGMENTS.index("HOUSEHOLD"), limit=10)
    assert list(r["key"]) == [101, 104]
    assert r["revenue"] == [1400000, 270000]


def test_oracle_q3_extension_golden(oracle_lib):
    # tests/extension.rs:391-472 -> (100, 1400), (102, 240)
    cust = [(1, "BUILDING"), (2, "HOUSEHOLD"), (3, "BUILDING")]
    orders = [(100, 1, "1995-03-10", 0), (101, 2, "1995-03-20", 1), (102, 3, "1995-03-05", 0),
              (103, 1, "1995-04-01", 2)]
    li = [(100, 1000.0, 0.05, "1995-03-30"), (100, 500.0, 0.10, "1995-04-01"), (101, 200.0, 0.00, "1995-03-28"),
          (102, 300.0, 0.20, "1995-03-26"), (103, 800.0, 0.15, "1995-03-30")]
    t = q3_tables(cust, orders, li, "1995-03-25")
    r = oracle_lib.q3(t, segment_code=1, limit=10)
    assert list(r["key"]) == [100, 102]
    assert r["revenue"] == [14000000, 2400000]


def q3_python(t, seg, limit):
    """Independent dictionary restatement of the config-4 query."""
    ok_c = {int(k) for k, s in zip(t.customer["c_custkey"], t.customer["c_mktsegment"]) if s == seg}
    orders = {}
    for k, c, d, p in zip(*(t.orders[x] for x in ("o_orderkey", "o_custkey", "o_orderdate", "o_shippriority"))):
        if d < t.date and int(c) in ok_c:
            orders[int(k)] = (int(d), int(p))
    rev = {}
    for k, pr, di, sd in zip(*(t.lineitem[x] for x in ("l_orderkey", "l_extendedprice", "l_discount",
                                                        "l_shipdate"))):
        if sd > t.date and int(k) in orders:
            rev[int(k)] = rev.get(int(k), 0) + int(pr) * (100 - int(di))
    rows = sorted(((-v, orders[k][0], k, v) for k, v in rev.items()))
    return [(r[2], r[3], r[1]) for r in rows[:limit]], len(rev)


def test_oracle_q3_random_vs_python(oracle_lib):
    t = W.q3(n_cust=300, n_ord=3000, seed_salt=7)
    want, groups = q3_python(t, 1, 25)
    r = oracle_lib.q3(t, segment_code=1, limit=25)
    assert r["groups"] == groups
    assert list(zip(r["key"].tolist(), r["revenue"], r["date"].tolist())) == want


@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.float32, np.float64])
@pytest.mark.parametrize("op", ["=", "<", "<=", ">", ">="])
def test_oracle_filter_vs_numpy(oracle_lib, dtype, op):
    r = np.random.default_rng(3)
    col = (r.integers(-50, 50, 5000) if np.dtype(dtype).kind == "i" else r.integers(-50, 50, 5000) / 4).astype(dtype)
    lit = 7 if np.dtype(dtype).kind == "i" else 1.75
    got = oracle_lib.filter_rows([(col, op, lit)])
    f = {"=": np.equal, "<": np.less, "<=": np.less_equal, ">": np.greater, ">=": np.greater_equal}[op]
    assert np.array_equal(got, np.nonzero(f(col, dtype(lit)))[0])


def test_oracle_filter_golden(oracle_lib):
    # tests/extension.rs:62-92: value > 2 over 1..5 -> 3, 4, 5
    col = np.array([1, 2, 3, 4, 5], np.int32)
    rows = oracle_lib.filter_rows([(col, ">", 2)])
    assert col[rows].tolist() == [3, 4, 5]
    # tests/extension.rs:132-162: x > 1 AND y < 50
    x = np.array([1, 2, 3, 4, 5], np.int32)
    y = np.array([10, 20, 30, 40, 50], np.int32)
    rows = oracle_lib.filter_rows([(x, ">", 1), (y, "<", 50)])
    assert list(zip(x[rows].tolist(), y[rows].tolist())) == [(2, 20), (3, 30), (4, 40)]


def test_oracle_projection_overflow(oracle_lib):
    col = np.array([1, 2, 300_000_000], np.int32)
    rows = np.arange(3)
    with pytest.raises(OverflowError):
        oracle_lib.gather(col, rows, "*", 10)
    assert oracle_lib.gather(col[:2], rows[:2], "*", 10).tolist() == [10, 20]


def test_oracle_sort_stable(oracle_lib):
    key = np.array([3, 1, 3, 2, 1], np.int32)
    rows = np.arange(5)
    assert oracle_lib.sort_rows(key, rows).tolist() == [1, 4, 3, 0, 2]
    assert oracle_lib.sort_rows(key, rows, desc=True).tolist() == [0, 2, 3, 1, 4]


def x87_avg(total: int, count: int) -> float:
    """(long double)total / (long double)count rounded to double, from first principles."""
    q = Fraction(total, count)
    if q == 0:
        return 0.0
    sign = -1 if q < 0 else 1
    q = abs(q)
    e = q.numerator.bit_length() - q.denominator.bit_length()
    while Fraction(2) ** e > q:
        e -= 1
    while Fraction(2) ** (e + 1) <= q:
        e += 1
    def rnd(x: Fraction, bits: int, exp: int) -> Fraction:
        scaled = x / Fraction(2) ** (exp - bits + 1)
        fl = scaled.numerator // scaled.denominator
        rem = scaled - fl
        if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and fl % 2 == 1):
            fl += 1
        return Fraction(fl) * Fraction(2) ** (exp - bits + 1)
    ld = rnd(q, 64, e)
    e2 = e + (1 if ld >= Fraction(2) ** (e + 1) else 0)
    d = rnd(ld, 53, e2)
    return sign * float(d)


def test_oracle_avg_matches_x87_model(oracle_lib):
    r = np.random.default_rng(11)
    for _ in range(2000):
        count = int(r.integers(1, 10**9))
        total = int(r.integers(-(10**18), 10**18))
        assert oracle_lib.avg_i128(total, count) == x87_avg(total, count)


def test_oracle_groupby_vs_python(oracle_lib):
    d = W.groupby(n=20000, groups=300, dist="zipf", seed_salt=2)
    res = oracle_lib.groupby_c3(d["k"], d["v"], d["f"], limit=-1)
    ref = {}
    for k, v, f in zip(d["k"].tolist(), d["v"].tolist(), d["f"].tolist()):
        g = ref.setdefault(k, [0, 0, 10**9, -1, Fraction(0), 2.0, -1.0])
        g[0] += v; g[1] += 1; g[2] = min(g[2], v); g[3] = max(g[3], v)
        g[4] += Fraction(f); g[5] = min(g[5], f); g[6] = max(g[6], f)
    assert res["groups"] == len(ref)
    assert res["k"].tolist() == sorted(ref)
    for i, k in enumerate(res["k"].tolist()):
        s, c, mn, mx, sf, mnf, mxf = ref[k]
        assert res["sum_v"][i] == s and res["cnt"][i] == c
        assert res["min_v"][i] == mn and res["max_v"][i] == mx
        assert res["avg_v"][i] == x87_avg(s, c)
        assert abs(res["sum_f"][i] - float(sf)) <= 1e-12 * max(1.0, float(sf))
        assert res["min_f"][i] == np.float32(mnf) and res["max_f"][i] == np.float32(mxf)


def test_oracle_groupby_topk_order(oracle_lib):
    k = np.array([5, 3, 5, 3, 9, 1], np.int64)
    v = np.array([10, 20, 10, 0, 20, 1], np.int64)
    f = np.zeros(6, np.float32)
    res = oracle_lib.groupby_c3(k, v, f, limit=3)
    # sums: 5 -> 20, 3 -> 20, 9 -> 20, 1 -> 1; ties broken by k ascending
    assert res["k"].tolist() == [3, 5, 9]


def test_civil_dates(oracle_lib):
    L = oracle_lib.lib()
    for y, m, d in [(1970, 1, 1), (1995, 3, 25), (2000, 2, 29), (1969, 12, 31), (1600, 3, 1)]:
        assert L.orc_days_from_civil(y, m, d) == (dt.date(y, m, d) - dt.date(1970, 1, 1)).days
