"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference benchmarks on TPC-H data produced by DuckDB's dbgen
(test/generate_tpch.py); neither DuckDB nor the network is available, so
these generators stand in, with the table shapes, sizes and value
distributions of the five configurations (numpy PCG64, fixed seeds):

* ``numbers``   — one INTEGER column uniform in [0, 10^6) (the plain small query);
* ``scan``      — a INTEGER U[0, 2^31), b BIGINT U[-2^62, 2^62), c FLOAT U[0,1),
                  d DATE and e TIMESTAMP uniform over seven years (filter scan);
* ``groupby``   — k BIGINT with G distinct keys, uniform or Zipf(s), key ids
                  hashed over int64; v BIGINT U[0, 10^6); f FLOAT U[0,1);
* ``q3``        — customer / orders / lineitem of the join -> filter -> group
                  -> top-K pipeline, DECIMAL(15,2) money as int64 cents.
"""
from __future__ import annotations

import datetime as _dt
from dataclasses import dataclass

import numpy as np

SEED_BASE = 0x4D45_54544C45
DAY0 = (_dt.date(1992, 1, 1) - _dt.date(1970, 1, 1)).days  # 1992-01-01 as days since epoch
SPAN_DAYS = (_dt.date(1999, 1, 1) - _dt.date(1992, 1, 1)).days  # seven years = 2557 days
SEGMENTS = ["AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY"]  # sorted: code 1 = BUILDING


def rng(config: int, salt: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(SEED_BASE + config + 1000 * salt))


def day_to_iso(days: int) -> str:
    return (_dt.date(1970, 1, 1) + _dt.timedelta(days=int(days))).isoformat()


# ------------------------------------------------------------------ config 1
def numbers(n: int = 1_000_000, seed_salt: int = 0) -> dict[str, np.ndarray]:
    r = rng(1, seed_salt)
    return {"value": r.integers(0, 1_000_000, n, dtype=np.int32)}


C1_SQL = "SELECT value, value * 10 AS scaled FROM numbers WHERE value > 500000 ORDER BY value"


# ------------------------------------------------------------------ config 2
def scan(n: int = 100_000_000, seed_salt: int = 0) -> dict[str, np.ndarray]:
    r = rng(2, seed_salt)
    us_day = 86_400_000_000
    return {
        "a": r.integers(0, 2**31, n, dtype=np.int64).astype(np.int32),
        "b": r.integers(-(2**62), 2**62, n, dtype=np.int64),
        "c": r.random(n, dtype=np.float32),
        "d": (DAY0 + r.integers(0, SPAN_DAYS, n, dtype=np.int32)).astype(np.int32),
        "e": DAY0 * us_day + r.integers(0, SPAN_DAYS * us_day, n, dtype=np.int64),
    }


def scan_literal(col: str, sel: float) -> str:
    """Literal k so that `col < k` keeps about `sel` of the rows."""
    if col == "a":
        return str(int(sel * 2**31))
    if col == "b":
        return str(int(-(2**62) + sel * 2**63))
    if col == "c":
        return repr(float(sel))
    if col == "d":
        return f"DATE '{day_to_iso(DAY0 + int(sel * SPAN_DAYS))}'"
    if col == "e":
        us = int(sel * SPAN_DAYS * 86_400_000_000)
        t = _dt.datetime(1992, 1, 1) + _dt.timedelta(microseconds=us)
        return f"TIMESTAMP '{t.strftime('%Y-%m-%d %H:%M:%S')}'"
    raise ValueError(col)


def scan_sql(col: str = "a", op: str = "<", sel: float = 0.5) -> str:
    """Filter/projection template: SELECT a, b + 5, c * 10, d, e FROM t WHERE <col> <op> <k>."""
    lit = scan_literal(col, sel if op in ("<", "<=") else 1.0 - sel)
    return f"SELECT a, b + 5 AS b5, c * 10 AS c10, d, e FROM t WHERE {col} {op} {lit}"


# ------------------------------------------------------------------ config 3
def _mix64(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64)
    x ^= x >> np.uint64(33)
    x *= np.uint64(0xFF51AFD7ED558CCD)
    x ^= x >> np.uint64(33)
    x *= np.uint64(0xC4CEB9FE1A85EC53)
    x ^= x >> np.uint64(33)
    return x.view(np.int64)


def groupby(n: int = 200_000_000, groups: int = 1000, dist: str = "uniform", s: float = 1.1,
            seed_salt: int = 0) -> dict[str, np.ndarray]:
    r = rng(3, seed_salt)
    if dist == "uniform":
        ids = r.integers(0, groups, n, dtype=np.int64)
    elif dist == "zipf":
        # exact bounded Zipf(s) over `groups` ranks: multinomial counts, then a shuffle
        w = 1.0 / np.power(np.arange(1, groups + 1, dtype=np.float64), s)
        counts = r.multinomial(n, w / w.sum())
        ids = np.repeat(np.arange(groups, dtype=np.int64), counts)
        r.shuffle(ids)
    else:
        raise ValueError(dist)
    return {
        "k": _mix64(ids),
        "v": r.integers(0, 1_000_000, n, dtype=np.int64),
        "f": r.random(n, dtype=np.float32),
    }


C3_SQL = ("SELECT k, SUM(v) AS sum_v, COUNT(*) AS cnt, MIN(v) AS min_v, MAX(v) AS max_v, AVG(v) AS avg_v, "
          "SUM(f) AS sum_f, MIN(f) AS min_f, MAX(f) AS max_f, AVG(f) AS avg_f FROM t GROUP BY k "
          "ORDER BY sum_v DESC, k LIMIT 100")


# ------------------------------------------------------------------ config 4
@dataclass
class Q3Tables:
    customer: dict
    orders: dict
    lineitem: dict
    date: int

    @property
    def lineitem_rows(self) -> int:
        return len(self.lineitem["l_orderkey"])


def _sparse_keys(r: np.random.Generator, n: int, dtype) -> np.ndarray:
    """n distinct keys spread over the whole range of dtype (both extremes
    and -1 included when n allows), in random order."""
    info = np.iinfo(dtype)
    special = np.array([-1, info.min, info.max], dtype=np.int64)[: min(3, n)]
    k = np.unique(r.integers(info.min, info.max, n + n // 8 + 16, dtype=np.int64, endpoint=True))
    k = np.setdiff1d(k, special)
    k = np.concatenate([special, r.choice(k, n - len(special), replace=False)])
    r.shuffle(k)
    return k.astype(dtype)


def q3(n_cust: int = 1_500_000, n_ord: int = 15_000_000, seed_salt: int = 0, keys: str = "dense") -> Q3Tables:
    """keys="dense": custkey 1..n_cust and orderkey 1..n_ord (the direct-mapped
    joins); "sparse32" / "sparse64": distinct INTEGER / BIGINT keys spread over
    the whole type range (-1 and both extremes included), so both joins take
    the open-addressing hash tables."""
    r = rng(4, seed_salt)
    if keys == "dense":
        cust_keys = np.arange(1, n_cust + 1, dtype=np.int32)
        order_keys = np.arange(1, n_ord + 1, dtype=np.int32)
    elif keys in ("sparse32", "sparse64"):
        dt = np.int32 if keys == "sparse32" else np.int64
        kr = rng(40, seed_salt)
        cust_keys = _sparse_keys(kr, n_cust, dt)
        order_keys = _sparse_keys(kr, n_ord, dt)
    else:
        raise ValueError(keys)
    customer = {
        "c_custkey": cust_keys,
        "c_mktsegment": r.integers(0, len(SEGMENTS), n_cust, dtype=np.int32),
    }
    orderdate = (DAY0 + r.integers(0, SPAN_DAYS, n_ord, dtype=np.int32)).astype(np.int32)
    orders = {
        "o_orderkey": order_keys,
        "o_custkey": cust_keys[r.integers(0, n_cust, n_ord)],
        "o_orderdate": orderdate,
        "o_shippriority": np.zeros(n_ord, dtype=np.int32),
    }
    lines = r.integers(1, 8, n_ord, dtype=np.int32)  # 1..7 lines per order, drawn first
    n_li = int(lines.sum())
    li_order = np.repeat(np.arange(n_ord, dtype=np.int64), lines)
    lineitem = {
        "l_orderkey": orders["o_orderkey"][li_order],
        "l_extendedprice": r.integers(90_000, 10_500_001, n_li, dtype=np.int64),
        "l_discount": r.integers(0, 11, n_li, dtype=np.int64),
        "l_shipdate": (orderdate[li_order] + r.integers(1, 122, n_li, dtype=np.int32)).astype(np.int32),
    }
    return Q3Tables(customer, orders, lineitem, DAY0 + SPAN_DAYS // 2)


def q3_sql(date: int, segment: str = "BUILDING", limit: int = 10) -> str:
    d = day_to_iso(date)
    return ("SELECT l_orderkey, SUM(l_extendedprice * (1 - l_discount)) AS revenue, o_orderdate, o_shippriority "
            "FROM customer, orders, lineitem "
            f"WHERE c_mktsegment = '{segment}' AND c_custkey = o_custkey AND l_orderkey = o_orderkey "
            f"AND o_orderdate < DATE '{d}' AND l_shipdate > DATE '{d}' "
            "GROUP BY l_orderkey, o_orderdate, o_shippriority "
            f"ORDER BY revenue DESC, o_orderdate LIMIT {limit}")


def q3_bytes(t: Q3Tables) -> int:
    """Algorithmic bytes of one config-4 query: every column the query names, read once."""
    kw = t.orders["o_orderkey"].dtype.itemsize
    return (len(t.customer["c_custkey"]) * (kw + 4) + len(t.orders["o_orderkey"]) * (kw + kw + 4 + 4)
            + t.lineitem_rows * (kw + 8 + 8 + 4))


def register_q3(conn, t: Q3Tables, upload: bool = True, borrow: bool = False):
    from . import _lib as L
    kt = L.T_BIGINT if t.orders["o_orderkey"].dtype == np.int64 else L.T_INTEGER
    conn.create_table("customer", {"c_custkey": (kt, t.customer["c_custkey"]),
                                   "c_mktsegment": (L.T_VARCHAR, t.customer["c_mktsegment"], SEGMENTS)})
    conn.create_table("orders", {"o_orderkey": (kt, t.orders["o_orderkey"]),
                                 "o_custkey": (kt, t.orders["o_custkey"]),
                                 "o_orderdate": (L.T_DATE, t.orders["o_orderdate"]),
                                 "o_shippriority": (L.T_INTEGER, t.orders["o_shippriority"])})
    conn.create_table("lineitem", {"l_orderkey": (kt, t.lineitem["l_orderkey"]),
                                   "l_extendedprice": (L.T_DECIMAL, t.lineitem["l_extendedprice"], 2),
                                   "l_discount": (L.T_DECIMAL, t.lineitem["l_discount"], 2),
                                   "l_shipdate": (L.T_DATE, t.lineitem["l_shipdate"])})
    for name in ("customer", "orders", "lineitem"):
        conn.gpu_register_table(name, upload=upload, borrow=borrow)


# ------------------------------------------------------------------ config 5
# Tables of the served mixed stream: (name, template, rows, generator kwargs).
SERVED_TABLES = [
    ("numbers", "c1", 1_000_000, {}),
    ("s1m", "c2", 1_000_000, {}),
    ("s10m", "c2", 10_000_000, {}),
    ("s60m", "c2", 60_000_000, {}),
    ("g1m", "c3", 1_000_000, {"groups": 1000, "dist": "uniform"}),
    ("g10m", "c3", 10_000_000, {"groups": 1_000_000, "dist": "zipf"}),
    ("g60m", "c3", 60_000_000, {"groups": 1000, "dist": "zipf"}),
]


def served_tables(salt: int = 5) -> dict[str, tuple[str, dict[str, np.ndarray]]]:
    out = {}
    for i, (name, tpl, n, kw) in enumerate(SERVED_TABLES):
        if tpl == "c1":
            out[name] = (tpl, numbers(n, seed_salt=salt + i))
        elif tpl == "c2":
            out[name] = (tpl, scan(n, seed_salt=salt + i))
        else:
            out[name] = (tpl, groupby(n, seed_salt=salt + i, **kw))
    return out


def _scan_value(col: str, q: float):
    """Numeric literal at quantile q of a scan column and its SQL spelling."""
    if col == "a":
        v = int(q * 2**31)
        return v, str(v)
    if col == "b":
        v = int(-(2**62) + q * 2**63)
        return v, str(v)
    if col == "c":
        # two-digit DECIMAL literal; compared as FLOAT(digits) / FLOAT(100)
        digits = int(round(q * 100))
        v = float(np.float32(digits) / np.float32(100))
        return v, f"{digits // 100}.{digits % 100:02d}"
    if col == "d":
        v = DAY0 + int(q * SPAN_DAYS)
        return v, f"DATE '{day_to_iso(v)}'"
    us_day = 86_400_000_000
    v = DAY0 * us_day + int(q * SPAN_DAYS * us_day) // 1_000_000 * 1_000_000
    t = _dt.datetime(1970, 1, 1) + _dt.timedelta(microseconds=v)
    return v, f"TIMESTAMP '{t.strftime('%Y-%m-%d %H:%M:%S')}'"


def served_stream(n: int = 2000, seed: int = 7) -> list[dict]:
    """The mixed query stream: templates of the plain small query, the scan
    and the grouped aggregate, with seeded constants and tables of 10^6 to
    6*10^7 rows. Each entry holds the SQL and the numeric form of its
    constants (for the CPU oracle)."""
    r = np.random.default_rng(seed)
    scans = [t for t, tpl, _, _ in SERVED_TABLES if tpl == "c2"]
    groups = [t for t, tpl, _, _ in SERVED_TABLES if tpl == "c3"]
    out = []
    for i in range(n):
        kind = int(r.integers(0, 3))
        if kind == 0:
            k = int(r.integers(0, 1_000_000))
            out.append({"tpl": "c1", "table": "numbers", "k": k,
                        "sql": f"SELECT value, value * 10 AS scaled FROM numbers WHERE value > {k} ORDER BY value"})
        elif kind == 1:
            table = scans[int(r.integers(0, len(scans)))]
            col = "abcde"[int(r.integers(0, 5))]
            op = ["<", "<=", ">", ">="][int(r.integers(0, 4))]
            sel = float(r.choice([0.01, 0.1, 0.5]))
            v, lit = _scan_value(col, sel if op in ("<", "<=") else 1.0 - sel)
            out.append({"tpl": "c2", "table": table, "col": col, "op": op, "v": v,
                        "sql": f"SELECT a, b + 5 AS b5, c * 10 AS c10, d, e FROM {table} WHERE {col} {op} {lit}"})
        else:
            table = groups[int(r.integers(0, len(groups)))]
            lim = int(r.integers(10, 101))
            out.append({"tpl": "c3", "table": table, "limit": lim,
                        "sql": C3_SQL.replace("FROM t", f"FROM {table}").replace("LIMIT 100", f"LIMIT {lim}")})
    return out
