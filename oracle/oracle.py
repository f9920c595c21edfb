"""Python wrapper of the CPU oracle (oracle/libmettle_oracle.so).

TEST INFRASTRUCTURE: the parity checker and the CPU baseline. Only tests/,
__graft_entry__.smoke() and bench.py's CPU legs import this module; the
product never does. See mettle_oracle.h for the semantics restated and the
reference files each function follows.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libmettle_oracle.so"
_lib = None

ORC_I32, ORC_I64, ORC_F32, ORC_F64 = 1, 2, 3, 4
OPS = {"=": 0, "<": 1, "<=": 2, ">": 3, ">=": 4}


def build() -> Path:
    """Compiles the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        P = C.c_void_p
        _lib.orc_filter.restype = C.c_int64
        _lib.orc_filter.argtypes = [C.c_int32, P, P, P, P, P, C.c_int64, P]
        for n in ("orc_gather_i32", "orc_gather_i64", "orc_gather_f32"):
            getattr(_lib, n).restype = C.c_int32
            getattr(_lib, n).argtypes = [P, P, C.c_int64, P]
        for n, kt in (("orc_gather_i32_mul", C.c_int32), ("orc_gather_i32_add", C.c_int32),
                      ("orc_gather_i64_add", C.c_int64), ("orc_gather_i64_mul", C.c_int64),
                      ("orc_gather_f32_mul", C.c_float)):
            getattr(_lib, n).restype = C.c_int32
            getattr(_lib, n).argtypes = [P, P, C.c_int64, kt, P]
        for n in ("orc_sort_rows_i32", "orc_sort_rows_i64"):
            getattr(_lib, n).restype = None
            getattr(_lib, n).argtypes = [P, P, C.c_int64, C.c_int32]
        _lib.orc_groupby_c3.restype = C.c_int64
        _lib.orc_groupby_c3.argtypes = [P, P, P, C.c_int64, C.c_int64, P] + [P] * 11
        _lib.orc_avg_i128.restype = C.c_double
        _lib.orc_avg_i128.argtypes = [C.c_uint64, C.c_int64, C.c_int64]
        _lib.orc_q3.restype = C.c_int64
        _lib.orc_q3.argtypes = [P, P, C.c_int64, P, P, P, P, C.c_int64, P, P, P, P, C.c_int64, C.c_int32,
                                C.c_int32, C.c_int64, P, P, P, P, P, P]
        _lib.orc_days_from_civil.restype = C.c_int32
        _lib.orc_days_from_civil.argtypes = [C.c_int32] * 3
        _lib.orc_threads.restype = C.c_int32
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


_TYPE = {np.dtype(np.int32): ORC_I32, np.dtype(np.int64): ORC_I64, np.dtype(np.float32): ORC_F32,
         np.dtype(np.float64): ORC_F64}


def filter_rows(preds: list[tuple[np.ndarray, str, float | int]]) -> np.ndarray:
    """Ascending row ids where every (column, op, literal) holds."""
    n = len(preds[0][0]) if preds else 0
    cols = (C.c_void_p * len(preds))(*[_p(p[0]) for p in preds])
    types = np.array([_TYPE[p[0].dtype] for p in preds], dtype=np.int32)
    ops = np.array([OPS[p[1]] for p in preds], dtype=np.int32)
    il = np.array([int(p[2]) if p[0].dtype.kind == "i" else 0 for p in preds], dtype=np.int64)
    fl = np.array([float(p[2]) for p in preds], dtype=np.float64)
    out = np.empty(max(n, 1), dtype=np.int64)
    k = lib().orc_filter(len(preds), cols, _p(types), _p(ops), _p(il), _p(fl), n, _p(out))
    return out[:k].copy()


def gather(col: np.ndarray, rows: np.ndarray, op: str | None = None, k=None) -> np.ndarray:
    """col[rows] (op None), or col[rows] op k with DuckDB types; raises OverflowError."""
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    out = np.empty(len(rows), dtype=col.dtype)
    L = lib()
    name = {np.dtype(np.int32): "i32", np.dtype(np.int64): "i64", np.dtype(np.float32): "f32"}[col.dtype]
    if op is None:
        rc = getattr(L, f"orc_gather_{name}")(_p(col), _p(rows), len(rows), _p(out))
    else:
        fn = getattr(L, f"orc_gather_{name}_{'add' if op == '+' else 'mul'}")
        rc = fn(_p(col), _p(rows), len(rows), k, _p(out))
    if rc:
        raise OverflowError("Overflow in integer arithmetic")
    return out


def sort_rows(key: np.ndarray, rows: np.ndarray, desc: bool = False) -> np.ndarray:
    rows = np.ascontiguousarray(rows, dtype=np.int64).copy()
    fn = lib().orc_sort_rows_i32 if key.dtype == np.int32 else lib().orc_sort_rows_i64
    fn(_p(key), _p(rows), len(rows), 1 if desc else 0)
    return rows


def groupby_c3(k: np.ndarray, v: np.ndarray, f: np.ndarray, limit: int = 100) -> dict[str, np.ndarray]:
    """Config-3 aggregate; limit < 0 returns every group ordered by k."""
    n = len(k)
    cap = n if limit < 0 else min(limit, n)
    cap = max(cap, 1)
    o = {"k": np.empty(cap, np.int64), "sum_lo": np.empty(cap, np.uint64), "sum_hi": np.empty(cap, np.int64),
         "cnt": np.empty(cap, np.int64), "min_v": np.empty(cap, np.int64), "max_v": np.empty(cap, np.int64),
         "avg_v": np.empty(cap, np.float64), "sum_f": np.empty(cap, np.float64),
         "min_f": np.empty(cap, np.float32), "max_f": np.empty(cap, np.float32),
         "avg_f": np.empty(cap, np.float64)}
    ng = C.c_int64(0)
    m = lib().orc_groupby_c3(_p(k), _p(v), _p(f), n, limit, C.addressof(ng),
                             *[_p(o[x]) for x in ("k", "sum_lo", "sum_hi", "cnt", "min_v", "max_v", "avg_v",
                                                  "sum_f", "min_f", "max_f", "avg_f")])
    out = {key: val[:m].copy() for key, val in o.items()}
    out["sum_v"] = [(int(h) << 64) | int(lo) for lo, h in zip(out["sum_lo"], out["sum_hi"])]
    out["groups"] = ng.value
    return out


def avg_i128(total: int, count: int) -> float:
    return lib().orc_avg_i128(total & ((1 << 64) - 1), total >> 64, count)


def q3(t, segment_code: int = 1, limit: int = 10) -> dict:
    """Config-4 pipeline on a workloads.Q3Tables; revenue at scale 4 as python ints."""
    c, o, li = t.customer, t.orders, t.lineitem
    cap = max(1, len(o["o_orderkey"]) if limit < 0 else limit)
    out = {"key": np.empty(cap, np.int32), "lo": np.empty(cap, np.uint64), "hi": np.empty(cap, np.int64),
           "date": np.empty(cap, np.int32), "prio": np.empty(cap, np.int32)}
    ng = C.c_int64(0)
    m = lib().orc_q3(_p(c["c_custkey"]), _p(c["c_mktsegment"]), len(c["c_custkey"]),
                     _p(o["o_orderkey"]), _p(o["o_custkey"]), _p(o["o_orderdate"]), _p(o["o_shippriority"]),
                     len(o["o_orderkey"]), _p(li["l_orderkey"]), _p(li["l_extendedprice"]), _p(li["l_discount"]),
                     _p(li["l_shipdate"]), len(li["l_orderkey"]), segment_code, t.date, limit, C.addressof(ng),
                     _p(out["key"]), _p(out["lo"]), _p(out["hi"]), _p(out["date"]), _p(out["prio"]))
    res = {k: v[:m].copy() for k, v in out.items()}
    res["revenue"] = [(int(h) << 64) | int(lo) for lo, h in zip(res["lo"], res["hi"])]
    res["groups"] = ng.value
    return res


def threads() -> int:
    return int(lib().orc_threads())


def _lookup(keys: np.ndarray, probe: np.ndarray) -> np.ndarray:
    """Row of each probe value in `keys` (distinct values), -1 when absent."""
    o = np.argsort(keys, kind="stable")
    s = keys[o]
    if len(s) == 0:
        return np.full(len(probe), -1, np.int64)
    i = np.minimum(np.searchsorted(s, probe), len(s) - 1)
    return np.where(s[i] == probe, o[i], -1)


def q3_numpy(t, limit: int = 10, segment_code: int = 1) -> list[tuple]:
    """Config-4 pipeline in numpy for keys of any integer width (orc_q3 takes
    INTEGER keys only): rows (orderkey, revenue at scale 4, orderdate,
    shippriority) ordered by revenue DESC, orderdate, orderkey. Same
    relational result as orc_q3; revenue per order fits int64 here (at most
    7 lines of at most 10,500,000 x 100)."""
    c, o, li = t.customer, t.orders, t.lineitem
    qual_cust = c["c_custkey"][c["c_mktsegment"] == segment_code]
    om = (o["o_orderdate"] < t.date) & np.isin(o["o_custkey"], qual_cust)
    ok = o["o_orderkey"][om]
    row = _lookup(ok, li["l_orderkey"])
    lm = (row >= 0) & (li["l_shipdate"] > t.date)
    keys, inv = np.unique(li["l_orderkey"][lm], return_inverse=True)
    rev = np.zeros(len(keys), np.int64)
    np.add.at(rev, inv, li["l_extendedprice"][lm] * (100 - li["l_discount"][lm]))
    orow = np.flatnonzero(om)[_lookup(ok, keys)]
    date = o["o_orderdate"][orow]
    prio = o["o_shippriority"][orow]
    order = np.lexsort((keys, date, -rev))
    if limit >= 0:
        order = order[:limit]
    return [(int(keys[i]), int(rev[i]), int(date[i]), int(prio[i])) for i in order]
