"""The SQL surface of the extension, mirrored over the C ABI.

The reference registers table functions on a DuckDB connection
(src/lib.rs:31-39): ``gpu_buffer_init``, ``gpu_register_table``,
``gpu_cache_status``, ``gpu_cache_reset`` and ``gpu_processing``. DuckDB is
not part of this build, so ``Connection`` plays the host role: it keeps a
small host catalog of tables (``CREATE TABLE`` / ``INSERT`` statements or
numpy arrays — the stand-in for DuckDB's catalog that ``gpu_register_table``
scans, src/pinned.rs:187-244) and routes ``CALL gpu_*`` statements to the
library. Queries handed to ``gpu_processing`` always run on the GPU; SQL
outside the offloaded subset raises ``MettleError`` with status UNSUPPORTED
(the reference falls back to DuckDB's CPU path there, src/processing.rs:
140-155, which a DuckDB host would do on that status).
"""
from __future__ import annotations

import ctypes as C
import datetime as _dt
import decimal
import re
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from ._lib import MettleError

EPOCH = _dt.date(1970, 1, 1)
EPOCH_TS = _dt.datetime(1970, 1, 1)

_TYPE_NAMES = {
    "integer": L.T_INTEGER, "int": L.T_INTEGER, "int4": L.T_INTEGER, "int32": L.T_INTEGER,
    "bigint": L.T_BIGINT, "int8": L.T_BIGINT, "int64": L.T_BIGINT, "long": L.T_BIGINT,
    "float": L.T_FLOAT, "real": L.T_FLOAT, "float4": L.T_FLOAT,
    "double": L.T_DOUBLE, "float8": L.T_DOUBLE,
    "date": L.T_DATE, "timestamp": L.T_TIMESTAMP, "datetime": L.T_TIMESTAMP,
    "varchar": L.T_VARCHAR, "text": L.T_VARCHAR, "string": L.T_VARCHAR,
    "decimal": L.T_DECIMAL, "numeric": L.T_DECIMAL,
}
_NP = {L.T_INTEGER: np.int32, L.T_BIGINT: np.int64, L.T_FLOAT: np.float32, L.T_DOUBLE: np.float64,
       L.T_DATE: np.int32, L.T_TIMESTAMP: np.int64, L.T_DECIMAL: np.int64, L.T_VARCHAR: np.int32}


def date_to_days(s: str) -> int:
    y, m, d = (int(x) for x in s.strip().split("-"))
    return (_dt.date(y, m, d) - EPOCH).days


def ts_to_micros(s: str) -> int:
    s = s.strip()
    fmt = "%Y-%m-%d %H:%M:%S.%f" if "." in s else ("%Y-%m-%d %H:%M:%S" if " " in s else "%Y-%m-%d")
    t = _dt.datetime.strptime(s, fmt)
    delta = t - EPOCH_TS
    return (delta.days * 86400 + delta.seconds) * 1_000_000 + delta.microseconds


@dataclass
class HostColumn:
    name: str
    type: int
    scale: int = 0
    values: list = field(default_factory=list)  # python values before materialization
    array: np.ndarray | None = None
    dictionary: list[str] | None = None

    def materialize(self) -> np.ndarray:
        if self.array is not None:
            return self.array
        if self.type == L.T_VARCHAR:
            d = sorted(set(self.values))
            idx = {v: i for i, v in enumerate(d)}
            self.dictionary = d
            self.array = np.array([idx[v] for v in self.values], dtype=np.int32)
        else:
            self.array = np.array(self.values, dtype=_NP[self.type])
        return self.array


@dataclass
class HostTable:
    name: str
    columns: list[HostColumn]

    @property
    def rows(self) -> int:
        if not self.columns:
            return 0
        c = self.columns[0]
        return len(c.array) if c.array is not None else len(c.values)


class _ResultOwner:
    """Frees the native result once no column view refers to it."""

    def __init__(self, lib, handle):
        self.lib, self.handle = lib, handle

    def __del__(self):
        if self.handle:
            try:
                self.lib.mtl_result_free(self.handle)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None


def _view(owner, ptr, nbytes, dtype):
    """Zero-copy numpy view of native result bytes, keeping ``owner`` alive."""
    buf = (C.c_uint8 * nbytes).from_address(ptr)
    buf._owner = owner
    arr = np.frombuffer(buf, dtype=dtype)
    arr.flags.writeable = False  # cached results share these bytes
    return arr


class Result:
    """A gpu_processing result with numpy columns and DuckDB-typed rows.

    Columns are read-only views of the native result's page-locked host
    buffers (no copy); the native result is freed when the last view goes.
    """

    def __init__(self, lib, handle):
        self.names: list[str] = []
        self.types: list[tuple[int, int]] = []
        self.columns: list[np.ndarray] = []
        self.valid: list[np.ndarray | None] = []
        self.dicts: list[list[str] | None] = []
        owner = _ResultOwner(lib, handle)
        self.rows = int(lib.mtl_result_rows(handle))
        self.device_ms = float(lib.mtl_result_device_ms(handle))
        for i in range(lib.mtl_result_columns(handle)):
            scale = C.c_int32(0)
            t = lib.mtl_result_column_type(handle, i, C.byref(scale))
            self.names.append(lib.mtl_result_column_name(handle, i).decode())
            self.types.append((t, scale.value))
            width = 16 if t in (L.T_HUGEINT, L.T_DECIMAL128) else (
                4 if t in (L.T_INTEGER, L.T_DATE, L.T_FLOAT, L.T_VARCHAR) else 8)
            ptr = lib.mtl_result_column_data(handle, i)
            dt = {L.T_FLOAT: np.float32, L.T_DOUBLE: np.float64}.get(
                t, np.int32 if width == 4 else np.int64)
            if self.rows and ptr:
                arr = _view(owner, ptr, self.rows * width, dt)
            else:
                arr = np.zeros(0, dtype=dt)
            if width == 16:
                arr = arr.reshape(-1, 2)
            self.columns.append(arr)
            vp = lib.mtl_result_column_valid(handle, i)
            self.valid.append(_view(owner, vp, self.rows, np.uint8) if vp and self.rows else None)
            if t == L.T_VARCHAR:
                d = []
                mx = int(arr.max()) if arr.size else -1
                for k in range(mx + 1):
                    s = lib.mtl_result_dict(handle, i, k)
                    d.append(s.decode() if s is not None else None)
                self.dicts.append(d)
            else:
                self.dicts.append(None)

    def value(self, col: int, row: int):
        t, scale = self.types[col]
        v = self.valid[col]
        if v is not None and not v[row]:
            return None
        a = self.columns[col]
        if t in (L.T_HUGEINT, L.T_DECIMAL128):
            lo, hi = int(a[row, 0]) & ((1 << 64) - 1), int(a[row, 1])
            x = (hi << 64) | lo
            return decimal.Decimal(x).scaleb(-scale) if t == L.T_DECIMAL128 else x
        x = a[row]
        if t == L.T_DATE:
            return EPOCH + _dt.timedelta(days=int(x))
        if t == L.T_TIMESTAMP:
            return EPOCH_TS + _dt.timedelta(microseconds=int(x))
        if t == L.T_DECIMAL:
            return decimal.Decimal(int(x)).scaleb(-scale)
        if t == L.T_VARCHAR:
            return self.dicts[col][int(x)]
        if t in (L.T_FLOAT, L.T_DOUBLE):
            return float(x)
        return int(x)

    def fetchall(self) -> list[tuple]:
        return [tuple(self.value(c, r) for c in range(len(self.names))) for r in range(self.rows)]


class Rows:
    """A small relation returned by ``Connection.execute``."""

    def __init__(self, names, rows, result: Result | None = None):
        self.names = names
        self.rows = rows
        self.result = result

    def fetchall(self):
        return list(self.rows)

    def fetchone(self):
        return self.rows[0] if self.rows else None


_CALL = re.compile(r"^\s*CALL\s+(\w+)\s*\((.*)\)\s*;?\s*$", re.I | re.S)


def _split_args(s: str) -> list[str]:
    """Splits CALL arguments on top-level commas (quotes respected)."""
    out, cur, q = [], "", False
    i = 0
    while i < len(s):
        ch = s[i]
        if ch == "'":
            if q and i + 1 < len(s) and s[i + 1] == "'":
                cur += "''"
                i += 2
                continue
            q = not q
        if ch == "," and not q:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
        i += 1
    if cur.strip():
        out.append(cur.strip())
    return out


def _unquote(s: str) -> str:
    s = s.strip()
    if len(s) >= 2 and s[0] == "'" and s[-1] == "'":
        return s[1:-1].replace("''", "'")
    return s


def _split_statements(sql: str) -> list[str]:
    out, cur, q = [], "", False
    for ch in sql:
        if ch == "'":
            q = not q
        if ch == ";" and not q:
            if cur.strip():
                out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


class Connection:
    """One host connection: catalog + the extension's SQL surface."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        self.device = device
        self.ctx = None
        self.tables: dict[str, HostTable] = {}
        self.budgets: L.Budgets | None = None

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if self.ctx:
            # requests and statements hold context resources: release them first
            for obj in list(getattr(self, "_children", ())):
                obj.close()
            self.lib.mtl_ctx_destroy(self.ctx)
            self.ctx = None

    def _adopt(self, obj):
        import weakref
        if not hasattr(self, "_children"):
            self._children = weakref.WeakSet()
        self._children.add(obj)
        return obj

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        L.check(rc, self.ctx)

    # ------------------------------------------------------------ host catalog
    def create_table(self, name: str, columns: dict[str, tuple]):
        """Adds a table from numpy arrays: {col: (type, array[, scale | dictionary])}."""
        cols = []
        for cname, spec in columns.items():
            t = spec[0] if isinstance(spec[0], int) else _TYPE_NAMES[spec[0].lower()]
            arr = spec[1]
            hc = HostColumn(cname.lower(), t)
            if t == L.T_VARCHAR:
                hc.dictionary = list(spec[2])
                hc.array = np.ascontiguousarray(arr, dtype=np.int32)
            else:
                if t == L.T_DECIMAL:
                    hc.scale = int(spec[2]) if len(spec) > 2 else 0
                hc.array = np.ascontiguousarray(arr, dtype=_NP[t])
            cols.append(hc)
        self.tables[name.lower()] = HostTable(name.lower(), cols)

    def _create_sql(self, sql: str):
        m = re.match(r"^\s*CREATE\s+TABLE\s+(\w+)\s*\((.*)\)\s*$", sql, re.I | re.S)
        if not m:
            raise MettleError(L.INVALID, f"unsupported statement: {sql[:60]}")
        cols = []
        for part in _split_args(m.group(2)):
            pm = re.match(r"^(\w+)\s+(\w+)\s*(?:\(\s*(\d+)\s*(?:,\s*(\d+))?\s*\))?$", part.strip(), re.I)
            if not pm:
                raise MettleError(L.INVALID, f"bad column definition: {part}")
            t = _TYPE_NAMES.get(pm.group(2).lower())
            if t is None:
                raise MettleError(L.INVALID, f"unsupported column type {pm.group(2)}")
            scale = int(pm.group(4) or 0) if t == L.T_DECIMAL else 0
            if t == L.T_DECIMAL and pm.group(3) is None:
                scale = 3  # DuckDB's DECIMAL default is DECIMAL(18,3)
            cols.append(HostColumn(pm.group(1).lower(), t, scale))
        self.tables[m.group(1).lower()] = HostTable(m.group(1).lower(), cols)

    def _parse_value(self, tok: str, col: HostColumn):
        tok = tok.strip()
        up = tok.upper()
        if up.startswith("DATE "):
            return date_to_days(_unquote(tok[5:]))
        if up.startswith("TIMESTAMP "):
            return ts_to_micros(_unquote(tok[10:]))
        if tok.startswith("'"):
            s = _unquote(tok)
            if col.type == L.T_DATE:
                return date_to_days(s)
            if col.type == L.T_TIMESTAMP:
                return ts_to_micros(s)
            return s
        if col.type in (L.T_INTEGER, L.T_BIGINT):
            return int(tok)
        if col.type == L.T_DECIMAL:
            return int(decimal.Decimal(tok).scaleb(col.scale).to_integral_value(decimal.ROUND_HALF_UP))
        return float(tok)

    def _insert_sql(self, sql: str):
        m = re.match(r"^\s*INSERT\s+INTO\s+(\w+)\s+VALUES\s*(.*)$", sql, re.I | re.S)
        if not m:
            raise MettleError(L.INVALID, f"unsupported statement: {sql[:60]}")
        t = self.tables[m.group(1).lower()]
        body = m.group(2).strip()
        tuples, depth, cur, q = [], 0, "", False
        for ch in body:
            if ch == "'":
                q = not q
            if not q and ch == "(":
                depth += 1
                if depth == 1:
                    cur = ""
                    continue
            if not q and ch == ")":
                depth -= 1
                if depth == 0:
                    tuples.append(cur)
                    continue
            if depth >= 1:
                cur += ch
        for tup in tuples:
            vals = _split_args(tup)
            if len(vals) != len(t.columns):
                raise MettleError(L.INVALID, "INSERT arity mismatch")
            for c, v in zip(t.columns, vals):
                if c.array is not None:
                    # appending to a materialized column: back to python values
                    c.values = ([c.dictionary[int(x)] for x in c.array] if c.type == L.T_VARCHAR
                                else c.array.tolist())
                    c.array = None
                c.values.append(self._parse_value(v, c))

    # ------------------------------------------------------------ SQL surface
    def execute(self, sql: str) -> Rows:
        """Runs one or more ';'-separated statements; returns the last result."""
        last = Rows([], [])
        for stmt in _split_statements(sql):
            last = self._execute_one(stmt)
        return last

    def _execute_one(self, stmt: str) -> Rows:
        head = stmt.lstrip().split(None, 1)[0].upper()
        if head == "CREATE":
            self._create_sql(stmt)
            return Rows([], [])
        if head == "INSERT":
            self._insert_sql(stmt)
            return Rows([], [])
        m = _CALL.match(stmt)
        if not m:
            raise MettleError(L.UNSUPPORTED, "only CALL gpu_* statements are routed to the extension")
        fn, args = m.group(1).lower(), _split_args(m.group(2))
        if fn == "gpu_buffer_init":
            return self.gpu_buffer_init(*self._init_args(args))
        if fn == "gpu_register_table":
            return self.gpu_register_table(_unquote(args[0]))
        if fn == "gpu_processing":
            r = self.gpu_processing(_unquote(args[0]) if args else "")
            return Rows(r.names, r.fetchall(), r)
        if fn == "gpu_cache_status":
            return self.gpu_cache_status()
        if fn == "gpu_cache_reset":
            return self.gpu_cache_reset()
        if fn == "gpu_rewrite_query":
            return Rows(["rewritten"], [(self.gpu_rewrite_query(_unquote(args[0])),)])
        raise MettleError(L.UNSUPPORTED, f"unknown table function {fn}")

    @staticmethod
    def _init_args(args):
        pos, pinned = [], None
        for a in args:
            nm = re.match(r"^(\w+)\s*(?::=|=)\s*(.*)$", a, re.S)
            if nm and not a.strip().startswith("'"):
                if nm.group(1).lower() == "pinned_memory_size":
                    pinned = _unquote(nm.group(2))
                continue
            pos.append(_unquote(a))
        return (pos[0] if pos else "", pos[1] if len(pos) > 1 else "", pinned)

    def gpu_buffer_init(self, cache: str, processing: str, pinned_memory_size: str | None = None) -> Rows:
        """CALL gpu_buffer_init (src/table_functions.rs:26-123)."""
        b = L.Budgets()
        err = C.create_string_buffer(512)
        rc = self.lib.mtl_parse_buffer_config(cache.encode(), processing.encode(),
                                              pinned_memory_size.encode() if pinned_memory_size else None,
                                              C.byref(b), err, 512)
        if rc != L.OK:
            raise MettleError(rc, err.value.decode())
        if self.ctx:
            self.lib.mtl_ctx_destroy(self.ctx)
            self.ctx = None
        h = C.c_void_p()
        self._check(self.lib.mtl_ctx_create(C.byref(b), self.device, C.byref(h)))
        self.ctx = h
        self.budgets = b
        name = C.create_string_buffer(256)
        backend = C.create_string_buffer(256)
        self._check(self.lib.mtl_device_info(self.ctx, name, 256, backend, 256, None, None))
        cols = ["status", "device_name", "cache_region_bytes", "processing_region_bytes", "pinned_region_bytes",
                "metal_backend"]
        return Rows(cols, [("initialized", name.value.decode(), b.cache_region_bytes, b.processing_region_bytes,
                            b.pinned_region_bytes, backend.value.decode())])

    def _require_ctx(self):
        if not self.ctx:
            raise MettleError(L.NOT_INITIALIZED, "call gpu_buffer_init before gpu_processing")

    def gpu_register_table(self, name: str, upload: bool = False, borrow: bool = False) -> Rows:
        """CALL gpu_register_table (src/table_functions.rs:132-199)."""
        self._require_ctx()
        t = self.tables.get(name.lower())
        if t is None:
            raise MettleError(L.INVALID, f"Table with name {name} does not exist!")
        descs = (L.ColumnDesc * max(1, len(t.columns)))()
        keep = []
        for i, c in enumerate(t.columns):
            arr = c.materialize()
            keep.append(arr)
            descs[i].name = c.name.encode()
            descs[i].type = c.type
            descs[i].scale = c.scale
            descs[i].data = arr.ctypes.data if arr.size else None
            if c.type == L.T_VARCHAR:
                d = (C.c_char_p * max(1, len(c.dictionary)))(*[s.encode() for s in c.dictionary])
                keep.append(d)
                descs[i].dict = C.cast(d, C.POINTER(C.c_char_p))
                descs[i].dict_size = len(c.dictionary)
        summary = L.PinSummary()
        flags = (L.PIN_UPLOAD if upload else 0) | (L.PIN_BORROW if borrow else 0)
        if borrow:
            self._borrowed = getattr(self, "_borrowed", {})
            self._borrowed[name.lower()] = keep
        self._check(self.lib.mtl_table_register(self.ctx, name.lower().encode(), t.rows, len(t.columns), descs,
                                                flags, C.byref(summary)))
        return Rows(["table_name", "row_count", "byte_count", "skipped_columns"],
                    [(name, summary.row_count, summary.byte_count, summary.skipped_columns.decode())])

    def gpu_processing(self, sql: str) -> Result:
        """CALL gpu_processing (src/processing.rs:55-143); always runs on the GPU."""
        if not sql.strip():
            raise MettleError(L.INVALID, "gpu_processing requires a non-empty SQL string")
        self._require_ctx()
        h = C.c_void_p()
        self._check(self.lib.mtl_processing(self.ctx, sql.encode(), C.byref(h)))
        return Result(self.lib, h)

    def last_execution_mode(self) -> str | None:
        """state::last_execution_mode (src/state.rs:103-111)."""
        if not self.ctx:
            return None
        m = self.lib.mtl_last_execution_mode(self.ctx).decode()
        return m or None

    def gpu_cache_status(self) -> Rows:
        """CALL gpu_cache_status (src/table_functions.rs:201-390): 19 columns."""
        self._require_ctx()
        s = L.CacheStats()
        self._check(self.lib.mtl_cache_stats_get(self.ctx, C.byref(s)))
        names = ["last_execution_mode", "metal_entries", "metal_cached_bytes", "metal_hits", "metal_misses",
                 "metal_evictions", "metal_bypasses", "metal_input_entries", "metal_input_cached_bytes",
                 "metal_selection_entries", "metal_selection_cached_bytes", "metal_join_result_entries",
                 "metal_join_result_cached_bytes", "source_selection_entries", "source_selection_bytes",
                 "grouped_topk_entries", "grouped_topk_bytes", "query_result_entries", "query_result_bytes"]
        vals = [self.last_execution_mode() or ""] + [getattr(s, f) for f, _ in L.CacheStats._fields_]
        return Rows(names, [tuple(vals)])

    def gpu_cache_reset(self) -> Rows:
        """CALL gpu_cache_reset (src/table_functions.rs:399-433)."""
        self._require_ctx()
        self._check(self.lib.mtl_cache_reset(self.ctx))
        return Rows(["status"], [("reset",)])

    def gpu_rewrite_query(self, sql: str) -> str:
        buf = C.create_string_buffer(max(4096, 4 * len(sql) + 256))
        self._check(self.lib.mtl_rewrite_query(self.ctx, sql.encode(), buf, len(buf)))
        return buf.value.decode()

    # ------------------------------------------------------------ scalar hooks
    def _hook(self, compare: bool, op: int, values: np.ndarray, scalar, type_code: int):
        self._require_ctx()
        arr = np.ascontiguousarray(values, dtype=_NP[type_code])
        out = np.empty(arr.shape, dtype=np.uint8 if compare else arr.dtype)
        ilit = int(scalar) if type_code not in (L.T_FLOAT, L.T_DOUBLE) else 0
        flit = float(scalar)
        fn = self.lib.mtl_scalar_compare if compare else self.lib.mtl_scalar_arith
        self._check(fn(self.ctx, op, type_code, arr.ctypes.data, arr.size, ilit, flit, out.ctypes.data))
        return out.astype(bool) if compare else out

    def gpu_add_scalar(self, values, scalar, type_code=L.T_INTEGER):
        return self._hook(False, L.HOOK_ADD, values, scalar, type_code)

    def gpu_mul_scalar(self, values, scalar, type_code=L.T_INTEGER):
        return self._hook(False, L.HOOK_MUL, values, scalar, type_code)

    def gpu_eq_scalar(self, values, scalar, type_code=L.T_INTEGER):
        return self._hook(True, 0, values, scalar, type_code)

    def gpu_lt_scalar(self, values, scalar, type_code=L.T_INTEGER):
        return self._hook(True, 1, values, scalar, type_code)

    def gpu_le_scalar(self, values, scalar, type_code=L.T_INTEGER):
        return self._hook(True, 2, values, scalar, type_code)

    def gpu_gt_scalar(self, values, scalar, type_code=L.T_INTEGER):
        return self._hook(True, 3, values, scalar, type_code)

    def gpu_ge_scalar(self, values, scalar, type_code=L.T_INTEGER):
        return self._hook(True, 4, values, scalar, type_code)

    # ------------------------------------------------------------ prepared / serving
    def prepare(self, sql: str) -> "Statement":
        self._require_ctx()
        return self._adopt(Statement(self, sql))

    def submit(self, sql: str) -> "Request":
        self._require_ctx()
        h = C.c_void_p()
        self._check(self.lib.mtl_query_submit(self.ctx, sql.encode(), C.byref(h)))
        return self._adopt(Request(self, h))

    def serve_stats(self) -> dict:
        s = L.ServeStats()
        self._check(self.lib.mtl_serve_stats_get(self.ctx, C.byref(s)))
        return {f: getattr(s, f) for f, _ in L.ServeStats._fields_}

    def set_serve_slots(self, n: int):
        self._check(self.lib.mtl_serve_set_slots(self.ctx, n))

    def autotune(self, sql: str, reps: int = 3) -> str:
        """Measures launch shapes and hash load factors for the query's steps
        and keeps the fastest per device (mtl_autotune); returns the report."""
        self._require_ctx()
        buf = C.create_string_buffer(16384)
        self._check(self.lib.mtl_autotune(self.ctx, sql.encode(), reps, buf, len(buf)))
        return buf.value.decode()


class Statement:
    """A prepared statement: launch() enqueues with no host sync."""

    def __init__(self, conn: Connection, sql: str):
        self.conn = conn
        self.h = C.c_void_p()
        conn._check(conn.lib.mtl_stmt_prepare(conn.ctx, sql.encode(), C.byref(self.h)))

    def launch(self, stream: int | None = None):
        self.conn._check(self.conn.lib.mtl_stmt_launch(self.h, C.c_void_p(stream) if stream else None))

    def fetch(self) -> Result:
        r = C.c_void_p()
        self.conn._check(self.conn.lib.mtl_stmt_fetch(self.h, C.byref(r)))
        return Result(self.conn.lib, r)

    def device_ms(self) -> float:
        return float(self.conn.lib.mtl_stmt_device_ms(self.h))

    def kernel_count(self) -> int:
        return int(self.conn.lib.mtl_stmt_kernel_count(self.h))

    def set_profiling(self, on: bool = True):
        self.conn._check(self.conn.lib.mtl_stmt_set_profiling(self.h, 1 if on else 0))

    def step_times(self) -> list[tuple[str, float]]:
        """(step name, device ms) of the last launch; needs set_profiling(True)."""
        lib = self.conn.lib
        return [(lib.mtl_stmt_step_name(self.h, i).decode(), float(lib.mtl_stmt_step_ms(self.h, i)))
                for i in range(lib.mtl_stmt_step_count(self.h))]

    def close(self):
        # after the connection closed, the context already released it
        if self.h and self.conn.ctx:
            self.conn.lib.mtl_stmt_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Request:
    """A request submitted to the serving loop."""

    def __init__(self, conn: Connection, h):
        self.conn = conn
        self.h = h

    def wait(self, timeout_s: float | None = None) -> Result:
        r = C.c_void_p()
        ns = -1 if timeout_s is None else int(timeout_s * 1e9)
        rc = self.conn.lib.mtl_request_wait(self.h, ns, C.byref(r))
        L.check(rc, self.conn.ctx)
        return Result(self.conn.lib, r)

    def latency_ms(self) -> float:
        return float(self.conn.lib.mtl_request_latency_ms(self.h))

    def close(self):
        if self.h and self.conn.ctx:
            self.conn.lib.mtl_request_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
