"""gpu_{add,mul}_scalar and gpu_{eq,lt,le,gt,ge}_scalar (README.md:57) on the
GPU against numpy with DuckDB's result types and overflow errors, and the
cache-status surface of the reference (tests/extension.rs:527-659)."""
import numpy as np
import pytest

from mettle_b200 import MettleError
from mettle_b200 import _lib as L


@pytest.mark.gpu
@pytest.mark.parametrize("type_code,dtype", [(L.T_INTEGER, np.int32), (L.T_BIGINT, np.int64),
                                             (L.T_FLOAT, np.float32), (L.T_DOUBLE, np.float64)])
def test_scalar_hooks(conn, type_code, dtype):
    conn.execute("CALL gpu_buffer_init('1 GB', '1 GB')")
    r = np.random.default_rng(1)
    x = r.integers(-1000, 1000, 100_000).astype(dtype)
    k = 7 if np.dtype(dtype).kind == "i" else 1.5
    assert np.array_equal(conn.gpu_add_scalar(x, k, type_code), (x + dtype(k)).astype(dtype))
    assert np.array_equal(conn.gpu_mul_scalar(x, k, type_code), (x * dtype(k)).astype(dtype))
    for name, f in [("eq", np.equal), ("lt", np.less), ("le", np.less_equal), ("gt", np.greater),
                    ("ge", np.greater_equal)]:
        got = getattr(conn, f"gpu_{name}_scalar")(x, k, type_code)
        assert np.array_equal(got, f(x, dtype(k)))


@pytest.mark.gpu
def test_scalar_hook_overflow(conn):
    conn.execute("CALL gpu_buffer_init('1 GB', '1 GB')")
    with pytest.raises(MettleError) as e:
        conn.gpu_mul_scalar(np.array([1, 2**30], np.int32), 4, L.T_INTEGER)
    assert e.value.code == L.OVERFLOW


@pytest.mark.gpu
def test_cache_status_and_reset(conn):
    # tests/extension.rs:527-604: a grouped top-K query fills the result cache,
    # the repeat is served from it, gpu_cache_reset clears it.
    conn.execute("CALL gpu_buffer_init('64 KB', '128 KB', pinned_memory_size = '256 KB')")
    conn.execute("""CREATE TABLE customer(c_custkey INTEGER, c_mktsegment VARCHAR);
        INSERT INTO customer VALUES (1, 'BUILDING'), (2, 'HOUSEHOLD'), (3, 'BUILDING');
        CREATE TABLE orders(o_orderkey INTEGER, o_custkey INTEGER, o_orderdate DATE, o_shippriority INTEGER);
        INSERT INTO orders VALUES (100, 1, DATE '1995-03-10', 0), (101, 2, DATE '1995-03-20', 1),
          (102, 3, DATE '1995-03-05', 0), (103, 1, DATE '1995-04-01', 2);
        CREATE TABLE lineitem(l_orderkey INTEGER, l_extendedprice DOUBLE, l_discount DOUBLE, l_shipdate DATE);
        INSERT INTO lineitem VALUES (100, 1000.0, 0.05, DATE '1995-03-30'), (100, 500.0, 0.10, DATE '1995-04-01'),
          (101, 200.0, 0.00, DATE '1995-03-28'), (102, 300.0, 0.20, DATE '1995-03-26'),
          (103, 800.0, 0.15, DATE '1995-03-30')""")
    for t in ("customer", "orders", "lineitem"):
        conn.execute(f"CALL gpu_register_table('{t}')")
    sql = ("CALL gpu_processing('SELECT l_orderkey, SUM(l_extendedprice * (1 - l_discount)) AS revenue, "
           "o_orderdate, o_shippriority FROM customer JOIN orders ON c_custkey = o_custkey "
           "JOIN lineitem ON l_orderkey = o_orderkey WHERE c_mktsegment = ''BUILDING'' "
           "AND o_orderdate < DATE ''1995-03-25'' AND l_shipdate > DATE ''1995-03-25'' "
           "GROUP BY l_orderkey, o_orderdate, o_shippriority ORDER BY revenue DESC LIMIT 10')")
    first = conn.execute(sql).fetchall()
    assert conn.last_execution_mode() == "cuda_generic_plan"
    st = conn.execute("CALL gpu_cache_status()").fetchone()
    assert len(st) == 19 and st[15] >= 1 and st[17] >= 1
    second = conn.execute(sql).fetchall()
    assert second == first
    assert conn.last_execution_mode() == "cuda_hot_query_cache"
    assert conn.execute("CALL gpu_cache_status()").fetchone()[0] == "cuda_hot_query_cache"
    assert conn.execute("CALL gpu_cache_reset()").fetchone() == ("reset",)
    st = conn.execute("CALL gpu_cache_status()").fetchone()
    assert st[0] == "" and st[15] == 0 and st[17] == 0


@pytest.mark.gpu
def test_buffer_init_row(conn):
    row = conn.execute("CALL gpu_buffer_init('1 GB', '2 GB', pinned_memory_size = '4 GB')").fetchone()
    assert row[0] == "initialized" and "B200" in row[1]
    assert row[2:5] == (1 << 30, 2 << 30, 4 << 30)
    assert row[5].startswith("cuda")
