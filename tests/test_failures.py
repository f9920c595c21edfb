"""Failure detection without a GPU fault: a bounded device wait that runs
out, a request wait that times out, and the column cache staying within its
budget. Every failure is made on the host (mtl_debug_inject) and ends in a
status the host reads; the context keeps working afterwards."""
import ctypes as C

import numpy as np
import pytest

from mettle_b200 import MettleError
from mettle_b200 import _lib as L

INJECT_NONE, INJECT_LOOKBACK_STALL, INJECT_HOLD_QUEUE = 0, 1, 2


def inject(conn, what, arg=0):
    assert conn.lib.mtl_debug_inject(conn.ctx, what, arg) == L.OK


def test_inject_rejects_unknown_kinds_without_a_context(built_lib):
    lib = L.load()
    assert lib.mtl_debug_inject(None, INJECT_LOOKBACK_STALL, 0) == L.NOT_INITIALIZED


@pytest.mark.gpu
def test_lookback_wait_runs_out_and_context_survives(conn):
    """The first tile of the order-preserving compaction never publishes its
    prefix: the tiles behind it give up after a few polls, the kernel ends,
    and the query reports the device wait that ran out. The same query then
    succeeds once the injection is cleared."""
    conn.execute("CALL gpu_buffer_init('1 GB', '1 GB')")
    n = 300_000
    x = np.arange(n, dtype=np.int32)
    conn.create_table("n", {"x": (L.T_INTEGER, x)})
    conn.gpu_register_table("n")
    sql = "SELECT x FROM n WHERE x >= 0"
    inject(conn, INJECT_LOOKBACK_STALL, 64)
    try:
        with pytest.raises(MettleError) as e:
            conn.gpu_processing(sql)
        assert e.value.code == L.DEVICE_ERROR
        assert "iteration limit" in str(e.value)
    finally:
        inject(conn, INJECT_NONE)
    conn.gpu_cache_reset()  # the failed query left no cached result, but be explicit
    r = conn.gpu_processing(sql)
    assert np.array_equal(r.columns[0], x)


@pytest.mark.gpu
def test_request_wait_times_out_then_completes(conn):
    conn.execute("CALL gpu_buffer_init('1 GB', '1 GB')")
    conn.create_table("n", {"x": (L.T_INTEGER, np.arange(1000, dtype=np.int32))})
    conn.gpu_register_table("n")
    inject(conn, INJECT_HOLD_QUEUE)
    try:
        req = conn.submit("SELECT x FROM n WHERE x < 10")
        with pytest.raises(MettleError) as e:
            req.wait(timeout_s=0.05)
        assert e.value.code == L.TIMEOUT
        assert conn.serve_stats()["queued"] >= 1
    finally:
        inject(conn, INJECT_NONE)
    r = req.wait(timeout_s=60)
    assert list(r.columns[0]) == list(range(10))
    req.close()


@pytest.mark.gpu
def test_column_cache_evicts_within_cache_region(conn):
    """Three 16 MB columns under a 40 MB cache region: using them in turn
    evicts the least recently used, the cached bytes never exceed the
    region, and every result stays correct."""
    conn.execute("CALL gpu_buffer_init('40 MB', '512 MB')")
    n = 4 * 1024 * 1024
    cols = {}
    for name in ("a", "b", "c"):
        cols[name] = np.random.default_rng(ord(name)).integers(0, 1000, n).astype(np.int32)
        conn.create_table(name, {"v": (L.T_INTEGER, cols[name])})
        conn.gpu_register_table(name)
    limit = 40 * 1024 * 1024
    def status():
        rows = conn.gpu_cache_status()
        return dict(zip(rows.names, rows.fetchall()[0]))

    for rnd in range(2):
        for name in ("a", "b", "c"):
            cut = 500 + rnd  # a new query text each round: no cached result
            r = conn.gpu_processing(f"SELECT COUNT(*), SUM(v) FROM {name} WHERE v < {cut}")
            m = cols[name] < cut
            assert r.fetchall() == [(int(m.sum()), int(cols[name][m].sum()))]
            assert status()["metal_cached_bytes"] <= limit
    assert status()["metal_evictions"] >= 3
