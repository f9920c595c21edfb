"""The C ABI without a GPU: the library loads, exports every declared symbol,
and its host-only entry points behave like the reference's."""
import ctypes as C

import pytest

from mettle_b200 import _lib as L


def test_library_exports_every_header_symbol(built_lib):
    lib = L.load()
    declared = L.header_symbols()
    assert len(declared) >= 35
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    bound = {name for name, _, _ in L.SIGNATURES}
    assert set(declared) == bound, set(declared) ^ bound


def parse(cache, processing, pinned=None):
    lib = L.load()
    b = L.Budgets()
    err = C.create_string_buffer(256)
    rc = lib.mtl_parse_buffer_config(cache.encode(), processing.encode(), pinned.encode() if pinned else None,
                                     C.byref(b), err, 256)
    return rc, b, err.value.decode()


def test_parse_human_sizes(built_lib):
    # src/config.rs:131-137
    for text, want in [("64", 64), ("64 KB", 64 * 1024), ("1.5 MB", 1_572_864), ("2gb", 2 * 1024 ** 3)]:
        rc, b, _ = parse(text, "1")
        assert rc == L.OK and b.cache_region_bytes == want


def test_pinned_defaults_to_sum(built_lib):
    # src/config.rs:139-144
    rc, b, _ = parse("1 KB", "2 KB")
    assert rc == L.OK
    assert (b.cache_region_bytes, b.processing_region_bytes, b.pinned_region_bytes) == (1024, 2048, 3072)


@pytest.mark.parametrize("cache,processing,msg", [
    ("0", "1", "non-zero cache region"), ("1", "0", "non-zero processing region"),
    ("", "1", "cannot be empty"), ("12 XB", "1", "unsupported size unit"), ("KB", "1", "missing numeric value"),
])
def test_buffer_config_errors(built_lib, cache, processing, msg):
    rc, _, err = parse(cache, processing)
    assert rc == L.INVALID and msg in err


def test_processing_requires_init(built_lib):
    # src/state.rs:42-54, test/sql/sirius-compat.test:7
    lib = L.load()
    out = C.c_void_p()
    rc = lib.mtl_processing(None, b"SELECT 42", C.byref(out))
    assert rc == L.NOT_INITIALIZED
    assert "call gpu_buffer_init before gpu_processing" in lib.mtl_last_error(None).decode()


def test_connection_requires_init(built_lib):
    from mettle_b200 import Connection, MettleError
    c = Connection()
    with pytest.raises(MettleError, match="call gpu_buffer_init before gpu_processing"):
        c.execute("CALL gpu_processing('SELECT 42 AS answer')")
    with pytest.raises(MettleError, match="non-empty SQL string"):
        c.gpu_processing("   ")


def test_rewrite_query_hooks(built_lib):
    lib = L.load()
    buf = C.create_string_buffer(1024)
    rc = lib.mtl_rewrite_query(None, b"SELECT value, value * 10 AS scaled FROM numbers WHERE value > 5 AND 3 >= x",
                               buf, 1024)
    assert rc == L.OK, lib.mtl_last_error(None)
    s = buf.value.decode()
    assert "gpu_mul_scalar(value, 10) AS \"scaled\"" in s
    assert "gpu_gt_scalar(value, 5)" in s and "gpu_le_scalar(x, 3)" in s


def test_host_catalog_parses_reference_setup(built_lib):
    from mettle_b200 import Connection
    c = Connection()
    c.execute("""CREATE TABLE events(id INTEGER, category VARCHAR, event_date DATE);
                 INSERT INTO events VALUES (1, 'A', DATE '2024-01-15'), (2, 'B', DATE '2024-02-20')""")
    t = c.tables["events"]
    assert t.rows == 2
    assert t.columns[1].materialize().tolist() == [0, 1] and t.columns[1].dictionary == ["A", "B"]
