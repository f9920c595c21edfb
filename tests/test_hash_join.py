"""Joins whose build keys span too wide a range for the direct-mapped map
take the open-addressing hash tables (build_insert / the probe in
k_pipeline.cu), the counterpart of the reference's hash_join_build_i32_v /
hash_join_probe_i32_v (src/metal/shaders/kernels.metal:786-837,
src/metal/runtime/join_ops.rs:22-125). These cases force that path: keys
drawn sparse over the INTEGER and BIGINT ranges, build keys equal to the
table's empty-slot sentinel (-1) and to both extremes of the type, probe
keys that match nothing, and the join -> filter -> group -> top-K pipeline
with both of its joins hashed. Results are compared with numpy and with the
CPU oracle; every integer result must be exact."""
import numpy as np
import pytest

import oracle as orc
from mettle_b200 import MettleError
from mettle_b200 import _lib as L
from mettle_b200 import workloads as W


def init(conn, size="8 GB"):
    conn.execute(f"CALL gpu_buffer_init('{size}', '{size}')")


def _sparse_build_probe(dtype, n_build, n_probe, seed, hit=0.7):
    r = np.random.default_rng(seed)
    info = np.iinfo(dtype)
    bk = W._sparse_keys(r, n_build, dtype)
    # probe keys: most drawn from the build keys (the specials among them),
    # the rest values that match nothing
    pk = bk[r.integers(0, n_build, n_probe)]
    miss = r.random(n_probe) >= hit
    absent = r.integers(info.min, info.max, int(miss.sum()), dtype=np.int64, endpoint=True).astype(dtype)
    absent = absent[~np.isin(absent, bk)]
    pk[np.flatnonzero(miss)[: len(absent)]] = absent
    specials = np.array([-1, info.min, info.max], dtype=dtype)
    pk[:3] = specials  # the first probe rows hit the special keys
    bv = r.integers(-10**12, 10**12, n_build).astype(np.int64)
    pv = r.integers(-10**9, 10**9, n_probe).astype(np.int64)
    return bk, bv, pk, pv


def _lookup(bk, pk):
    """Build row of every probe key, -1 when it has none."""
    o = np.argsort(bk, kind="stable")
    s = bk[o]
    i = np.searchsorted(s, pk)
    i_c = np.minimum(i, len(s) - 1)
    found = s[i_c] == pk
    return np.where(found, o[i_c], -1)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,ltype", [(np.int32, L.T_INTEGER), (np.int64, L.T_BIGINT)])
def test_hash_join_sparse_keys_materialize(conn, dtype, ltype):
    init(conn)
    bk, bv, pk, pv = _sparse_build_probe(dtype, 300_000, 2_000_000, seed=11 + ltype)
    conn.create_table("bt", {"bk": (ltype, bk), "bv": (L.T_BIGINT, bv)})
    conn.create_table("pt", {"pk": (ltype, pk), "pv": (L.T_BIGINT, pv)})
    conn.gpu_register_table("bt")
    conn.gpu_register_table("pt")
    res = conn.gpu_processing("SELECT pk, pv, bv FROM pt, bt WHERE pk = bk")
    b = _lookup(bk, pk)
    m = b >= 0
    assert res.rows == int(m.sum())
    # the probe table drives the scan: rows come out in its row order
    assert np.array_equal(res.columns[0], pk[m])
    assert np.array_equal(res.columns[1], pv[m])
    assert np.array_equal(res.columns[2], bv[b[m]])
    assert res.rows >= 3 and list(res.columns[0][:3]) == [-1, np.iinfo(dtype).min, np.iinfo(dtype).max]


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,ltype", [(np.int32, L.T_INTEGER), (np.int64, L.T_BIGINT)])
def test_hash_join_filters_on_both_sides(conn, dtype, ltype):
    """Filters on the build side leave gaps in the build; filters on the probe
    side run before the probe."""
    init(conn)
    bk, bv, pk, pv = _sparse_build_probe(dtype, 200_000, 1_500_000, seed=21 + ltype)
    conn.create_table("bt", {"bk": (ltype, bk), "bv": (L.T_BIGINT, bv)})
    conn.create_table("pt", {"pk": (ltype, pk), "pv": (L.T_BIGINT, pv)})
    conn.gpu_register_table("bt")
    conn.gpu_register_table("pt")
    res = conn.gpu_processing("SELECT pv, bv FROM pt, bt WHERE pk = bk AND bv > 0 AND pv < 500000000")
    b = _lookup(bk, pk)
    m = (b >= 0) & (pv < 500_000_000)
    m &= np.where(b >= 0, bv[np.maximum(b, 0)] > 0, False)
    assert res.rows == int(m.sum())
    assert np.array_equal(res.columns[0], pv[m])
    assert np.array_equal(res.columns[1], bv[b[m]])


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,ltype", [(np.int32, L.T_INTEGER), (np.int64, L.T_BIGINT)])
def test_hash_join_group_by_build_key_topk(conn, dtype, ltype):
    """GROUP BY the build key groups by the build's slot (the representative
    row), probed through the hash table; then a fused top-K."""
    init(conn)
    bk, bv, pk, pv = _sparse_build_probe(dtype, 250_000, 2_000_000, seed=31 + ltype)
    pv = np.abs(pv) % 1000  # many equal sums: ties ordered by the key
    conn.create_table("bt", {"bk": (ltype, bk), "bv": (L.T_BIGINT, bv)})
    conn.create_table("pt", {"pk": (ltype, pk), "pv": (L.T_BIGINT, pv)})
    conn.gpu_register_table("bt")
    conn.gpu_register_table("pt")
    for limit in (10, 100):
        res = conn.gpu_processing(f"SELECT bk, SUM(pv) AS s, COUNT(*) AS c FROM pt, bt WHERE pk = bk "
                                  f"GROUP BY bk ORDER BY s DESC, bk LIMIT {limit}")
        b = _lookup(bk, pk)
        m = b >= 0
        keys, inv = np.unique(pk[m], return_inverse=True)
        sums = np.bincount(inv, weights=pv[m].astype(np.float64)).astype(np.int64)
        cnts = np.bincount(inv)
        order = np.lexsort((keys, -sums))[:limit]
        rows = res.fetchall()
        assert [r[0] for r in rows] == keys[order].tolist()
        assert [int(r[1]) for r in rows] == sums[order].tolist()
        assert [r[2] for r in rows] == cnts[order].tolist()


@pytest.mark.gpu
def test_hash_join_group_by_build_column(conn):
    """A hashed join feeding a grouped aggregate over a build-side column."""
    init(conn)
    bk, bv, pk, pv = _sparse_build_probe(np.int64, 100_000, 1_000_000, seed=41)
    bg = (np.abs(bv) % 37).astype(np.int32)
    conn.create_table("bt", {"bk": (L.T_BIGINT, bk), "bg": (L.T_INTEGER, bg)})
    conn.create_table("pt", {"pk": (L.T_BIGINT, pk), "pv": (L.T_BIGINT, pv)})
    conn.gpu_register_table("bt")
    conn.gpu_register_table("pt")
    res = conn.gpu_processing("SELECT bg, COUNT(*), SUM(pv), MIN(pv), MAX(pv) FROM pt, bt WHERE pk = bk "
                              "GROUP BY bg ORDER BY bg")
    b = _lookup(bk, pk)
    m = b >= 0
    g = bg[b[m]]
    v = pv[m]
    rows = res.fetchall()
    want = sorted(set(g.tolist()))
    assert [r[0] for r in rows] == want
    for r in rows:
        sel = g == r[0]
        assert r[1] == int(sel.sum())
        assert int(r[2]) == int(v[sel].sum())
        assert r[3] == int(v[sel].min()) and r[4] == int(v[sel].max())


@pytest.mark.gpu
def test_hash_join_duplicate_build_key_is_rejected(conn):
    """A build side whose key repeats is outside the subset: the query is
    refused with an error (never answered with wrong rows)."""
    init(conn)
    bk = np.array([5, -1, 2**40, 5, 7], dtype=np.int64)  # 5 twice
    conn.create_table("bt", {"bk": (L.T_BIGINT, bk), "bv": (L.T_BIGINT, np.arange(5, dtype=np.int64))})
    conn.create_table("pt", {"pk": (L.T_BIGINT, np.array([5, 7, -1, 9, 2**40, 5] * 1000, dtype=np.int64))})
    conn.gpu_register_table("bt")
    conn.gpu_register_table("pt")
    with pytest.raises(MettleError) as e:
        conn.gpu_processing("SELECT pk, bv FROM pt, bt WHERE pk = bk")
    assert e.value.code == L.UNSUPPORTED
    assert "unique key on its build side" in str(e.value)


def _q3_rows(res):
    import datetime as dt
    return [(k, int(rev.scaleb(4)), (d - dt.date(1970, 1, 1)).days, p) for k, rev, d, p in res.fetchall()]


@pytest.mark.gpu
@pytest.mark.parametrize("keys", ["sparse32", "sparse64"])
@pytest.mark.parametrize("scale", [0.01, 0.1])
def test_c4_pipeline_hashed_joins(conn, keys, scale):
    """The config-4 pipeline with both joins on open-addressing tables: keys
    spread over the whole INTEGER or BIGINT range."""
    init(conn, "16 GB")
    t = W.q3(n_cust=int(1_500_000 * scale), n_ord=int(15_000_000 * scale), seed_salt=7, keys=keys)
    W.register_q3(conn, t)
    for limit in (10, 1000):
        got = _q3_rows(conn.gpu_processing(W.q3_sql(t.date, limit=limit)))
        want = orc.q3_numpy(t, limit=limit)
        assert got == want
        if keys == "sparse32":
            # the C oracle joins through its own hash maps: the same rows
            w = orc.q3(t, segment_code=1, limit=limit)
            assert got == list(zip(w["key"].tolist(), w["revenue"], w["date"].tolist(), w["prio"].tolist()))


@pytest.mark.gpu
def test_c4_pipeline_hashed_joins_full_size(conn):
    """Full size (customer 1.5M, orders 15M, lineitem ~60M) with BIGINT keys
    over the whole int64 range."""
    init(conn, "24 GB")
    t = W.q3(keys="sparse64")
    W.register_q3(conn, t, upload=True)
    got = _q3_rows(conn.gpu_processing(W.q3_sql(t.date, limit=10)))
    assert got == orc.q3_numpy(t, limit=10)


def test_q3_numpy_agrees_with_the_oracle():
    """The numpy restatement used above gives the oracle's rows (dense and
    sparse INTEGER keys)."""
    for keys in ("dense", "sparse32"):
        t = W.q3(n_cust=3000, n_ord=30_000, seed_salt=5, keys=keys)
        w = orc.q3(t, segment_code=1, limit=50)
        assert orc.q3_numpy(t, limit=50) == list(zip(w["key"].tolist(), w["revenue"], w["date"].tolist(),
                                                  w["prio"].tolist()))
