"""mtl_topk_noalloc: the top-K entry point for callers that cannot allocate
device memory when they need the result. For example, a host may have
given all device memory to its own pool, or may not allow cudaMalloc or
cudaFree to synchronize the device.

The entry point is checked against the existing path, gpu_processing with
ORDER BY ... LIMIT, and against numpy's stable argsort, on two calls in a
row. The two calls share the fixed
scratch array, so the second call also shows that what the first one left
there does no harm. This file sorts last, so a run that stops at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from mettle_b200 import _lib as L


def _existing(conn, desc: bool, k: int):
    order = "DESC" if desc else "ASC"
    res = conn.gpu_processing(f"SELECT v, i FROM t ORDER BY v {order} LIMIT {k}")
    return res.columns[0].copy(), res.columns[1].copy()


def _noalloc(lib, torch, v_dev, n: int, desc: bool, k: int):
    rows = torch.full((k,), -1, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = lib.mtl_topk_noalloc(L.T_BIGINT, C.c_void_p(v_dev.data_ptr()), n, k, 1 if desc else 0,
                              C.c_void_p(rows.data_ptr()), C.c_void_p(count.data_ptr()),
                              C.c_void_p(stream.cuda_stream))
    assert rc == L.OK, lib.mtl_last_error(None)
    torch.cuda.synchronize()
    m = int(count.item())
    return rows[:m].cpu().numpy().view(np.uint32).astype(np.int64)


@pytest.mark.gpu
def test_topk_noalloc_matches_gpu_processing_twice(conn):
    import torch

    lib = L.load()
    n = 3_000_000
    r = np.random.default_rng(2024)
    v = r.integers(-50_000, 50_000, n, dtype=np.int64)  # many ties
    i = np.arange(n, dtype=np.int64)
    conn.execute("CALL gpu_buffer_init('2 GB', '2 GB')")
    conn.create_table("t", {"v": (L.T_BIGINT, v), "i": (L.T_BIGINT, i)})
    conn.gpu_register_table("t", upload=True)
    v_dev = torch.from_numpy(v).cuda()

    for desc, k in ((True, 10), (False, 32)):
        want_v, want_rows = _existing(conn, desc, k)
        got_rows = _noalloc(lib, torch, v_dev, n, desc, k)
        assert len(got_rows) == k
        np.testing.assert_array_equal(got_rows, want_rows)
        np.testing.assert_array_equal(v[got_rows], want_v)
        # and a CPU reference that shares no code with either GPU path
        np.testing.assert_array_equal(got_rows, np.argsort(-v if desc else v, kind="stable")[:k])


@pytest.mark.gpu
@pytest.mark.parametrize("n,k", [(20_000_000, 32), (7_000_001, 25)])
def test_topk_noalloc_large_n_matches_numpy(built_lib, n, k):
    """Sizes whose full-occupancy grid would need more candidate lists than
    the fixed array holds: the grid is capped and every row still counts.
    Checked against numpy's stable argsort (ties: the lower row first),
    descending then ascending, two calls in a row on the same array."""
    import torch

    lib = L.load()
    r = np.random.default_rng(n)
    v = r.integers(-(2**40), 2**40, n, dtype=np.int64)
    v[r.integers(0, n, 64)] = 2**40 + 7  # repeated maxima: ties decided by row number
    v[r.integers(0, n, 64)] = -(2**40) - 7
    v_dev = torch.from_numpy(v).cuda()
    for desc in (True, False):
        want = np.argsort(-v if desc else v, kind="stable")[:k]
        got = _noalloc(lib, torch, v_dev, n, desc, k)
        np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_topk_noalloc_rejects_sizes_beyond_its_limits(conn):
    import torch

    lib = L.load()
    v_dev = torch.zeros(8, dtype=torch.int64, device="cuda")
    rows = torch.zeros(64, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    args = (C.c_void_p(rows.data_ptr()), C.c_void_p(count.data_ptr()), None)
    assert lib.mtl_topk_noalloc(L.T_BIGINT, C.c_void_p(v_dev.data_ptr()), 8, 33, 1, *args) == L.INVALID
    assert b"k must be between 1 and 32" in lib.mtl_last_error(None)
    assert lib.mtl_topk_noalloc(L.T_BIGINT, C.c_void_p(v_dev.data_ptr()), 2**32, 4, 1, *args) == L.INVALID
    assert lib.mtl_topk_noalloc(L.T_INTEGER, C.c_void_p(v_dev.data_ptr()), 8, 4, 1, *args) == L.UNSUPPORTED
    # a small input still works after the rejections
    assert lib.mtl_topk_noalloc(L.T_BIGINT, C.c_void_p(v_dev.data_ptr()), 8, 4, 1, *args) == L.OK
    torch.cuda.synchronize()
    assert int(count.item()) == 4
    assert rows[:4].cpu().tolist() == [0, 1, 2, 3]  # all values tie: lowest row numbers first
