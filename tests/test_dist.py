"""The N>1 host path of bench.py on CPU: two gloo ranks, each a replica.

The offloaded path has no exchange step (replicas only): every rank runs the
whole workload on its own GPU and the benchmark reduces times with a max and
rows with a sum over ranks. These are the collectives exercised here."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    ws, r, local = bench.dist_env()
    dist = bench.dist_init(ws, backend="gloo")
    t_max = bench.reduce_max(dist, 10.0 + r)
    rows = bench.reduce_sum(dist, 1000.0 * (r + 1))
    bench.barrier(dist)
    q.put((r, ws, local, t_max, rows))
    dist.destroy_process_group()


def test_two_rank_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2 for o in out)
    assert all(o[3] == 11.0 for o in out)      # max over ranks
    assert all(o[4] == 3000.0 for o in out)    # whole-job rows


def test_single_rank_is_identity():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    assert bench.reduce_max(None, 5.0) == 5.0 and bench.reduce_sum(None, 7.0) == 7.0
    assert bench.dist_init(1) is None
