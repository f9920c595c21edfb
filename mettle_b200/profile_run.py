"""Runs one benchmark workload as a prepared statement a few times and prints
the per-step device times; small enough to run under a profiler.

  python -m mettle_b200.profile_run --config c4 --scale 0.25 --launches 3
"""
from __future__ import annotations

import argparse
import sys

from . import Connection, workloads as W
from . import _lib as L


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c4", choices=["c1", "c2", "c3", "c4"])
    ap.add_argument("--scale", type=float, default=0.25)
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--groups", type=int, default=1_000_000)
    ap.add_argument("--dist", default="uniform")
    a = ap.parse_args(argv)
    conn = Connection()
    conn.execute("CALL gpu_buffer_init('16 GB', '16 GB', pinned_memory_size = '32 GB')")
    if a.config == "c4":
        t = W.q3(n_cust=int(1_500_000 * a.scale), n_ord=int(15_000_000 * a.scale))
        W.register_q3(conn, t, upload=True)
        sql = W.q3_sql(t.date)
    elif a.config == "c1":
        d = W.numbers(int(1_000_000 * a.scale))
        conn.create_table("numbers", {"value": (L.T_INTEGER, d["value"])})
        conn.gpu_register_table("numbers", upload=True)
        sql = W.C1_SQL
    elif a.config == "c2":
        d = W.scan(int(100_000_000 * a.scale))
        conn.create_table("t", {"a": (L.T_INTEGER, d["a"]), "b": (L.T_BIGINT, d["b"]), "c": (L.T_FLOAT, d["c"]),
                                "d": (L.T_DATE, d["d"]), "e": (L.T_TIMESTAMP, d["e"])})
        conn.gpu_register_table("t", upload=True)
        sql = W.scan_sql("a", "<", 0.5)
    else:
        d = W.groupby(int(200_000_000 * a.scale), groups=a.groups, dist=a.dist)
        conn.create_table("t", {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]), "f": (L.T_FLOAT, d["f"])})
        conn.gpu_register_table("t", upload=True)
        sql = W.C3_SQL
    st = conn.prepare(sql)
    st.set_profiling(True)
    for i in range(a.launches):
        st.launch()
        res = st.fetch()
        steps = st.step_times()
        print(f"launch {i}: rows={res.rows} device_ms={st.device_ms():.3f} kernels={st.kernel_count()}")
        for name, ms in steps:
            print(f"  {name:40s} {ms:8.4f} ms")
    st.close()
    conn.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
