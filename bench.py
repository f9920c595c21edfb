#!/usr/bin/env python
"""Benchmark of the B200 execution path for mettle's offloaded SQL subset.

Default workload (the headline): the join -> filter -> group -> top-K
pipeline at 60M fact rows (customer 1.5M, orders 15M, lineitem ~60M;
DECIMAL(15,2) money as int64 cents, exact scale-4 revenue). Other workloads:
--config c1 (plain small query, 10^6 rows), c2 (filter/projection scan,
10^8 rows), c3 (grouped aggregate + top-100, 2*10^8 rows), c5 (served mixed
stream vs plain launches).

`value` is device throughput with the tables resident in HBM: K launches of
the prepared query back to back on one stream, timed with CUDA events on
that stream. `e2e` is the same metric through the public API with host
buffers: every step registers the tables from pinned host memory (H2D
copies), runs gpu_processing and downloads the result. Multi-GPU runs are
independent replicas (the path has no exchange step): every rank runs the
full workload on its own GPU, times are the max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mettle|reference] [--config c4]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

from mettle_b200 import workloads as W  # noqa: E402

FALLBACK_HBM_GBS = 6650.0


# ------------------------------------------------------------------ ranks
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws: int, backend: str = "nccl"):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    return dist


def barrier(dist, device=None):
    if dist is not None:
        if device is not None:
            dist.barrier(device_ids=[device])
        else:
            dist.barrier()


def reduce_max(dist, x: float, device: str = "cpu") -> float:
    """Max of a per-rank scalar over all ranks (identity for one rank)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(dist, x: float, device: str = "cpu") -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


def measured_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(name: str) -> float | None:
    """DRAM bytes per launch of the dominant kernel from a committed ncu summary."""
    for f in (ROOT / "profiles").glob("*.md"):
        m = re.search(rf"^traffic\[{re.escape(name)}\]:\s*([0-9.eE+]+)", f.read_text(), re.M)
        if m:
            return float(m.group(1))
    return None


# ------------------------------------------------------------------ workloads
class Workload:
    """A benchmark configuration: tables, SQL, fact rows, algorithmic bytes.
    `scale` shrinks the tables (profiling runs on a small case); `groups` and
    `dist` pick the config-3 key distribution; `keys` the config-4 join keys."""

    def __init__(self, name: str, scale: float = 1.0, groups: int | None = None, dist: str | None = None,
                 keys: str = "dense"):
        self.name = name
        if name == "c4":
            self.t = W.q3(n_cust=int(1_500_000 * scale), n_ord=int(15_000_000 * scale), keys=keys)
            self.sql = W.q3_sql(self.t.date)
            self.rows = self.t.lineitem_rows
            self.bytes = W.q3_bytes(self.t)
            self.dom_step = "pipeline:agg_slot:lineitem"
            kw = self.t.orders["o_orderkey"].dtype.itemsize
            self.dom_bytes = self.rows * (kw + 8 + 8 + 4)
            self.desc = (f"c4 join->filter->group->top-10: customer {len(self.t.customer['c_custkey'])}, "
                         f"orders {len(self.t.orders['o_orderkey'])}, lineitem {self.rows} rows; "
                         "DECIMAL(15,2) as int64 cents, revenue exact int128 at scale 4"
                         + ("" if keys == "dense" else f"; {keys} join keys (open-addressing hash joins)"))
        elif name == "c1":
            self.d = W.numbers(1_000_000)
            self.sql = W.C1_SQL
            self.rows = 1_000_000
            sel = int((self.d["value"] > 500000).sum())
            self.bytes = 4 * self.rows + sel * 8
            self.dom_step = "pipeline:materialize:numbers"
            self.dom_bytes = 4 * self.rows + sel * 8
            # order-preserving compaction: one pass with a look-back, or a
            # count pass, a scan and a write pass (the autotuner picks)
            self.dom_candidates = [("pipeline:materialize:numbers", self.dom_bytes),
                                   ("pipeline:mat_write:numbers", self.dom_bytes),
                                   ("pipeline:mat_count:numbers", 4 * self.rows), ("radix_sort", 8 * sel),
                                   ("gather_outs", 16 * sel)]
            self.desc = "c1 numbers 1M rows: SELECT value, value*10 WHERE value > 500000 ORDER BY value"
        elif name == "c2":
            self.rows = int(100_000_000 * scale)
            self.d = W.scan(self.rows)
            self.sql = W.scan_sql("a", "<", 0.5)
            sel = int((self.d["a"] < int(0.5 * 2**31)).sum())
            self.bytes = 4 * self.rows + sel * (28 - 4) + sel * 28
            self.dom_step = "pipeline:materialize:t"
            self.dom_bytes = self.bytes
            # the write pass of the two-pass compaction reads `a` again and
            # moves every selected row: the query's bytes; the count pass
            # reads `a` only
            self.dom_candidates = [("pipeline:materialize:t", self.bytes), ("pipeline:mat_write:t", self.bytes),
                                   ("pipeline:mat_count:t", 4 * self.rows), ("gather_outs", 56 * sel)]
            self.desc = f"c2 scan {self.rows} rows (a,b,c,d,e): SELECT a, b+5, c*10, d, e WHERE a < 2^30 (50%)"
        elif name == "c3":
            g = groups or int(os.environ.get("C3_GROUPS", "1000000"))
            dist = dist or os.environ.get("C3_DIST", "uniform")
            self.rows = int(200_000_000 * scale)
            self.d = W.groupby(self.rows, groups=g, dist=dist)
            self.sql = W.C3_SQL
            self.bytes = 20 * self.rows
            self.dom_step = "pipeline:agg_"
            self.dom_bytes = self.bytes
            # The query reads 20 B per row (k, v, f). Many groups take the
            # partitioned aggregation, whose kernels move intermediate records
            # too (count pass: reads k; scatter pass: reads k, v, f and writes
            # a 32-byte record; per-partition aggregation: reads the record);
            # those per-kernel figures are reported as diagnostics, while the
            # roofline fraction is the query's 20 B per row over the whole
            # query's time.
            self.dom_candidates = [("pipeline:agg_", self.bytes), ("agg_few", self.bytes),
                                   ("pipeline:part_count", 8 * self.rows),
                                   ("pipeline:part_scatter", 52 * self.rows), ("part_agg", 32 * self.rows)]
            self.query_frac_is_roofline = True
            self.desc = f"c3 group-by {self.rows} rows, G={g} {dist}: SUM/COUNT/MIN/MAX/AVG x2, top-100"
        else:
            raise SystemExit(f"unknown config {name}")

    def register(self, conn, upload=True, borrow=False):
        from mettle_b200 import _lib as L
        if self.name == "c4":
            W.register_q3(conn, self.t, upload=upload, borrow=borrow)
        elif self.name == "c1":
            conn.create_table("numbers", {"value": (L.T_INTEGER, self.d["value"])})
            conn.gpu_register_table("numbers", upload=upload, borrow=borrow)
        elif self.name == "c2":
            conn.create_table("t", {"a": (L.T_INTEGER, self.d["a"]), "b": (L.T_BIGINT, self.d["b"]),
                                    "c": (L.T_FLOAT, self.d["c"]), "d": (L.T_DATE, self.d["d"]),
                                    "e": (L.T_TIMESTAMP, self.d["e"])})
            conn.gpu_register_table("t", upload=upload, borrow=borrow)
        else:
            conn.create_table("t", {"k": (L.T_BIGINT, self.d["k"]), "v": (L.T_BIGINT, self.d["v"]),
                                    "f": (L.T_FLOAT, self.d["f"])})
            conn.gpu_register_table("t", upload=upload, borrow=borrow)

    def host_arrays(self) -> list[np.ndarray]:
        if self.name == "c4":
            return [*self.t.customer.values(), *self.t.orders.values(), *self.t.lineitem.values()]
        return list(self.d.values())

    def replace_arrays(self, arrays: list[np.ndarray]):
        it = iter(arrays)
        if self.name == "c4":
            for tab in (self.t.customer, self.t.orders, self.t.lineitem):
                for k in tab:
                    tab[k] = next(it)
        else:
            for k in self.d:
                self.d[k] = next(it)

    # ---- CPU (oracle port) execution of the same query
    def cpu_run(self):
        import oracle as orc
        if self.name == "c4":
            if self.t.orders["o_orderkey"].dtype == np.int64:
                return orc.q3_numpy(self.t, limit=10)
            return orc.q3(self.t, segment_code=1, limit=10)
        if self.name == "c1":
            rows = orc.filter_rows([(self.d["value"], ">", 500000)])
            rows = orc.sort_rows(self.d["value"], rows)
            return orc.gather(self.d["value"], rows), orc.gather(self.d["value"], rows, "*", 10)
        if self.name == "c2":
            rows = orc.filter_rows([(self.d["a"], "<", int(0.5 * 2**31))])
            return [orc.gather(self.d["a"], rows), orc.gather(self.d["b"], rows, "+", 5),
                    orc.gather(self.d["c"], rows, "*", np.float32(10)), orc.gather(self.d["d"], rows),
                    orc.gather(self.d["e"], rows)]
        return orc.groupby_c3(self.d["k"], self.d["v"], self.d["f"], limit=100)

    def parity(self, res) -> bool:
        want = self.cpu_run()
        rows = res.fetchall()
        if self.name == "c4":
            got = [(r[0], int(r[1].scaleb(4)), r[3]) for r in rows]
            if isinstance(want, list):
                return got == [(k, rev, p) for k, rev, _, p in want]
            exp = list(zip(want["key"].tolist(), want["revenue"], want["prio"].tolist()))
            return got == exp
        if self.name == "c1":
            return np.array_equal(res.columns[0], want[0]) and np.array_equal(res.columns[1], want[1])
        if self.name == "c2":
            return all(np.array_equal(res.columns[i], want[i]) for i in range(5))
        # every column: integers and AVG(BIGINT) (DuckDB's extended-precision
        # quotient) exact, FLOAT sums and averages within 1e-6 relative
        ok = len(rows) == len(want["k"])
        for i, r in enumerate(rows[: len(want["k"])]):
            k, sum_v, cnt, min_v, max_v, avg_v, sum_f, min_f, max_f, avg_f = r
            ok &= k == want["k"][i] and sum_v == want["sum_v"][i] and cnt == want["cnt"][i]
            ok &= min_v == want["min_v"][i] and max_v == want["max_v"][i] and avg_v == want["avg_v"][i]
            ok &= abs(sum_f - want["sum_f"][i]) <= 1e-6 * abs(want["sum_f"][i])
            ok &= np.float32(min_f) == want["min_f"][i] and np.float32(max_f) == want["max_f"][i]
            ok &= abs(avg_f - want["avg_f"][i]) <= 1e-6 * abs(want["avg_f"][i])
        return bool(ok)


def cpu_baseline(wl: Workload, seconds: float) -> dict:
    import oracle as orc
    wl.cpu_run()  # warm
    n, t0 = 0, time.perf_counter()
    while True:
        wl.cpu_run()
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 200:
            break
    return {"value": wl.rows * n / el, "unit": "rows/s", "cores": orc.threads(), "kind": "port",
            "sample": f"{n} full runs of the {wl.name} workload ({wl.rows} fact rows each), {el:.1f} s, "
                      f"OpenMP oracle (oracle/mettle_oracle.c)"}


# ------------------------------------------------------------------ arms
def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    import oracle as orc
    if args.config == "c5":
        tables = W.served_tables()
        stream = W.served_stream(args.c5_queries)
        budget = 60.0  # bounded sample of the stream
        t0, k = time.perf_counter(), 0
        while time.perf_counter() - t0 < budget and k < len(stream):
            _oracle_query(stream[k], tables)
            k += 1
        el = time.perf_counter() - t0
        value = k / el
        line = {"impl": "reference", "metric": "served queries/s", "value": value, "unit": "queries/s",
                "n_gpus": args.gpus, "steps": k, "warmup": 0, "ms_per_step": el * 1e3 / max(k, 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                "data": "synthetic", "config": {"workload": f"c5 served mixed stream, first {k} of {len(stream)} queries"},
                "cpu_baseline": {"value": value, "unit": "queries/s", "cores": orc.threads(), "kind": "port",
                                 "sample": f"first {k} queries of the stream back to back on the host cores "
                                           f"({el:.1f} s); the reference itself (Rust + Apple Metal) cannot run "
                                           "on this box"},
                "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    wl = Workload(args.config)
    for _ in range(min(args.warmup, 1)):
        wl.cpu_run()
    steps = max(1, min(args.steps, 20))
    t0 = time.perf_counter()
    for _ in range(steps):
        wl.cpu_run()
    el = time.perf_counter() - t0
    value = wl.rows * steps / el
    line = {"impl": "reference", "metric": "pipeline rows/s", "value": value, "unit": "rows/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": min(args.warmup, 1), "ms_per_step": el * 1e3 / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": {"workload": wl.desc},
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": orc.threads(), "kind": "port",
                             "sample": f"{steps} timed full runs of {wl.name} (of {args.steps} requested; bounded "
                                       "to keep the run within minutes) on the host cores; the reference itself "
                                       "(Rust + Apple Metal) cannot run on this box"},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _budget_sql(wl) -> str:
    # scratch for the largest plans: partition records (32 B per row) and a
    # one-key table of twice the groups at 64 B per entry
    gb = max(16, int(wl.bytes * 8 / 2**30) + 8)
    return f"CALL gpu_buffer_init('{gb} GB', '{gb} GB', pinned_memory_size = '{2 * gb} GB')"


def measure(wl, args, dist, local: int, with_e2e: bool, cpu_seconds: float) -> dict:
    """One configuration's bench figures: K launches of the prepared
    statement timed with CUDA events on the launching stream (max over
    ranks), parity of the measured statement against the oracle, per-step
    device times, the roofline of the dominant kernel, and optionally the
    end-to-end figure through the public API with host buffers."""
    import torch
    from mettle_b200 import Connection
    ws, rank, _ = dist_env()
    conn = Connection(device=local)
    conn.execute(_budget_sql(wl))
    wl.register(conn, upload=True)
    tune_report = None
    if args.autotune:
        # the autotuner measures this query's launch shapes, hash load factors
        # and aggregation strategy, and the statement below is compiled with
        # its choices (untimed)
        tune_report = conn.autotune(wl.sql, reps=3)
        print(tune_report, file=sys.stderr, flush=True)
    stmt = conn.prepare(wl.sql)
    # A dedicated (non-default) stream: the library enqueues on it and the
    # CUDA events below are recorded on the same stream.
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream

    # parity of the measured statement (rank 0, once)
    stmt.launch(sp)
    first = stmt.fetch()
    parity = wl.parity(first) if rank == 0 else None
    del first

    for _ in range(args.warmup):
        stmt.launch(sp)
    torch.cuda.synchronize()

    # ---- timed region: K launches, events on the launching stream
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier(dist, local)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")  # lets ncu select the timed launches (--nvtx-include timed/)
        e0.record(stream)
        for _ in range(args.steps):
            stmt.launch(sp)
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        barrier(dist, local)
    ms = e0.elapsed_time(e1)
    ms = reduce_max(dist, ms, f"cuda:{local}")
    clocks = clk.summary()
    total_rows = reduce_sum(dist, float(wl.rows * args.steps), f"cuda:{local}")
    value = total_rows / (ms / 1e3)
    kernels = stmt.kernel_count()

    # ---- per-step device times of the same launches (dominant kernel)
    stmt.set_profiling(True)
    prof_runs = max(3, min(args.steps, 50))
    cands = getattr(wl, "dom_candidates", [(wl.dom_step, wl.dom_bytes)])
    per = {p: [] for p, _ in cands}
    totals = {}
    for _ in range(prof_runs):
        stmt.launch(sp)
        steps = stmt.step_times()
        for name, t in steps:
            totals[name] = totals.get(name, 0.0) + t
        for p, _ in cands:
            per[p].append(sum(t for n, t in steps if n.startswith(p)))
    stmt.set_profiling(False)
    dom_prefix, dom_bytes = max(cands, key=lambda c: statistics.mean(per[c[0]]))
    dom_ms = max(statistics.mean(per[dom_prefix]), 1e-9)
    peak, peak_src = measured_peak()
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = profile_traffic(f"{wl.name}:{dom_prefix}")
    query_ms = ms / args.steps
    query_gbs = wl.bytes / (query_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": dom_prefix, "kernel_ms": dom_ms, "algorithmic_bytes": dom_bytes,
            "peak_source": peak_src, "query_gbs": query_gbs, "query_frac": query_gbs / peak,
            "query_algorithmic_bytes": wl.bytes}
    if getattr(wl, "query_frac_is_roofline", False):
        # the query's own bytes over the whole query's time; the dominant
        # kernel's figure (which counts intermediate records) is a diagnostic
        roof.update({"achieved": query_gbs, "frac": query_gbs / peak, "kernel": "whole query",
                     "kernel_ms": query_ms, "algorithmic_bytes": wl.bytes,
                     "dominant_kernel": {"name": dom_prefix, "ms": dom_ms, "bytes": dom_bytes,
                                         "frac": achieved / peak}})
    out = {"value": value, "ms_per_step": query_ms, "roofline": roof, "gpu_launches": kernels * args.steps,
           "clocks": clocks, "parity": parity, "autotuned": tune_report is not None,
           "step_ms": {k: v / prof_runs for k, v in sorted(totals.items(), key=lambda kv: -kv[1])[:8]}}
    stmt.close()
    conn.close()

    # ---- e2e through the public API with host buffers
    if with_e2e:
        os.environ["METTLE_DISABLE_QUERY_CACHE"] = "1"
        pinned = [torch.from_numpy(a).pin_memory() for a in wl.host_arrays()]
        wl.replace_arrays([p.numpy() for p in pinned])
        h2d = sum(a.nbytes for a in wl.host_arrays())
        e2e_steps = max(3, min(args.steps, 10))
        conn2 = Connection(device=local)
        conn2.execute(_budget_sql(wl))
        wl.register(conn2, upload=False, borrow=True)
        r = conn2.gpu_processing(wl.sql)  # warm (plans, stats)
        barrier(dist, local)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            wl.register(conn2, upload=False, borrow=True)  # new table version: H2D on first use
            r = conn2.gpu_processing(wl.sql)
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        e2e_s = reduce_max(dist, e2e_s, f"cuda:{local}")
        d2h = sum(c.nbytes for c in r.columns) + 12
        e2e_value = reduce_sum(dist, float(wl.rows), f"cuda:{local}") / e2e_s
        out["e2e"] = {"value": e2e_value, "unit": "rows/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                      "ms_per_step": e2e_s * 1e3, "steps": e2e_steps}
        del r
        conn2.close()
        os.environ.pop("METTLE_DISABLE_QUERY_CACHE", None)

    out["cpu_baseline"] = (cpu_baseline(wl, cpu_seconds)
                           if (rank == 0 and ws == 1 and cpu_seconds > 0) else None)
    return out


# Extra configurations measured beside the headline in the default run:
# (key, config, kwargs).
EXTRA_CONFIGS = [
    ("c1_plain_small", "c1", {}),
    ("c2_scan_a_lt_2e30", "c2", {}),
    ("c3_groups_1e6_uniform", "c3", {"groups": 1_000_000, "dist": "uniform"}),
    ("c3_groups_5e7_uniform", "c3", {"groups": 50_000_000, "dist": "uniform"}),
]


def run_profile(args):
    """Runs one workload as a prepared statement a few times and prints the
    per-step device times: a small case for a profiler to capture."""
    from mettle_b200 import Connection
    wl = Workload(args.config, scale=args.scale, keys=args.keys, groups=args.groups, dist=args.dist)
    conn = Connection()
    conn.execute(_budget_sql(wl))
    wl.register(conn, upload=True)
    st = conn.prepare(wl.sql)
    st.set_profiling(True)
    for i in range(args.launches):
        st.launch()
        res = st.fetch()
        steps = st.step_times()
        print(f"launch {i}: rows={res.rows} device_ms={st.device_ms():.3f} kernels={st.kernel_count()}")
        for name, t in steps:
            print(f"  {name:40s} {t:8.4f} ms")
    st.close()
    conn.close()


def run_mettle(args):
    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = dist_init(ws)
    wl = Workload(args.config, scale=args.scale, keys=args.keys, groups=args.groups, dist=args.dist)
    m = measure(wl, args, dist, local, with_e2e=True, cpu_seconds=args.cpu_seconds)
    desc = wl.desc
    extra = {}
    if args.config == "c4" and args.scale == 1.0 and args.keys == "dense" and not args.no_extra:
        del wl
        for key, cfg, kw in EXTRA_CONFIGS:
            x = Workload(cfg, **kw)
            r = measure(x, args, dist, local, with_e2e=False, cpu_seconds=min(args.cpu_seconds, 5.0))
            l2 = ("inputs (4 MB) fit in L2 and stay there between launches: a latency-bound small query"
                  if cfg == "c1" else "inputs larger than L2 (126 MB); no flush")
            extra[key] = {"workload": x.desc, "metric": "pipeline rows/s", "unit": "rows/s", "l2": l2, **r}
            del x
    if rank == 0:
        line = {
            "metric": "pipeline rows/s", "value": m["value"], "unit": "rows/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": desc,
                       "l2": "inputs larger than L2 (126 MB); no flush",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU"},
            "roofline": m["roofline"], "cpu_baseline": m["cpu_baseline"], "e2e": m["e2e"],
            "gpu_launches": m["gpu_launches"], "clocks": m["clocks"], "parity": m["parity"],
            "step_ms": m["step_ms"],
        }
        if extra:
            line["extra_configs"] = extra
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ------------------------------------------------------------------ served stream
def _checksum(res) -> tuple:
    """Size-independent digest of a result: row count, exact integer sums
    per column (wrapping), float sums, and the first rows' bytes."""
    import hashlib
    ints, floats = [], []
    head = hashlib.blake2b(digest_size=16)
    for c in res.columns:
        if c.dtype.kind == "f":
            floats.append(float(c.astype(np.float64).sum()))
        else:
            v = c.reshape(-1)
            ints.append(int(v.sum(dtype=np.int64)) if v.itemsize == 4 else int(v.view(np.int64).sum()))
            head.update(np.ascontiguousarray(v[:512]).tobytes())
    return res.rows, tuple(ints), tuple(floats), head.hexdigest()


def _same(a: tuple, b: tuple, rel: float = 1e-6) -> bool:
    if a[0] != b[0] or a[1] != b[1] or a[3] != b[3]:
        return False
    return all(abs(x - y) <= rel * max(abs(x), abs(y), 1e-300) for x, y in zip(a[2], b[2]))


def _oracle_query(q: dict, tables: dict):
    import oracle as orc
    tpl, d = tables[q["table"]]
    if q["tpl"] == "c1":
        rows = orc.sort_rows(d["value"], orc.filter_rows([(d["value"], ">", q["k"])]))
        return orc.gather(d["value"], rows)
    if q["tpl"] == "c2":
        rows = orc.filter_rows([(d[q["col"]], q["op"], q["v"])])
        return orc.gather(d["a"], rows)
    return orc.groupby_c3(d["k"], d["v"], d["f"], limit=q["limit"])


def _run_stream(conn, stream, arrivals, served: bool):
    """Runs the stream with the given arrival offsets (s). Returns per-query
    latency (arrival -> result on the host, ms), makespan (s) and digests."""
    import queue
    n = len(stream)
    lat = [0.0] * n
    digests = [None] * n
    done_at = [0.0] * n
    t0 = time.perf_counter()
    if served:
        q: "queue.Queue" = queue.Queue()

        def waiter():
            while True:
                item = q.get()
                if item is None:
                    return
                i, req, t_sub = item
                res = req.wait(timeout_s=600)
                t_done = time.perf_counter()
                done_at[i] = t_done
                lat[i] = (t_done - (t0 + arrivals[i])) * 1e3
                digests[i] = _checksum(res)
                req.close()

        th = threading.Thread(target=waiter)
        th.start()
        for i, qq in enumerate(stream):
            wait = t0 + arrivals[i] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            q.put((i, conn.submit(qq["sql"]), time.perf_counter()))
        q.put(None)
        th.join()
    else:
        for i, qq in enumerate(stream):
            wait = t0 + arrivals[i] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            res = conn.gpu_processing(qq["sql"])
            t_done = time.perf_counter()
            done_at[i] = t_done
            lat[i] = (t_done - (t0 + arrivals[i])) * 1e3
            digests[i] = _checksum(res)
    makespan = max(done_at) - t0
    return lat, makespan, digests


def run_served(args):
    """Served mixed stream (2,000 queries, Poisson arrivals at swept rates)
    against the same stream as plain one-query-at-a-time launches."""
    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = dist_init(ws)
    from mettle_b200 import Connection
    from mettle_b200 import _lib as L
    os.environ["METTLE_DISABLE_QUERY_CACHE"] = "1"  # every query runs on the device
    tables = W.served_tables()
    stream = W.served_stream(args.c5_queries)
    conn = Connection(device=local)
    conn.execute("CALL gpu_buffer_init('40 GB', '20 GB')")
    for name, (tpl, d) in tables.items():
        if tpl == "c1":
            conn.create_table(name, {"value": (L.T_INTEGER, d["value"])})
        elif tpl == "c2":
            conn.create_table(name, {"a": (L.T_INTEGER, d["a"]), "b": (L.T_BIGINT, d["b"]),
                                     "c": (L.T_FLOAT, d["c"]), "d": (L.T_DATE, d["d"]),
                                     "e": (L.T_TIMESTAMP, d["e"])})
        else:
            conn.create_table(name, {"k": (L.T_BIGINT, d["k"]), "v": (L.T_BIGINT, d["v"]),
                                     "f": (L.T_FLOAT, d["f"])})
        conn.gpu_register_table(name, upload=True)
    # warm: plans, statistics and column uploads for every template/table
    seen = set()
    for qq in stream:
        key = (qq["tpl"], qq["table"], qq.get("col"))
        if key not in seen:
            seen.add(key)
            conn.gpu_processing(qq["sql"])
    # oracle spot checks of the first queries of each template
    parity_oracle = True
    if rank == 0:
        checked = set()
        for qq in stream:
            if qq["tpl"] in checked or (qq["tpl"] != "c3" and tables[qq["table"]][1].get("a", np.empty(0)).size > 20_000_000):
                continue
            checked.add(qq["tpl"])
            res = conn.gpu_processing(qq["sql"])
            want = _oracle_query(qq, tables)
            if qq["tpl"] == "c3":
                parity_oracle &= bool(np.array_equal(res.columns[0], want["k"]) and
                                      np.array_equal(res.columns[2], want["cnt"]))
            else:
                parity_oracle &= bool(np.array_equal(res.columns[0], want))
    # the closed-loop plain capacity on the whole stream (its full mix of
    # templates and table sizes) sets the swept rates
    _, mk, _ = _run_stream(conn, stream, [0.0] * len(stream), served=False)
    plain_cap = len(stream) / mk
    rng = np.random.default_rng(11)
    sweep = []
    for factor in args.c5_rates:
        rate = plain_cap * factor
        gaps = rng.exponential(1.0 / rate, len(stream))
        arrivals = np.cumsum(gaps) - gaps[0]
        barrier(dist, local)
        pl, pmk, pdig = _run_stream(conn, stream, arrivals, served=False)
        barrier(dist, local)
        sl, smk, sdig = _run_stream(conn, stream, arrivals, served=True)
        same = all(_same(a, b) for a, b in zip(pdig, sdig))
        n = len(stream)
        sweep.append({
            "offered_qps": rate, "rate_factor": factor,
            "served": {"qps": n / smk, "p50_ms": float(np.percentile(sl, 50)), "p99_ms": float(np.percentile(sl, 99))},
            "plain": {"qps": n / pmk, "p50_ms": float(np.percentile(pl, 50)), "p99_ms": float(np.percentile(pl, 99))},
            "identical": same})
    top = sweep[-1]
    served_qps = reduce_sum(dist, top["served"]["qps"], f"cuda:{local}")
    st = conn.serve_stats()
    cpu = None
    if rank == 0 and ws == 1 and args.cpu_seconds > 0:
        import oracle as orc
        t0, k = time.perf_counter(), 0
        while time.perf_counter() - t0 < args.cpu_seconds and k < len(stream):
            _oracle_query(stream[k], tables)
            k += 1
        el = time.perf_counter() - t0
        cpu = {"value": k / el, "unit": "queries/s", "cores": orc.threads(), "kind": "port",
               "sample": f"first {k} queries of the stream run back to back through the OpenMP oracle "
                         f"({el:.1f} s; scan queries gather one column)"}
    if rank == 0:
        line = {
            "metric": "served queries/s", "value": served_qps, "unit": "queries/s", "n_gpus": ws,
            "steps": len(stream), "warmup": len(seen), "ms_per_step": 1e3 / top["served"]["qps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "config": {"workload": f"c5 served mixed stream: {len(stream)} queries (templates c1/c2/c3, tables 1M-60M "
                                   "rows), Poisson arrivals swept as multiples of the plain closed-loop rate; "
                                   "gpu_buffer_init('40 GB','20 GB')",
                       "l2": "tables larger than L2 (126 MB) except the 1M-row ones; no flush",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU"},
            "p50_ms": top["served"]["p50_ms"], "p99_ms": top["served"]["p99_ms"],
            "plain": top["plain"], "sweep": sweep, "identical": all(s["identical"] for s in sweep),
            "parity_oracle": parity_oracle, "plain_closed_loop_qps": plain_cap,
            "roofline": None, "cpu_baseline": cpu,
            "e2e": {"value": served_qps, "unit": "queries/s", "h2d_bytes_per_step": len(stream[0]["sql"]),
                    "d2h_bytes_per_step": None,
                    "note": "columns resident in the HBM column cache (the served form); results downloaded"},
            "gpu_launches": None, "serve_stats": st,
        }
        print(json.dumps(line), flush=True)
    conn.close()
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="mettle", choices=["mettle", "reference"])
    ap.add_argument("--config", default="c4", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--c5-queries", type=int, default=2000)
    ap.add_argument("--c5-rates", type=float, nargs="+", default=[0.25, 0.5, 0.75, 0.9])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--scale", type=float, default=1.0, help="table size factor (profiling runs use a small case)")
    ap.add_argument("--keys", default="dense", choices=["dense", "sparse32", "sparse64"],
                    help="config-4 join keys: dense (direct-mapped joins) or sparse (hash joins)")
    ap.add_argument("--launches", type=int, default=0,
                    help="profile mode: run the prepared statement this many times and print per-step times")
    ap.add_argument("--no-extra", action="store_true", help="measure the headline configuration only")
    ap.add_argument("--autotune", action="store_true",
                    help="run the autotuner on each measured query first (untimed) and measure its choices")
    ap.add_argument("--groups", type=int, default=None, help="config-3 group count (default 10^6)")
    ap.add_argument("--dist", default=None, choices=["uniform", "zipf"], help="config-3 key distribution")
    args = ap.parse_args()
    if args.launches > 0:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config == "c5":
        run_served(args)
    else:
        run_mettle(args)


if __name__ == "__main__":
    main()
