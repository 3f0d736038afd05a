"""Python side of the serving layer (velo_server_* in libvelo_obl.so).

* ``ServedTables`` builds the seeded resident tables on the device: a fact
  table (lineitem-shaped columns plus an int64 foreign key), a dimension table
  (unique int64 keys, a date) and a second fact table whose foreign key points
  at fact rows.  At full scale they hold 60 M, 15 M and 150 M rows.
* ``query_stream`` draws a seeded mix of queries: 50 % filter + group-by
  (config-1 shape), 35 % two-way join + group-by + top-10 (config-2 shape),
  15 % three-way join chain, each over public slice sizes that vary.
* ``Server`` wraps the C ABI; ``run_open_loop`` submits queries at Poisson
  arrival times from one thread and collects them from another.
"""
from __future__ import annotations

import ctypes as C
import threading
import time

import numpy as np
import torch

from . import workloads as W
from ._lib import (VeloJoinPred, VeloLineitem, VeloLineitemPred, VeloQuery, VeloQueryResult, VeloServedTables,
                   VeloServerConfig, VeloServerStats, check, lib)

Q_FILTER_GROUPBY, Q_JOIN_TOPK, Q_JOIN3 = 1, 2, 3
SHAPE_NAMES = {Q_FILTER_GROUPBY: "filter_groupby", Q_JOIN_TOPK: "join2_topk", Q_JOIN3: "join3_chain"}

FULL_SCALE = dict(fact_n=60_000_000, dim_n=15_000_000, fact2_n=150_000_000)


class ServedTables:
    def __init__(self, fact_n: int, dim_n: int, fact2_n: int, seed: int = W.SEED_SERVE, device="cuda"):
        self.fact_n, self.dim_n, self.fact2_n = fact_n, dim_n, fact2_n
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        li = W.lineitem(fact_n, seed=seed)
        self.fact = {k: t(v) for k, v in li.items()}
        dim_key = (W.permutation(seed, dim_n, 20) + 1).astype(np.int64)
        fk = W.uniform_int(seed, fact_n, 21, 1, dim_n, np.int64)
        self.fact_fk = t(fk)
        self.fact_fk32 = t(fk.astype(np.int32))
        self.dim_key = t(dim_key)
        self.dim_key32 = t(dim_key.astype(np.int32))
        self.dim_date = t(W.uniform_int(seed, dim_n, 22, 0, 2556, np.int32))
        self.fact2_fk = t(W.uniform_int(seed, fact2_n, 23, 0, fact_n - 1, np.int64))
        self.fact2_price = t(W.uniform_int(seed, fact2_n, 24, 90_000, 10_500_000, np.int64))
        self.bytes = sum(x.numel() * x.element_size() for x in
                         list(self.fact.values()) + [self.fact_fk, self.fact_fk32, self.dim_key, self.dim_key32,
                                                     self.dim_date, self.fact2_fk, self.fact2_price])

    def struct(self) -> VeloServedTables:
        f = self.fact
        li = VeloLineitem(*[f[k].data_ptr() for k in ("qty", "price", "disc", "tax", "shipdate", "flag1", "flag2")])
        return VeloServedTables(li, self.fact_fk.data_ptr(), self.fact_fk32.data_ptr(), self.fact_n,
                                self.dim_key.data_ptr(), self.dim_key32.data_ptr(), self.dim_date.data_ptr(),
                                self.dim_n, self.fact2_fk.data_ptr(), self.fact2_price.data_ptr(), self.fact2_n)


class HostSlices:
    """Host copies of the slices a query reads, generated from the same
    seeded streams as ``ServedTables`` without building the whole tables (the
    dimension keys, a permutation, are generated once in full)."""

    def __init__(self, fact_n: int, dim_n: int, fact2_n: int, seed: int = W.SEED_SERVE):
        self.fact_n, self.dim_n, self.fact2_n, self.seed = fact_n, dim_n, fact2_n, seed
        self._dim_key = None

    def dim_key(self):
        if self._dim_key is None:
            self._dim_key = (W.permutation(self.seed, self.dim_n, 20) + 1).astype(np.int64)
        return self._dim_key

    def lineitem(self, o: int, n: int) -> dict:
        return W.lineitem(n, seed=self.seed, start=o)

    def join_inputs(self, q):
        s, o, n, do, dn = self.seed, q.offset, q.n, q.dim_offset, q.dim_n
        dim = dict(key=self.dim_key()[do:do + dn].astype(np.int32),
                   date=W.uniform_int(s, dn, 22, 0, 2556, np.int32, do))
        fact = dict(fk=W.uniform_int(s, n, 21, 1, self.dim_n, np.int64, o).astype(np.int32),
                    price=W.uniform_int(s, n, 1, 90_000, 10_500_000, np.int64, o))
        return dim, fact


def query_stream(tables, count: int, seed: int = W.SEED_SERVE, lo_log2: float = 16.0,
                 hi_log2: float = 22.0):
    """Seeded query mix (50 % filter + group-by, 35 % two-way join, 15 %
    three-way chain) with public slice sizes log-uniform in [2^lo, 2^hi]."""
    u = W.splitmix64(seed, count, 100).astype(np.float64) / 2.0**64
    v = W.splitmix64(seed, 4 * count, 101).astype(np.float64) / 2.0**64
    out = []
    for i in range(count):
        shape = Q_FILTER_GROUPBY if u[i] < 0.50 else (Q_JOIN_TOPK if u[i] < 0.85 else Q_JOIN3)
        size = lambda j, cap: int(min(cap, np.floor(2.0 ** (lo_log2 + v[4 * i + j] * (hi_log2 - lo_log2)))))  # noqa
        n = size(0, tables.fact_n)
        dn = size(1, tables.dim_n)
        f2 = size(2, tables.fact2_n)
        o = int(v[4 * i + 3] * (tables.fact_n - n + 1))
        do = int(v[4 * i + 3] * (tables.dim_n - dn + 1))
        fo = int(v[4 * i + 3] * (tables.fact2_n - f2 + 1))
        q = VeloQuery()
        q.shape = shape
        q.offset, q.n = o, n
        q.dim_offset, q.dim_n = do, dn
        q.f2_offset, q.f2_n = fo, f2
        p = W.LINEITEM_PRED
        q.pred = VeloLineitemPred(p["ship_lo"], p["ship_hi"], p["disc_lo"], p["disc_hi"], p["qty_lo"], p["qty_hi"])
        q.jpred = VeloJoinPred(W.JOIN_PRED["date_hi"], 0, W.JOIN_PRED["price_hi"])
        out.append(q)
    return out


def arrivals(count: int, rate_qps: float, seed: int = W.SEED_SERVE) -> np.ndarray:
    """Poisson arrival times (seconds from start) at `rate_qps`."""
    u = (W.splitmix64(seed, count, 200).astype(np.float64) + 0.5) / 2.0**64
    return np.cumsum(-np.log(u) / rate_qps)


SERVE_PERSISTENT = 1


class Server:
    """The serving layer (velo_server_*); persistent=True runs the admitted
    queries as jobs of one persistent command queue instead of per-slot
    streams."""

    def __init__(self, tables: ServedTables, slots: int, budget_bytes: int, device: int = 0,
                 persistent: bool = False, idle_us: int = 0):
        self.tables = tables
        self._tab = tables.struct()
        self.ptr = C.c_void_p()
        cfg = VeloServerConfig(device, slots, budget_bytes, SERVE_PERSISTENT if persistent else 0, idle_us)
        check(lib().velo_server_create(C.byref(cfg), C.byref(self._tab), C.byref(self.ptr)), "velo_server_create")

    def submit(self, q: VeloQuery) -> int:
        qid = C.c_uint64()
        check(lib().velo_server_submit(self.ptr, C.byref(q), C.byref(qid)), "velo_server_submit")
        return qid.value

    def wait(self, qid: int, timeout_s: float = 120.0) -> VeloQueryResult:
        r = VeloQueryResult()
        check(lib().velo_server_wait(self.ptr, qid, int(timeout_s * 1e9), C.byref(r)), "velo_server_wait")
        return r

    def stats(self) -> dict:
        s = VeloServerStats()
        check(lib().velo_server_stats(self.ptr, C.byref(s)), "velo_server_stats")
        return {k: int(getattr(s, k)) for k, _ in s._fields_}

    def close(self, timeout_ms: int = 60_000):
        if self.ptr:
            check(lib().velo_server_destroy(self.ptr, timeout_ms), "velo_server_destroy")
            self.ptr = None


def result_key(r: VeloQueryResult):
    """The deterministic part of a result (outputs and counts)."""
    return (int(r.shape), tuple(int(x) for x in r.out), tuple(int(x) for x in r.counts))


def run_closed_one_at_a_time(srv: Server, queries):
    """The plain path: each query submitted after the previous finished."""
    res = []
    t0 = time.perf_counter()
    for q in queries:
        res.append(srv.wait(srv.submit(q)))
    return res, time.perf_counter() - t0


def run_open_loop(srv: Server, queries, times):
    """Submits query i at times[i] (seconds) from one thread, collects from
    another; returns (results in query order, makespan seconds)."""
    qids = [None] * len(queries)
    ready = [threading.Event() for _ in queries]
    results = [None] * len(queries)
    t0 = time.perf_counter()

    def submitter():
        for i, (q, t) in enumerate(zip(queries, times)):
            d = t0 + t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            qids[i] = srv.submit(q)
            ready[i].set()

    def collector():
        for i in range(len(queries)):
            ready[i].wait()
            results[i] = srv.wait(qids[i])

    a = threading.Thread(target=submitter)
    b = threading.Thread(target=collector)
    a.start()
    b.start()
    a.join()
    b.join()
    return results, time.perf_counter() - t0


def latency_stats(results):
    lat = np.asarray([r.end_ms - r.submit_ms for r in results])
    return dict(p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                mean_ms=float(lat.mean()), max_ms=float(lat.max()))
