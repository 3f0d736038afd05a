#!/usr/bin/env python3
"""Benchmark of the oblivious operator hot path on B200.

Default workload: oblivious filter + group-by over the synthetic
6,001,215-row lineitem-shaped fact table (predicate -> ORCompact -> bitonic
sort on (flag1, flag2) -> segmented int64 sums, output padded to 8 groups).
One step = one pass of that pipeline over one batch of input.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload groupby|sort|batch|serve|join]

Workloads: groupby (6,001,215-row filter + group-by, the default), sort
(plain 2^20-row sort), join (1.5 M x 6 M-row PK-FK join + group-by + top-10), batch (512 uneven sorts/compactions in one persistent
launch replayed from a CUDA graph, beside 512 plain launch sequences), serve
(query stream over resident 60 M / 15 M / 150 M-row tables: served vs plain
one-at-a-time throughput and p50/p99 latency).

Multi-GPU: one process per GPU (torchrun); the path does not shard, so every
rank runs an independent replica of the workload ("replicas only") and the
aggregate throughput is the total rows of all ranks over the slowest rank's
time.  `--impl reference` times the reference's CPU algorithm (the C oracle
port in the reference's network order, all host cores) on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")

# DRAM bytes (read + write) per launch of the dominant kernel from one ncu
# capture (the mean over the tile, global and merge passes of one sort), or
# None when the workload's launch is too large to capture.
TRAFFIC = {"groupby": 210.1e6, "sort": 12.65e6, "batch": None}
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# --------------------------------------------------------------------------
# pass-count model (mirrors plan_sort / plan_compact of the library)
# --------------------------------------------------------------------------

# levels fused per global pass: plain (u64, u32) sorts keep 32 contiguous rows
# per warp (lmax = lt - 5); the pipelines' 8-byte records use 16 (lt - 4)
PIPE_LMAX = 8


def sort_passes(logn: int, lt: int, lmax: int) -> int:
    p = 1
    for k in range(lt + 1, logn + 1):
        p += -(-(k - lt) // lmax) + 1
    return p


def compact_passes(logn: int, lt: int, lmax: int) -> int:
    return 1 + (-(-(max(0, logn - lt)) // lmax) if logn > lt else 0)


def rdm_psort(np_rows: int) -> int:
    """Pass count of the survey's algorithmic-bytes model: T = 2^13, L = 8."""
    m = max(0, int(np.log2(np_rows)) - 13)
    return 1 + sum(-(-i // 8) + 1 for i in range(1, m + 1))


def rdm_pcomp(np_rows: int) -> int:
    m = max(0, int(np.log2(np_rows)) - 13)
    return 1 + -(-m // 8)


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"velo_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# workloads (ours)
# --------------------------------------------------------------------------

class GroupBy:
    """Config-1 shape: filter + group-by over 6,001,215 rows."""
    name = "filter_groupby"

    def __init__(self, torch, capi, W, device):
        self.torch, self.capi = torch, capi
        self.n = W.LINEITEM_ROWS
        self.pred = W.LINEITEM_PRED
        self.G = W.LINEITEM_GROUP_BOUND
        self.host = W.lineitem(self.n)
        self.pinned = {k: torch.from_numpy(v).pin_memory() for k, v in self.host.items()}
        self.dev = {k: torch.empty_like(v, device=device) for k, v in self.pinned.items()}
        for k in self.dev:
            self.dev[k].copy_(self.pinned[k])
        self.scratch = torch.empty(capi.filter_groupby_scratch_bytes(self.n, self.G), dtype=torch.uint8,
                                   device=device)
        self.out = torch.empty((self.G, 6), dtype=torch.int64, device=device)
        self.counts = torch.empty(2, dtype=torch.int64, device=device)
        self.out_host = torch.empty((self.G, 6), dtype=torch.int64).pin_memory()
        self.counts_host = torch.empty(2, dtype=torch.int64).pin_memory()
        self.in_bytes = sum(v.numel() * v.element_size() for v in self.pinned.values())
        self.np_rows = 1 << int(np.ceil(np.log2(self.n)))
        self.rec_bytes = 16  # 2-word records (the predicate's bands fit the packed layout)
        self.flush_l2 = False  # inputs (156 MB) and records (134 MB) exceed the 126 MB L2

    def step(self):
        self.capi.filter_groupby(self.dev, self.n, self.pred, self.G, scratch=self.scratch, out=self.out,
                                 counts=self.counts)

    def step_e2e(self):
        for k in self.dev:
            self.dev[k].copy_(self.pinned[k], non_blocking=True)
        self.step()
        self.out_host.copy_(self.out, non_blocking=True)
        self.counts_host.copy_(self.counts, non_blocking=True)

    def d2h_bytes(self):
        return self.out.numel() * 8 + self.counts.numel() * 8

    def launches(self):
        logn = int(np.log2(self.np_rows))
        return 2 + compact_passes(logn, 12, PIPE_LMAX) + sort_passes(logn, 12, PIPE_LMAX) + 4

    def rdm_bytes(self):
        npr = self.np_rows
        pred = self.n * 9
        comp = self.n * 5 + 2 * npr * 24 * rdm_pcomp(npr)
        srt = 2 * npr * 40 * rdm_psort(npr)
        heads = 2 * npr * 40
        return pred + comp + srt + heads

    def check(self, orc):
        g, keys, sums = orc.filter_groupby(self.host, self.pred, self.G)
        out = self.out.cpu().numpy()
        cnt = self.counts.cpu().numpy()
        ok = int(cnt[1]) == g and np.array_equal(out[:g, 0], keys.astype(np.int64)) and np.array_equal(
            out[:g, 1:], sums)
        return bool(ok)

    def dominant(self, device):
        """The dominant kernel is the bitonic pass kernel of the pipeline's
        sort stage (about 70 % of the step in the ncu launch list).  Its
        launches are timed inside the pipeline itself: with stage timing on,
        velo_filter_groupby records CUDA events on its stream around each
        stage, and the sort stage's time is divided by its launch count.  The
        records are 2 words (16 B: the predicate's quantity and discount bands
        fit the packed layout) over next_pow2(6,001,215) = 2^23 rows, and
        every launch reads and writes every record once: 2 x 2^23 x 16 B."""
        capi = self.capi
        logn = int(np.log2(self.np_rows))
        launches = sort_passes(logn, 12, PIPE_LMAX)
        capi.set_stage_timing(True)
        ts = []
        try:
            for i in range(6):
                self.step()
                st = capi.last_stage_times()
                if i:
                    ts.append(st[2])
        finally:
            capi.set_stage_timing(False)
        return {"kernel": "k_sort_pass<RowRec<2,1,false,KEY_HI32>,8,4> (bitonic passes of the sort stage, "
                          "2^23 x 16 B records)",
                "launches_per_sort": launches, "avg_launch_us": float(np.mean(ts)) * 1e3 / launches,
                "bytes_per_launch": int(2 * self.np_rows * 16)}


def dominant_timing(torch, run, reset, launches, bytes_per_launch, name, reps=5):
    """Average launch duration of the dominant kernel from CUDA events around
    whole sorts (each sort = `launches` launches of the kernel), with the
    input restored between sorts outside the timed events."""
    ts = []
    for i in range(reps + 1):
        reset()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        run()
        e.record()
        torch.cuda.synchronize()
        if i:
            ts.append(s.elapsed_time(e))
    per_launch_ms = float(np.mean(ts)) / launches
    return {"kernel": name, "launches_per_sort": launches, "avg_launch_us": per_launch_ms * 1e3,
            "bytes_per_launch": int(bytes_per_launch)}


class JoinTopK:
    """Config-2 shape: oblivious PK-FK join of a 1,500,000-row dimension
    table and a 6,000,000-row fact table (~50 % filters on each side),
    group-by fk over the joined rows, top-10 groups by sum(price).  Throughput
    counts the 7.5 M input rows."""
    name = "join_groupby_top10"

    def __init__(self, torch, capi, W, device):
        self.torch, self.capi = torch, capi
        dim, fact = W.join_tables()
        self.host = (dim, fact)
        self.nd, self.nf = len(dim["key"]), len(fact["fk"])
        self.n = self.nd + self.nf
        self.pred = W.JOIN_PRED
        self.k = W.JOIN_TOPK
        self.pinned = {"dim_key": torch.from_numpy(dim["key"]).pin_memory(),
                       "dim_date": torch.from_numpy(dim["date"]).pin_memory(),
                       "fact_fk": torch.from_numpy(fact["fk"]).pin_memory(),
                       "fact_price": torch.from_numpy(fact["price"]).pin_memory()}
        self.dev = {k: v.to(device) for k, v in self.pinned.items()}
        self.scratch = torch.empty(capi.join_groupby_topk_scratch_bytes(self.nd, self.nf), dtype=torch.uint8,
                                   device=device)
        self.out = torch.empty((self.k, 3), dtype=torch.int64, device=device)
        self.counts = torch.empty(2, dtype=torch.int64, device=device)
        self.out_host = torch.empty((self.k, 3), dtype=torch.int64).pin_memory()
        self.counts_host = torch.empty(2, dtype=torch.int64).pin_memory()
        self.in_bytes = sum(v.numel() * v.element_size() for v in self.pinned.values())
        self.np_rows = 1 << int(np.ceil(np.log2(self.n)))
        self.rec_bytes = 16
        self.flush_l2 = False  # inputs (60 MB) plus union records (268 MB) exceed the 126 MB L2

    def step(self):
        self.capi.join_groupby_topk(self.dev, self.pred, self.k, scratch=self.scratch, out=self.out,
                                    counts=self.counts)

    def step_e2e(self):
        for key in self.dev:
            self.dev[key].copy_(self.pinned[key], non_blocking=True)
        self.step()
        self.out_host.copy_(self.out, non_blocking=True)
        self.counts_host.copy_(self.counts, non_blocking=True)

    def d2h_bytes(self):
        return self.out.numel() * 8 + self.counts.numel() * 8

    def launches(self):
        u = int(np.log2(self.np_rows))
        top = int(np.log2(1 << int(np.ceil(np.log2(self.nd)))))
        # pack, union sort, fill, count+scan, compaction, aggregation, count+scan,
        # group compaction, top-k pack, tile pass, candidates, candidate sort, out
        cand = int(np.log2((1 << max(0, top - 12)) * 16)) if top > 12 else 0
        topk = (1 + 1 + sort_passes(cand, 12, PIPE_LMAX)) if top > 12 else sort_passes(top, 12, PIPE_LMAX)
        return (1 + sort_passes(u, 12, PIPE_LMAX) + 3 + 2 + compact_passes(u, 12, PIPE_LMAX) + 3 + 2
                + compact_passes(u, 12, PIPE_LMAX) + 1 + topk + 1)

    def rdm_bytes(self):
        """The algorithmic-bytes model of the join pipeline: union sort
        (24 B), compaction to the fact bound, sort by fk (16 B), compaction of
        the group heads, top-k sort over the dimension bound (16 B), plus one
        streaming read and write of the union for the fill and the scan."""
        u = self.np_rows
        d = 1 << int(np.ceil(np.log2(self.nd)))
        return (2 * u * 24 * rdm_psort(u) + self.nf * 5 + 2 * u * 24 * rdm_pcomp(u) + 2 * u * 16 * rdm_psort(u)
                + 2 * u * 24 * rdm_pcomp(u) + 2 * d * 16 * rdm_psort(d) + 2 * 2 * u * 24)

    def check(self, orc):
        dim, fact = self.host
        g, ofk, osum, ocnt = orc.join_groupby_topk(dim, fact, self.pred, self.k)
        out = self.out.cpu().numpy()
        cnt = self.counts.cpu().numpy()
        m = min(g, self.k)
        return bool(int(cnt[1]) == g and np.array_equal(out[:m, 0], ofk) and np.array_equal(out[:m, 1], osum)
                    and np.array_equal(out[:m, 2], ocnt))

    def dominant(self, device):
        """The dominant kernel is the bitonic pass kernel of the union sort
        (next_pow2(7.5 M) = 2^23 records of 2 words, 4096-row tiles), timed
        live through the pipeline's stage timer (stage 2 = the union sort)."""
        capi = self.capi
        launches = sort_passes(int(np.log2(self.np_rows)), 12, PIPE_LMAX)
        capi.set_stage_timing(True)
        ts = []
        try:
            for i in range(6):
                self.step()
                st = capi.last_stage_times()
                if i:
                    ts.append(st[1])
        finally:
            capi.set_stage_timing(False)
        return {"kernel": "k_sort_pass<RowRec<2,1,false,KEY_FULL>,8,4> (union sort, 2^23 x 16 B records)",
                "launches_per_sort": launches, "avg_launch_us": float(np.mean(ts)) * 1e3 / launches,
                "bytes_per_launch": int(2 * self.np_rows * 16)}


def make_workload(name, torch, capi, W, device):
    if name == "groupby":
        return GroupBy(torch, capi, W, device)
    if name == "join":
        return JoinTopK(torch, capi, W, device)
    if name == "sort":
        return SortKP(torch, capi, W, device)
    if name == "batch":
        return Batched(torch, capi, W, device)
    raise SystemExit(f"unknown workload {name}")


class Batched:
    """Config-3 shape: 512 independent instances (log-uniform 2^10..2^22
    rows; even = sort of (u64 key, u32 payload), odd = compaction with
    Bernoulli(0.3) keep flags), each padded to its own power of two, run by
    ONE persistent launch captured in a CUDA graph, tile configuration picked
    by the autotuner.  The plain path (one launch sequence per instance,
    back to back) is timed beside it."""
    name = "batched_512"

    def __init__(self, torch, capi, W, device):
        self.torch, self.capi = torch, capi
        insts = W.batch_instances()
        self.items = []
        self.host = []
        for it in insts:
            n = it["n"]
            cap = capi.next_pow2(n)
            d = dict(kind=it["kind"], n=n, keys=capi.to_dev_u64(it["keys"], cap),
                     pay=capi.to_dev_u32(it["pay"], cap))
            if it["kind"] == "compact":
                d["marks"] = capi.to_dev_u8(it["marks"], cap)
                d["count"] = torch.zeros(1, dtype=torch.int64, device=device)
            self.items.append(d)
            self.host.append(it)
        self.n = int(sum(it["n"] for it in insts))
        self.np_rows = int(sum(capi.next_pow2(it["n"]) for it in insts))
        self.rec_bytes = 12
        self.flush_l2 = False  # 3.4 GB of instances, far beyond L2
        self.in_bytes = int(sum(it["n"] * (12 + (1 if it["kind"] == "compact" else 0)) for it in insts))
        self.tune, self.tune_ms = capi.batch_autotune(self.items, reps=1)
        self.batch = capi.Batch(self.items, tune=self.tune)
        self.stream = torch.cuda.Stream()
        self.batch.launch(stream=self.stream)
        self.batch.status(stream=self.stream)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            self.batch.launch(stream=self.stream)
        self.pinned = [(torch.from_numpy(h["keys"].view(np.int64)).pin_memory(),
                        torch.from_numpy(h["pay"].view(np.int32)).pin_memory(),
                        torch.from_numpy(h["marks"]).pin_memory() if h["kind"] == "compact" else None)
                       for h in insts]
        self.count_host = torch.zeros(len(self.items), dtype=torch.int64).pin_memory()

    def step(self):
        self.graph.replay()

    def step_plain(self):
        for it in self.items:
            if it["kind"] == "sort":
                self.capi.osort_kp(it["keys"], it["pay"], it["n"], tune=self.tune)
            else:
                self.capi.ocompact_kpm(it["keys"], it["pay"], it["marks"], it["n"], tune=self.tune)

    def step_e2e(self):
        for it, (k, p, m) in zip(self.items, self.pinned):
            it["keys"][: it["n"]].copy_(k, non_blocking=True)
            it["pay"][: it["n"]].copy_(p, non_blocking=True)
            if m is not None:
                it["marks"][: it["n"]].copy_(m, non_blocking=True)
        self.step()
        for i, it in enumerate(self.items):
            if "count" in it:
                self.count_host[i: i + 1].copy_(it["count"], non_blocking=True)

    def d2h_bytes(self):
        return 8 * sum(1 for it in self.items if "count" in it)

    def launches(self):
        return 1  # one persistent kernel per step (plus one counter memset)

    def rdm_bytes(self):
        tot = 0
        for it in self.items:
            npr = self.capi.next_pow2(it["n"])
            if it["kind"] == "sort":
                tot += 2 * npr * 12 * rdm_psort(npr)
            else:
                tot += it["n"] * 5 + 2 * npr * 13 * rdm_pcomp(npr)
        return tot

    def check(self, orc):
        self.batch.status(stream=self.stream)
        ok = True
        for it, h in list(zip(self.items, self.host))[:24]:
            if it["kind"] == "sort":
                k = it["keys"].cpu().numpy().view(np.uint64)[: it["n"]]
                o = np.sort(h["keys"])
                ok &= bool(np.array_equal(k, o))
            else:
                c = int(it["count"].item())
                ok &= c == int(h["marks"].sum())
                k = it["keys"].cpu().numpy().view(np.uint64)[:c]
                ok &= bool(np.array_equal(k, h["keys"][h["marks"].astype(bool)]))
        return ok

    def dominant(self, device):
        """The persistent scheduler kernel is the only kernel of the step;
        its algorithmic bytes per launch are the batch's network bytes."""
        torch = self.torch
        ts = []
        for i in range(4):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            self.graph.replay()
            e.record()
            torch.cuda.synchronize()
            if i:
                ts.append(s.elapsed_time(e))
        bytes_ = 0
        for it in self.items:
            npr = self.capi.next_pow2(it["n"])
            lt = self.tune[0]
            lmax = min(8, lt - 5)
            if it["kind"] == "sort":
                bytes_ += 2 * npr * 12 * sort_passes(int(np.log2(npr)), lt, lmax)
            else:
                bytes_ += 2 * npr * 13 * compact_passes(int(np.log2(npr)), lt, lmax) + npr * 5
        return {"kernel": f"k_sched (persistent, tile 2^{self.tune[0]} x {self.tune[1]} threads)",
                "launches_per_sort": 1, "avg_launch_us": float(np.mean(ts)) * 1e3, "bytes_per_launch": int(bytes_)}


class SortKP:
    """Config-0 shape: plain oblivious sort of 2^20 (u64 key, u32 payload) rows."""
    name = "plain_sort_2^20"

    def __init__(self, torch, capi, W, device):
        self.torch, self.capi = torch, capi
        self.n = 1 << 20
        keys, pay = W.sort_kp(self.n)
        self.pinned_k = torch.from_numpy(keys.view(np.int64)).pin_memory()
        self.pinned_p = torch.from_numpy(pay.view(np.int32)).pin_memory()
        self.k0 = self.pinned_k.to(device)
        self.p0 = self.pinned_p.to(device)
        self.k = torch.empty_like(self.k0)
        self.p = torch.empty_like(self.p0)
        self.kh = torch.empty_like(self.pinned_k).pin_memory()
        self.ph = torch.empty_like(self.pinned_p).pin_memory()
        self.in_bytes = self.n * 12
        self.np_rows = self.n
        self.rec_bytes = 12
        self.flush_l2 = True  # 12.6 MB fits in L2: flushed between steps

    def step(self):
        # the network sorts in place: restore the unsorted input first (the
        # restore is a device copy inside the timed step)
        self.k.copy_(self.k0)
        self.p.copy_(self.p0)
        self.capi.osort_kp(self.k, self.p, self.n)

    def step_e2e(self):
        self.k.copy_(self.pinned_k, non_blocking=True)
        self.p.copy_(self.pinned_p, non_blocking=True)
        self.capi.osort_kp(self.k, self.p, self.n)
        self.kh.copy_(self.k, non_blocking=True)
        self.ph.copy_(self.p, non_blocking=True)

    def d2h_bytes(self):
        return self.n * 12

    def launches(self):
        return sort_passes(20, 12, 7)

    def rdm_bytes(self):
        return 2 * self.n * 12 * rdm_psort(self.n)

    def check(self, orc):
        k = self.k.cpu().numpy().view(np.uint64)
        p = self.p.cpu().numpy().view(np.uint32)
        ok_, op_ = orc.bitonic_kp(self.k0.cpu().numpy().view(np.uint64), self.p0.cpu().numpy().view(np.uint32))
        return bool(np.array_equal(k, ok_) and np.array_equal(p, op_))

    def dominant(self, device):
        """The bitonic pass kernel is the only kernel of the step; every
        launch reads and writes every (8 B key + 4 B payload) row once."""
        run = lambda: self.capi.osort_kp(self.k, self.p, self.n)  # noqa: E731

        def reset():
            self.k.copy_(self.k0)
            self.p.copy_(self.p0)

        return dominant_timing(self.torch, run, reset, self.launches(), 2 * self.n * 12,
                               "k_sort_pass<RowKP> (bitonic passes, 2^20 x 12 B rows)")


# --------------------------------------------------------------------------

def time_steps(torch, fn, steps, flush=None, stream=None):
    """Per-step CUDA-event durations (ms) of `fn`, flushing L2 between steps
    outside the timed events when asked."""
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for s, e in evs:
        if flush is not None:
            flush()
        s.record()
        fn()
        e.record()
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in evs]


def cpu_baseline_groupby(W, orc):
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    n = 1 << 21
    cols = W.lineitem(n)
    t0 = time.perf_counter()
    reps = 0
    while True:
        orc.filter_groupby(cols, W.LINEITEM_PRED, 8, n_threads=cores)
        reps += 1
        if time.perf_counter() - t0 > 10.0 or reps >= 50:
            break
    dt = (time.perf_counter() - t0) / reps
    del mp
    return {"value": n / dt / 1e6, "unit": "Mrows/s", "cores": cores, "kind": "port",
            "sample": f"first {n} rows of the 6,001,215-row table, {reps} runs, OpenMP over all cores"}


def cpu_baseline_sort(W, orc):
    cores = os.cpu_count() or 1
    n = 1 << 20
    keys, pay = W.sort_kp(n)
    t0 = time.perf_counter()
    reps = 0
    while True:
        orc.bitonic_kp(keys, pay, n_threads=cores)
        reps += 1
        if time.perf_counter() - t0 > 10.0 or reps >= 200:
            break
    dt = (time.perf_counter() - t0) / reps
    return {"value": n / dt / 1e6, "unit": "Mrows/s", "cores": cores, "kind": "port",
            "sample": f"full 2^20-row sort, {reps} runs, OpenMP over all cores"}


def cpu_baseline_join(W, orc):
    cores = os.cpu_count() or 1
    dim, fact = W.join_tables()
    t0 = time.perf_counter()
    reps = 0
    while True:
        orc.join_groupby_topk(dim, fact, W.JOIN_PRED, W.JOIN_TOPK, n_threads=cores)
        reps += 1
        if time.perf_counter() - t0 > 10.0 or reps >= 20:
            break
    dt = (time.perf_counter() - t0) / reps
    n = len(dim["key"]) + len(fact["fk"])
    return {"value": n / dt / 1e6, "unit": "Mrows/s", "cores": cores, "kind": "port",
            "sample": f"full 1.5 M + 6 M-row join, {reps} runs, OpenMP over all cores"}


def cpu_baseline_batch(W, orc):
    """The oracle on instances of the 512 in a fixed stride order until about
    10 s of CPU work: sorts on all cores, compactions single-threaded."""
    cores = os.cpu_count() or 1
    insts = W.batch_instances()
    rows, t_tot, used = 0, 0.0, 0
    for i in range(len(insts)):
        it = insts[(i * 97) % len(insts)]
        if it["kind"] == "sort":
            t0 = time.perf_counter()
            orc.bitonic_kp(it["keys"], it["pay"], n_threads=cores)
        else:
            r = np.zeros((it["n"], 16), np.uint8)
            r[:, :8] = it["keys"].view(np.uint8).reshape(-1, 8)
            r[:, 8:12] = it["pay"].view(np.uint8).reshape(-1, 4)
            t0 = time.perf_counter()
            orc.ocompact(r, it["marks"])
        t_tot += time.perf_counter() - t0
        rows += it["n"]
        used += 1
        if t_tot > 10.0:
            break
    return {"value": rows / t_tot / 1e6, "unit": "Mrows/s", "cores": cores, "kind": "port",
            "sample": f"{used} of the 512 instances (stride 97 through the list, {rows} rows); sorts on all "
                      f"cores, compactions single-threaded"}


def run_reference(args, rank):
    """CPU reference arm: the reference's algorithm for the path (the oracle
    port in the reference's network order) on all host cores, rank 0 only.
    Each step is a bounded sample of the workload: the whole table for
    groupby and sort, one instance of the 512 for batch, one query of the
    stream for serve."""
    if rank != 0:
        return
    import oracle as orc
    from velodb_b200 import workloads as W

    orc.lib()
    cores = os.cpu_count() or 1
    unit = "Mrows/s"
    if args.workload == "sort":
        n = 1 << 20
        keys, pay = W.sort_kp(n)
        steps = [(lambda: orc.bitonic_kp(keys, pay, n_threads=cores), n)]
        sample, wl = "full 2^20-row sort per step", "plain_sort_2^20"
    elif args.workload == "batch":
        insts = W.batch_instances()
        order = [(i * 97) % len(insts) for i in range(len(insts))]

        def inst_fn(it):
            if it["kind"] == "sort":
                return lambda: orc.bitonic_kp(it["keys"], it["pay"], n_threads=cores)
            rows = np.zeros((it["n"], 16), np.uint8)
            rows[:, :8] = it["keys"].view(np.uint8).reshape(-1, 8)
            rows[:, 8:12] = it["pay"].view(np.uint8).reshape(-1, 4)
            return lambda: orc.ocompact(rows, it["marks"])

        steps = [(inst_fn(insts[i]), insts[i]["n"]) for i in order]
        sample = "one of the 512 instances per step (stride 97 through the list); sorts on all cores, " \
                 "compactions single-threaded"
        wl = "batched_512"
    elif args.workload == "join":
        dim, fact = W.join_tables()
        steps = [(lambda: orc.join_groupby_topk(dim, fact, W.JOIN_PRED, W.JOIN_TOPK, n_threads=cores),
                  len(dim["key"]) + len(fact["fk"]))]
        sample, wl = "full 1.5 M + 6 M-row join per step", "join_groupby_top10"
    elif args.workload == "serve":
        from velodb_b200 import serving as S

        hs = S.HostSlices(**S.FULL_SCALE)
        lo, hi = SERVE_DISTS["short"]
        qs = [q for q in S.query_stream(hs, 4 * (args.steps + args.warmup) + 8, seed=0xB200000000000004,
                                        lo_log2=lo, hi_log2=hi) if q.shape != S.Q_JOIN3]

        def q_fn(q):
            if q.shape == S.Q_FILTER_GROUPBY:
                cols = hs.lineitem(q.offset, q.n)
                return lambda: orc.filter_groupby(cols, W.LINEITEM_PRED, 8, n_threads=cores)
            dim, fact = hs.join_inputs(q)
            return lambda: orc.join_groupby_topk(dim, fact, W.JOIN_PRED, 10, n_threads=cores)

        steps = [(q_fn(q), 1) for q in qs]
        unit = "queries/s"
        sample = "one query per step from the served stream (sizes 2^10..2^18), filter+group-by and " \
                 "two-way join shapes (the three-way chain has no oracle pipeline)"
        wl = "served_stream"
    else:
        # the reference reveals the filtered count and sorts next_pow2(count)
        # rows (src/operator/filter_compaction_operator.cpp:171-178)
        n = W.LINEITEM_ROWS
        cols = W.lineitem(n)
        steps = [(lambda: orc.filter_groupby(cols, W.LINEITEM_PRED, 8, n_threads=cores), n)]
        sample, wl = "full 6,001,215-row table per step (filtered count revealed)", "filter_groupby"
    for i in range(args.warmup):
        steps[i % len(steps)][0]()
    ts, units = [], 0
    for i in range(args.steps):
        fn, u = steps[(args.warmup + i) % len(steps)]
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
        units += u
    total = float(np.sum(ts))
    ms = 1e3 * total / args.steps
    value = units / total / (1e6 if unit == "Mrows/s" else 1.0)
    line = {
        "impl": "reference", "metric": metric_name(args.workload), "value": value, "unit": unit,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": wl},
        "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# served query stream (resident tables, continuous admission)
# --------------------------------------------------------------------------

SERVE_DISTS = {"short": (10.0, 18.0), "analytic": (14.0, 22.0)}
SERVE_LOADS = (0.5, 0.9, 1.5, 3.0, 6.0)


def _lat(results, t_key="submit_ms"):
    lat = np.asarray([r.end_ms - getattr(r, t_key) for r in results])
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}


def run_serve(args, world, rank, local):
    """Config-4 shape: a seeded query stream (50 % filter + group-by, 35 %
    two-way join + top-10, 15 % three-way chain) over resident tables of
    60 M / 15 M / 150 M rows, admitted by a 120 GB HBM budget.  The plain
    path is the same request loop with one slot, each query submitted after
    the previous one returned; the served path admits up to 16 queries at a
    time on their own streams.  Latency is submit -> result in host memory on
    the host clock (the request loop spans many streams, so no single device
    event brackets it); `value` is the served throughput at saturation."""
    import torch
    import torch.distributed as dist

    from velodb_b200 import serving as S

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)
    t0 = time.perf_counter()
    tab = S.ServedTables(**S.FULL_SCALE)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(120 << 30, free - (4 << 30)))
    nq = max(128, 32 * args.steps)
    slots = 16
    out = {}
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    for dname, (lo, hi) in SERVE_DISTS.items():
        qs = S.query_stream(tab, nq, seed=0xB200000000000004, lo_log2=lo, hi_log2=hi)
        srv = S.Server(tab, slots=1, budget_bytes=budget)
        S.run_closed_one_at_a_time(srv, qs[: max(8, args.warmup)])
        plain_res, plain_s = S.run_closed_one_at_a_time(srv, qs)
        plain_qps = nq / plain_s
        plain_loads = {}
        for f in (0.5, 0.9):
            r, _ = S.run_open_loop(srv, qs, S.arrivals(nq, f * plain_qps, seed=int(f * 1000)))
            plain_loads[f"{f}x"] = {"offered_qps": f * plain_qps, **_lat(r)}
        srv.close()
        srv = S.Server(tab, slots=slots, budget_bytes=budget)
        S.run_open_loop(srv, qs[: max(16, args.warmup)], np.zeros(max(16, args.warmup)))
        sat_res, sat_s = S.run_open_loop(srv, qs, np.zeros(nq))
        served_qps = nq / sat_s
        loads = {}
        for f in SERVE_LOADS:
            r, s = S.run_open_loop(srv, qs, S.arrivals(nq, f * plain_qps, seed=int(f * 1000)))
            loads[f"{f}x"] = {"offered_qps": f * plain_qps, "achieved_qps": nq / s, **_lat(r)}
        st = srv.stats()
        srv.close()
        same = all(S.result_key(a) == S.result_key(b) and a.status == 0 and b.status == 0
                   for a, b in zip(plain_res, sat_res))
        shapes = {S.SHAPE_NAMES[k]: int(sum(1 for q in qs if q.shape == k)) for k in S.SHAPE_NAMES}
        out[dname] = {
            "sizes_log2": [lo, hi], "queries": nq, "mix": shapes,
            "plain": {"qps": plain_qps, **_lat(plain_res), "under_poisson": plain_loads},
            "served": {"qps_saturation": served_qps, **_lat(sat_res), "slots": slots,
                       "peak_inflight": st["peak_inflight"], "peak_arena_bytes": st["peak_arena_bytes"],
                       "poisson": loads},
            "speedup_served_vs_plain": served_qps / plain_qps,
            "results_identical_alone_and_in_mix": bool(same),
        }
    clk = clocks.stop()
    head = out["short"]
    value = head["served"]["qps_saturation"]
    value, _ = aggregate_throughput(1.0, 1e3 / value, world, device, scale=1.0)
    from velodb_b200._lib import VeloQuery, VeloQueryResult

    line = {
        "metric": metric_name("serve"), "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": nq, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": "served_stream", "tables_rows": dict(S.FULL_SCALE),
                   "resident_bytes": int(tab.bytes), "table_build_s": build_s, "hbm_budget_bytes": budget,
                   "headline_sizes_log2": list(SERVE_DISTS["short"]), "parallelism": f"replicas{world}",
                   "timing": "host clock, submit -> result in host memory",
                   "l2": "inputs larger than L2 (resident tables 4.9 GB)"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": C_sizeof(VeloQuery),
                "d2h_bytes_per_step": C_sizeof(VeloQueryResult),
                "note": "the served numbers are end to end: a query descriptor in, a result struct out"},
        "serve": out, "clocks": clk,
        "gpu_launches": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def C_sizeof(t):
    import ctypes

    return ctypes.sizeof(t)


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The slowest rank's value (every rank takes part; identity at N = 1)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_throughput(units_per_rank: float, ms: float, world: int, device=None, scale: float = 1e6) -> tuple:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    ms_max = max_over_ranks(ms, world, device)
    return world * units_per_rank / (ms_max / 1e3) / scale, ms_max


def metric_name(workload):
    if workload == "join":
        return "oblivious PK-FK join + group-by + top-10 input throughput (1.5 M dim + 6 M fact rows)"
    if workload == "serve":
        return "served query throughput at saturation (queries/s; p50/p99 vs plain one-at-a-time)"
    if workload == "batch":
        return "batched oblivious sorts+compactions throughput (512 instances, 2^10..2^22 rows)"
    if workload == "sort":
        return "oblivious bitonic sort throughput (2^20 rows, u64 key + u32 payload)"
    return "oblivious filter+group-by input throughput (6,001,215-row fact table)"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="groupby", choices=["groupby", "sort", "batch", "serve", "join"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "serve":
        run_serve(args, world, rank, local)
        return

    import torch
    import torch.distributed as dist

    from velodb_b200 import capi, workloads as W

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=device)

    wl = make_workload(args.workload, torch, capi, W, device)
    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device=device) if wl.flush_l2 else None
    flush = (lambda: l2_flush.fill_(1)) if l2_flush is not None else None

    for _ in range(args.warmup):
        wl.step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ts = time_steps(torch, wl.step, args.steps, flush)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    rows_per_step = wl.n
    value, ms = aggregate_throughput(rows_per_step, float(np.mean(ts)), world, device)

    # end to end through the public API with host buffers
    for _ in range(2):
        wl.step_e2e()
    torch.cuda.synchronize()
    te = time_steps(torch, wl.step_e2e, max(3, args.steps // 2))
    e2e_value, ems = aggregate_throughput(rows_per_step, float(np.mean(te)), world, device)
    e2e = {"value": e2e_value, "unit": "Mrows/s",
           "h2d_bytes_per_step": int(wl.in_bytes), "d2h_bytes_per_step": int(wl.d2h_bytes()), "ms_per_step": ems}

    if hasattr(wl, "step_plain"):
        for _ in range(2):
            wl.step_plain()
        torch.cuda.synchronize()
        tp = time_steps(torch, wl.step_plain, max(3, args.steps // 2))
        pms = float(np.mean(tp))
        plain = {"ms_per_step": pms, "value": world * rows_per_step / (pms / 1e3) / 1e6,
                 "speedup_batched_vs_plain": pms / ms, "tune": list(wl.tune),
                 "autotune_ms": {f"{k[0]}x{k[1]}": v for k, v in wl.tune_ms.items()}}
    else:
        plain = None

    # the result of the last step is checked against the oracle (rank 0)
    peak, peak_kind = hbm_peak()
    rdm = wl.rdm_bytes()
    line = {
        "metric": metric_name(args.workload), "value": value, "unit": "Mrows/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": wl.name, "rows": rows_per_step, "padded_rows": wl.np_rows,
                   "record_bytes": wl.rec_bytes, "parallelism": f"replicas{world}",
                   "l2": "flushed between steps" if wl.flush_l2 else "inputs larger than L2"},
        "e2e": e2e,
        "gpu_launches": int(wl.launches() * args.steps),
        "rdm": {"bytes_per_step": int(rdm), "achieved_gbs": rdm / (ms / 1e3) / 1e9,
                "frac_of_hbm": rdm / (ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind},
        "clocks": clk,
    }
    if plain is not None:
        line["plain_path"] = plain
    dom = wl.dominant(device)
    achieved = dom["bytes_per_launch"] / (dom["avg_launch_us"] / 1e6) / 1e9
    line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                        if peak_kind == "measured" else "fallback", "traffic": TRAFFIC.get(args.workload),
                        "kernel": dom["kernel"], "avg_launch_us": dom["avg_launch_us"],
                        "algorithmic_bytes_per_launch": dom["bytes_per_launch"]}
    if rank == 0:
        import oracle as orc

        orc.lib()
        line["checked_against_oracle"] = wl.check(orc)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = {"groupby": cpu_baseline_groupby, "sort": cpu_baseline_sort,
                                    "batch": cpu_baseline_batch, "join": cpu_baseline_join}[args.workload](W, orc)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
