#!/usr/bin/env python3
"""Benchmark of the oblivious operator hot path on B200.

Headline workload (the default): the oblivious PK-FK sort-merge join of a
1,500,000-row dimension table and a 6,000,000-row fact table, followed by an
oblivious group-by on the foreign key and the top-10 groups by sum(price)
(union -> bitonic sort on (key, tag) -> forward fill -> ORCompact -> segmented
sums -> bitonic top-k).  One step = one pass of that pipeline over the two
tables.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload join|sort|groupby|batch|serve] [--extras all|none]

At N = 1 the same run also measures, each in its own key of `extras` and
each checked against the oracle: the plain sort of 2^20 (u64 key, u32
payload) rows and of 2^24 rows (inputs far beyond L2: the HBM case), the
filter + group-by over the 6,001,215-row fact table, the batch of 512 uneven
sorts and compactions (one persistent launch from a CUDA graph, and as jobs of
the persistent command queue, against 512 plain launch sequences), and the
served query stream (p50/p99 latency and throughput, served on per-query
streams and through the persistent command queue, against plain
one-at-a-time).

Every network pass is also timed on its own with CUDA events (the library's
pass timer) and the line reports the achieved HBM bandwidth per pass kind:
tile sort, in-tile merge, fused global levels, ORCompact tile and global
passes.

`e2e` is the same pipeline through the public API from pinned host buffers,
every step's host -> device and device -> host copies inside the timed
region, with three input/output sets in flight so that the copies of
neighbouring steps overlap the pipeline; `e2e.serial` is the one step at a
time form (copy in, pipeline, copy out).

Multi-GPU: one process per GPU (torchrun); the path does not shard, so every
rank runs an independent replica of the headline workload ("replicas only")
and the aggregate throughput is the total rows of all ranks over the slowest
rank's time.  `--impl reference` times the CPU oblivious path on rank 0: the
oracle's oblivious pipeline (network sorts over all next_pow2(n) rows in the
reference's network order, ORCompact, segmented sums) on all host cores.
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
FALLBACK_HBM_GBS = 6650.0
METRIC = "obliv sort & join Mrows/s (frac of HBM peak); p50/p99 latency served vs plain"

# DRAM bytes (read + write) per launch of the dominant kernel from one ncu
# capture of the same pipeline (the mean over its sort passes), or None when
# no capture of that launch exists.
TRAFFIC = {"groupby": 210.1e6, "sort": 12.65e6, "join": 210.6e6, "batch": None}

# warm-up runs at least this long (seconds) so that the clock samples taken
# from the end of the warm-up through the timed steps show the GPU under load
SOAK_S = 1.5


def hbm_peak():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# --------------------------------------------------------------------------
# pass-count models
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
    """Pass count of the algorithmic-bytes model: T = 2^13, L = 8."""
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
        self.path = os.path.join("/tmp", f"velo_clocks_{os.getpid()}_{index}.csv")

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
                "reasons": sorted(reasons), "samples": len(sm),
                "window": f"the last {SOAK_S} s of the warm-up and the timed steps"}


# --------------------------------------------------------------------------
# workloads (ours)
# --------------------------------------------------------------------------

class JoinTopK:
    """Oblivious PK-FK join of a 1,500,000-row dimension table and a
    6,000,000-row fact table (~50 % filters on each side), group-by fk over
    the joined rows, top-10 groups by sum(price).  Throughput counts the
    7.5 M input rows."""
    name = "join_groupby_top10"
    key = "join"

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
        self.kernel = ("k_sort_pass<RowRec<2,1,false,KEY_FULL>,8,4,PK,2> (union sort: 2^23 two-word records, "
                       "4096-row tiles, two CTAs per SM)")

    def step(self):
        self.capi.join_groupby_topk(self.dev, self.pred, self.k, scratch=self.scratch, out=self.out,
                                    counts=self.counts)

    def step_e2e(self):
        for key in self.dev:
            self.dev[key].copy_(self.pinned[key], non_blocking=True)
        self.step()
        self.out_host.copy_(self.out, non_blocking=True)
        self.counts_host.copy_(self.counts, non_blocking=True)

    # one input/output set of the pipelined end-to-end form
    def e2e_set(self):
        t = self.torch
        return {"dev": {k: t.empty_like(v, device=self.out.device) for k, v in self.pinned.items()},
                "out": t.empty_like(self.out), "counts": t.empty_like(self.counts),
                "out_host": t.empty_like(self.out_host).pin_memory(),
                "counts_host": t.empty_like(self.counts_host).pin_memory()}

    def e2e_in(self, b):
        for key in b["dev"]:
            b["dev"][key].copy_(self.pinned[key], non_blocking=True)

    def e2e_run(self, b):
        self.capi.join_groupby_topk(b["dev"], self.pred, self.k, scratch=self.scratch, out=b["out"],
                                    counts=b["counts"])

    def e2e_out(self, b):
        b["out_host"].copy_(b["out"], non_blocking=True)
        b["counts_host"].copy_(b["counts"], non_blocking=True)

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
        """The oracle's pipeline, and an independent numpy join + bincount."""
        dim, fact = self.host
        g, ofk, osum, ocnt = orc.join_groupby_topk(dim, fact, self.pred, self.k)
        out = self.out.cpu().numpy()
        cnt = self.counts.cpu().numpy()
        m = min(g, self.k)
        ok = int(cnt[1]) == g and np.array_equal(out[:m, 0], ofk) and np.array_equal(out[:m, 1], osum) \
            and np.array_equal(out[:m, 2], ocnt)
        nfk, nsum, ncnt, ng = numpy_join_topk(dim, fact, self.pred, self.k)
        ok = ok and ng == g and np.array_equal(out[:m, 0], nfk) and np.array_equal(out[:m, 1], nsum) \
            and np.array_equal(out[:m, 2], ncnt)
        return bool(ok)


def numpy_join_topk(dim, fact, pred, k):
    """The join + group-by + top-k computed directly with numpy (no oracle
    code): dimension rows passing the date filter, fact rows passing the price
    filter and whose key has a passing dimension row, sums by bincount, the k
    largest sums with ties to the smaller key."""
    nd = len(dim["key"])
    keep_dim = np.zeros(nd + 2, bool)
    keep_dim[dim["key"][dim["date"] < pred["date_hi"]]] = True
    fk = fact["fk"].astype(np.int64)
    joined = (fact["price"] < pred["price_hi"]) & keep_dim[fk]
    cnts = np.bincount(fk[joined], minlength=nd + 2).astype(np.int64)
    psum = np.zeros(nd + 2, np.int64)
    np.add.at(psum, fk[joined], fact["price"][joined])
    groups = np.nonzero(cnts)[0]
    order = np.lexsort((groups, -psum[groups]))[:k]
    top = groups[order]
    return top.astype(np.int64), psum[top], cnts[top], int(len(groups))


class GroupBy:
    """Filter + group-by over the 6,001,215-row fact table."""
    name = "filter_groupby"
    key = "groupby"

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
        self.kernel = ("k_sort_pass<RowRec<2,1,false,KEY_HI32>,8,4,PK,3> (sort stage: 2^23 two-word records, "
                       "4096-row tiles, three CTAs per SM)")

    def step(self):
        self.capi.filter_groupby(self.dev, self.n, self.pred, self.G, scratch=self.scratch, out=self.out,
                                 counts=self.counts)

    def step_e2e(self):
        for k in self.dev:
            self.dev[k].copy_(self.pinned[k], non_blocking=True)
        self.step()
        self.out_host.copy_(self.out, non_blocking=True)
        self.counts_host.copy_(self.counts, non_blocking=True)

    def e2e_set(self):
        t = self.torch
        return {"dev": {k: t.empty_like(v, device=self.out.device) for k, v in self.pinned.items()},
                "out": t.empty_like(self.out), "counts": t.empty_like(self.counts),
                "out_host": t.empty_like(self.out_host).pin_memory(),
                "counts_host": t.empty_like(self.counts_host).pin_memory()}

    def e2e_in(self, b):
        for k in b["dev"]:
            b["dev"][k].copy_(self.pinned[k], non_blocking=True)

    def e2e_run(self, b):
        self.capi.filter_groupby(b["dev"], self.n, self.pred, self.G, scratch=self.scratch, out=b["out"],
                                 counts=b["counts"])

    def e2e_out(self, b):
        b["out_host"].copy_(b["out"], non_blocking=True)
        b["counts_host"].copy_(b["counts"], non_blocking=True)

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


class SortKP:
    """Plain oblivious sort of n (u64 key, u32 payload) rows."""
    key = "sort"

    def __init__(self, torch, capi, W, device, n=1 << 20):
        self.torch, self.capi = torch, capi
        self.n = n
        self.name = f"plain_sort_2^{int(np.log2(n))}"
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
        # up to 2^23 rows (100 MB) the rows fit in L2 and it is flushed
        # between steps; 2^24 rows (201 MB) exceed it
        self.flush_l2 = self.n * 12 < (126 << 20)
        self.kernel = (f"k_sort_pass<RowKP,8,4,PK,{3 if n >= (1 << 21) else 2}> (2^{int(np.log2(n))} rows of "
                       f"12 B, 4096-row tiles)")

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

    def e2e_set(self):
        t = self.torch
        return {"k": t.empty_like(self.k), "p": t.empty_like(self.p), "kh": t.empty_like(self.kh).pin_memory(),
                "ph": t.empty_like(self.ph).pin_memory()}

    def e2e_in(self, b):
        b["k"].copy_(self.pinned_k, non_blocking=True)
        b["p"].copy_(self.pinned_p, non_blocking=True)

    def e2e_run(self, b):
        self.capi.osort_kp(b["k"], b["p"], self.n)

    def e2e_out(self, b):
        b["kh"].copy_(b["k"], non_blocking=True)
        b["ph"].copy_(b["p"], non_blocking=True)

    def d2h_bytes(self):
        return self.n * 12

    def launches(self):
        return sort_passes(int(np.log2(self.n)), 12, 7)

    def rdm_bytes(self):
        return 2 * self.n * 12 * rdm_psort(self.n)

    def check(self, orc):
        k = self.k.cpu().numpy().view(np.uint64)
        p = self.p.cpu().numpy().view(np.uint32)
        if self.n <= (1 << 20):
            ok_, op_ = orc.bitonic_kp(self.k0.cpu().numpy().view(np.uint64), self.p0.cpu().numpy().view(np.uint32))
            return bool(np.array_equal(k, ok_) and np.array_equal(p, op_))
        # every (key, payload) row is unique, so the sorted output is the
        # lexicographic sort of the input
        k0 = self.k0.cpu().numpy().view(np.uint64)
        p0 = self.p0.cpu().numpy().view(np.uint32)
        o = np.lexsort((p0, k0))
        return bool(np.array_equal(k, k0[o]) and np.array_equal(p, p0[o]))


class Batched:
    """512 independent instances (log-uniform 2^10..2^22 rows; even = sort of
    (u64 key, u32 payload), odd = compaction with Bernoulli(0.3) keep flags),
    each padded to its own power of two, run by ONE persistent launch captured
    in a CUDA graph, tile configuration picked by the autotuner.  The plain
    path (one launch sequence per instance, back to back) is timed beside
    it."""
    name = "batched_512"
    key = "batch"

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
        self.kernel = "k_sched (persistent)"

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

    def network_bytes(self):
        """Bytes the batch's passes read and write, by the library's own pass
        plan for the chosen tile."""
        tot = 0
        for it in self.items:
            npr = self.capi.next_pow2(it["n"])
            lt = self.tune[0]
            lmax = min(8, lt - 5)
            if it["kind"] == "sort":
                tot += 2 * npr * 12 * sort_passes(int(np.log2(npr)), lt, lmax)
            else:
                tot += 2 * npr * 13 * compact_passes(int(np.log2(npr)), lt, lmax) + npr * 5
        return tot

    def check(self, orc):
        """Every instance against numpy; a stride sample against the oracle."""
        self.batch.status(stream=self.stream)
        ok = True
        for i, (it, h) in enumerate(zip(self.items, self.host)):
            if it["kind"] == "sort":
                k = it["keys"].cpu().numpy().view(np.uint64)[: it["n"]]
                ok &= bool(np.array_equal(k, np.sort(h["keys"])))
                if i % 61 == 0 and it["n"] <= (1 << 20):
                    ok_, _ = orc.bitonic_kp(h["keys"], h["pay"])
                    ok &= bool(np.array_equal(k, ok_[: it["n"]]))
            else:
                c = int(it["count"].item())
                ok &= c == int(h["marks"].sum())
                k = it["keys"].cpu().numpy().view(np.uint64)[:c]
                ok &= bool(np.array_equal(k, h["keys"][h["marks"].astype(bool)]))
        return bool(ok)


# --------------------------------------------------------------------------
# timing
# --------------------------------------------------------------------------

def time_steps(torch, fn, steps, flush=None):
    """Per-step CUDA-event durations (ms) of `fn` on the current stream,
    flushing L2 between steps outside the timed events when asked."""
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for s, e in evs:
        if flush is not None:
            flush()
        s.record()
        fn()
        e.record()
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in evs]


def warm(torch, fn, warmup, min_s=SOAK_S):
    """At least `warmup` untimed steps, continuing until `min_s` seconds of
    work have run, so the clock samples see the GPU under steady load."""
    t0 = time.perf_counter()
    i = 0
    while i < warmup or time.perf_counter() - t0 < min_s:
        fn()
        i += 1
        if i % 8 == 0:
            torch.cuda.synchronize()
    torch.cuda.synchronize()
    return i


PASS_KINDS = ("tile_sort", "merge", "global", "compact_tile", "compact_global")


def pass_roofline(torch, capi, run, peak, reps=3, reset=None):
    """Every network pass of `run` timed on its own (the library's pass timer:
    CUDA events around each pass, on the pass's stream) and grouped by pass
    kind.  Algorithmic bytes of a pass: every row read and written once,
    2 x rows x row bytes."""
    rows = []
    for _ in range(reps):
        if reset is not None:
            reset()
        torch.cuda.synchronize()
        capi.set_pass_timing(True)
        try:
            run()
            torch.cuda.synchronize()
            rows.extend(capi.last_pass_times())
        finally:
            capi.set_pass_timing(False)
    out = {}
    for kind in PASS_KINDS:
        xs = [(2 * (1 << lg) * rb, ms) for (k, lg, rb, ms) in rows if k == kind and ms > 0]
        if not xs:
            continue
        byt = sum(b for b, _ in xs)
        t = sum(m for _, m in xs)
        fr = [b / (m / 1e3) / 1e9 / peak for b, m in xs]
        out[kind] = {"launches_per_step": len(xs) // reps, "avg_launch_us": t / len(xs) * 1e3,
                     "achieved_gbs": byt / (t / 1e3) / 1e9, "frac": byt / (t / 1e3) / 1e9 / peak,
                     "min_frac": min(fr), "max_frac": max(fr)}
    # the dominant sort: the sort passes of the largest padded size
    sorts = [(lg, rb, ms) for (k, lg, rb, ms) in rows if k in ("tile_sort", "merge", "global") and ms > 0]
    dom = None
    if sorts:
        lg_max = max(lg for lg, _, _ in sorts)
        xs = [(2 * (1 << lg) * rb, ms) for lg, rb, ms in sorts if lg == lg_max]
        dom = {"launches_per_step": len(xs) // reps, "avg_launch_us": sum(m for _, m in xs) / len(xs) * 1e3,
               "algorithmic_bytes_per_launch": xs[0][0], "log2_rows": lg_max}
    return out, dom


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


E2E_SETS = 3


def e2e_pipelined_ms(torch, wl, steps):
    """The end-to-end form with E2E_SETS input/output sets in flight: step
    i's host -> device copy (one copy stream) and step i-1's device -> host
    copy (another) run while a pipeline runs on the compute stream.  Every
    step still moves all its bytes through PCIe; the two copy directions and
    the SMs work at once.  With three sets a set's round trip (copy in,
    pipeline, copy out) may take up to three steps, so a step is bound by
    the slowest of the three, not by their sum over two steps.  Returns ms
    per step (CUDA events on the compute stream around `steps` steps, the
    last result copy included)."""
    n = E2E_SETS
    sets = [wl.e2e_set() for _ in range(n)]
    hs, ds = torch.cuda.Stream(), torch.cuda.Stream()
    ms = torch.cuda.current_stream()
    ev_in = [torch.cuda.Event() for _ in range(n)]
    ev_done = [torch.cuda.Event() for _ in range(n)]
    ev_free = [torch.cuda.Event() for _ in range(n)]

    def run(k, start=None):
        for i in range(k):
            b = i % n
            with torch.cuda.stream(hs):
                if start is not None and i == 0:
                    hs.wait_event(start)
                if i >= n:
                    hs.wait_event(ev_free[b])  # set b's result has left the device
                wl.e2e_in(sets[b])
                ev_in[b].record(hs)
            ms.wait_event(ev_in[b])
            wl.e2e_run(sets[b])
            ev_done[b].record(ms)
            with torch.cuda.stream(ds):
                ds.wait_event(ev_done[b])
                wl.e2e_out(sets[b])
                ev_free[b].record(ds)
        for b in range(min(k, n)):
            ms.wait_event(ev_free[b])

    run(2 * n)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(ms)
    run(steps, start=s)
    e.record(ms)
    torch.cuda.synchronize()
    return s.elapsed_time(e) / steps


def measure(torch, capi, wl, args, world, device, peak, peak_kind, with_e2e=True):
    """Warm-up, K timed steps (max over ranks), the end-to-end form through
    the public API with host buffers, and the algorithmic-bytes model."""
    import torch.distributed as dist

    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device=device) if wl.flush_l2 else None
    flush = (lambda: l2_flush.fill_(1)) if l2_flush is not None else None
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    warm(torch, wl.step, args.warmup)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ts = time_steps(torch, wl.step, args.steps, flush)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    value, ms = aggregate_throughput(wl.n, float(np.mean(ts)), world, device)
    res = {"value": value, "unit": "Mrows/s", "ms_per_step": ms, "clocks": clk,
           "l2": "flushed between steps" if wl.flush_l2 else "inputs larger than L2",
           "config": {"workload": wl.name, "rows": int(wl.n), "padded_rows": int(wl.np_rows),
                      "record_bytes": wl.rec_bytes}}
    if with_e2e:
        for _ in range(2):
            wl.step_e2e()
        torch.cuda.synchronize()
        te = time_steps(torch, wl.step_e2e, max(3, args.steps // 2))
        serial_value, serial_ms = aggregate_throughput(wl.n, float(np.mean(te)), world, device)
        serial_form = "copy in, pipeline, copy out, one step after the other"
        e2e = {"unit": "Mrows/s", "h2d_bytes_per_step": int(wl.in_bytes),
               "d2h_bytes_per_step": int(wl.d2h_bytes())}
        if hasattr(wl, "e2e_set"):
            e2e_value, ems = aggregate_throughput(wl.n, e2e_pipelined_ms(torch, wl, max(4, args.steps)), world,
                                                  device)
            e2e.update(value=e2e_value, ms_per_step=ems,
                       form=(f"{E2E_SETS} input/output sets in flight: step i's host-to-device copy and step "
                             "i-1's device-to-host copy overlap the pipeline"),
                       serial={"value": serial_value, "ms_per_step": serial_ms, "form": serial_form})
        else:
            # the batch replays one captured graph over fixed buffers and
            # keeps the serial form only
            e2e.update(value=serial_value, ms_per_step=serial_ms, form=serial_form)
        res["e2e"] = e2e
    rdm = wl.rdm_bytes()
    res["rdm"] = {"bytes_per_step": int(rdm), "achieved_gbs": rdm / (ms / 1e3) / 1e9,
                  "frac_of_hbm": rdm / (ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind}
    res["gpu_launches"] = int(wl.launches() * args.steps)
    return res


def roofline_of(torch, capi, wl, peak, peak_kind):
    """The `roofline` object: the dominant kernel (the bitonic pass kernel of
    the workload's largest sort) and every pass kind."""
    reset = None
    run = wl.step
    if isinstance(wl, SortKP):
        def reset():
            wl.k.copy_(wl.k0)
            wl.p.copy_(wl.p0)

        def run():
            wl.capi.osort_kp(wl.k, wl.p, wl.n)
    kinds, dom = pass_roofline(torch, capi, run, peak, reset=reset)
    if dom is None:
        return None
    achieved = dom["algorithmic_bytes_per_launch"] / (dom["avg_launch_us"] / 1e6) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
            "traffic": TRAFFIC.get(wl.key), "kernel": wl.kernel, "avg_launch_us": dom["avg_launch_us"],
            "launches_per_step": dom["launches_per_step"],
            "algorithmic_bytes_per_launch": dom["algorithmic_bytes_per_launch"],
            "timing": "each pass bracketed by CUDA events on its stream (library pass timer), mean of 3 runs",
            "by_pass_kind": kinds}


# --------------------------------------------------------------------------
# CPU baselines (the oracle's oblivious pipelines, all host cores)
# --------------------------------------------------------------------------

def _timed_reps(fn, min_s, max_reps):
    t0 = time.perf_counter()
    reps = 0
    while True:
        fn()
        reps += 1
        if time.perf_counter() - t0 > min_s or reps >= max_reps:
            break
    return (time.perf_counter() - t0) / reps, reps


def _batch_compact_rows(orc, it):
    """An instance's (key, payload | mark << 32) records over next_pow2(n)
    rows for the CPU ORCompact (pads unmarked)."""
    npr = int(orc.next_pow2(it["n"]))
    r = np.full((npr, 2), np.uint64(2**64 - 1), np.uint64)
    r[: it["n"], 0] = it["keys"]
    r[: it["n"], 1] = it["pay"].astype(np.uint64) | (it["marks"].astype(np.uint64) << np.uint64(32))
    r[it["n"]:, 1] = np.uint64(0)
    return r


def cpu_baseline(wl_key, W, orc, budget_s=10.0):
    cores = os.cpu_count() or 1
    if wl_key == "join":
        dim, fact = W.join_tables()
        n = len(dim["key"]) + len(fact["fk"])
        dt, reps = _timed_reps(lambda: orc.join_groupby_topk(dim, fact, W.JOIN_PRED, W.JOIN_TOPK,
                                                             n_threads=cores, oblivious=True), budget_s, 20)
        rdt, rreps = _timed_reps(lambda: orc.join_groupby_topk(dim, fact, W.JOIN_PRED, W.JOIN_TOPK,
                                                               n_threads=cores), budget_s / 4, 5)
        return {"value": n / dt / 1e6, "unit": "Mrows/s", "cores": cores, "kind": "port", "same_config": True,
                "sample": f"the full 1.5 M + 6 M-row join per run, {reps} runs, oblivious: network sort of all "
                          f"2^23 union rows in the reference's network order (OpenMP, cache-blocked levels), "
                          f"chunked forward fill, ORCompact (parallel halves), chunked segmented sums, ORCompact "
                          f"of the groups, network sort of 2^21 group records; the chunk-carry steps are serial",
                "revealing_reference_semantics": {
                    "value": n / rdt / 1e6, "unit": "Mrows/s", "runs": rreps,
                    "what": "the same join with the joined rows found by a serial branching scan (the count "
                            "is revealed and only the joined groups are sorted)"}}
    if wl_key == "groupby":
        n = W.LINEITEM_ROWS
        cols = W.lineitem(n)
        dt, reps = _timed_reps(lambda: orc.filter_groupby(cols, W.LINEITEM_PRED, 8, n_threads=cores,
                                                          oblivious=True), budget_s, 20)
        rdt, rreps = _timed_reps(lambda: orc.filter_groupby(cols, W.LINEITEM_PRED, 8, n_threads=cores),
                                 budget_s / 4, 20)
        return {"value": n / dt / 1e6, "unit": "Mrows/s", "cores": cores, "kind": "port", "same_config": True,
                "sample": f"the full 6,001,215-row table per run, {reps} runs, oblivious: predicate, ORCompact "
                          f"of all 2^23 rows (parallel halves), network sort of all 2^23 rows (OpenMP, "
                          f"cache-blocked levels), chunked segmented sums into 8 ranked slots",
                "revealing_reference_semantics": {
                    "value": n / rdt / 1e6, "unit": "Mrows/s", "runs": rreps,
                    "what": "filter by a serial stable scatter, then a network sort of only the rows that "
                            "pass (the count is revealed, as src/operator/filter_compaction_operator.cpp:"
                            "171-178 does)"}}
    if wl_key == "sort":
        n = 1 << 20
        keys, pay = W.sort_kp(n)
        dt, reps = _timed_reps(lambda: orc.bitonic_kp(keys, pay, n_threads=cores), budget_s, 200)
        return {"value": n / dt / 1e6, "unit": "Mrows/s", "cores": cores, "kind": "port", "same_config": True,
                "sample": f"full 2^20-row network sort in the reference's network order, {reps} runs, OpenMP "
                          f"over all cores"}
    if wl_key == "batch":
        insts = W.batch_instances()
        rows, t_tot, used = 0, 0.0, 0
        for i in range(len(insts)):
            it = insts[(i * 97) % len(insts)]
            if it["kind"] == "sort":
                t0 = time.perf_counter()
                orc.bitonic_kp(it["keys"], it["pay"], n_threads=cores)
            else:
                r = _batch_compact_rows(orc, it)
                t0 = time.perf_counter()
                orc.obl_compact_rec2(r, 1, 32, 0, n_threads=cores)
            t_tot += time.perf_counter() - t0
            rows += it["n"]
            used += 1
            if t_tot > budget_s:
                break
        return {"value": rows / t_tot / 1e6, "unit": "Mrows/s", "cores": cores, "kind": "port",
                "same_config": False,
                "sample": f"{used} of the 512 instances (stride 97 through the list, {rows} rows): network sorts "
                          f"and ORCompact over each instance's next_pow2(n) rows, OpenMP over all cores"}
    return None


# --------------------------------------------------------------------------
# served query stream (resident tables, continuous admission)
# --------------------------------------------------------------------------

SERVE_SIZES_LOG2 = (10.0, 18.0)


def _lat(results, t_key="submit_ms"):
    lat = np.asarray([r.end_ms - getattr(r, t_key) for r in results])
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}


def _served_form(S, tab, qs, qs_poisson, budget, slots, plain_qps, persistent, loads):
    """One server form at saturation (every query of `qs` offered at once) and
    under Poisson arrivals of `qs_poisson` at the given multiples of the plain
    capacity."""
    nq = len(qs)
    srv = S.Server(tab, slots=slots, budget_bytes=budget, persistent=persistent)
    S.run_open_loop(srv, qs[:32], np.zeros(32))
    sat_res, sat_s = S.run_open_loop(srv, qs, np.zeros(nq))
    out_loads = {}
    for f in loads:
        r, s = S.run_open_loop(srv, qs_poisson, S.arrivals(len(qs_poisson), f * plain_qps, seed=int(f * 1000)))
        out_loads[f"{f}x_plain_capacity"] = {"offered_qps": f * plain_qps, "achieved_qps": len(qs_poisson) / s,
                                             **_lat(r)}
    st = srv.stats()
    srv.close()
    form = {"qps_saturation": nq / sat_s, **_lat(sat_res), "slots": slots,
            "peak_inflight": st["peak_inflight"], "peak_arena_bytes": st["peak_arena_bytes"], "poisson": out_loads}
    return form, sat_res


def measure_serve(torch, nq=256, n_poisson=1024, slots=16, persistent_slots=64):
    """A seeded query stream (50 % filter + group-by, 35 % two-way join +
    top-10, 15 % three-way chain; slice sizes 2^10..2^18) over resident tables
    of 60 M / 15 M / 150 M rows, admitted by a 120 GB HBM budget.

    Plain = the same request loop with one slot: each query submitted after
    the previous one returned (its capacity), and Poisson arrivals at 0.9x
    that capacity.  Served = up to 16 queries in flight on their own streams;
    served_persistent = up to 64 queries in flight as jobs of one persistent
    command queue.  Each form at saturation (256 queries offered at once) and
    under Poisson arrivals (1024 queries) at multiples of the plain capacity.
    Latency is submit -> result in host memory, on the host clock.  `target`
    compares each load point against the plain path's p99 under Poisson
    arrivals at 0.9x its capacity (the same arrival process) and against its
    closed-loop p99 (no queueing at all)."""
    from velodb_b200 import serving as S

    t0 = time.perf_counter()
    tab = S.ServedTables(**S.FULL_SCALE)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(120 << 30, free - (4 << 30)))
    lo, hi = SERVE_SIZES_LOG2
    qs = S.query_stream(tab, nq, seed=0xB200000000000004, lo_log2=lo, hi_log2=hi)
    qp = S.query_stream(tab, n_poisson, seed=0xB200000000000005, lo_log2=lo, hi_log2=hi)
    srv = S.Server(tab, slots=1, budget_bytes=budget)
    S.run_closed_one_at_a_time(srv, qs[:16])
    plain_res, plain_s = S.run_closed_one_at_a_time(srv, qs)
    plain_qps = nq / plain_s
    r09, _ = S.run_open_loop(srv, qp, S.arrivals(n_poisson, 0.9 * plain_qps, seed=900))
    srv.close()
    plain = {"qps": plain_qps, **_lat(plain_res), "poisson_0.9x": {"offered_qps": 0.9 * plain_qps, **_lat(r09)}}
    served, sat_res = _served_form(S, tab, qs, qp, budget, slots, plain_qps, False, (0.9, 3.0))
    served_p, sat_p = _served_form(S, tab, qs, qp, budget, persistent_slots, plain_qps, True,
                                   (0.9, 3.0, 4.0, 5.0, 6.0))

    def same(rs):
        return bool(all(S.result_key(a) == S.result_key(b) and a.status == 0 and b.status == 0
                        for a, b in zip(plain_res, rs)))

    def target(form):
        # load points with >= 3x the plain throughput and a p99 no higher than
        # the plain path's
        pts = {k: v for k, v in form["poisson"].items() if v["achieved_qps"] >= 3.0 * plain_qps}
        best = max(pts.items(), key=lambda kv: kv[1]["achieved_qps"], default=(None, None))
        return {
            "loads_at_3x_plain_throughput": sorted(pts),
            "p99_vs_plain_poisson_0.9x": {k: v["p99_ms"] <= plain["poisson_0.9x"]["p99_ms"] for k, v in pts.items()},
            "p99_vs_plain_closed_loop": {k: v["p99_ms"] <= plain["p99_ms"] for k, v in pts.items()},
            "best": best[0],
        }

    shapes = {S.SHAPE_NAMES[k]: int(sum(1 for q in qs if q.shape == k)) for k in S.SHAPE_NAMES}
    out = {
        "tables_rows": dict(S.FULL_SCALE), "resident_bytes": int(tab.bytes), "table_build_s": build_s,
        "hbm_budget_bytes": budget, "sizes_log2": [lo, hi], "queries": nq, "poisson_queries": n_poisson,
        "mix": shapes,
        "plain": plain,
        "served": served,
        "served_persistent": served_p,
        "speedup_served_vs_plain": served["qps_saturation"] / plain_qps,
        "speedup_served_persistent_vs_plain": served_p["qps_saturation"] / plain_qps,
        "target_served": target(served),
        "target_served_persistent": target(served_p),
        "results_identical_alone_and_in_mix": same(sat_res) and same(sat_p),
        "timing": "host clock, submit -> result in host memory",
    }
    del tab
    torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------------
# reference arm
# --------------------------------------------------------------------------

def run_reference(args, rank):
    """CPU reference arm: the reference's algorithm for the path as the
    oracle's oblivious pipeline (network sorts in the reference's network
    order over all next_pow2(n) rows, ORCompact, segmented sums) on all host
    cores, rank 0 only, on the same workload as our arm.  Each step is one run
    of the whole workload (one instance of the batch, one query of the stream
    for serve)."""
    if rank != 0:
        return
    import oracle as orc
    from velodb_b200 import workloads as W

    orc.lib()
    cores = os.cpu_count() or 1
    unit = "Mrows/s"
    extra = None
    if args.workload == "sort":
        n = 1 << 20
        keys, pay = W.sort_kp(n)
        steps = [(lambda: orc.bitonic_kp(keys, pay, n_threads=cores), n)]
        sample, wl = "full 2^20-row network sort per step", "plain_sort_2^20"
    elif args.workload == "batch":
        insts = W.batch_instances()
        order = [(i * 97) % len(insts) for i in range(len(insts))]

        def inst_fn(it):
            if it["kind"] == "sort":
                return lambda: orc.bitonic_kp(it["keys"], it["pay"], n_threads=cores)
            r = _batch_compact_rows(orc, it)
            return lambda: orc.obl_compact_rec2(r, 1, 32, 0, n_threads=cores)

        steps = [(inst_fn(insts[i]), insts[i]["n"]) for i in order]
        sample = "one of the 512 instances per step (stride 97 through the list); network sorts and ORCompact " \
                 "over next_pow2(n) rows, all cores"
        wl = "batched_512"
    elif args.workload == "groupby":
        n = W.LINEITEM_ROWS
        cols = W.lineitem(n)
        steps = [(lambda: orc.filter_groupby(cols, W.LINEITEM_PRED, 8, n_threads=cores, oblivious=True), n)]
        sample, wl = "full 6,001,215-row table per step, oblivious pipeline", "filter_groupby"
        extra = ("revealing_reference_semantics",
                 lambda: orc.filter_groupby(cols, W.LINEITEM_PRED, 8, n_threads=cores), n)
    elif args.workload == "serve":
        from velodb_b200 import serving as S

        hs = S.HostSlices(**S.FULL_SCALE)
        lo, hi = SERVE_SIZES_LOG2
        qs = [q for q in S.query_stream(hs, 4 * (args.steps + args.warmup) + 8, seed=0xB200000000000004,
                                        lo_log2=lo, hi_log2=hi) if q.shape != S.Q_JOIN3]

        def q_fn(q):
            if q.shape == S.Q_FILTER_GROUPBY:
                cols = hs.lineitem(q.offset, q.n)
                return lambda: orc.filter_groupby(cols, W.LINEITEM_PRED, 8, n_threads=cores, oblivious=True)
            dim, fact = hs.join_inputs(q)
            return lambda: orc.join_groupby_topk(dim, fact, W.JOIN_PRED, 10, n_threads=cores, oblivious=True)

        steps = [(q_fn(q), 1) for q in qs]
        unit = "queries/s"
        sample = "one query per step from the served stream (sizes 2^10..2^18), filter+group-by and " \
                 "two-way join shapes (the three-way chain has no oracle pipeline), oblivious pipelines"
        wl = "served_stream"
    else:
        dim, fact = W.join_tables()
        n = len(dim["key"]) + len(fact["fk"])
        steps = [(lambda: orc.join_groupby_topk(dim, fact, W.JOIN_PRED, W.JOIN_TOPK, n_threads=cores,
                                                oblivious=True), n)]
        sample, wl = "full 1.5 M + 6 M-row join per step, oblivious pipeline", "join_groupby_top10"
        extra = ("revealing_reference_semantics",
                 lambda: orc.join_groupby_topk(dim, fact, W.JOIN_PRED, W.JOIN_TOPK, n_threads=cores), n)
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
        "impl": "reference", "metric": METRIC, "value": value, "unit": unit,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": wl},
        "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if extra is not None:
        name, fn, u = extra
        dt, reps = _timed_reps(fn, 3.0, 5)
        line[name] = {"value": u / dt / 1e6, "unit": unit, "runs": reps,
                      "what": "the reference's count-revealing semantics (the filtered or joined rows found by "
                              "a serial scan, only those sorted)"}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------

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


def batch_persistent(torch, capi, wl, reps=5):
    """The same 512 instances as jobs of one persistent command queue
    (velo_batch_submit on a VELO_QUEUE_PERSISTENT context: the instances run
    beside each other, every CTA of the consumer claiming work items of any
    of them).  Host clock from the submission to the last completion, best
    of `reps`."""
    scr = []
    cmds = []
    for it in wl.items:
        if it["kind"] == "sort":
            cmds.append(capi.make_cmd("OSORT_KP", it["keys"], it["pay"], it["n"], it["keys"].numel()))
        else:
            cap = it["keys"].numel()
            sc = torch.empty(capi.compact_scratch_bytes(cap), dtype=torch.uint8, device=it["keys"].device)
            scr.append(sc)
            cmds.append(capi.make_cmd("OCOMPACT_KPM", it["keys"], it["pay"], it["marks"], it["n"], cap,
                                      it["count"], sc, sc.numel()))
    torch.cuda.synchronize()
    best = None
    with capi.Queue(persistent=True) as q:
        for r in range(reps + 1):
            t0 = time.perf_counter()
            tix = q.submit_batch(cmds)
            for t in tix:
                q.wait(t)
            dt = time.perf_counter() - t0
            if r > 0:
                best = dt if best is None else min(best, dt)
        launches = q.launches()
    return {"ms_per_step": best * 1e3, "value": wl.n / best / 1e6, "unit": "Mrows/s", "runs": reps,
            "consumer_launches": launches,
            "timing": "host clock, velo_batch_submit of the 512 commands -> last velo_wait returned"}


def batch_plain(torch, wl, args):
    """The plain path of the batch (512 launch sequences back to back) and the
    batch's network bytes against both."""
    peak, _ = hbm_peak()
    for _ in range(2):
        wl.step_plain()
    torch.cuda.synchronize()
    tp = time_steps(torch, wl.step_plain, max(3, args.steps // 2))
    pms = float(np.mean(tp))
    tb = time_steps(torch, wl.step, max(3, args.steps // 2))
    bms = float(np.mean(tb))
    nb = wl.network_bytes()
    return {"plain_path": {"ms_per_step": pms, "value": wl.n / (pms / 1e3) / 1e6,
                           "network_frac_of_hbm": nb / (pms / 1e3) / 1e9 / peak},
            "batched_ms_per_step": bms, "speedup_batched_vs_plain": pms / bms,
            "batched_network_frac_of_hbm": nb / (bms / 1e3) / 1e9 / peak,
            "network_bytes_per_step": int(nb), "tune": list(wl.tune),
            "autotune_ms": {f"{k[0]}x{k[1]}": v for k, v in wl.tune_ms.items()}}


def measure_join_algorithms(torch, capi, W, steps):
    """The three oblivious equi-joins on the 1.5 M-row dimension keys and the
    6 M-row fact foreign keys (join only, no group-by): the union-sort PK-FK
    join, the bin-padded hash join and the many-to-many sort-merge join
    (bound 6 M pairs).  Each is timed with CUDA events over `steps` calls and
    its pair set checked against numpy."""
    dim, fact = W.join_tables()
    bk = torch.from_numpy(dim["key"]).cuda()
    pk = torch.from_numpy(fact["fk"]).cuda()
    n = len(dim["key"]) + len(fact["fk"])
    keyset = np.zeros(len(dim["key"]) + 2, np.int64) - 1
    keyset[dim["key"]] = np.arange(len(dim["key"]))
    want = int((keyset[fact["fk"]] >= 0).sum())
    out = {}
    algos = {"pkfk_union_sort": lambda: capi.ojoin_pkfk(bk, None, pk, None, 4),
             "hash_bin_padded": lambda: capi.ohash_join(bk, None, pk, None, 4),
             "many_to_many_sort_merge": lambda: capi.ojoin_mn(bk, None, pk, None, 4, len(fact["fk"]))}
    for name, fn in algos.items():
        try:
            for _ in range(2):
                fn()
            torch.cuda.synchronize()
            ts = time_steps(torch, fn, max(3, steps // 2))
            ob, op, cnt = fn()
            torch.cuda.synchronize()
            m = int(cnt[0].item())
            o_b, o_p = ob.cpu().numpy()[:m], op.cpu().numpy()[:m]
            ok = m == want and bool(np.array_equal(keyset[fact["fk"][o_p]], o_b))
            ms = float(np.mean(ts))
            out[name] = {"ms": ms, "input_mrows_per_s": n / (ms / 1e3) / 1e6, "pairs": m, "checked": ok}
        except Exception as e:  # noqa: BLE001
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
    out["note"] = ("times include each call's scratch allocation by the caching allocator (no cudaMalloc after "
                   "the first call)")
    return out


def run_extras(torch, capi, W, device, args, peak, peak_kind, orc):
    """The other configurations, each measured and checked on its own (N = 1
    only).  A failure is recorded in its key instead of ending the run."""
    out = {}
    sub = argparse.Namespace(steps=args.steps, warmup=args.warmup)

    def one(key, mk, cpu_key=None):
        try:
            wl = mk()
            r = measure(torch, capi, wl, sub, 1, device, peak, peak_kind)
            r["roofline"] = roofline_of(torch, capi, wl, peak, peak_kind)
            r["checked_against_oracle"] = wl.check(orc)
            if cpu_key is not None:
                r["cpu_baseline"] = cpu_baseline(cpu_key, W, orc, budget_s=5.0)
            out[key] = r
            del wl
        except Exception as e:  # noqa: BLE001
            out[key] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()

    if args.workload != "sort":
        one("sort_2^20", lambda: SortKP(torch, capi, W, device, 1 << 20), "sort")
    one("sort_2^24", lambda: SortKP(torch, capi, W, device, 1 << 24))
    if args.workload != "groupby":
        one("filter_groupby", lambda: GroupBy(torch, capi, W, device), "groupby")
    if args.workload != "batch":
        try:
            wl = Batched(torch, capi, W, device)
            r = measure(torch, capi, wl, sub, 1, device, peak, peak_kind, with_e2e=False)
            r.update(batch_plain(torch, wl, sub))
            r["persistent_queue"] = batch_persistent(torch, capi, wl)
            r["speedup_persistent_queue_vs_plain"] = r["plain_path"]["ms_per_step"] / r["persistent_queue"]["ms_per_step"]
            r["checked_against_oracle"] = wl.check(orc)
            out["batched"] = r
            del wl
        except Exception as e:  # noqa: BLE001
            out["batched"] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
    try:
        out["joins_1.5Mx6M"] = measure_join_algorithms(torch, capi, W, args.steps)
    except Exception as e:  # noqa: BLE001
        out["joins_1.5Mx6M"] = {"error": f"{type(e).__name__}: {e}"}
    try:
        out["served"] = measure_serve(torch)
    except Exception as e:  # noqa: BLE001
        out["served"] = {"error": f"{type(e).__name__}: {e}"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="join", choices=["join", "sort", "groupby", "batch", "serve"])
    ap.add_argument("--extras", default="all", choices=["all", "none"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist

    from velodb_b200 import capi, workloads as W

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=device)
    peak, peak_kind = hbm_peak()

    if args.workload == "serve":
        import ctypes

        from velodb_b200._lib import VeloQuery, VeloQueryResult

        res = measure_serve(torch)
        # the served stream through the persistent command queue
        value, _ = aggregate_throughput(res["served_persistent"]["qps_saturation"], 1e3, world, device, scale=1.0)
        line = {"metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": res["queries"],
                "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int64", "data": "synthetic",
                "config": {"workload": "served_stream", "parallelism": f"replicas{world}",
                           "l2": "inputs larger than L2 (resident tables 4.9 GB)"},
                "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": ctypes.sizeof(VeloQuery),
                        "d2h_bytes_per_step": ctypes.sizeof(VeloQueryResult)},
                "serve": res, "gpu_launches": None}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    wl = make_workload(args.workload, torch, capi, W, device)
    res = measure(torch, capi, wl, args, world, device, peak, peak_kind)
    line = {
        "metric": METRIC, "value": res["value"], "unit": "Mrows/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": dict(res["config"], parallelism=f"replicas{world}", l2=res["l2"]),
        "e2e": res["e2e"], "gpu_launches": res["gpu_launches"], "rdm": res["rdm"], "clocks": res["clocks"],
    }
    line["roofline"] = roofline_of(torch, capi, wl, peak, peak_kind)
    if isinstance(wl, Batched):
        line.update(batch_plain(torch, wl, args))
    orc = None
    if rank == 0:
        import oracle as orc

        orc.lib()
        line["checked_against_oracle"] = wl.check(orc)
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(wl.key, W, orc)
    if world == 1 and args.extras == "all":
        del wl
        torch.cuda.empty_cache()
        line["extras"] = run_extras(torch, capi, W, device, args, peak, peak_kind, orc)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
