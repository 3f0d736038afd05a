"""One invocation of one operator on seeded input, for profilers.

    python -m velodb_b200.cases sort_kp --log2 23
    python -m velodb_b200.cases sort_records --log2 23 --words 3
    python -m velodb_b200.cases compact_kpm --log2 23
    python -m velodb_b200.cases filter_groupby
    python -m velodb_b200.cases join_topk
    python -m velodb_b200.cases batch

Each case uploads its input, runs the operator `--reps` times (the network
sorts in place, so later repetitions see sorted input; the access pattern of
an oblivious network does not depend on the data) and synchronizes.  The
inputs are the seeded workloads of ``velodb_b200.workloads``.
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

from . import capi
from . import workloads as W


def case_sort_kp(a):
    n = 1 << a.log2
    keys, pay = W.sort_kp(n)
    k, p = capi.to_dev_u64(keys), capi.to_dev_u32(pay)
    for _ in range(a.reps):
        capi.osort_kp(k, p, n, tune=a.tune)


def case_sort_records(a):
    n = 1 << a.log2
    ws = [capi.to_dev_u64(W.splitmix64(7, n, i)) for i in range(a.words)]
    for _ in range(a.reps):
        capi.osort_records(ws, n, 0xFFFF800000000000, tune=a.tune)


def case_compact_kpm(a):
    n = 1 << a.log2
    keys, pay = W.sort_kp(n)
    marks = (W.lemire(W.splitmix64(5, n, 0), 10) < 3).astype(np.uint8)
    k, p, m = capi.to_dev_u64(keys), capi.to_dev_u32(pay), capi.to_dev_u8(marks)
    for _ in range(a.reps):
        capi.ocompact_kpm(k, p, m, n, tune=a.tune)


def case_filter_groupby(a):
    cols = W.lineitem()
    d = capi.lineitem_to_device(cols)
    for _ in range(a.reps):
        capi.filter_groupby(d, W.LINEITEM_ROWS, W.LINEITEM_PRED, W.LINEITEM_GROUP_BOUND)


def case_join_topk(a):
    dim, fact = W.join_tables()
    dt = capi.join_to_device(dim, fact)
    for _ in range(a.reps):
        capi.join_groupby_topk(dt, W.JOIN_PRED, W.JOIN_TOPK)


def case_batch(a):
    insts = W.batch_instances(count=a.count, max_log2=a.max_log2)
    items = []
    for it in insts:
        cap = capi.next_pow2(it["n"])
        d = dict(kind=it["kind"], n=it["n"], keys=capi.to_dev_u64(it["keys"], cap),
                 pay=capi.to_dev_u32(it["pay"], cap))
        if it["kind"] == "compact":
            d["marks"] = capi.to_dev_u8(it["marks"], cap)
            d["count"] = torch.zeros(1, dtype=torch.int64, device="cuda")
        items.append(d)
    b = capi.Batch(items, tune=a.tune)
    for _ in range(a.reps):
        b.launch()


CASES = {k[5:]: v for k, v in globals().items() if k.startswith("case_")}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--log2", type=int, default=20)
    ap.add_argument("--words", type=int, default=3)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--max-log2", type=float, default=22.0)
    ap.add_argument("--tile-log2", type=int, default=0)
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args(argv)
    a.tune = (a.tile_log2, a.threads) if a.tile_log2 else None
    torch.cuda.set_device(0)
    CASES[a.case](a)
    torch.cuda.synchronize()
    print(f"{a.case}: ok")


if __name__ == "__main__":
    main()
