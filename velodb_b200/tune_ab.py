"""A/B timing of one load tune of the network passes against the plain
kernels, on the seeded workloads, with CUDA events on the launching stream.

    python -m velodb_b200.tune_ab tensor_tile_loads
    python -m velodb_b200.tune_ab merge_pipeline

For each workload (the 1.5 M x 6 M join + group-by + top-10, the 6 M-row
filter + group-by, key-payload sorts of 2^20, 2^23 and 2^24 rows) and each
setting (off, on): 3 warm-up calls, the mean of 10 timed calls, then one call
with the library's pass timer for the per-pass-kind means, and whether the
outputs of the two settings are identical.  Prints one JSON object.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import capi
from . import workloads as W


def _timed(fn, reps=10):
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def _pass_means(fn):
    capi.set_pass_timing(True)
    capi.clear_pass_times()
    fn()
    torch.cuda.synchronize()
    pt = capi.last_pass_times()
    capi.set_pass_timing(False)
    out = {}
    for kind in ("tile_sort", "merge", "global", "compact_tile", "compact_global"):
        ms = [p[3] for p in pt if p[0] == kind]
        if ms:
            out[kind] = {"passes": len(ms), "mean_us": float(np.mean(ms)) * 1e3}
    return out


def _workloads():
    """(name, call, reset): reset restores the input of an in-place sort."""
    dim, fact = W.join_tables()
    dt = capi.join_to_device(dim, fact)
    jsc = torch.empty(capi.join_groupby_topk_scratch_bytes(len(dim["key"]), len(fact["fk"])), dtype=torch.uint8,
                      device="cuda")
    yield "join_groupby_top10", lambda: capi.join_groupby_topk(dt, W.JOIN_PRED, W.JOIN_TOPK, scratch=jsc), None
    cols = W.lineitem()
    dc = capi.lineitem_to_device(cols)
    n = W.LINEITEM_ROWS
    gsc = torch.empty(capi.filter_groupby_scratch_bytes(n, W.LINEITEM_GROUP_BOUND), dtype=torch.uint8, device="cuda")
    yield ("filter_groupby",
           lambda: capi.filter_groupby(dc, n, W.LINEITEM_PRED, W.LINEITEM_GROUP_BOUND, scratch=gsc), None)
    for lg in (20, 23, 24):
        keys, pay = W.sort_kp(1 << lg, seed=lg)
        k0, p0 = capi.to_dev_u64(keys), capi.to_dev_u32(pay)
        k, p = k0.clone(), p0.clone()

        def sort(k=k, p=p, lg=lg):
            capi.osort_kp(k, p, 1 << lg)
            return k, p

        def reset(k=k, p=p, k0=k0, p0=p0):
            k.copy_(k0)
            p.copy_(p0)

        yield f"sort_kp_2^{lg}", sort, reset


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("tune", choices=sorted(capi.TUNES))
    a = ap.parse_args(argv)
    switch = capi.TUNES[a.tune]
    res = {"tune": a.tune, "workloads": {}}
    try:
        for name, fn, reset in _workloads():
            row, outs = {}, {}
            for on in (False, True):
                switch(on)
                if reset is not None:
                    reset()
                out = fn()
                torch.cuda.synchronize()
                outs[on] = [t.clone() for t in out]
                row["on" if on else "off"] = {"ms": _timed(fn), "passes": _pass_means(fn)}
            # the sorts run in place: the checked call of each setting sorts
            # the same input, the timed calls re-sort sorted rows (the same
            # passes: the network does not depend on the data)
            row["identical"] = all(torch.equal(x, y) for x, y in zip(outs[False], outs[True]))
            res["workloads"][name] = row
            torch.cuda.empty_cache()
    finally:
        switch(False)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
