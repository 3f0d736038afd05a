"""Obliviousness: the recorded global-memory address trace and the launch
sequence of each operator are identical for different inputs of the same
public size.

The operators run from the instrumented test build libvelo_obl_trace.so
(every global load/store site of the oblivious path folds (site, address)
into a hash chain per logical thread; every kernel logs (kernel, grid, block,
dynamic smem)).  Each case runs the same call on several inputs through the
same device buffers and compares the chain digest and the launch log; a
different public size must change the trace (the check is not vacuous)."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from velodb_b200 import _lib, workloads as W

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "velodb_b200")
TRACE_LIB = os.path.join(PKG, "libvelo_obl_trace.so")
SLOTS = 1 << 22
LAUNCH_CAP = 1 << 14


@pytest.fixture(scope="module")
def T(cuda):
    if not os.path.exists(TRACE_LIB):
        from velodb_b200 import build as B

        B.build_trace()
    L = C.CDLL(TRACE_LIB)
    for name, (res, args) in _lib.PROTOS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    assert L.velo_trace_enabled() == 1
    return L


def trace_of(T, fn):
    torch.cuda.synchronize()
    assert T.velo_trace_begin(SLOTS, LAUNCH_CAP) == 0, T.velo_last_error_text()
    fn()
    torch.cuda.synchronize()
    digest, touched, nl = C.c_uint64(), C.c_uint64(), C.c_uint64()
    log = np.zeros(4 * LAUNCH_CAP, np.uint64)
    assert T.velo_trace_end(C.byref(digest), C.byref(touched), log.ctypes.data, LAUNCH_CAP, C.byref(nl)) == 0
    n = int(nl.value)
    assert 0 < n <= LAUNCH_CAP and touched.value > 0
    return int(digest.value), int(touched.value), log[: 4 * n].reshape(n, 4).copy()


def assert_same_trace(traces):
    d0, t0, l0 = traces[0]
    for d, t, l in traces[1:]:
        assert np.array_equal(l, l0), "launch sequence differs"
        assert t == t0, "number of logical threads with accesses differs"
        assert d == d0, "address trace differs"


def dev_copy(dst, src_np):
    dst[: len(src_np)].copy_(torch.from_numpy(np.ascontiguousarray(src_np)))


# ---- plain sort -----------------------------------------------------------------

def test_sort_trace_is_data_independent(T):
    n = (1 << 16) + 123
    cap = 1 << 17
    k = torch.empty(cap, dtype=torch.int64, device="cuda")
    p = torch.empty(cap, dtype=torch.int32, device="cuda")
    inputs = [W.sort_kp(n, seed=1), W.sort_kp(n, seed=2),
              (np.full(n, 7, np.uint64), np.zeros(n, np.uint32)),  # all-equal keys
              (np.arange(n, dtype=np.uint64)[::-1].copy(), np.arange(n, dtype=np.uint32))]  # reversed

    def run(keys, pay, nn=n):
        def f():
            dev_copy(k, keys.view(np.int64))
            dev_copy(p, pay.view(np.int32))
            torch.cuda.synchronize()
            assert T.velo_osort_kp(k.data_ptr(), p.data_ptr(), nn, cap, None, None) == 0, T.velo_last_error_text()
        return f

    traces = [trace_of(T, run(*x)) for x in inputs]
    assert_same_trace(traces)
    # sensitivity: one row more is a different public size and a different trace
    other = trace_of(T, run(*W.sort_kp(n + 1, seed=1), nn=n + 1))
    assert other[0] != traces[0][0]


# ---- compaction ---------------------------------------------------------------------

def test_compaction_trace_is_data_independent(T):
    n = (1 << 16) + 5
    cap = 1 << 17
    k = torch.empty(cap, dtype=torch.int64, device="cuda")
    p = torch.empty(cap, dtype=torch.int32, device="cuda")
    m = torch.empty(cap, dtype=torch.uint8, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    sb = T.velo_compact_scratch_bytes(cap, None)
    scratch = torch.empty(sb, dtype=torch.uint8, device="cuda")
    keys, pay = W.sort_kp(n, seed=3)
    rng = np.random.default_rng(0)
    marks = [np.zeros(n, np.uint8), np.ones(n, np.uint8), (rng.random(n) < 0.3).astype(np.uint8),
             (np.arange(n) % 2).astype(np.uint8)]

    def run(mk):
        def f():
            dev_copy(k, keys.view(np.int64))
            dev_copy(p, pay.view(np.int32))
            dev_copy(m, mk)
            torch.cuda.synchronize()
            assert T.velo_ocompact_kpm(k.data_ptr(), p.data_ptr(), m.data_ptr(), n, cap, cnt.data_ptr(),
                                       scratch.data_ptr(), sb, None, None) == 0, T.velo_last_error_text()
        return f

    assert_same_trace([trace_of(T, run(x)) for x in marks])


# ---- filter + group-by ---------------------------------------------------------------

def test_filter_groupby_trace_is_data_independent(T):
    n = 100_003
    G = 8
    tabs = [W.lineitem(n, seed=5), W.lineitem(n, seed=6)]
    all_pass = W.lineitem(n, seed=7)  # every row passes the predicate
    all_pass["shipdate"][:] = 10
    all_pass["disc"][:] = 10
    all_pass["qty"][:] = 5
    none_pass = W.lineitem(n, seed=8)  # no row passes
    none_pass["disc"][:] = 3
    tabs += [all_pass, none_pass]
    cols = {k: torch.from_numpy(v).cuda() for k, v in tabs[0].items()}
    li = _lib.VeloLineitem(*[cols[k].data_ptr() for k in ("qty", "price", "disc", "tax", "shipdate", "flag1",
                                                          "flag2")])
    pr = W.LINEITEM_PRED
    pred = _lib.VeloLineitemPred(pr["ship_lo"], pr["ship_hi"], pr["disc_lo"], pr["disc_hi"], pr["qty_lo"],
                                 pr["qty_hi"])
    sb = T.velo_filter_groupby_scratch_bytes(n, G)
    scratch = torch.empty(sb, dtype=torch.uint8, device="cuda")
    out = torch.empty((G, 6), dtype=torch.int64, device="cuda")
    counts = torch.empty(2, dtype=torch.int64, device="cuda")

    def run(tab):
        def f():
            for key, v in tab.items():
                cols[key].copy_(torch.from_numpy(v))
            torch.cuda.synchronize()
            assert T.velo_filter_groupby(C.byref(li), n, C.byref(pred), G, 0, out.data_ptr(), counts.data_ptr(),
                                         scratch.data_ptr(), sb, None) == 0, T.velo_last_error_text()
        return f

    assert_same_trace([trace_of(T, run(t)) for t in tabs])


# ---- join + group-by + top-k -----------------------------------------------------------

def test_join_topk_trace_is_data_independent(T):
    nd, nf = 20_000, 80_000
    sets = [W.join_tables(nd, nf, seed=s) for s in (11, 12)]
    d3, f3 = W.join_tables(nd, nf, seed=13)
    f3["fk"][:] = d3["key"][0]  # every fact row on one key
    sets.append((d3, f3))
    d4, f4 = W.join_tables(nd, nf, seed=14)
    f4["fk"][:] = nd + 5  # no fact row joins
    sets.append((d4, f4))
    dk = torch.empty(nd, dtype=torch.int32, device="cuda")
    dd = torch.empty(nd, dtype=torch.int32, device="cuda")
    ff = torch.empty(nf, dtype=torch.int32, device="cuda")
    fp = torch.empty(nf, dtype=torch.int64, device="cuda")
    tab = _lib.VeloJoinTables(dk.data_ptr(), dd.data_ptr(), nd, ff.data_ptr(), fp.data_ptr(), nf)
    pred = _lib.VeloJoinPred(W.JOIN_PRED["date_hi"], 0, W.JOIN_PRED["price_hi"])
    sb = T.velo_join_groupby_topk_scratch_bytes(nd, nf)
    scratch = torch.empty(sb, dtype=torch.uint8, device="cuda")
    out = torch.empty((10, 3), dtype=torch.int64, device="cuda")
    counts = torch.empty(2, dtype=torch.int64, device="cuda")

    def run(dim, fact):
        def f():
            dk.copy_(torch.from_numpy(dim["key"]))
            dd.copy_(torch.from_numpy(dim["date"]))
            ff.copy_(torch.from_numpy(fact["fk"]))
            fp.copy_(torch.from_numpy(fact["price"]))
            torch.cuda.synchronize()
            assert T.velo_join_groupby_topk(C.byref(tab), C.byref(pred), 10, out.data_ptr(), counts.data_ptr(),
                                            scratch.data_ptr(), sb, None) == 0, T.velo_last_error_text()
        return f

    assert_same_trace([trace_of(T, run(d, f)) for d, f in sets])


# ---- batched persistent launch -----------------------------------------------------------

def test_batched_launch_trace_is_data_independent(T):
    sizes = [3000, 70_000, 1 << 15, 12_345, 1 << 16, 999]
    bufs = []
    for i, n in enumerate(sizes):
        cap = int(T.velo_next_pow2(n))
        bufs.append(dict(n=n, cap=cap, kind=1 if i % 2 == 0 else 2,  # sort / compaction items
                         k=torch.empty(cap, dtype=torch.int64, device="cuda"),
                         p=torch.empty(cap, dtype=torch.int32, device="cuda"),
                         m=torch.empty(cap, dtype=torch.uint8, device="cuda"),
                         c=torch.zeros(1, dtype=torch.int64, device="cuda")))
    items = (_lib.VeloBatchItem * len(bufs))()
    for it, b in zip(items, bufs):
        it.kind = b["kind"]
        it.d_keys = b["k"].data_ptr()
        it.d_payload = b["p"].data_ptr()
        it.d_marks = b["m"].data_ptr() if b["kind"] == 2 else None
        it.n = b["n"]
        it.capacity = b["cap"]
        it.d_count = b["c"].data_ptr() if b["kind"] == 2 else None
    h = C.c_void_p()
    tune = _lib.VeloTune(12, 256)
    assert T.velo_batch_create(items, len(bufs), C.byref(tune), C.byref(h)) == 0, T.velo_last_error_text()

    def run(seed, dens):
        def f():
            rng = np.random.default_rng(seed)
            for b in bufs:
                keys = rng.integers(0, 2**63, b["n"], dtype=np.int64) if seed else np.zeros(b["n"], np.int64)
                dev_copy(b["k"], keys)
                dev_copy(b["p"], np.arange(b["n"], dtype=np.int32))
                dev_copy(b["m"], (rng.random(b["n"]) < dens).astype(np.uint8))
            torch.cuda.synchronize()
            assert T.velo_batch_launch(h, None) == 0
            assert T.velo_batch_status(h, None) == 0
        return f

    try:
        assert_same_trace([trace_of(T, run(s, d)) for s, d in ((1, 0.3), (2, 0.9), (0, 0.0))])
    finally:
        T.velo_batch_destroy(h)


# ---- oblivious shuffle, gather, join, column compaction -------------------------------------

def test_shuffle_gather_join_traces_are_data_independent(T):
    n = 50_000
    m = torch.empty(n, dtype=torch.int32, device="cuda")
    sb = T.velo_oshuffle_scratch_bytes(n)
    s = torch.empty(sb, dtype=torch.uint8, device="cuda")

    def shuf(seed):
        def f():
            dev_copy(m, np.random.default_rng(seed).permutation(n).astype(np.int32))
            torch.cuda.synchronize()
            assert T.velo_oshuffle_position_map(m.data_ptr(), n, 123, 7, s.data_ptr(), sb, None) == 0
        return f

    assert_same_trace([trace_of(T, shuf(x)) for x in (1, 2)])

    tn, rn = 30_000, 20_000
    table = torch.empty(tn, dtype=torch.int64, device="cuda")
    rids = torch.empty(rn, dtype=torch.int32, device="cuda")
    out = torch.empty(rn, dtype=torch.int64, device="cuda")
    gb = T.velo_ogather_scratch_bytes(tn, rn)
    gs = torch.empty(gb, dtype=torch.uint8, device="cuda")

    def gather(seed, dup):
        def f():
            rng = np.random.default_rng(seed)
            dev_copy(table, rng.integers(0, 2**62, tn, dtype=np.int64))
            r = np.full(rn, 17, np.int32) if dup else rng.integers(0, tn + 100, rn).astype(np.int32)
            dev_copy(rids, r)
            torch.cuda.synchronize()
            assert T.velo_ogather_u64(table.data_ptr(), tn, rids.data_ptr(), rn, out.data_ptr(), gs.data_ptr(), gb,
                                      None) == 0
        return f

    assert_same_trace([trace_of(T, gather(x, d)) for x, d in ((3, False), (4, False), (5, True))])

    bn, pn = 10_000, 40_000
    bk = torch.empty(bn, dtype=torch.int64, device="cuda")
    pk = torch.empty(pn, dtype=torch.int64, device="cuda")
    ob = torch.empty(pn, dtype=torch.int64, device="cuda")
    op = torch.empty(pn, dtype=torch.int64, device="cuda")
    jc = torch.empty(2, dtype=torch.int64, device="cuda")
    jb = T.velo_ojoin_scratch_bytes(bn, pn)
    js = torch.empty(jb, dtype=torch.uint8, device="cuda")

    def join(seed, miss):
        def f():
            rng = np.random.default_rng(seed)
            dev_copy(bk, rng.permutation(bn).astype(np.int64))
            fk = rng.integers(bn, 2 * bn, pn) if miss else rng.integers(0, bn, pn)
            dev_copy(pk, fk.astype(np.int64))
            torch.cuda.synchronize()
            assert T.velo_ojoin_pkfk(bk.data_ptr(), None, bn, pk.data_ptr(), None, pn, 5, ob.data_ptr(),
                                     op.data_ptr(), jc.data_ptr(), js.data_ptr(), jb, None) == 0
        return f

    assert_same_trace([trace_of(T, join(x, mm)) for x, mm in ((6, False), (7, False), (8, True))])


def test_column_compaction_trace_is_data_independent(T):
    n = 70_001
    a = torch.empty(n, dtype=torch.int32, device="cuda")
    b = torch.empty(n, dtype=torch.int64, device="cuda")
    va = torch.empty(n, dtype=torch.uint8, device="cuda")
    mask = torch.empty(n, dtype=torch.uint8, device="cuda")
    cnt = torch.empty(1, dtype=torch.int64, device="cuda")
    sb = T.velo_ocompact_columns_scratch_bytes(n)
    s = torch.empty(sb, dtype=torch.uint8, device="cuda")
    cols = (C.c_void_p * 2)(a.data_ptr(), b.data_ptr())
    types = (C.c_uint32 * 2)(4, 5)
    valid = (C.c_void_p * 2)(va.data_ptr(), None)

    def run(seed, dens):
        def f():
            rng = np.random.default_rng(seed)
            dev_copy(a, rng.integers(-100, 100, n).astype(np.int32))
            dev_copy(b, rng.integers(0, 2**40, n).astype(np.int64))
            dev_copy(va, (rng.random(n) < 0.5).astype(np.uint8))
            dev_copy(mask, (rng.random(n) < dens).astype(np.uint8))
            torch.cuda.synchronize()
            assert T.velo_ocompact_columns(cols, types, valid, 2, mask.data_ptr(), n, cnt.data_ptr(), s.data_ptr(),
                                           sb, None) == 0
        return f

    assert_same_trace([trace_of(T, run(x, d)) for x, d in ((1, 0.0), (2, 0.5), (3, 1.0))])


def test_ogroupby_trace_is_data_independent(T):
    n = 60_001
    keys = torch.empty(n, dtype=torch.int32, device="cuda")
    vals = torch.empty(n, dtype=torch.int64, device="cuda")
    mask = torch.empty(n, dtype=torch.uint8, device="cuda")
    bound = 1000
    ok = torch.empty(bound, dtype=torch.int64, device="cuda")
    os_ = torch.empty(bound, dtype=torch.int64, device="cuda")
    oc = torch.empty(bound, dtype=torch.int64, device="cuda")
    cnt = torch.empty(2, dtype=torch.int64, device="cuda")
    sb = T.velo_ogroupby_scratch_bytes(n)
    s = torch.empty(sb, dtype=torch.uint8, device="cuda")
    sums = (C.c_void_p * 2)(vals.data_ptr(), None)
    outs = (C.c_void_p * 2)(os_.data_ptr(), None)

    def run(k, dens):
        def f():
            rng = np.random.default_rng(int(dens * 100))
            dev_copy(keys, k)
            dev_copy(vals, rng.integers(0, 1000, n).astype(np.int64))
            dev_copy(mask, (rng.random(n) < dens).astype(np.uint8))
            torch.cuda.synchronize()
            assert T.velo_ogroupby(keys.data_ptr(), 4, sums, 1, 1, mask.data_ptr(), n, bound, ok.data_ptr(), outs,
                                   oc.data_ptr(), cnt.data_ptr(), s.data_ptr(), sb, None) == 0, \
                T.velo_last_error_text()
        return f

    rng = np.random.default_rng(0)
    cases = [(rng.integers(0, 50, n).astype(np.int32), 0.5),      # few groups
             (np.arange(n, dtype=np.int32), 1.0),                  # every row its own group
             (np.zeros(n, np.int32), 0.0)]                         # one key, nothing selected
    assert_same_trace([trace_of(T, run(k, d)) for k, d in cases])


def test_mn_join_trace_is_data_independent(T):
    bn, pn, mp = 6_000, 20_000, 50_000
    bk = torch.empty(bn, dtype=torch.int32, device="cuda")
    pk = torch.empty(pn, dtype=torch.int32, device="cuda")
    bm = torch.empty(bn, dtype=torch.uint8, device="cuda")
    ob = torch.empty(mp, dtype=torch.int64, device="cuda")
    op = torch.empty(mp, dtype=torch.int64, device="cuda")
    jc = torch.empty(2, dtype=torch.int64, device="cuda")
    sb = T.velo_ojoin_mn_scratch_bytes(bn, pn, mp)
    s = torch.empty(sb, dtype=torch.uint8, device="cuda")

    def join(seed, span, all_masked=False):
        def f():
            rng = np.random.default_rng(seed)
            dev_copy(bk, rng.integers(0, span, bn).astype(np.int32))
            dev_copy(pk, rng.integers(0, span, pn).astype(np.int32))
            dev_copy(bm, np.zeros(bn, np.uint8) if all_masked else (rng.random(bn) < 0.7).astype(np.uint8))
            torch.cuda.synchronize()
            assert T.velo_ojoin_mn(bk.data_ptr(), bm.data_ptr(), bn, pk.data_ptr(), None, pn, 4, mp, ob.data_ptr(),
                                   op.data_ptr(), jc.data_ptr(), s.data_ptr(), sb, None) == 0
        return f

    # many matches per key, one key only (overflowing the bound), no key
    # matching at all, every build row left out
    assert_same_trace([trace_of(T, join(x, sp, am)) for x, sp, am in
                       ((1, 3000, False), (2, 3000, False), (3, 1, False), (4, 10**9, False), (5, 3000, True))])


def test_hash_join_trace_is_data_independent(T):
    bn, pn = 5_000, 20_000
    bk = torch.empty(bn, dtype=torch.int64, device="cuda")
    pk = torch.empty(pn, dtype=torch.int64, device="cuda")
    ob = torch.empty(pn, dtype=torch.int64, device="cuda")
    op = torch.empty(pn, dtype=torch.int64, device="cuda")
    jc = torch.empty(3, dtype=torch.int64, device="cuda")
    sb = T.velo_ohash_join_scratch_bytes(bn, pn)
    s = torch.empty(sb, dtype=torch.uint8, device="cuda")

    def join(seed, miss):
        def f():
            rng = np.random.default_rng(seed)
            dev_copy(bk, rng.permutation(bn).astype(np.int64))
            fk = rng.integers(bn, 2 * bn, pn) if miss else rng.integers(0, bn, pn)
            dev_copy(pk, fk.astype(np.int64))
            torch.cuda.synchronize()
            assert T.velo_ohash_join(bk.data_ptr(), None, bn, pk.data_ptr(), None, pn, 5, 99, ob.data_ptr(),
                                     op.data_ptr(), jc.data_ptr(), s.data_ptr(), sb, None) == 0
        return f

    assert_same_trace([trace_of(T, join(x, mm)) for x, mm in ((6, False), (7, False), (8, True))])


def test_ogroupby_bigint_trace_is_data_independent(T):
    n = 40_001
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    vals = torch.empty(n, dtype=torch.int64, device="cuda")
    mask = torch.empty(n, dtype=torch.uint8, device="cuda")
    bound = 500
    ok = torch.empty(bound, dtype=torch.int64, device="cuda")
    os_ = torch.empty(bound, dtype=torch.int64, device="cuda")
    oc = torch.empty(bound, dtype=torch.int64, device="cuda")
    cnt = torch.empty(2, dtype=torch.int64, device="cuda")
    sb = T.velo_ogroupby_scratch_bytes(n)
    s = torch.empty(sb, dtype=torch.uint8, device="cuda")
    sums = (C.c_void_p * 2)(vals.data_ptr(), None)
    outs = (C.c_void_p * 2)(os_.data_ptr(), None)

    def run(k, dens):
        def f():
            rng = np.random.default_rng(int(dens * 100) + 1)
            dev_copy(keys, k)
            dev_copy(vals, rng.integers(0, 1000, n).astype(np.int64))
            dev_copy(mask, (rng.random(n) < dens).astype(np.uint8))
            torch.cuda.synchronize()
            assert T.velo_ogroupby(keys.data_ptr(), 5, sums, 1, 1, mask.data_ptr(), n, bound, ok.data_ptr(), outs,
                                   oc.data_ptr(), cnt.data_ptr(), s.data_ptr(), sb, None) == 0, \
                T.velo_last_error_text()
        return f

    rng = np.random.default_rng(1)
    cases = [(rng.integers(-(2**63), 2**63 - 1, n, dtype=np.int64), 0.5),              # distinct, extreme range
             (np.full(n, 2**63 - 1, np.int64), 1.0),                                    # one key, the maximum
             (rng.choice(np.array([-(2**63), 0, 2**63 - 1], np.int64), n), 0.0)]        # nothing selected
    assert_same_trace([trace_of(T, run(k, d)) for k, d in cases])


# ---- persistent command queue ---------------------------------------------------------------

def test_persistent_queue_traces_are_data_independent(T):
    # a filter + group-by and a (key, payload) sort run as jobs of a fresh
    # persistent queue: logical threads are numbered by the item within its
    # job, so the trace does not depend on which CTA takes which item
    from velodb_b200 import capi

    n = 60_001
    G = 8
    tabs = [W.lineitem(n, seed=21), W.lineitem(n, seed=22)]
    none_pass = W.lineitem(n, seed=23)
    none_pass["disc"][:] = 3
    tabs.append(none_pass)
    cols = {k: torch.from_numpy(v).cuda() for k, v in tabs[0].items()}
    li = _lib.VeloLineitem(*[cols[k].data_ptr() for k in capi.LINEITEM_COLS])
    pr = W.LINEITEM_PRED
    pred = _lib.VeloLineitemPred(pr["ship_lo"], pr["ship_hi"], pr["disc_lo"], pr["disc_hi"], pr["qty_lo"],
                                 pr["qty_hi"])
    sb = T.velo_filter_groupby_scratch_bytes(n, G)
    scratch = torch.empty(sb, dtype=torch.uint8, device="cuda")
    out = torch.empty((G, 6), dtype=torch.int64, device="cuda")
    counts = torch.empty(2, dtype=torch.int64, device="cuda")
    ns = 70_001
    cap = 1 << 17
    k = torch.empty(cap, dtype=torch.int64, device="cuda")
    p = torch.empty(cap, dtype=torch.int32, device="cuda")

    def run(i, tab):
        def f():
            for key, v in tab.items():
                cols[key].copy_(torch.from_numpy(v))
            keys, pay = W.sort_kp(ns, seed=i + 1) if i < 2 else (np.zeros(ns, np.uint64), np.zeros(ns, np.uint32))
            dev_copy(k, keys.view(np.int64))
            dev_copy(p, pay.view(np.int32))
            torch.cuda.synchronize()
            q = C.c_void_p()
            # a long idle time: one consumer launch for the whole run
            assert T.velo_init(C.byref(_lib.VeloConfig(0, 0, capi.QUEUE_PERSISTENT, 10_000_000)), C.byref(q)) == 0
            t1, t2 = C.c_uint64(), C.c_uint64()
            g = capi.make_cmd("FILTER_GROUPBY", C.addressof(li), n, C.addressof(pred), G, out, counts, scratch, sb)
            s = capi.make_cmd("OSORT_KP", k, p, ns, cap)
            assert T.velo_submit(q, C.byref(g), C.byref(t1)) == 0, T.velo_last_error_text()
            assert T.velo_submit(q, C.byref(s), C.byref(t2)) == 0, T.velo_last_error_text()
            assert T.velo_wait(q, t2.value, 30_000_000_000) == 0
            assert T.velo_shutdown(q, 30_000) == 0
        return f

    assert_same_trace([trace_of(T, run(i, t)) for i, t in enumerate(tabs)])
