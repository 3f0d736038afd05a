"""Parity of the batched and served configurations at their full sizes.

* The batch of 512 instances (log-uniform 2^10..2^22 rows, even instances
  sorts of (u64 key, u32 payload), odd ones compactions with Bernoulli(0.3)
  keep flags), run as one persistent launch replayed from a CUDA graph and as
  jobs of the persistent command queue, must equal the plain path (one launch
  sequence per instance) bit for bit on every instance, and a stride sample
  of instances must equal the oracle.
* The served stream over the full resident tables (60 M-row fact table, 15 M
  dimension rows, 150 M-row second fact table) must give every query the same
  result alone and in the mix -- on per-query streams and through the
  persistent command queue -- and a sample of each query shape must equal the
  oracle (filter + group-by, two-way join) or a numpy computation (three-way
  chain).
"""
import numpy as np
import pytest
import torch

from velodb_b200 import capi, serving as S, workloads as W

pytestmark = pytest.mark.gpu


def _upload(insts, device):
    items = []
    for it in insts:
        cap = capi.next_pow2(it["n"])
        d = dict(kind=it["kind"], n=it["n"], keys=capi.to_dev_u64(it["keys"], cap),
                 pay=capi.to_dev_u32(it["pay"], cap))
        if it["kind"] == "compact":
            d["marks"] = capi.to_dev_u8(it["marks"], cap)
            d["count"] = torch.full((1,), -1, dtype=torch.int64, device=device)
        items.append(d)
    return items


def _restore(items, insts):
    for d, it in zip(items, insts):
        n = it["n"]
        d["keys"][:n].copy_(torch.from_numpy(it["keys"].view(np.int64)))
        d["pay"][:n].copy_(torch.from_numpy(it["pay"].view(np.int32)))
        if "marks" in d:
            d["marks"][:n].copy_(torch.from_numpy(it["marks"]))


def test_batch_512_instances_graph_replay_matches_plain_and_oracle(cuda, orc):
    insts = W.batch_instances()
    assert len(insts) == 512
    assert min(it["n"] for it in insts) >= 1 << 10 and max(it["n"] for it in insts) <= 1 << 22
    items = _upload(insts, cuda)
    ref = [{k: (v.clone() if torch.is_tensor(v) else v) for k, v in d.items()} for d in items]
    # the plain path: one launch sequence per instance
    for d in ref:
        if d["kind"] == "sort":
            capi.osort_kp(d["keys"], d["pay"], d["n"])
        else:
            d["count"].copy_(capi.ocompact_kpm(d["keys"], d["pay"], d["marks"], d["n"]))
    torch.cuda.synchronize()
    # the batched path: one persistent launch, captured in a CUDA graph
    b = capi.Batch(items)
    s = torch.cuda.Stream()
    b.launch(stream=s)  # first launch outside the graph sets the kernel up
    b.status(stream=s)
    torch.cuda.synchronize()
    _restore(items, insts)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.launch(stream=s)
    g.replay()
    b.status(stream=s)
    torch.cuda.synchronize()
    for d, r in zip(items, ref):
        cap = capi.next_pow2(d["n"])
        for k in ("keys", "pay", "marks"):
            if k in d:
                assert torch.equal(d[k][:cap], r[k][:cap]), (d["kind"], d["n"], k)
        if "count" in d:
            assert int(d["count"].item()) == int(r["count"].item())
    # a stride sample against the oracle
    for i in range(0, 512, 37):
        it, d = insts[i], items[i]
        n = it["n"]
        if it["kind"] == "sort" and n <= 1 << 20:
            ok, op = orc.bitonic_kp(it["keys"], it["pay"])
            assert np.array_equal(capi.host_u64(d["keys"], len(ok)), ok)
            assert np.array_equal(capi.host_u32(d["pay"], len(op)), op)
        elif it["kind"] == "compact" and n <= 1 << 18:
            cap = capi.next_pow2(n)
            rec = np.zeros((cap, 16), np.uint8)
            kk = np.full(cap, np.uint64(2**64 - 1))
            pp = np.full(cap, np.uint32(2**32 - 1))
            kk[:n], pp[:n] = it["keys"], it["pay"]
            rec[:, :8] = kk.view(np.uint8).reshape(cap, 8)
            rec[:, 8:12] = pp.view(np.uint8).reshape(cap, 4)
            mm = np.zeros(cap, np.uint8)
            mm[:n] = it["marks"]
            od, _, cnt = orc.ocompact(rec, mm)
            assert int(d["count"].item()) == cnt == int(it["marks"].sum())
            assert np.array_equal(capi.host_u64(d["keys"], cap),
                                  np.ascontiguousarray(od[:, :8]).view(np.uint64).reshape(-1))
    del g
    b.close()
    # the same 512 instances as jobs of one persistent command queue
    _restore(items, insts)
    scr, cmds = [], []
    for d in items:
        cap = capi.next_pow2(d["n"])
        if d["kind"] == "sort":
            cmds.append(capi.make_cmd("OSORT_KP", d["keys"], d["pay"], d["n"], cap))
        else:
            sc = torch.empty(capi.compact_scratch_bytes(cap), dtype=torch.uint8, device=cuda)
            scr.append(sc)
            d["count"].fill_(-1)
            cmds.append(capi.make_cmd("OCOMPACT_KPM", d["keys"], d["pay"], d["marks"], d["n"], cap, d["count"], sc,
                                      sc.numel()))
    torch.cuda.synchronize()
    with capi.Queue(persistent=True) as q:
        for t in q.submit_batch(cmds):
            q.wait(t)
    for d, r in zip(items, ref):
        cap = capi.next_pow2(d["n"])
        for k in ("keys", "pay", "marks"):
            if k in d:
                assert torch.equal(d[k][:cap], r[k][:cap]), ("persistent queue", d["kind"], d["n"], k)
        if "count" in d:
            assert int(d["count"].item()) == int(r["count"].item())


@pytest.fixture(scope="module")
def full_tables(cuda):
    t = S.ServedTables(**S.FULL_SCALE)
    torch.cuda.synchronize()
    yield t
    del t
    torch.cuda.empty_cache()


def _check_query(orc, tab, q, r):
    o, n = q.offset, q.n
    if q.shape == S.Q_FILTER_GROUPBY:
        cols = {k: v[o:o + n].cpu().numpy() for k, v in tab.fact.items()}
        g, keys, sums = orc.filter_groupby(cols, W.LINEITEM_PRED, 8)
        out = np.asarray(r.out[:48]).reshape(8, 6)
        assert int(r.counts[1]) == g
        assert np.array_equal(out[:g, 0], keys.astype(np.int64)) and np.array_equal(out[:g, 1:], sums)
        return
    dsl = slice(q.dim_offset, q.dim_offset + q.dim_n)
    dk = tab.dim_key[dsl].cpu().numpy()
    dd = tab.dim_date[dsl].cpu().numpy()
    fk = tab.fact_fk[o:o + n].cpu().numpy()
    fp = tab.fact["price"][o:o + n].cpu().numpy()
    if q.shape == S.Q_JOIN_TOPK:
        dim = dict(key=dk.astype(np.int32), date=dd)
        fct = dict(fk=fk.astype(np.int32), price=fp)
        g, ofk, osum, ocnt = orc.join_groupby_topk(dim, fct, W.JOIN_PRED, 10)
        out = np.asarray(r.out[:30]).reshape(10, 3)
        m = min(g, 10)
        assert int(r.counts[1]) == g
        assert np.array_equal(out[:m, 0], ofk) and np.array_equal(out[:m, 1], osum)
        assert np.array_equal(out[:m, 2], ocnt)
        return
    ok_keys = dk[dd < W.JOIN_PRED["date_hi"]]
    ok_fact = np.nonzero((fp < W.JOIN_PRED["price_hi"]) & np.isin(fk, ok_keys))[0] + o
    f2 = tab.fact2_fk[q.f2_offset:q.f2_offset + q.f2_n].cpu().numpy()
    f2p = tab.fact2_price[q.f2_offset:q.f2_offset + q.f2_n].cpu().numpy()
    hit = np.isin(f2, ok_fact)
    assert int(r.counts[0]) == int(hit.sum())
    assert int(r.out[0]) == int(f2p[hit].sum())


def test_served_full_tables_alone_and_in_the_mix(full_tables, orc):
    tab = full_tables
    assert (tab.fact_n, tab.dim_n, tab.fact2_n) == (60_000_000, 15_000_000, 150_000_000)
    qs = S.query_stream(tab, 48, seed=21, lo_log2=14, hi_log2=20)
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(120 << 30, free - (4 << 30)))
    alone = S.Server(tab, slots=1, budget_bytes=budget)
    ra, _ = S.run_closed_one_at_a_time(alone, qs)
    alone.close()
    mix = S.Server(tab, slots=16, budget_bytes=budget)
    rm, _ = S.run_open_loop(mix, qs, np.zeros(len(qs)))  # all arrive at once
    st = mix.stats()
    mix.close()
    assert st["peak_inflight"] > 1
    for a, m in zip(ra, rm):
        assert a.status == 0 and m.status == 0
        assert S.result_key(a) == S.result_key(m)
    seen = {S.Q_FILTER_GROUPBY: 0, S.Q_JOIN_TOPK: 0, S.Q_JOIN3: 0}
    for q, r in zip(qs, rm):
        if seen[q.shape] < 3:
            _check_query(orc, tab, q, r)
            seen[q.shape] += 1
    assert all(v > 0 for v in seen.values())
    # the same stream through one persistent command queue: every result as alone
    pq = S.Server(tab, slots=64, budget_bytes=budget, persistent=True)
    rp, _ = S.run_open_loop(pq, qs, np.zeros(len(qs)))
    st = pq.stats()
    pq.close()
    assert st["peak_inflight"] > 1
    for a, p in zip(ra, rp):
        assert p.status == 0 and S.result_key(a) == S.result_key(p)
