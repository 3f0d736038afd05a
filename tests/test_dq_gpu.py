"""GPU tests of the persistent command queue (velo_init with
VELO_QUEUE_PERSISTENT): every command it runs gives bit for bit the result of
the direct entry point on the same inputs, many jobs run at once and in
order where ordered, the consumer exits when idle and is relaunched, and
every wait is bounded."""
import ctypes as C
import time

import numpy as np
import pytest
import torch

from velodb_b200 import capi, workloads as W
from velodb_b200._lib import VeloJoinPred, VeloJoinTables, VeloLineitem, VeloLineitemPred

pytestmark = pytest.mark.gpu

ETIMEDOUT, ENOTSUP = -4, -7


def ready():
    """Inputs (and outputs pre-filled) by torch kernels must be complete
    before a command reads or writes them: the consumer runs on a stream of
    its own, and while it runs other streams' kernels wait for SMs."""
    torch.cuda.synchronize()


@pytest.fixture
def pq(cuda):
    q = capi.Queue(persistent=True, idle_us=2000)
    yield q
    q.close()


def kp_case(n, seed):
    keys, pay = W.sort_kp(n, seed=seed)
    cap = capi.next_pow2(n)
    return keys, pay, capi.to_dev_u64(keys, cap), capi.to_dev_u32(pay, cap)


def test_sorts_and_compactions_match_direct_path(pq, orc):
    cmds, checks, keep = [], [], []
    for i, n in enumerate([1, 2, 1000, 4096, 4097, 70_001, 300_000, 1 << 20, (1 << 21) + 3]):
        keys, pay, k, p = kp_case(n, 7000 + i)
        k2, p2 = k.clone(), p.clone()
        if i % 2 == 0:
            cmds.append(capi.make_cmd("OSORT_KP", k, p, n, k.numel()))
            capi.osort_kp(k2, p2, n)
            checks.append((k, p, k2, p2, None, None))
        else:
            marks = (W.lemire(W.splitmix64(7100 + i, n, 0), 10) < 3).astype(np.uint8)
            cap = capi.next_pow2(n)
            m, m2 = capi.to_dev_u8(marks, cap), capi.to_dev_u8(marks, cap)
            cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
            sc = torch.empty(capi.compact_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
            cmds.append(capi.make_cmd("OCOMPACT_KPM", k, p, m, n, cap, cnt, sc, sc.numel()))
            cnt2 = capi.ocompact_kpm(k2, p2, m2, n)
            checks.append((k, p, k2, p2, cnt, cnt2))
            keep += [m, m2, sc]
    ready()
    tix = pq.submit_batch(cmds)
    for t in tix:
        pq.wait(t)
    torch.cuda.synchronize()
    for k, p, k2, p2, cnt, cnt2 in checks:
        assert torch.equal(k, k2) and torch.equal(p, p2)
        if cnt is not None:
            assert int(cnt.item()) == int(cnt2.item())
    # and one against the oracle
    keys, pay, k, p = kp_case(123_457, 99)
    ready()
    pq.wait(pq.submit(capi.make_cmd("OSORT_KP", k, p, 123_457, k.numel())))
    ok, op = orc.bitonic_kp(keys, pay)
    assert np.array_equal(capi.host_u64(k, len(ok)), ok) and np.array_equal(capi.host_u32(p, len(op)), op)


def test_ordered_commands_see_each_others_results(pq):
    # sort, then compact the sorted rows, then permute them: each command
    # reads what the one before wrote
    n = 200_003
    keys, pay, k, p = kp_case(n, 31)
    cap = capi.next_pow2(n)
    marks = (W.lemire(W.splitmix64(32, cap, 0), 4) == 0).astype(np.uint8)
    m = capi.to_dev_u8(marks, cap)
    k2, p2, m2 = k.clone(), p.clone(), m.clone()
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    sc = torch.empty(capi.compact_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
    idx = torch.from_numpy(np.random.default_rng(3).permutation(n).astype(np.int64)).cuda()
    out = torch.zeros(n, dtype=torch.int64, device="cuda")
    ready()
    t1 = pq.submit(capi.make_cmd("OSORT_KP", k, p, n, cap))
    t2 = pq.submit(capi.make_cmd("OCOMPACT_KPM", k, p, m, n, cap, cnt, sc, sc.numel()))
    t3 = pq.submit(capi.make_cmd("PERMUTE", out, k, idx, n, 5))  # BIGINT
    assert t1 < t2 < t3
    pq.wait(t3)
    capi.osort_kp(k2, p2, n)
    cnt2 = capi.ocompact_kpm(k2, p2, m2, n)
    out2 = torch.zeros(n, dtype=torch.int64, device="cuda")
    capi.permute(out2, k2, idx, n, 5)
    torch.cuda.synchronize()
    assert int(cnt.item()) == int(cnt2.item())
    assert torch.equal(k, k2) and torch.equal(p, p2) and torch.equal(out, out2)


def groupby_cmd(dcols, n, pred, G):
    cols = VeloLineitem(*[dcols[c].data_ptr() for c in capi.LINEITEM_COLS])
    pr = VeloLineitemPred(*[int(pred[c]) for c in ("ship_lo", "ship_hi", "disc_lo", "disc_hi", "qty_lo", "qty_hi")])
    out = torch.full((G, 6), 7, dtype=torch.int64, device="cuda")
    counts = torch.full((2,), 7, dtype=torch.int64, device="cuda")
    sc = torch.empty(capi.filter_groupby_scratch_bytes(n, G), dtype=torch.uint8, device="cuda")
    cmd = capi.make_cmd("FILTER_GROUPBY", C.addressof(cols), n, C.addressof(pr), G, out, counts, sc, sc.numel())
    return cmd, (cols, pr, sc), out, counts


@pytest.mark.parametrize("n", [1, 999, 4096, 50_000, 1 << 20, 3_000_001])
def test_filter_groupby_matches_direct_path(pq, n):
    cols = W.lineitem(n, seed=W.SEED_LINEITEM + n)
    dcols = capi.lineitem_to_device(cols)
    # bands too wide for the two-word layout: three-word records
    wide = dict(ship_lo=100, ship_hi=2400, disc_lo=0, disc_hi=10, qty_lo=-100_000, qty_hi=100_000)
    for pred in (W.LINEITEM_PRED, wide):
        cmd, keep, out, counts = groupby_cmd(dcols, n, pred, 8)
        ready()
        pq.wait(pq.submit(cmd))
        out2, counts2 = capi.filter_groupby(dcols, n, pred, 8)
        torch.cuda.synchronize()
        assert torch.equal(counts, counts2) and torch.equal(out, out2)


def join_cmd(dt, pred, k):
    nd, nf = dt["dim_key"].numel(), dt["fact_fk"].numel()
    tabs = VeloJoinTables(dt["dim_key"].data_ptr(), dt["dim_date"].data_ptr(), nd, dt["fact_fk"].data_ptr(),
                          dt["fact_price"].data_ptr(), nf)
    pr = VeloJoinPred(int(pred["date_hi"]), 0, int(pred["price_hi"]))
    out = torch.full((k, 3), 7, dtype=torch.int64, device="cuda")
    counts = torch.full((2,), 7, dtype=torch.int64, device="cuda")
    sc = torch.empty(capi.join_groupby_topk_scratch_bytes(nd, nf), dtype=torch.uint8, device="cuda")
    cmd = capi.make_cmd("JOIN_GROUPBY_TOPK", C.addressof(tabs), C.addressof(pr), k, out, counts, sc, sc.numel())
    return cmd, (tabs, pr, sc), out, counts


@pytest.mark.parametrize("nd,nf,k", [(1, 1, 10), (100, 1000, 10), (20_000, 80_000, 10), (20_000, 80_000, 100),
                                     (1_500_000, 6_000_000, 10)])
def test_join_topk_matches_direct_path(pq, nd, nf, k):
    dim, fact = W.join_tables(nd, nf, seed=W.SEED_JOIN + nd + nf)
    dt = capi.join_to_device(dim, fact)
    cmd, keep, out, counts = join_cmd(dt, W.JOIN_PRED, k)
    ready()
    pq.wait(pq.submit(cmd))
    out2, counts2 = capi.join_groupby_topk(dt, W.JOIN_PRED, k)
    torch.cuda.synchronize()
    assert torch.equal(counts, counts2) and torch.equal(out, out2)


@pytest.mark.parametrize("key_type", [4, 5])  # INTEGER, BIGINT
@pytest.mark.parametrize("bn,pn", [(1, 1), (0, 10), (1000, 5000), (100_000, 400_001)])
def test_pkfk_join_matches_direct_path(pq, key_type, bn, pn):
    rng = np.random.default_rng(bn + pn + key_type)
    dt = np.int32 if key_type == 4 else np.int64
    bk = rng.permutation(max(bn, 1))[:bn].astype(dt) * 3 - 7
    pk = rng.choice(bk, pn) if bn else rng.integers(-5, 5, pn).astype(dt)
    pk = np.where(rng.random(pn) < 0.2, rng.integers(-10**6, 10**6, pn), pk).astype(dt)
    bm = (rng.random(max(bn, 1)) < 0.8).astype(np.uint8)[:bn]
    pm = (rng.random(pn) < 0.8).astype(np.uint8)
    tb = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda() if len(a) else torch.zeros(1, dtype=torch.int64, device="cuda")  # noqa: E731
    dbk, dpk, dbm, dpm = tb(bk), tb(pk), tb(bm), tb(pm)
    ob = torch.full((max(pn, 1),), 9, dtype=torch.int64, device="cuda")
    op = torch.full((max(pn, 1),), 9, dtype=torch.int64, device="cuda")
    cnt = torch.full((2,), 9, dtype=torch.int64, device="cuda")
    sc = torch.empty(max(capi.lib().velo_ojoin_scratch_bytes(bn, pn), 1), dtype=torch.uint8, device="cuda")
    ready()
    pq.wait(pq.submit(capi.make_cmd("OJOIN_PKFK", dbk, dbm, bn, dpk, dpm, pn, key_type, ob, op, cnt, sc,
                                    sc.numel())))
    dbk2 = dbk[:bn] if bn else dbk[:0]
    ob2, op2, cnt2 = capi.ojoin_pkfk(dbk2, dbm if bn else None, dpk, dpm, key_type)
    torch.cuda.synchronize()
    assert torch.equal(cnt, cnt2)
    assert torch.equal(ob[:pn], ob2[:pn]) and torch.equal(op[:pn], op2[:pn])


@pytest.mark.parametrize("tn,rn", [(1, 1), (5000, 12_345), (300_000, 1_000_003)])
def test_ogather_and_shuffle_match_direct_path(pq, tn, rn):
    rng = np.random.default_rng(tn + rn)
    table = torch.from_numpy(W.splitmix64(tn, tn, 0).view(np.int64)).cuda()
    rids = rng.integers(0, tn + 3, rn).astype(np.uint32)  # some past the table
    drids = torch.from_numpy(rids.view(np.int32)).cuda()
    out = torch.zeros(rn, dtype=torch.int64, device="cuda")
    sc = torch.empty(capi.lib().velo_ogather_scratch_bytes(tn, rn), dtype=torch.uint8, device="cuda")
    ready()
    pq.wait(pq.submit(capi.make_cmd("OGATHER", table, tn, drids, rn, out, sc, sc.numel())))
    out2 = torch.zeros(rn, dtype=torch.int64, device="cuda")
    capi.ogather_u64(table, tn, drids, rn, out2)
    # position-map shuffle
    pmap = torch.from_numpy(np.arange(rn, dtype=np.uint32).view(np.int32)).cuda()
    pmap2 = pmap.clone()
    ss = torch.empty(capi.lib().velo_oshuffle_scratch_bytes(rn), dtype=torch.uint8, device="cuda")
    ready()
    pq.wait(pq.submit(capi.make_cmd("OSHUFFLE", pmap, rn, 0x1234, 77, ss, ss.numel())))
    capi.oshuffle_position_map(pmap2, rn, 0x1234, 77)
    torch.cuda.synchronize()
    assert torch.equal(out, out2)
    assert torch.equal(pmap, pmap2)
    assert np.array_equal(np.sort(pmap.cpu().numpy().view(np.uint32)), np.arange(rn, dtype=np.uint32))


def test_reference_command_set_matches_direct_path(pq):
    rng = np.random.default_rng(11)
    n = 100_003
    x = torch.from_numpy(rng.integers(0, 1000, n).astype(np.int32)).cuda()
    y = torch.from_numpy(np.where(rng.random(n) < 0.5, x.cpu().numpy(), 5).astype(np.int32)).cuda()
    idx64 = torch.from_numpy(rng.permutation(n).astype(np.int64)).cuda()
    mask = torch.from_numpy((rng.random(n) < 0.3).astype(np.uint8)).cuda()
    sidx = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    scnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ssc = torch.empty(capi.lib().velo_scatter_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    perm_out = torch.zeros(n, dtype=torch.int32, device="cuda")
    eq_out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    u32 = lambda a: torch.from_numpy(a.astype(np.uint32).view(np.int32)).cuda()  # noqa: E731
    old, sigma = u32(rng.permutation(n)), u32(rng.permutation(n))
    comp = torch.zeros(n, dtype=torch.int32, device="cuda")
    enr = torch.zeros(n, dtype=torch.int32, device="cuda")
    gat = torch.zeros(n, dtype=torch.int32, device="cuda")
    ready()
    t = pq.submit_batch([
        capi.make_cmd("PERMUTE", perm_out, x, idx64, n, 4),
        capi.make_cmd("COMPARE_EQ", x, y, eq_out, n, 4),
        capi.make_cmd("SCATTER", mask, n, sidx, scnt, ssc, ssc.numel()),
        capi.make_cmd("COMPOSE_POSITION_MAP", old, sigma, comp, n),
        capi.make_cmd("ENRICH_POSITIONS", sigma, old, enr, n),
    ])
    # a gather by the scatter's indices runs after the batch (ordered)
    t.append(pq.submit(capi.make_cmd("GATHER", gat, x, sidx, mask, n, 4)))
    for tk in t:
        pq.wait(tk)
    perm2 = torch.zeros(n, dtype=torch.int32, device="cuda")
    capi.permute(perm2, x, idx64, n, 4)
    eq2 = torch.zeros(n, dtype=torch.uint8, device="cuda")
    capi.compare_eq(x, y, eq2, n, 4)
    sidx2 = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    scnt2 = capi.scatter(mask, n, sidx2)
    comp2 = torch.zeros(n, dtype=torch.int32, device="cuda")
    capi.compose_position_map(old, sigma, comp2, n)
    enr2 = torch.zeros(n, dtype=torch.int32, device="cuda")
    capi.enrich_positions(sigma, old, enr2, n)
    gat2 = torch.zeros(n, dtype=torch.int32, device="cuda")
    capi.gather(gat2, x, sidx2, mask, n, 4)
    torch.cuda.synchronize()
    assert torch.equal(perm_out, perm2) and torch.equal(eq_out, eq2) and torch.equal(comp, comp2)
    assert torch.equal(enr, enr2) and torch.equal(sidx, sidx2) and int(scnt.item()) == int(scnt2.item())
    assert torch.equal(gat, gat2)


def test_many_jobs_in_flight_wrap_the_ring(pq):
    # more unordered jobs than ring slots, of uneven sizes
    cases, cmds = [], []
    for i in range(300):
        n = int(W.lemire(W.splitmix64(i, 1, 5), 20_000)[0]) + 1
        keys, pay, k, p = kp_case(n, 50_000 + i)
        cases.append((n, keys, pay, k, p))
        cmds.append(capi.make_cmd("OSORT_KP", k, p, n, k.numel(), flags=capi.CMD_UNORDERED))
    ready()
    tix = [pq.submit(c) for c in cmds]
    for t in tix:
        pq.wait(t)
    for n, keys, pay, k, p in cases:
        order = np.lexsort((pay, keys))
        assert np.array_equal(capi.host_u64(k, n), keys[order]) and np.array_equal(capi.host_u32(p, n), pay[order])


def test_consumer_exits_when_idle_and_is_relaunched(pq):
    keys, pay, k, p = kp_case(50_000, 5)
    ready()
    pq.wait(pq.submit(capi.make_cmd("OSORT_KP", k, p, 50_000, k.numel())))
    first = pq.launches()
    assert first >= 1
    # well past the 2 ms idle time the consumer's stream is idle: it exited
    st = torch.cuda.ExternalStream(capi.lib().velo_ctx_stream(pq._c))
    deadline = time.time() + 5.0
    while not st.query():
        assert time.time() < deadline, "the consumer did not exit when idle"
        time.sleep(0.002)
    keys, pay, k, p = kp_case(60_000, 6)
    ready()
    pq.wait(pq.submit(capi.make_cmd("OSORT_KP", k, p, 60_000, k.numel())))
    assert pq.launches() > first
    order = np.lexsort((pay, keys))
    assert np.array_equal(capi.host_u64(k, 60_000), keys[order])


def test_wait_is_bounded_and_unsupported_opcodes_are_refused(pq):
    n = 1 << 24
    keys, pay, k, p = kp_case(n, 1)
    ready()
    t = pq.submit(capi.make_cmd("OSORT_KP", k, p, n, k.numel()))
    assert pq.wait_raw(t, 1000) == ETIMEDOUT  # 1 us: the sort cannot be done yet
    pq.wait(t)
    assert pq.submit_raw(capi.make_cmd("OJOIN_MN")) == ENOTSUP
    assert pq.wait_raw(10**9, 1000) == -1  # unknown ticket


def test_rapid_publication_of_tiny_jobs(pq):
    # thousands of tiny jobs published back to back while the consumer runs:
    # every one is ingested once, runs, and reports success
    n = 3
    keys = [torch.from_numpy(W.splitmix64(i, 4, 9).view(np.int64)).cuda() for i in range(2000)]
    pays = [torch.from_numpy(np.arange(4, dtype=np.int32)).cuda() for _ in range(2000)]
    ready()
    tix = [pq.submit(capi.make_cmd("OSORT_KP", k, p, n, 4, flags=capi.CMD_UNORDERED)) for k, p in zip(keys, pays)]
    for t in tix:
        pq.wait(t)
    for i, k in enumerate(keys):
        h = k.cpu().numpy().view(np.uint64)
        assert np.array_equal(h[:3], np.sort(W.splitmix64(i, 4, 9)[:3]))
