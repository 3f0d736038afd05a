"""GPU tests of the reference command-set operators (same semantics as the
reference) and of the oblivious shuffle, gather and PK-FK join."""
import numpy as np
import pytest
import torch

from velodb_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu

TYPES = {1: np.uint8, 2: np.int8, 3: np.int16, 4: np.int32, 5: np.int64, 6: np.float32, 7: np.float64, 8: np.uint64,
         10: np.uint32}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).to("cuda")


def host(t, dtype, n):
    return t.cpu().numpy().view(dtype)[:n]


@pytest.mark.parametrize("type_id", sorted(TYPES))
def test_permute_and_gather(cuda, type_id):
    rng = np.random.default_rng(type_id)
    n = 10_007
    dt = TYPES[type_id]
    x = (rng.integers(0, 100, n)).astype(dt)
    idx = rng.permutation(n).astype(np.int64)
    out = torch.zeros(n * x.itemsize, dtype=torch.uint8, device=cuda)
    capi.permute(out, dev(x), torch.from_numpy(idx).to(cuda), n, type_id)
    assert np.array_equal(host(out, dt, n), x[idx])
    mask = (rng.random(n) < 0.4).astype(np.uint8)
    dmask = torch.from_numpy(mask).to(cuda)
    sidx = torch.full((n,), -1, dtype=torch.int32, device=cuda)
    cnt = capi.scatter(dmask, n, sidx)
    assert int(cnt.item()) == int(mask.sum())
    si = sidx.cpu().numpy()
    assert np.array_equal(si[mask.astype(bool)], np.arange(int(mask.sum())))
    assert (si[~mask.astype(bool)] == -1).all()  # untouched
    g = torch.zeros(n * x.itemsize, dtype=torch.uint8, device=cuda)
    capi.gather(g, dev(x), sidx, dmask, n, type_id)
    assert np.array_equal(host(g, dt, int(mask.sum())), x[mask.astype(bool)])


def test_compare_eq_reference_semantics(cuda):
    rng = np.random.default_rng(2)
    n = 5000
    for type_id, dt in TYPES.items():
        a = rng.integers(0, 3, n).astype(dt)
        b = rng.integers(0, 3, n).astype(dt)
        out = torch.full((n,), 7, dtype=torch.uint8, device=cuda)
        capi.compare_eq(dev(a), dev(b), out, n, type_id)
        got = out.cpu().numpy()
        if type_id in (1, 8):  # BOOLEAN, VARCHAR: the reference writes zeros
            assert not got.any()
        elif type_id == 10:  # DATE compares as int32
            assert np.array_equal(got, (a.view(np.int32) == b.view(np.int32)).astype(np.uint8))
        else:
            assert np.array_equal(got, (a == b).astype(np.uint8))


def test_compose_and_enrich(cuda):
    rng = np.random.default_rng(3)
    n = 100_000
    old = rng.permutation(n).astype(np.uint32)
    sigma = rng.permutation(n).astype(np.uint32)
    new = torch.empty(n, dtype=torch.int32, device=cuda)
    capi.compose_position_map(dev(old), dev(sigma), new, n)
    assert np.array_equal(host(new, np.uint32, n), old[sigma])
    rids = rng.integers(0, n, 30_000).astype(np.uint32)
    pos = torch.empty(30_000, dtype=torch.int32, device=cuda)
    capi.enrich_positions(dev(rids), dev(old), pos, 30_000)
    assert np.array_equal(host(pos, np.uint32, 30_000), old[rids])


@pytest.mark.parametrize("n", [1, 2, 1000, 8192, 65_537, 1 << 20])
def test_oblivious_shuffle(cuda, orc, n):
    pmap = np.random.default_rng(n).permutation(n).astype(np.uint32)
    d = dev(pmap).view(torch.int32)
    key, counter = 0x0123456789ABCDEF, 42
    capi.oshuffle_position_map(d, n, key, counter)
    got = host(d, np.uint32, n)
    assert np.array_equal(got, orc.shuffle_position_map(pmap, key, counter))
    assert np.array_equal(np.sort(got), np.sort(pmap))  # still a permutation
    # a different counter gives a different permutation
    d2 = dev(pmap).view(torch.int32)
    capi.oshuffle_position_map(d2, n, key, counter + 1)
    if n > 8:
        assert not np.array_equal(host(d2, np.uint32, n), got)


@pytest.mark.parametrize("tn,rn", [(1, 1), (10, 100), (5000, 3000), (100_000, 250_000), (1 << 20, 1 << 18)])
def test_oblivious_gather(cuda, tn, rn):
    rng = np.random.default_rng(tn + rn)
    table = W.splitmix64(tn, tn, 0)
    rids = rng.integers(0, tn + max(1, tn // 10), rn).astype(np.uint32)  # duplicates and out-of-range ids
    out = torch.empty(rn, dtype=torch.int64, device=cuda)
    capi.ogather_u64(dev(table).view(torch.int64), tn, dev(rids).view(torch.int32), rn, out)
    exp = np.where(rids < tn, table[np.minimum(rids, tn - 1)], 0).astype(np.uint64)
    assert np.array_equal(out.cpu().numpy().view(np.uint64), exp)


def join_expected(bk, bm, pk, pm):
    pos = {}
    for i, (k, m) in enumerate(zip(bk.tolist(), bm.tolist())):
        pos[k] = (i, m)
    pairs = []
    for j, (k, m) in enumerate(zip(pk.tolist(), pm.tolist())):
        if m and k in pos and pos[k][1]:
            pairs.append((pos[k][0], j))
    return pairs


@pytest.mark.parametrize("key_type", [4, 5])
@pytest.mark.parametrize("bn,pn", [(1, 1), (10, 50), (1000, 5000), (60_000, 250_000)])
def test_oblivious_pkfk_join_pairs(cuda, key_type, bn, pn):
    rng = np.random.default_rng(bn * 7 + pn + key_type)
    dt = np.int32 if key_type == 4 else np.int64
    bk = (rng.permutation(bn * 2)[:bn] - bn).astype(dt)  # unique, signed
    pk = rng.choice(np.concatenate([bk, np.arange(bn * 2, bn * 2 + 50).astype(dt)]), pn).astype(dt)
    bm = (rng.random(bn) < 0.8).astype(np.uint8)
    pm = (rng.random(pn) < 0.7).astype(np.uint8)
    ob, op, cnt = capi.ojoin_pkfk(dev(bk).view(torch.int32 if dt == np.int32 else torch.int64),
                                  torch.from_numpy(bm).to(cuda),
                                  dev(pk).view(torch.int32 if dt == np.int32 else torch.int64),
                                  torch.from_numpy(pm).to(cuda), key_type)
    torch.cuda.synchronize()
    exp = join_expected(bk, bm, pk, pm)
    c = int(cnt[0].item())
    assert c == len(exp) and int(cnt[1].item()) == 0
    got_b, got_p = ob.cpu().numpy()[:pn], op.cpu().numpy()[:pn]
    assert sorted(zip(got_b[:c].tolist(), got_p[:c].tolist())) == sorted(exp)
    assert (got_b[c:] == -1).all() and (got_p[c:] == -1).all()
    keys = bk[got_b[:c]].astype(np.int64)
    assert np.all(keys[:-1] <= keys[1:])  # pairs come in key order


def test_oblivious_join_reports_duplicate_build_keys(cuda):
    bk = np.array([5, 7, 5, 9], np.int32)
    pk = np.array([5, 9, 1], np.int32)
    ob, op, cnt = capi.ojoin_pkfk(dev(bk).view(torch.int32), None, dev(pk).view(torch.int32), None, 4)
    assert int(cnt[1].item()) == 1
