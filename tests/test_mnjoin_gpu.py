"""GPU parity of the oblivious many-to-many equi-join (velo_ojoin_mn) with the
reference sort-merge join's output (the oracle's restatement of
include/cuda/sort_merge_join.cuh:63-199): every pair of rows with equal keys,
in (key, probe row id, build row id) order, padded to the public bound."""
import numpy as np
import pytest
import torch

from velodb_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu

INTEGER, BIGINT = 4, 5


def run(build, bmask, probe, pmask, key_type, max_pairs):
    dt = torch.int32 if key_type == INTEGER else torch.int64
    bk = torch.from_numpy(np.ascontiguousarray(build)).to(dtype=dt, device="cuda")
    pk = torch.from_numpy(np.ascontiguousarray(probe)).to(dtype=dt, device="cuda")
    bm = None if bmask is None else torch.from_numpy(bmask.astype(np.uint8)).cuda()
    pm = None if pmask is None else torch.from_numpy(pmask.astype(np.uint8)).cuda()
    ob, op, cnt = capi.ojoin_mn(bk, bm, pk, pm, key_type, max_pairs)
    torch.cuda.synchronize()
    return ob.cpu().numpy(), op.cpu().numpy(), cnt.cpu().numpy()


def check(orc, build, bmask, probe, pmask, key_type=INTEGER, max_pairs=None):
    ol, orr, total = orc.smj_pairs(probe, pmask, build, bmask)
    mp = max(total, 1) if max_pairs is None else max_pairs
    ob, op, cnt = run(build, bmask, probe, pmask, key_type, mp)
    assert int(cnt[0]) == total
    assert int(cnt[1]) == (1 if total > mp else 0)
    m = min(total, mp)
    assert np.array_equal(op[:m], ol[:m])
    assert np.array_equal(ob[:m], orr[:m])
    assert (op[m:] == -1).all() and (ob[m:] == -1).all()
    return total


def keys(seed, n, lo, hi, dtype=np.int32):
    return W.uniform_int(seed, n, 0, lo, hi, dtype)


def mask(seed, n, tenths):
    return W.lemire(W.splitmix64(seed, n, 9), 10) < tenths


@pytest.mark.parametrize("nb,np_,span", [(1, 1, 1), (3, 5, 2), (100, 300, 20), (1000, 1000, 1000),
                                         (5000, 20_000, 3000), (40_000, 100_000, 50_000)])
def test_mn_join_duplicates_both_sides(cuda, orc, nb, np_, span):
    b = keys(nb, nb, 1, span)
    p = keys(np_ + 7, np_, 1, span)
    total = check(orc, b, None, p, None)
    # with masks on both sides and a bound above the pair count
    check(orc, b, mask(1, nb, 7), p, mask(2, np_, 6), max_pairs=total + 123)


def test_mn_join_cross_product_and_no_match(cuda, orc):
    b = np.full(300, 42, np.int32)
    p = np.full(200, 42, np.int32)
    assert check(orc, b, None, p, None) == 60_000
    assert check(orc, b, None, p + 1, None) == 0


def test_mn_join_overflow_keeps_the_first_pairs(cuda, orc):
    b = keys(3, 2000, 1, 50)
    p = keys(4, 3000, 1, 50)
    check(orc, b, None, p, None, max_pairs=10_000)  # far fewer than the ~120 k pairs
    check(orc, b, None, p, None, max_pairs=1)


def test_mn_join_bigint_extremes(cuda, orc):
    big = np.array([-(2**63), 2**63 - 1, -1, 0, 1, 2**40, -(2**40)], np.int64)
    b = np.concatenate([big, big[:4], big[2:]])
    p = np.concatenate([big[::-1], big, big[3:]])
    check(orc, b, None, p, None, key_type=BIGINT)
    b = W.splitmix64(5, 30_000, 0).view(np.int64) // (2**51)
    p = W.splitmix64(6, 30_000, 1).view(np.int64) // (2**51)
    check(orc, b, mask(7, 30_000, 5), p, None, key_type=BIGINT)


def test_mn_join_pkfk_matches_pkfk_operator(cuda, orc):
    dim, fact = W.join_tables(20_000, 80_000, seed=12)
    total = check(orc, dim["key"], None, fact["fk"], None)
    bk = torch.from_numpy(dim["key"]).cuda()
    pk = torch.from_numpy(fact["fk"]).cuda()
    ob, op, cnt = capi.ojoin_pkfk(bk, None, pk, None, INTEGER)
    torch.cuda.synchronize()
    m = int(cnt[0].item())
    assert m == total
    a = set(zip(ob.cpu().numpy()[:m].tolist(), op.cpu().numpy()[:m].tolist()))
    mb, mpr, _ = run(dim["key"], None, fact["fk"], None, INTEGER, total)
    assert a == set(zip(mb.tolist(), mpr.tolist()))


def test_mn_join_larger(cuda, orc):
    b = keys(8, 300_000, 1, 200_000)
    p = keys(9, 1_000_000, 1, 200_000)
    check(orc, b, mask(10, 300_000, 8), p, mask(11, 1_000_000, 9))
