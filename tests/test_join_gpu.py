"""GPU parity of the oblivious PK-FK join + group-by + top-k against the
oracle (exact int64 sums, ties broken by fk), through the C ABI."""
import numpy as np
import pytest
import torch

from velodb_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu


def check(orc, dim, fact, pred, k=10):
    dt = capi.join_to_device(dim, fact)
    out, counts = capi.join_groupby_topk(dt, pred, k)
    torch.cuda.synchronize()
    out, counts = out.cpu().numpy(), counts.cpu().numpy()
    g, fk, s, c = orc.join_groupby_topk(dim, fact, pred, k)
    assert int(counts[1]) == g
    m = min(g, k)
    assert np.array_equal(out[:m, 0], fk.astype(np.int64))
    assert np.array_equal(out[:m, 1], s)
    assert np.array_equal(out[:m, 2], c)
    assert not out[m:].any()
    dv = dim["date"] < pred["date_hi"]
    ok_keys = set(dim["key"][dv].tolist())
    joined = int(((fact["price"] < pred["price_hi"]) & np.isin(fact["fk"], list(ok_keys))).sum())
    assert int(counts[0]) == joined


@pytest.mark.parametrize("nd,nf", [(1, 1), (1, 5), (10, 3), (100, 1000), (3000, 10000), (20000, 80000),
                                   (100_000, 500_000)])
def test_join_small(cuda, orc, nd, nf):
    dim, fact = W.join_tables(nd, nf, seed=W.SEED_JOIN + nd)
    check(orc, dim, fact, W.JOIN_PRED)
    check(orc, dim, fact, dict(date_hi=10**6, price_hi=10**12))  # everything joins


def test_join_ties_and_no_matches(cuda, orc):
    dim, fact = W.join_tables(500, 4000, seed=3)
    fact["price"] = np.full(4000, 100_000, np.int64)  # many equal sums: fk breaks ties
    check(orc, dim, fact, dict(date_hi=10**6, price_hi=10**12), k=50)
    check(orc, dim, fact, dict(date_hi=-1, price_hi=10**12))  # no dimension row passes


@pytest.mark.parametrize("k", [1, 15, 16, 17, 100, 1024])
def test_join_topk_sizes(cuda, orc, k):
    # candidates a tile keeps: 16 up to k = 16, then next_pow2(k); 1024 keeps whole tiles
    dim, fact = W.join_tables(5000, 40000, seed=11)
    check(orc, dim, fact, W.JOIN_PRED, k=k)
    check(orc, dim, fact, dict(date_hi=10**6, price_hi=10**12), k=k)


def test_join_config2_full(cuda, orc):
    dim, fact = W.join_tables()  # 1.5 M x 6 M
    check(orc, dim, fact, W.JOIN_PRED)
