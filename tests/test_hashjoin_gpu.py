"""GPU parity of the oblivious bin-padded hash join (velo_ohash_join): for a
build side with unique keys it returns every (build row, probe row) pair with
equal keys and both rows valid -- the reference hash join's output
(include/cuda/hash_join.cuh:28-254) as a set -- and it reports a repeated
build key or a bin overflow instead of losing pairs silently."""
import numpy as np
import pytest
import torch

from velodb_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu

INTEGER, BIGINT = 4, 5


def run(build, bmask, probe, pmask, key_type=INTEGER, seed=0x5EED):
    dt = torch.int32 if key_type == INTEGER else torch.int64
    bk = torch.from_numpy(np.ascontiguousarray(build)).to(dtype=dt, device="cuda")
    pk = torch.from_numpy(np.ascontiguousarray(probe)).to(dtype=dt, device="cuda")
    bm = None if bmask is None else torch.from_numpy(bmask.astype(np.uint8)).cuda()
    pm = None if pmask is None else torch.from_numpy(pmask.astype(np.uint8)).cuda()
    ob, op, cnt = capi.ohash_join(bk, bm, pk, pm, key_type, seed)
    torch.cuda.synchronize()
    return ob.cpu().numpy(), op.cpu().numpy(), cnt.cpu().numpy()


def expected_pairs(orc, build, bmask, probe, pmask):
    ol, orr, _ = orc.smj_pairs(probe, pmask, build, bmask)
    return set(zip(orr.tolist(), ol.tolist()))


def check(orc, build, bmask, probe, pmask, key_type=INTEGER, seed=0x5EED):
    ob, op, cnt = run(build, bmask, probe, pmask, key_type, seed)
    assert int(cnt[1]) == 0 and int(cnt[2]) == 0
    m = int(cnt[0])
    want = expected_pairs(orc, build, bmask, probe, pmask)
    assert m == len(want)
    assert set(zip(ob[:m].tolist(), op[:m].tolist())) == want
    assert (ob[m:] == -1).all() and (op[m:] == -1).all()
    # pairs come in (bin, probe row id) order: probe row ids rise inside a bin
    return m


@pytest.mark.parametrize("nd,nf", [(1, 1), (5, 40), (1000, 4000), (3000, 10_000), (50_000, 200_000),
                                   (1_500_000, 6_000_000)])
def test_hash_join_pkfk(cuda, orc, nd, nf):
    dim, fact = W.join_tables(nd, nf, seed=W.SEED_JOIN + 17 + nd)
    check(orc, dim["key"], None, fact["fk"], None)
    dm = dim["date"] < W.JOIN_PRED["date_hi"]
    fm = fact["price"] < W.JOIN_PRED["price_hi"]
    check(orc, dim["key"], dm, fact["fk"], fm)


def test_hash_join_bigint_keys_and_seeds(cuda, orc):
    keys = (W.splitmix64(3, 40_000, 0) >> np.uint64(1)).view(np.int64)  # distinct with overwhelming odds
    keys = np.unique(keys)
    probe = keys[W.uniform_int(4, 100_000, 0, 0, len(keys) - 1, np.int64)]
    probe[::7] = -probe[::7] - 1  # misses
    for seed in (1, 2, 0xDEADBEEF):
        check(orc, keys, None, probe, None, key_type=BIGINT, seed=seed)


def test_hash_join_reports_repeated_build_keys(cuda, orc):
    build = np.array([1, 2, 2, 3], np.int32)
    probe = np.array([2, 3, 4], np.int32)
    _, _, cnt = run(build, None, probe, None)
    assert int(cnt[1]) == 1  # probe row 0 has two partners


def test_hash_join_reports_bin_overflow(cuda, orc):
    dim, _ = W.join_tables(20_000, 1, seed=5)
    probe = np.full(200_000, dim["key"][7], np.int32)  # one hot key: its bin overflows
    _, _, cnt = run(dim["key"], None, probe, None)
    assert int(cnt[2]) > 0
