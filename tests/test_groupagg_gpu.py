"""GPU parity of the generic oblivious GROUP BY (velo_ogroupby) against exact
host group sums and against the oracle's restatement of the reference's
oblivious group-by (scalable_oblivious_join.c:221-232)."""
import numpy as np
import pytest
import torch

from velodb_b200 import capi

pytestmark = pytest.mark.gpu

INTEGER, BIGINT = 4, 5


def expected(keys, vals, mask):
    k = keys[mask]
    uk, inv = np.unique(k, return_inverse=True)
    sums = [np.zeros(len(uk), np.int64) for _ in vals]
    for s, v in zip(sums, vals):
        np.add.at(s, inv, v[mask])
    cnt = np.bincount(inv, minlength=len(uk)).astype(np.int64)
    return uk.astype(np.int64), sums, cnt


def run(keys, key_type, vals, with_count, mask=None, bound=None):
    n = len(keys)
    dk = torch.from_numpy(keys).cuda()
    dv = [torch.from_numpy(v).cuda() for v in vals]
    dm = torch.from_numpy(mask.astype(np.uint8)).cuda() if mask is not None else None
    ok, osum, ocnt, cnt = capi.ogroupby(dk, key_type, n, dv, with_count, dm, bound)
    torch.cuda.synchronize()
    return (ok.cpu().numpy(), [s.cpu().numpy() for s in osum], None if ocnt is None else ocnt.cpu().numpy(),
            cnt.cpu().numpy())


@pytest.mark.parametrize("n", [1, 7, 100, 2048, 4097, 70_001, 300_000])
@pytest.mark.parametrize("combo", [(0, True), (1, True), (1, False), (2, False)])
def test_ogroupby_matches_exact_sums(cuda, n, combo):
    ns, with_count = combo
    rng = np.random.default_rng(n * 7 + ns)
    keys = rng.integers(-50, 50, n).astype(np.int32) if n > 100 else rng.integers(-2**31, 2**31, n).astype(np.int32)
    vals = [rng.integers(-10**9, 10**9, n).astype(np.int64) for _ in range(ns)]
    mask = rng.random(n) < 0.7
    ok, osum, ocnt, cnt = run(keys, INTEGER, vals, with_count, mask)
    ek, es, ec = expected(keys, vals, mask)
    g = len(ek)
    assert int(cnt[0]) == g and int(cnt[1]) == 0
    assert np.array_equal(ok[:g], ek)
    for a, b in zip(osum, es):
        assert np.array_equal(a[:g], b)
    if with_count:
        assert np.array_equal(ocnt[:g], ec)
    assert not ok[g:].any() and all(not a[g:].any() for a in osum)


EXTREMES = np.array([-(2**63), -(2**63) + 1, -(2**62) - 1, -(2**62), -5, 0, 7, 2**62 - 1, 2**62, 2**63 - 2,
                     2**63 - 1], np.int64)


@pytest.mark.parametrize("combo", [(0, True), (1, True), (1, False), (2, False)])
def test_ogroupby_bigint_full_range(cuda, combo):
    # every BIGINT value is a key, the extremes included, with and without a
    # mask; a key whose rows are all left out forms no group
    ns, with_count = combo
    n = 50_000
    rng = np.random.default_rng(3 + ns)
    keys = rng.choice(EXTREMES, n)
    vals = [rng.integers(-10**12, 10**12, n).astype(np.int64) for _ in range(ns)]
    for mask in (None, rng.random(n) < 0.6, keys != 2**63 - 1):
        ok, osum, ocnt, cnt = run(keys, BIGINT, vals, with_count, mask)
        ek, es, ec = expected(keys, vals, np.ones(n, bool) if mask is None else mask)
        g = len(ek)
        assert int(cnt[0]) == g and int(cnt[1]) == 0
        assert np.array_equal(ok[:g], ek)
        for a, b in zip(osum, es):
            assert np.array_equal(a[:g], b)
        if with_count:
            assert np.array_equal(ocnt[:g], ec)
        assert not ok[g:].any()


@pytest.mark.parametrize("n", [1, 4097, 300_000])
def test_ogroupby_bigint_random(cuda, n):
    rng = np.random.default_rng(n)
    keys = (rng.integers(-(2**63), 2**63 - 1, n, dtype=np.int64) // (2**60)) * (2**60)  # 16 distinct values
    keys[: n // 3] = rng.integers(-(2**63), 2**63 - 1, n // 3, dtype=np.int64)
    vals = [rng.integers(-10**9, 10**9, n).astype(np.int64)]
    mask = rng.random(n) < 0.8
    ok, osum, ocnt, cnt = run(keys, BIGINT, vals, True, mask)
    ek, es, ec = expected(keys, vals, mask)
    g = len(ek)
    assert int(cnt[0]) == g
    assert np.array_equal(ok[:g], ek) and np.array_equal(osum[0][:g], es[0]) and np.array_equal(ocnt[:g], ec)


def test_ogroupby_public_bound(cuda):
    n = 10_000
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 1000, n).astype(np.int32)
    vals = [np.ones(n, np.int64)]
    ok, osum, ocnt, cnt = run(keys, INTEGER, vals, True, bound=16)
    ek, es, ec = expected(keys, vals, np.ones(n, bool))
    assert int(cnt[0]) == len(ek) and len(ok) == 16
    assert np.array_equal(ok, ek[:16]) and np.array_equal(osum[0], es[0][:16]) and np.array_equal(ocnt, ec[:16])


def test_ogroupby_nothing_selected(cuda):
    keys = np.arange(5000, dtype=np.int32)
    ok, osum, ocnt, cnt = run(keys, INTEGER, [], True, np.zeros(5000, bool))
    assert int(cnt[0]) == 0 and not ok.any() and not ocnt.any()


def test_ogroupby_matches_oracle_restatement(cuda, orc):
    n = 20_000
    rng = np.random.default_rng(9)
    keys = rng.integers(0, 300, n).astype(np.int32)
    vals = [rng.integers(-1000, 1000, n).astype(np.int64), rng.integers(0, 10**12, n).astype(np.int64)]
    ok, osum, _, cnt = run(keys, INTEGER, vals, False)
    order = np.argsort(keys, kind="stable")
    gk, gs = orc.groupby_sorted(keys[order].astype(np.uint64), np.stack([v[order] for v in vals], axis=1))
    g = len(gk)
    assert int(cnt[0]) == g
    assert np.array_equal(ok[:g], gk.astype(np.int64))
    assert np.array_equal(osum[0][:g], gs[:, 0]) and np.array_equal(osum[1][:g], gs[:, 1])
