"""GPU parity of the network sorts with each load tune switched on: the
bulk-copy merge prefetch (velo_set_merge_pipeline) and the tensor-map tile
loads of the merge and fused global passes (velo_set_tensor_tile_loads).
Both keep the network, so the results are bit-exact against the oracle, and
the pipelines that sort inside (join, group-by) equal their plain runs."""
import numpy as np
import pytest
import torch

from velodb_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu

ALL_ONES = 2**64 - 1


@pytest.fixture(params=sorted(capi.TUNES))
def tune(request):
    switch = capi.TUNES[request.param]
    switch(True)
    try:
        yield request.param
    finally:
        switch(False)
    assert capi.tensor_tile_status() == 0


def gpu_sort_kp(keys, pay):
    n = len(keys)
    cap = capi.next_pow2(n)
    k, p = capi.to_dev_u64(keys, cap), capi.to_dev_u32(pay, cap)
    capi.osort_kp(k, p, n)
    torch.cuda.synchronize()
    return capi.host_u64(k, cap), capi.host_u32(p, cap)


def gpu_sort_records(words, mask, strict):
    n = len(words[0])
    cap = capi.next_pow2(n)
    ds = [capi.to_dev_u64(w, cap) for w in words]
    capi.osort_records(ds, n, mask, strict=strict)
    torch.cuda.synchronize()
    return [capi.host_u64(d, cap) for d in ds]


# 2^13 rows: one global pass of one level; 65,537 and 300,001 rows: a
# partial last tile; 2^20: global passes of 1..8 levels
@pytest.mark.parametrize("n", [8192, 65_537, 300_001, 1 << 20])
def test_sort_kp_with_tune(cuda, orc, tune, n):
    keys, pay = W.sort_kp(n, seed=W.SEED_SORT + 3 * n)
    keys[: n // 3] = keys[n // 2]  # ties: the arrangement of equal keys is the network's
    gk, gp = gpu_sort_kp(keys, pay)
    ok, op = orc.bitonic_kp(keys, pay)
    assert np.array_equal(gk, ok) and np.array_equal(gp, op)


def record_case(words, seed):
    n = (1 << 19) + 123
    ws = [W.splitmix64(seed + x, n, x) for x in range(words)]
    ws[0] = ws[0] & np.uint64(0xFFFF0000FFFFFFFF)  # equal masked keys
    return ws


# Strict record sorts order ties as the oracle's network does, so they are
# bit-exact against it; the default (non-strict) sorts may exchange equal keys
# in descending blocks, so their keys match the oracle's and their whole rows
# match the same sort with the tune off.
@pytest.mark.parametrize("words,mask", [(2, 0xFFFFFFFF00000000), (2, ALL_ONES), (3, 0xFFFF800000000000)])
@pytest.mark.parametrize("strict", [True, False])
def test_sort_records_with_tune(cuda, orc, tune, words, mask, strict):
    ws = record_case(words, 11)
    got = gpu_sort_records(ws, mask, strict)
    want = orc.bitonic_records(ws, 1, [mask], [ALL_ONES] * words)
    if strict:
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
        return
    assert np.array_equal(got[0] & np.uint64(mask), want[0] & np.uint64(mask))
    capi.TUNES[tune](False)
    plain = gpu_sort_records(ws, mask, strict)
    for g, w in zip(got, plain):
        assert np.array_equal(g, w)


@pytest.mark.parametrize("words,mask", [(1, ALL_ONES), (2, 0xFFFFFFFF00000000), (3, 0xFFFF800000000000)])
def test_sort_records_strict_without_tune(cuda, orc, words, mask):
    ws = record_case(words, 29)
    got = gpu_sort_records(ws, mask, True)
    want = orc.bitonic_records(ws, 1, [mask], [ALL_ONES] * words)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_join_and_groupby_with_tune(cuda, tune):
    dim, fact = W.join_tables()
    dt = capi.join_to_device(dim, fact)
    cols = W.lineitem()
    dc = capi.lineitem_to_device(cols)
    n = W.LINEITEM_ROWS

    def both():
        jo, jc = capi.join_groupby_topk(dt, W.JOIN_PRED, W.JOIN_TOPK)
        go, gc = capi.filter_groupby(dc, n, W.LINEITEM_PRED, W.LINEITEM_GROUP_BOUND)
        torch.cuda.synchronize()
        return [t.cpu().numpy() for t in (jo, jc, go, gc)]

    with_tune = both()
    capi.TUNES[tune](False)
    plain = both()
    for a, b in zip(with_tune, plain):
        assert np.array_equal(a, b)
