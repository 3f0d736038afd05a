"""GPU parity of the oblivious filter + group-by pipeline against the oracle
(exact int64 sums), through the C ABI."""
import numpy as np
import pytest
import torch

from velodb_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu


def run_gpu(cols, pred, G=8, reveal=False):
    n = len(cols["qty"])
    d = capi.lineitem_to_device(cols)
    out, counts = capi.filter_groupby(d, n, pred, G, reveal_count=reveal)
    torch.cuda.synchronize()
    return out.cpu().numpy(), counts.cpu().numpy()


def check(orc, cols, pred, G=8, reveal=False):
    out, counts = run_gpu(cols, pred, G, reveal)
    g, keys, sums = orc.filter_groupby(cols, pred, max_groups=G)
    mask = ((cols["shipdate"] >= pred["ship_lo"]) & (cols["shipdate"] <= pred["ship_hi"])
            & (cols["disc"] >= pred["disc_lo"]) & (cols["disc"] <= pred["disc_hi"])
            & (cols["qty"] >= pred["qty_lo"]) & (cols["qty"] <= pred["qty_hi"]))
    assert int(counts[0]) == int(mask.sum())
    assert int(counts[1]) == g
    m = min(g, G)
    assert np.array_equal(out[:m, 0], keys[:m].astype(np.int64))
    assert np.array_equal(out[:m, 1:], sums[:m])
    assert not out[m:].any()


@pytest.mark.parametrize("n", [1, 7, 100, 2047, 2048, 4096, 5000, 65536, 100_003])
def test_filter_groupby_small(cuda, orc, n):
    cols = W.lineitem(n, seed=W.SEED_LINEITEM + n)
    check(orc, cols, W.LINEITEM_PRED)
    check(orc, cols, dict(ship_lo=0, ship_hi=2556, disc_lo=0, disc_hi=10, qty_lo=1, qty_hi=50))  # everything


def test_filter_groupby_selectivities(cuda, orc):
    cols = W.lineitem(300_000, seed=99)
    for pred in [dict(ship_lo=0, ship_hi=-1, disc_lo=0, disc_hi=10, qty_lo=1, qty_hi=50),  # nothing passes
                 dict(ship_lo=5, ship_hi=6, disc_lo=3, disc_hi=3, qty_lo=1, qty_hi=2),      # a handful
                 W.LINEITEM_PRED]:
        check(orc, cols, pred)
        check(orc, cols, pred, reveal=True)


def test_filter_groupby_bound_smaller_than_groups(cuda, orc):
    cols = W.lineitem(50_000, seed=5)
    check(orc, cols, W.LINEITEM_PRED, G=4)  # 6 groups, 4 slots: first 4 in key order, count says 6


def test_filter_groupby_config1_full(cuda, orc):
    cols = W.lineitem()  # 6,001,215 rows
    check(orc, cols, W.LINEITEM_PRED)
    check(orc, cols, W.LINEITEM_PRED, reveal=True)


def test_filter_groupby_wide_bands_use_three_word_records(cuda, orc):
    # bands too wide for the packed two-word layout: the three-word path
    cols = W.lineitem(70_000, seed=17)
    check(orc, cols, dict(ship_lo=0, ship_hi=2000, disc_lo=-(1 << 20), disc_hi=1 << 20, qty_lo=-(2**31),
                          qty_hi=2**31 - 1))


def test_filter_groupby_band_edges_in_packed_layout(cuda, orc):
    # qty band of 10 bits and disc band of 5 bits (15 packed bits, the limit),
    # with values at both edges of each band
    n = 20_000
    rng = np.random.default_rng(4)
    cols = W.lineitem(n, seed=23)
    cols["qty"] = rng.choice(np.array([-7, -7 + 1023, 100], np.int32), n)
    cols["disc"] = rng.choice(np.array([3, 3 + 31, 10], np.int32), n)
    check(orc, cols, dict(ship_lo=0, ship_hi=2556, disc_lo=3, disc_hi=34, qty_lo=-7, qty_hi=1016))


def test_stage_timing_reports_four_stages(cuda):
    cols = W.lineitem(100_000, seed=3)
    d = capi.lineitem_to_device(cols)
    capi.set_stage_timing(True)
    try:
        capi.filter_groupby(d, 100_000, W.LINEITEM_PRED)
        t = capi.last_stage_times()
    finally:
        capi.set_stage_timing(False)
    assert len(t) == 4 and all(x >= 0 for x in t) and sum(t) > 0
