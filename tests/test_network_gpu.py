"""GPU parity of the two oblivious networks against the oracle, through the C ABI.

Bit-exact: the GPU bitonic network and the oracle's reference-order network
perform the same compare-exchanges, so outputs match element for element
(including sentinel pads and the arrangement of equal keys); ORCompact is
compared over the padded rows element for element, and against the golden
outputs of the reference's liboblivious o_compact.
"""
import numpy as np
import pytest
import torch

from velodb_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu

TUNES = [(11, 256), (11, 512), (11, 1024), (12, 256), (12, 512), (12, 1024), (13, 256), (13, 512), (13, 1024)]


def gpu_sort_kp(keys, pay, tune=None):
    n = len(keys)
    cap = capi.next_pow2(n)
    k = capi.to_dev_u64(keys, cap)
    p = capi.to_dev_u32(pay, cap)
    capi.osort_kp(k, p, n, tune=tune)
    torch.cuda.synchronize()
    return capi.host_u64(k, cap), capi.host_u32(p, cap)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 32, 33, 100, 1000, 2047, 2048, 2049, 4096, 8191, 8192, 8193, 16384,
                               65537, 300_000])
def test_osort_kp_bit_exact(cuda, orc, n):
    keys, pay = W.sort_kp(n, seed=W.SEED_SORT + n)
    gk, gp = gpu_sort_kp(keys, pay)
    ok, op = orc.bitonic_kp(keys, pay)
    assert np.array_equal(gk, ok) and np.array_equal(gp, op)


def test_osort_kp_config0_full_size(cuda, orc):
    keys, pay = W.sort_kp()  # 2^20 rows, the plain-sort workload
    gk, gp = gpu_sort_kp(keys, pay)
    ok, op = orc.bitonic_kp(keys, pay)
    assert np.array_equal(gk, ok) and np.array_equal(gp, op)
    o = np.lexsort((pay, keys))
    assert np.array_equal(gk, keys[o]) and np.array_equal(gp, pay[o])


@pytest.mark.parametrize("tune", TUNES)
def test_osort_kp_all_tunes(cuda, orc, tune):
    for n in [5000, 70_000, 1 << 18]:
        keys, pay = W.sort_kp(n, seed=W.SEED_SORT ^ n)
        gk, gp = gpu_sort_kp(keys, pay, tune)
        ok, op = orc.bitonic_kp(keys, pay)
        assert np.array_equal(gk, ok) and np.array_equal(gp, op), (tune, n)


def test_osort_kp_ties_keep_network_arrangement(cuda, orc):
    rng = np.random.default_rng(1)
    for n in [777, 10_000, 1 << 17]:
        keys = rng.integers(0, 5, n).astype(np.uint64)
        pay = rng.integers(0, 3, n).astype(np.uint32)
        gk, gp = gpu_sort_kp(keys, pay)
        ok, op = orc.bitonic_kp(keys, pay)
        assert np.array_equal(gk, ok) and np.array_equal(gp, op)


@pytest.mark.parametrize("logn", [21, 22])
def test_osort_kp_three_cta_form_bit_exact(cuda, orc, logn):
    # from 2^21 rows the passes run in their three-CTA-per-SM form
    n = 1 << logn
    keys, pay = W.sort_kp(n, seed=W.SEED_SORT + logn)
    gk, gp = gpu_sort_kp(keys, pay)
    ok, op = orc.bitonic_kp(keys, pay)
    assert np.array_equal(gk, ok) and np.array_equal(gp, op)
    rng = np.random.default_rng(logn)
    keys = rng.integers(0, 5, n).astype(np.uint64)  # ties: the network's own arrangement
    pay = rng.integers(0, 3, n).astype(np.uint32)
    gk, gp = gpu_sort_kp(keys, pay)
    ok, op = orc.bitonic_kp(keys, pay)
    assert np.array_equal(gk, ok) and np.array_equal(gp, op)


def test_osort_kp_large_property(cuda):
    # 2^23 rows: beyond what the oracle does in seconds; check order + multiset
    n = 1 << 23
    keys, pay = W.sort_kp(n, seed=12345)
    gk, gp = gpu_sort_kp(keys, pay)
    assert np.all((gk[:-1] < gk[1:]) | ((gk[:-1] == gk[1:]) & (gp[:-1] <= gp[1:])))
    assert np.array_equal(np.sort(gp), np.sort(pay))
    assert np.bitwise_xor.reduce(gk) == np.bitwise_xor.reduce(keys)


# ---- ORCompact ---------------------------------------------------------------

def gpu_compact(keys, pay, marks, tune=None):
    n = len(keys)
    cap = capi.next_pow2(n)
    k = capi.to_dev_u64(keys, cap)
    p = capi.to_dev_u32(pay, cap)
    m = capi.to_dev_u8(marks, cap)
    cnt = capi.ocompact_kpm(k, p, m, n, tune=tune)
    torch.cuda.synchronize()
    return capi.host_u64(k, cap), capi.host_u32(p, cap), m.cpu().numpy(), int(cnt.item())


def oracle_compact_padded(orc, keys, pay, marks):
    """ORCompact restatement over the next_pow2(n) padded rows (pads are
    (UINT64_MAX, UINT32_MAX, unmarked), as the kernel pads them)."""
    n = len(keys)
    np_ = capi.next_pow2(n)
    rec = np.zeros((np_, 16), np.uint8)
    kk = np.full(np_, np.uint64(2**64 - 1))
    pp = np.full(np_, np.uint32(2**32 - 1))
    kk[:n] = keys
    pp[:n] = pay
    rec[:, :8] = kk.view(np.uint8).reshape(np_, 8)
    rec[:, 8:12] = pp.view(np.uint8).reshape(np_, 4)
    mm = np.zeros(np_, np.uint8)
    mm[:n] = marks
    d, m, cnt = orc.ocompact(rec, mm)
    return (np.ascontiguousarray(d[:, :8]).view(np.uint64).reshape(-1),
            np.ascontiguousarray(d[:, 8:12]).view(np.uint32).reshape(-1), m, cnt)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 100, 1000, 2048, 5000, 8192, 8193, 65536, 100_000, 1 << 19])
@pytest.mark.parametrize("density", [0.0, 0.3, 1.0])
def test_ocompact_bit_exact(cuda, orc, n, density):
    rng = np.random.default_rng(n)
    keys = W.splitmix64(77, n, 0)
    pay = np.arange(n, dtype=np.uint32)
    marks = (rng.random(n) < density).astype(np.uint8)
    gk, gp, gm, cnt = gpu_compact(keys, pay, marks)
    ok, op, om, ocnt = oracle_compact_padded(orc, keys, pay, marks)
    assert cnt == ocnt == int(marks.sum())
    assert np.array_equal(gk, ok) and np.array_equal(gp, op) and np.array_equal(gm, om)
    assert np.array_equal(gk[:cnt], keys[marks.astype(bool)])


@pytest.mark.parametrize("tune", [(11, 256), (12, 512), (13, 512), (13, 1024), (12, 1024)])
def test_ocompact_tunes(cuda, orc, tune):
    rng = np.random.default_rng(9)
    for n in [3000, 1 << 16, 300_001]:
        keys = W.splitmix64(78, n, 0)
        pay = np.arange(n, dtype=np.uint32)
        marks = (rng.random(n) < 0.3).astype(np.uint8)
        gk, gp, gm, cnt = gpu_compact(keys, pay, marks, tune)
        ok, op, om, ocnt = oracle_compact_padded(orc, keys, pay, marks)
        assert cnt == ocnt and np.array_equal(gk, ok) and np.array_equal(gp, op), tune


def test_ocompact_matches_liboblivious_golden(cuda):
    """The reference library's own outputs (o_compact over n rows, tests/golden):
    for power-of-two n the whole output is identical; otherwise the marked
    prefix (order-preserving) and the count are."""
    import importlib.util
    import os

    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(gold, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d = np.load(os.path.join(gold, "liboblivious_compact.npz"))
    off = np.concatenate([[0], np.cumsum(d["sizes"])])
    for case, n in enumerate(d["sizes"]):
        n = int(n)
        perm = d["perm"][off[case]:off[case + 1]].astype(np.int64)
        vals, marks = mg.compact_inputs(n, case)
        gk, gp, gm, cnt = gpu_compact(vals, np.arange(n, dtype=np.uint32), marks)
        assert cnt == int(marks.sum())
        assert np.array_equal(gp[:cnt].astype(np.int64), perm[:cnt])
        if n & (n - 1) == 0:
            assert np.array_equal(gp[:n].astype(np.int64), perm)


def test_ocompact_large_property(cuda):
    n = 6_001_215
    keys = W.splitmix64(5, n, 0)
    marks = (W.lemire(W.splitmix64(5, n, 1), 100) < 2).astype(np.uint8)
    gk, gp, gm, cnt = gpu_compact(keys, np.arange(n, dtype=np.uint32), marks)
    assert cnt == int(marks.sum())
    assert np.array_equal(gp[:cnt], np.nonzero(marks)[0].astype(np.uint32))
    assert not gm[cnt:].any()


# ---- reference OP_SORT contract (multi-column) --------------------------------

def test_sort_columns_matches_reference_network(cuda, orc):
    rng = np.random.default_rng(21)
    cases = [
        ([orc.INTEGER], [True]), ([orc.INTEGER], [False]), ([orc.BIGINT, orc.INTEGER], [True, False]),
        ([orc.BOOLEAN, orc.VARCHAR], [True, True]), ([orc.DOUBLE], [True]), ([orc.FLOAT, orc.SMALLINT], [False, True]),
        ([orc.DATE, orc.TINYINT, orc.BIGINT], [True, False, True]),
        ([orc.BIGINT, orc.BIGINT, orc.DOUBLE], [True, True, False]),
        ([orc.BIGINT] * 5, [True, False, True, False, True]),
    ]
    for types, asc in cases:
        for n in [1, 2, 5, 1000, 5000, 40_000]:
            cols = []
            for t in types:
                dt = orc.NP_OF_TYPE[t]
                if dt in (np.float32, np.float64):
                    c = rng.integers(-5, 5, n).astype(dt) * dt(0.5)
                else:
                    info = np.iinfo(dt)
                    c = rng.integers(max(info.min, -4), min(info.max, 4), n, endpoint=True).astype(dt)
                cols.append(c)
            ocols, oidx = orc.bitonic_sort_cols(cols, types, asc, n)
            np_ = capi.next_pow2(n)
            dcols = []
            for c in cols:
                t = torch.zeros(np_ * c.itemsize, dtype=torch.uint8, device=cuda)
                t[: c.nbytes].copy_(torch.from_numpy(c.view(np.uint8)))
                dcols.append(t)
            idx = capi.sort_columns(dcols, types, asc, n)
            torch.cuda.synchronize()
            assert np.array_equal(idx.cpu().numpy()[:np_], oidx[:np_]), (types, asc, n)
            for t, oc, c in zip(dcols, ocols, cols):
                got = t.cpu().numpy().view(c.dtype)[:np_]
                assert np.array_equal(got.view(np.uint8), oc[:np_].view(np.uint8)), (types, asc, n)


def test_sort_columns_order_by_known_answers(cuda, orc):
    from tests.test_oracle import order_by_cases

    for cols, types, asc, check in order_by_cases(orc):
        n = len(cols[0])
        np_ = capi.next_pow2(n)
        dcols = []
        for c in cols:
            c = np.asarray(c)
            t = torch.zeros(np_ * c.itemsize, dtype=torch.uint8, device=cuda)
            t[: c.nbytes].copy_(torch.from_numpy(c.view(np.uint8)))
            dcols.append(t)
        idx = capi.sort_columns(dcols, types, asc, n)
        torch.cuda.synchronize()
        outs = [t.cpu().numpy().view(np.asarray(c).dtype)[:n] for t, c in zip(dcols, cols)]
        assert check(outs, idx.cpu().numpy()[:n])
