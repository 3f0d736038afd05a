"""GPU tests of the serving layer: every query's result is identical when it
runs alone (one query at a time) and when it runs in the mix (continuous
admission, overlapping on the device); results match the oracle; admission
respects the HBM budget; waits are bounded."""
import numpy as np
import pytest

from velodb_b200 import serving as S, workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tables(cuda):
    return S.ServedTables(300_000, 60_000, 500_000, seed=77)


def test_results_identical_alone_and_in_the_mix(tables):
    qs = S.query_stream(tables, 40, seed=5, lo_log2=12, hi_log2=17)
    alone = S.Server(tables, slots=1, budget_bytes=2 << 30)
    ra, _ = S.run_closed_one_at_a_time(alone, qs)
    alone.close()
    mix = S.Server(tables, slots=8, budget_bytes=2 << 30)
    rm, _ = S.run_open_loop(mix, qs, np.zeros(len(qs)))  # all arrive at once
    st = mix.stats()
    mix.close()
    assert st["peak_inflight"] > 1  # queries really overlapped
    for a, m in zip(ra, rm):
        assert a.status == 0 and m.status == 0
        assert S.result_key(a) == S.result_key(m)


def test_persistent_queue_results_identical_alone_and_in_the_mix(tables):
    # the same stream served through one persistent command queue: every
    # query's result equals its result alone on the stream path
    qs = S.query_stream(tables, 40, seed=6, lo_log2=10, hi_log2=17)
    alone = S.Server(tables, slots=1, budget_bytes=2 << 30)
    ra, _ = S.run_closed_one_at_a_time(alone, qs)
    alone.close()
    mix = S.Server(tables, slots=16, budget_bytes=2 << 30, persistent=True)
    rm, _ = S.run_open_loop(mix, qs, np.zeros(len(qs)))
    st = mix.stats()
    mix.close()
    assert st["peak_inflight"] > 1
    for a, m in zip(ra, rm):
        assert a.status == 0 and m.status == 0
        assert S.result_key(a) == S.result_key(m)


def test_results_match_oracle(tables, orc):
    qs = [q for q in S.query_stream(tables, 12, seed=9, lo_log2=12, hi_log2=16)]
    srv = S.Server(tables, slots=4, budget_bytes=1 << 30)
    res, _ = S.run_open_loop(srv, qs, np.zeros(len(qs)))
    srv.close()
    fact = {k: v.cpu().numpy() for k, v in tables.fact.items()}
    fk = tables.fact_fk.cpu().numpy()
    dk = tables.dim_key.cpu().numpy()
    dd = tables.dim_date.cpu().numpy()
    f2fk = tables.fact2_fk.cpu().numpy()
    f2p = tables.fact2_price.cpu().numpy()
    for q, r in zip(qs, res):
        o, n = q.offset, q.n
        if q.shape == S.Q_FILTER_GROUPBY:
            cols = {k: v[o:o + n] for k, v in fact.items()}
            g, keys, sums = orc.filter_groupby(cols, W.LINEITEM_PRED, 8)
            out = np.asarray(r.out[:48]).reshape(8, 6)
            assert int(r.counts[1]) == g
            assert np.array_equal(out[:g, 0], keys.astype(np.int64)) and np.array_equal(out[:g, 1:], sums)
        elif q.shape == S.Q_JOIN_TOPK:
            dim = dict(key=dk[q.dim_offset:q.dim_offset + q.dim_n].astype(np.int32),
                       date=dd[q.dim_offset:q.dim_offset + q.dim_n])
            fct = dict(fk=fk[o:o + n].astype(np.int32), price=fact["price"][o:o + n])
            g, ofk, osum, ocnt = orc.join_groupby_topk(dim, fct, W.JOIN_PRED, 10)
            out = np.asarray(r.out[:30]).reshape(10, 3)
            m = min(g, 10)
            assert int(r.counts[1]) == g
            assert np.array_equal(out[:m, 0], ofk) and np.array_equal(out[:m, 1], osum)
        else:
            dsl = slice(q.dim_offset, q.dim_offset + q.dim_n)
            ok_keys = set(dk[dsl][dd[dsl] < W.JOIN_PRED["date_hi"]].tolist())
            fsl_fk, fsl_p = fk[o:o + n], fact["price"][o:o + n]
            ok_fact = set((np.nonzero((fsl_p < W.JOIN_PRED["price_hi"]) & np.isin(fsl_fk, list(ok_keys)))[0]
                           + o).tolist())
            f2 = f2fk[q.f2_offset:q.f2_offset + q.f2_n]
            hit = np.isin(f2, list(ok_fact))
            assert int(r.counts[0]) == int(hit.sum())
            assert int(r.out[0]) == int(f2p[q.f2_offset:q.f2_offset + q.f2_n][hit].sum())


def test_admission_respects_budget(tables):
    qs = S.query_stream(tables, 16, seed=11, lo_log2=15, hi_log2=17)
    budget = 160 << 20  # room for only a few queries at a time
    srv = S.Server(tables, slots=16, budget_bytes=budget)
    res, _ = S.run_open_loop(srv, qs, np.zeros(len(qs)))
    st = srv.stats()
    srv.close()
    assert all(r.status == 0 for r in res)
    assert st["peak_arena_bytes"] <= budget and st["completed"] == len(qs)


def test_oversized_query_is_rejected(tables):
    srv = S.Server(tables, slots=2, budget_bytes=1 << 20)
    q = S.query_stream(tables, 1, seed=1, lo_log2=17, hi_log2=17)[0]
    import velodb_b200

    with pytest.raises(velodb_b200.VeloError) as e:
        srv.submit(q)
    assert e.value.status == -2  # VELO_ENOMEM: larger than the whole budget
    srv.close()
