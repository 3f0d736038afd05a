// Tests of the C++ operator layer (include/velo_operator.hpp) on the device.
//
// Written after the behaviour the reference's own tests pin for these
// operators: ORDER BY directions, multi-column keys, mixed ASC/DESC and ties
// (tests/query/test_order_by.cpp), filter semantics (tests/query/test_filter*),
// join cardinality (tests/query/test_join_execution.cpp,
// tests/query/test_multi_join.cpp), materialization by row id
// (tests/operator/test_oblivious_materialization.cpp), LIMIT/OFFSET.  The
// expected results come from plain host code, and for the sort's arrangement
// of equal keys from the oracle's restatement of the reference network
// (oracle/oracle.h, linked by this test only).
//
//   operator_tests            run every test (needs a GPU)
//   operator_tests --list     print the test names
//   operator_tests --no-device  checks that need no GPU (context errors)
#include "velo_operator.hpp"

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <random>
#include <string>
#include <vector>

extern "C" {
#include "oracle.h"
}

using namespace velo_b200;

static int g_failures = 0;

#define EXPECT(cond)                                                                                                   \
    do {                                                                                                               \
        if (!(cond)) {                                                                                                 \
            std::fprintf(stderr, "  %s:%d: expectation failed: %s\n", __FILE__, __LINE__, #cond);                     \
            throw std::runtime_error("expectation failed");                                                            \
        }                                                                                                              \
    } while (0)

// an operator that replays prepared batches (the child of the tested operator)
class BatchSource : public UnaryOperator {
public:
    BatchSource(ExecutionContext& ctx, Schema s, std::vector<RowBatch> batches, bool fail = false)
        : UnaryOperator(ctx, std::move(s), nullptr)
        , batches_(std::move(batches))
        , fail_(fail)
    {
    }
    Result<RowBatch> next() override
    {
        if (fail_)
            return Result<RowBatch>::failure("source failed on purpose");
        if (i_ >= batches_.size())
            return Result<RowBatch>::success(RowBatch());
        return Result<RowBatch>::success(std::move(batches_[i_++]));
    }

private:
    std::vector<RowBatch> batches_;
    size_t i_ = 0;
    bool fail_;
};

static std::vector<RowBatch> drain(AbstractOperator& op)
{
    std::vector<RowBatch> out;
    for (;;) {
        Result<RowBatch> r = op.next();
        if (!r)
            throw std::runtime_error("operator failed: " + r.error());
        RowBatch b = std::move(r).value();
        if (b.getRowCount() == 0)
            return out;
        out.push_back(std::move(b));
    }
}

template <class T>
static std::vector<T> col_host(ExecutionContext& ctx, std::vector<RowBatch>& bs, size_t c)
{
    std::vector<T> out;
    for (auto& b : bs) {
        auto v = b.getColumn(c).toHost<T>(ctx);
        out.insert(out.end(), v.begin(), v.end());
    }
    return out;
}

static std::vector<uint8_t> valid_host(ExecutionContext& ctx, std::vector<RowBatch>& bs, size_t c)
{
    std::vector<uint8_t> out;
    for (auto& b : bs) {
        auto v = b.getColumn(c).validityToHost(ctx);
        out.insert(out.end(), v.begin(), v.end());
    }
    return out;
}

static Schema schema_of(std::vector<std::pair<std::string, DataTypeId>> cols)
{
    std::vector<ColumnInfo> v;
    for (auto& c : cols)
        v.push_back({ c.first, c.second });
    return Schema(std::move(v));
}

// ---- ORDER BY ----------------------------------------------------------------

// sorts through SortOperator and checks key columns and the permutation of
// every other column against the oracle network (reference tie order)
static void check_sort(ExecutionContext& ctx, const std::vector<int32_t>& a, const std::vector<int64_t>& b,
                       std::vector<size_t> order, std::vector<bool> asc, size_t split = 0)
{
    const size_t n = a.size();
    std::vector<int64_t> rowid(n);
    for (size_t i = 0; i < n; i++)
        rowid[i] = (int64_t)i;
    Schema s = schema_of({ { "t.a", VELO_INTEGER }, { "t.b", VELO_BIGINT }, { "t.id", VELO_BIGINT } });
    std::vector<RowBatch> in;
    // one batch, or two (exercises collectBatches)
    auto make = [&](size_t lo, size_t hi) {
        std::vector<int32_t> a2(a.begin() + lo, a.begin() + hi);
        std::vector<int64_t> b2(b.begin() + lo, b.begin() + hi), r2(rowid.begin() + lo, rowid.begin() + hi);
        RowBatch rb;
        rb.addColumn(Column::fromHost(ctx, VELO_INTEGER, a2));
        rb.addColumn(Column::fromHost(ctx, VELO_BIGINT, b2));
        rb.addColumn(Column::fromHost(ctx, VELO_BIGINT, r2));
        return rb;
    };
    if (split && split < n) {
        in.push_back(make(0, split));
        in.push_back(make(split, n));
    } else {
        in.push_back(make(0, n));
    }
    auto src = std::make_unique<BatchSource>(ctx, s, std::move(in));
    SortOperator op(ctx, s, std::move(src), order, asc);
    auto out = drain(op);
    auto ga = col_host<int32_t>(ctx, out, 0);
    auto gb = col_host<int64_t>(ctx, out, 1);
    auto gid = col_host<int64_t>(ctx, out, 2);
    EXPECT(ga.size() == n);

    // oracle: the reference network over the key columns
    const size_t np = orc_next_pow2(n);
    std::vector<int32_t> oa(np);
    std::vector<int64_t> ob(np), idx(np);
    std::copy(a.begin(), a.end(), oa.begin());
    std::copy(b.begin(), b.end(), ob.begin());
    std::vector<void*> cols;
    std::vector<int> types;
    std::vector<uint8_t> ascv;
    for (size_t k = 0; k < order.size(); k++) {
        cols.push_back(order[k] == 0 ? (void*)oa.data() : (void*)ob.data());
        types.push_back(order[k] == 0 ? VELO_INTEGER : VELO_BIGINT);
        ascv.push_back(asc[k] ? 1 : 0);
    }
    EXPECT(orc_bitonic_sort_cols((int)cols.size(), cols.data(), types.data(), ascv.data(), n, np, idx.data()) == 0);
    for (size_t i = 0; i < n; i++) {
        EXPECT(gid[i] == idx[i]);
        EXPECT(ga[i] == a[(size_t)idx[i]]);
        EXPECT(gb[i] == b[(size_t)idx[i]]);
    }
}

static void test_order_by_single_column(ExecutionContext& ctx)
{
    std::mt19937_64 rng(1);
    std::vector<int32_t> a(5000);
    std::vector<int64_t> b(5000);
    for (auto& x : a)
        x = (int32_t)(rng() % 100000) - 50000;
    for (auto& x : b)
        x = (int64_t)rng();
    check_sort(ctx, a, b, { 0 }, { true });
    check_sort(ctx, a, b, { 0 }, { false });
    check_sort(ctx, a, b, { 1 }, { true }, 1234);
}

static void test_order_by_mixed_directions_and_ties(ExecutionContext& ctx)
{
    std::mt19937_64 rng(2);
    std::vector<int32_t> a(3001);
    std::vector<int64_t> b(3001);
    for (auto& x : a)
        x = (int32_t)(rng() % 7);
    for (auto& x : b)
        x = (int64_t)(rng() % 5) - 2;
    check_sort(ctx, a, b, { 0, 1 }, { true, false });
    check_sort(ctx, a, b, { 1, 0 }, { false, true }, 1000);
    check_sort(ctx, a, b, { 0 }, { true }); // ties: network arrangement
}

static void test_order_by_known_answer(ExecutionContext& ctx)
{
    // ORDER BY dept ASC, salary DESC on a small table
    std::vector<int32_t> dept = { 3, 1, 2, 1, 3, 2, 1 };
    std::vector<int64_t> salary = { 50, 70, 65, 90, 40, 65, 60 };
    check_sort(ctx, dept, salary, { 0, 1 }, { true, false });
    Schema s = schema_of({ { "dept", VELO_INTEGER }, { "salary", VELO_BIGINT } });
    RowBatch rb;
    rb.addColumn(Column::fromHost(ctx, VELO_INTEGER, dept));
    rb.addColumn(Column::fromHost(ctx, VELO_BIGINT, salary));
    std::vector<RowBatch> in;
    in.push_back(std::move(rb));
    SortOperator op(ctx, s, std::make_unique<BatchSource>(ctx, s, std::move(in)), { 0, 1 }, { true, false });
    auto out = drain(op);
    auto d = col_host<int32_t>(ctx, out, 0);
    auto sal = col_host<int64_t>(ctx, out, 1);
    EXPECT((d == std::vector<int32_t> { 1, 1, 1, 2, 2, 3, 3 }));
    EXPECT((sal == std::vector<int64_t> { 90, 70, 60, 65, 65, 50, 40 }));
}

static void test_sort_carries_nulls(ExecutionContext& ctx)
{
    std::vector<int32_t> k = { 5, 1, 4, 2, 3 };
    std::vector<int64_t> v = { 50, 10, 40, 20, 30 };
    std::vector<uint8_t> valid = { 1, 0, 1, 1, 0 };
    Schema s = schema_of({ { "k", VELO_INTEGER }, { "v", VELO_BIGINT } });
    RowBatch rb;
    rb.addColumn(Column::fromHost(ctx, VELO_INTEGER, k));
    rb.addColumn(Column::fromHost(ctx, VELO_BIGINT, v, &valid));
    std::vector<RowBatch> in;
    in.push_back(std::move(rb));
    SortOperator op(ctx, s, std::make_unique<BatchSource>(ctx, s, std::move(in)), { 0 }, { true });
    auto out = drain(op);
    EXPECT((col_host<int64_t>(ctx, out, 1) == std::vector<int64_t> { 10, 20, 30, 40, 50 }));
    EXPECT((valid_host(ctx, out, 1) == std::vector<uint8_t> { 0, 1, 0, 1, 1 }));
}

static void test_sort_empty_input(ExecutionContext& ctx)
{
    Schema s = schema_of({ { "k", VELO_INTEGER } });
    SortOperator op(ctx, s, std::make_unique<BatchSource>(ctx, s, std::vector<RowBatch> {}), { 0 }, { true });
    EXPECT(drain(op).empty());
}

// ---- scan + filter compaction --------------------------------------------------

static Table make_table(ExecutionContext& ctx, size_t n, uint64_t seed, std::vector<int32_t>& a,
                        std::vector<int64_t>& b, std::vector<uint32_t>& d)
{
    std::mt19937_64 rng(seed);
    a.resize(n);
    b.resize(n);
    d.resize(n);
    for (size_t i = 0; i < n; i++) {
        a[i] = (int32_t)(rng() % 1000);
        b[i] = (int64_t)(rng() % 2000000) - 1000000;
        d[i] = (uint32_t)(rng() % 2557);
    }
    Table t;
    t.schema = schema_of({ { "t.a", VELO_INTEGER }, { "t.b", VELO_BIGINT }, { "t.d", VELO_DATE } });
    t.columns.push_back(Column::fromHost(ctx, VELO_INTEGER, a));
    t.columns.push_back(Column::fromHost(ctx, VELO_BIGINT, b));
    t.columns.push_back(Column::fromHost(ctx, VELO_DATE, d));
    t.rows = n;
    return t;
}

static Schema scan_schema()
{
    return schema_of({ { "t.a", VELO_INTEGER }, { "t.b", VELO_BIGINT }, { "t.d", VELO_DATE },
                       { "t.$_rowid", VELO_BIGINT }, { "t.$_mask", VELO_BOOLEAN } });
}

static void test_scan_filter_compaction(ExecutionContext& ctx)
{
    for (size_t n : { (size_t)1, (size_t)777, (size_t)4096, (size_t)100003 }) {
        std::vector<int32_t> a;
        std::vector<int64_t> b;
        std::vector<uint32_t> d;
        Table t = make_table(ctx, n, 10 + n, a, b, d);
        std::vector<RangePredicate> pred = { { 0, 100, 499 }, { 2, 0, 1277 } };
        auto scan = std::make_unique<SeqScanOperator>(ctx, t, scan_schema(), pred);
        FilterCompactionOperator op(ctx, scan_schema(), std::move(scan));
        auto out = drain(op);
        std::vector<int32_t> ea;
        std::vector<int64_t> eb, eid;
        for (size_t i = 0; i < n; i++)
            if (a[i] >= 100 && a[i] <= 499 && d[i] <= 1277) {
                ea.push_back(a[i]);
                eb.push_back(b[i]);
                eid.push_back((int64_t)i);
            }
        EXPECT(col_host<int32_t>(ctx, out, 0) == ea);
        EXPECT(col_host<int64_t>(ctx, out, 1) == eb);
        EXPECT(col_host<int64_t>(ctx, out, 3) == eid);
        auto m = col_host<uint8_t>(ctx, out, 4);
        EXPECT(std::all_of(m.begin(), m.end(), [](uint8_t x) { return x == 1; }));
    }
}

static void test_filter_nothing_and_everything(ExecutionContext& ctx)
{
    std::vector<int32_t> a;
    std::vector<int64_t> b;
    std::vector<uint32_t> d;
    Table t = make_table(ctx, 5000, 3, a, b, d);
    {
        auto scan = std::make_unique<SeqScanOperator>(ctx, t, scan_schema(),
                                                      std::vector<RangePredicate> { { 0, 2000, 3000 } });
        FilterCompactionOperator op(ctx, scan_schema(), std::move(scan));
        auto r = op.next();
        EXPECT((bool)r && r.value().getRowCount() == 0); // empty batch: end of stream
    }
    {
        auto scan = std::make_unique<SeqScanOperator>(ctx, t, scan_schema());
        FilterCompactionOperator op(ctx, scan_schema(), std::move(scan));
        auto out = drain(op);
        EXPECT(col_host<int32_t>(ctx, out, 0) == a);
    }
}

static void test_filter_keeps_nulls_and_uncompacted_columns(ExecutionContext& ctx)
{
    std::vector<int32_t> a = { 1, 2, 3, 4, 5, 6 };
    std::vector<int16_t> c = { 10, 20, 30, 40, 50, 60 };
    std::vector<uint8_t> valid = { 1, 0, 1, 0, 1, 0 };
    std::vector<uint8_t> mask = { 0, 1, 1, 0, 0, 1 };
    Schema s = schema_of({ { "a", VELO_INTEGER }, { "c", VELO_SMALLINT }, { "$_mask", VELO_BOOLEAN } });
    RowBatch rb;
    rb.addColumn(Column::fromHost(ctx, VELO_INTEGER, a, &valid));
    rb.addColumn(Column::fromHost(ctx, VELO_SMALLINT, c));
    rb.addColumn(Column::fromHost(ctx, VELO_BOOLEAN, mask));
    std::vector<RowBatch> in;
    in.push_back(std::move(rb));
    FilterCompactionOperator op(ctx, s, std::make_unique<BatchSource>(ctx, s, std::move(in)), { true, false, true });
    auto r = op.next();
    EXPECT((bool)r);
    RowBatch& b = r.value();
    EXPECT(b.getRowCount() == 3);
    EXPECT((b.getColumn(0).toHost<int32_t>(ctx) == std::vector<int32_t> { 2, 3, 6 }));
    EXPECT((b.getColumn(0).validityToHost(ctx) == std::vector<uint8_t> { 0, 1, 0 }));
    EXPECT((b.getColumn(1).toHost<int16_t>(ctx) == std::vector<int16_t> { 10, 20, 30 })); // not compacted
}

static void test_filter_propagates_child_failure(ExecutionContext& ctx)
{
    Schema s = schema_of({ { "$_mask", VELO_BOOLEAN } });
    FilterCompactionOperator op(ctx, s, std::make_unique<BatchSource>(ctx, s, std::vector<RowBatch> {}, true));
    auto r = op.next();
    EXPECT(!r && r.error() == "source failed on purpose");
    SortOperator so(ctx, s, std::make_unique<BatchSource>(ctx, s, std::vector<RowBatch> {}, true), { 0 }, { true });
    bool threw = false;
    try {
        so.next();
    } catch (const ExecutionError&) {
        threw = true;
    }
    EXPECT(threw);
}

// ---- joins -----------------------------------------------------------------------

struct JoinInput {
    std::vector<int32_t> dkey, ddate;
    std::vector<int32_t> ffk;
    std::vector<int64_t> fprice;
};

static JoinInput make_join(size_t nd, size_t nf, uint64_t seed)
{
    std::mt19937_64 rng(seed);
    JoinInput j;
    j.dkey.resize(nd);
    for (size_t i = 0; i < nd; i++)
        j.dkey[i] = (int32_t)(i * 3 + 1);
    std::shuffle(j.dkey.begin(), j.dkey.end(), rng);
    j.ddate.resize(nd);
    for (auto& x : j.ddate)
        x = (int32_t)(rng() % 2557);
    j.ffk.resize(nf);
    j.fprice.resize(nf);
    for (size_t i = 0; i < nf; i++) {
        j.ffk[i] = (int32_t)(rng() % (3 * nd + 5)); // some match no dimension key
        j.fprice[i] = (int64_t)(rng() % 10000000);
    }
    return j;
}

static void run_join_test(ExecutionContext& ctx, bool hash, size_t nd, size_t nf, uint64_t seed)
{
    JoinInput j = make_join(nd, nf, seed);
    Schema ls = schema_of({ { "d.key", VELO_INTEGER }, { "d.date", VELO_INTEGER }, { "d.$_mask", VELO_BOOLEAN } });
    Schema rs = schema_of({ { "f.fk", VELO_INTEGER }, { "f.price", VELO_BIGINT }, { "f.$_mask", VELO_BOOLEAN } });
    std::vector<uint8_t> dm(nd), fm(nf);
    for (size_t i = 0; i < nd; i++)
        dm[i] = j.ddate[i] < 1278;
    for (size_t i = 0; i < nf; i++)
        fm[i] = j.fprice[i] < 5000000;
    RowBatch lb, rb;
    lb.addColumn(Column::fromHost(ctx, VELO_INTEGER, j.dkey));
    lb.addColumn(Column::fromHost(ctx, VELO_INTEGER, j.ddate));
    lb.addColumn(Column::fromHost(ctx, VELO_BOOLEAN, dm));
    rb.addColumn(Column::fromHost(ctx, VELO_INTEGER, j.ffk));
    rb.addColumn(Column::fromHost(ctx, VELO_BIGINT, j.fprice));
    rb.addColumn(Column::fromHost(ctx, VELO_BOOLEAN, fm));
    std::vector<RowBatch> li, ri;
    li.push_back(std::move(lb));
    ri.push_back(std::move(rb));
    Schema os = schema_of({ { "d.key", VELO_INTEGER }, { "d.date", VELO_INTEGER }, { "d.$_mask", VELO_BOOLEAN },
                            { "f.fk", VELO_INTEGER }, { "f.price", VELO_BIGINT }, { "f.$_mask", VELO_BOOLEAN } });
    std::unique_ptr<AbstractOperator> op;
    auto L = std::make_unique<BatchSource>(ctx, ls, std::move(li));
    auto R = std::make_unique<BatchSource>(ctx, rs, std::move(ri));
    if (hash)
        op = std::make_unique<HashJoinOperator>(ctx, os, std::move(L), std::move(R), std::make_pair(0ul, 0ul),
                                                std::make_pair(2l, 2l));
    else
        op = std::make_unique<SortMergeJoinOperator>(ctx, os, std::move(L), std::move(R), std::make_pair(0ul, 0ul));
    auto out = drain(*op);
    // expected: for each fact row whose fk has a dimension row (and both masks
    // pass for the hash join), one pair; output in key order
    std::map<int32_t, size_t> dim_of;
    for (size_t i = 0; i < nd; i++)
        dim_of[j.dkey[i]] = i;
    std::multiset<std::pair<int32_t, int64_t>> expect;
    for (size_t i = 0; i < nf; i++) {
        auto it = dim_of.find(j.ffk[i]);
        if (it == dim_of.end())
            continue;
        if (hash && (!dm[it->second] || !fm[i]))
            continue;
        expect.insert({ j.ffk[i], j.fprice[i] });
    }
    auto gk = col_host<int32_t>(ctx, out, 0);
    auto gdate = col_host<int32_t>(ctx, out, 1);
    auto gfk = col_host<int32_t>(ctx, out, 3);
    auto gp = col_host<int64_t>(ctx, out, 4);
    EXPECT(gk.size() == expect.size());
    std::multiset<std::pair<int32_t, int64_t>> got;
    for (size_t i = 0; i < gk.size(); i++) {
        EXPECT(gk[i] == gfk[i]);
        EXPECT(gdate[i] == j.ddate[dim_of[gk[i]]]);
        // the sort-merge join emits key order; the hash join bin order
        if (i && !hash)
            EXPECT(gk[i - 1] <= gk[i]);
        got.insert({ gfk[i], gp[i] });
    }
    EXPECT(got == expect);
}

static void test_sort_merge_join_cardinality(ExecutionContext& ctx)
{
    run_join_test(ctx, false, 1, 1, 1);
    run_join_test(ctx, false, 1000, 5000, 2);
    run_join_test(ctx, false, 30000, 120000, 3);
}

static void test_hash_join_with_masks(ExecutionContext& ctx)
{
    run_join_test(ctx, true, 1000, 5000, 4);
    run_join_test(ctx, true, 20000, 70001, 5);
}

// repeated build keys: every pair, as the reference's sort-merge join writes
// the cross product of each run of equal keys
static void run_many_to_many(ExecutionContext& ctx, bool hash)
{
    Schema s = schema_of({ { "k", VELO_INTEGER }, { "v", VELO_BIGINT } });
    std::vector<int32_t> lk, rk;
    std::vector<int64_t> lv, rv;
    std::mt19937_64 rng(hash ? 11 : 12);
    for (int i = 0; i < 3000; i++) {
        lk.push_back((int32_t)(rng() % 400));
        lv.push_back(i);
    }
    for (int i = 0; i < 5000; i++) {
        rk.push_back((int32_t)(rng() % 400));
        rv.push_back(100000 + i);
    }
    RowBatch lb, rb;
    lb.addColumn(Column::fromHost(ctx, VELO_INTEGER, lk));
    lb.addColumn(Column::fromHost(ctx, VELO_BIGINT, lv));
    rb.addColumn(Column::fromHost(ctx, VELO_INTEGER, rk));
    rb.addColumn(Column::fromHost(ctx, VELO_BIGINT, rv));
    std::vector<RowBatch> li, ri;
    li.push_back(std::move(lb));
    ri.push_back(std::move(rb));
    Schema os = schema_of({ { "l.k", VELO_INTEGER }, { "l.v", VELO_BIGINT }, { "r.k", VELO_INTEGER },
                            { "r.v", VELO_BIGINT } });
    std::unique_ptr<AbstractOperator> op;
    auto L = std::make_unique<BatchSource>(ctx, s, std::move(li));
    auto R = std::make_unique<BatchSource>(ctx, s, std::move(ri));
    if (hash)
        op = std::make_unique<HashJoinOperator>(ctx, os, std::move(L), std::move(R), std::make_pair(0ul, 0ul),
                                                std::make_pair(-1l, -1l));
    else
        op = std::make_unique<SortMergeJoinOperator>(ctx, os, std::move(L), std::move(R), std::make_pair(0ul, 0ul));
    auto out = drain(*op);
    std::multiset<std::pair<int64_t, int64_t>> expect, got;
    for (size_t a = 0; a < lk.size(); a++)
        for (size_t b = 0; b < rk.size(); b++)
            if (lk[a] == rk[b])
                expect.insert({ lv[a], rv[b] });
    auto gl = col_host<int64_t>(ctx, out, 1);
    auto gr = col_host<int64_t>(ctx, out, 3);
    auto gkl = col_host<int32_t>(ctx, out, 0);
    auto gkr = col_host<int32_t>(ctx, out, 2);
    EXPECT(gl.size() == expect.size());
    for (size_t i = 0; i < gl.size(); i++) {
        EXPECT(gkl[i] == gkr[i]);
        got.insert({ gl[i], gr[i] });
    }
    EXPECT(got == expect);
}

static void test_join_many_to_many(ExecutionContext& ctx)
{
    run_many_to_many(ctx, false);
    run_many_to_many(ctx, true);
}

static void test_join_empty_side(ExecutionContext& ctx)
{
    Schema s = schema_of({ { "k", VELO_INTEGER } });
    RowBatch rb;
    rb.addColumn(Column::fromHost(ctx, VELO_INTEGER, std::vector<int32_t> { 2, 1 }));
    std::vector<RowBatch> ri;
    ri.push_back(std::move(rb));
    SortMergeJoinOperator op(ctx, schema_of({ { "l.k", VELO_INTEGER }, { "r.k", VELO_INTEGER } }),
                             std::make_unique<BatchSource>(ctx, s, std::vector<RowBatch> {}),
                             std::make_unique<BatchSource>(ctx, s, std::move(ri)), { 0, 0 });
    EXPECT(drain(op).empty());
}

// ---- materialization + limit ------------------------------------------------------------

static void test_materialization(ExecutionContext& ctx)
{
    std::vector<int32_t> a;
    std::vector<int64_t> b;
    std::vector<uint32_t> d;
    Table t = make_table(ctx, 10000, 77, a, b, d);
    std::vector<uint8_t> bvalid(10000);
    for (size_t i = 0; i < 10000; i++)
        bvalid[i] = (i % 7) != 0;
    t.columns[1] = Column::fromHost(ctx, VELO_BIGINT, b, &bvalid);
    std::mt19937_64 rng(8);
    std::vector<int64_t> rid(3001);
    for (auto& r : rid)
        r = (int64_t)(rng() % 10020) - 10; // some below 0, some >= rows
    rid[0] = rid[1] = 42;                  // duplicates
    Schema s = schema_of({ { "x.$_rowid", VELO_BIGINT } });
    RowBatch rb;
    rb.addColumn(Column::fromHost(ctx, VELO_BIGINT, rid));
    std::vector<RowBatch> in;
    in.push_back(std::move(rb));
    MaterializationOperator op(
        ctx, schema_of({ { "t.a", VELO_INTEGER }, { "t.b", VELO_BIGINT }, { "t.d", VELO_DATE } }),
        std::make_unique<BatchSource>(ctx, s, std::move(in)),
        { { 0, &t, 0 }, { 0, &t, 1 }, { 0, &t, 2 } });
    auto out = drain(op);
    auto ga = col_host<int32_t>(ctx, out, 0);
    auto gb = col_host<int64_t>(ctx, out, 1);
    auto gd = col_host<uint32_t>(ctx, out, 2);
    auto va = valid_host(ctx, out, 0);
    auto vb = valid_host(ctx, out, 1);
    EXPECT(ga.size() == rid.size());
    for (size_t i = 0; i < rid.size(); i++) {
        const bool in_range = rid[i] >= 0 && rid[i] < 10000;
        if (in_range) {
            EXPECT(ga[i] == a[(size_t)rid[i]] && gd[i] == d[(size_t)rid[i]] && va[i] == 1);
            EXPECT(vb[i] == bvalid[(size_t)rid[i]]);
            if (vb[i])
                EXPECT(gb[i] == b[(size_t)rid[i]]);
        } else {
            EXPECT(va[i] == 0 && vb[i] == 0);
        }
    }
}

static void test_limit_offset(ExecutionContext& ctx)
{
    Schema s = schema_of({ { "k", VELO_INTEGER } });
    std::vector<RowBatch> in;
    for (int b = 0; b < 3; b++) {
        std::vector<int32_t> v(10);
        for (int i = 0; i < 10; i++)
            v[i] = b * 10 + i;
        RowBatch rb;
        rb.addColumn(Column::fromHost(ctx, VELO_INTEGER, v));
        in.push_back(std::move(rb));
    }
    LimitOperator op(ctx, s, std::make_unique<BatchSource>(ctx, s, std::move(in)), 12, 15);
    auto out = drain(op);
    std::vector<int32_t> e;
    for (int i = 15; i < 27; i++)
        e.push_back(i);
    EXPECT(col_host<int32_t>(ctx, out, 0) == e);
}

// ---- plan: scan -> filter -> sort -> limit ---------------------------------------------------

static void test_plan_scan_filter_sort_limit(ExecutionContext& ctx)
{
    std::vector<int32_t> a;
    std::vector<int64_t> b;
    std::vector<uint32_t> d;
    Table t = make_table(ctx, 50000, 99, a, b, d);
    auto scan = std::make_unique<SeqScanOperator>(ctx, t, scan_schema(),
                                                  std::vector<RangePredicate> { { 2, 100, 900 } });
    auto filt = std::make_unique<FilterCompactionOperator>(ctx, scan_schema(), std::move(scan));
    auto sort = std::make_unique<SortOperator>(ctx, scan_schema(), std::move(filt), std::vector<size_t> { 1, 3 },
                                               std::vector<bool> { false, true });
    LimitOperator lim(ctx, scan_schema(), std::move(sort), 100);
    auto out = drain(lim);
    std::vector<std::pair<int64_t, int64_t>> rows;
    for (size_t i = 0; i < a.size(); i++)
        if (d[i] >= 100 && d[i] <= 900)
            rows.push_back({ -b[i], (int64_t)i });
    std::sort(rows.begin(), rows.end());
    auto gb = col_host<int64_t>(ctx, out, 1);
    auto gid = col_host<int64_t>(ctx, out, 3);
    EXPECT(gb.size() == 100);
    for (size_t i = 0; i < 100; i++)
        EXPECT(gb[i] == -rows[i].first && gid[i] == rows[i].second);
}

// ---- aggregate ------------------------------------------------------------------------------

static void test_aggregate_sum_count_with_mask(ExecutionContext& ctx)
{
    std::vector<int32_t> a;
    std::vector<int64_t> b;
    std::vector<uint32_t> d;
    Table t = make_table(ctx, 60000, 31, a, b, d);
    // GROUP BY a with SUM(b), COUNT(*), SUM(d) over the rows the scan's
    // predicate keeps ($_mask), three aggregates (two calls underneath)
    auto scan = std::make_unique<SeqScanOperator>(ctx, t, scan_schema(),
                                                  std::vector<RangePredicate> { { 2, 0, 1999 } });
    Schema os = schema_of({ { "a", VELO_BIGINT }, { "sum_b", VELO_BIGINT }, { "cnt", VELO_BIGINT },
                            { "sum_d", VELO_BIGINT } });
    AggregateOperator op(ctx, os, std::move(scan), 0,
                         { { AggKind::SUM, 1 }, { AggKind::COUNT, 0 }, { AggKind::SUM, 2 } });
    auto out = drain(op);
    std::map<int32_t, std::array<int64_t, 3>> e;
    for (size_t i = 0; i < a.size(); i++)
        if (d[i] <= 1999) {
            auto& x = e[a[i]];
            x[0] += b[i];
            x[1] += 1;
            x[2] += d[i];
        }
    auto gk = col_host<int64_t>(ctx, out, 0);
    auto s0 = col_host<int64_t>(ctx, out, 1);
    auto c = col_host<int64_t>(ctx, out, 2);
    auto s1 = col_host<int64_t>(ctx, out, 3);
    EXPECT(gk.size() == e.size());
    size_t i = 0;
    for (auto& kv : e) {
        EXPECT(gk[i] == kv.first && s0[i] == kv.second[0] && c[i] == kv.second[1] && s1[i] == kv.second[2]);
        i++;
    }
}

static void test_aggregate_bound_and_bigint_keys(ExecutionContext& ctx)
{
    std::vector<int64_t> k(5000), v(5000);
    std::mt19937_64 rng(6);
    for (size_t i = 0; i < k.size(); i++) {
        k[i] = (int64_t)(rng() % 400) - 200;
        v[i] = (int64_t)(rng() % 1000);
    }
    Schema s = schema_of({ { "k", VELO_BIGINT }, { "v", VELO_BIGINT } });
    RowBatch rb;
    rb.addColumn(Column::fromHost(ctx, VELO_BIGINT, k));
    rb.addColumn(Column::fromHost(ctx, VELO_BIGINT, v));
    std::vector<RowBatch> in;
    in.push_back(std::move(rb));
    AggregateOperator op(ctx, schema_of({ { "k", VELO_BIGINT }, { "s", VELO_BIGINT } }),
                         std::make_unique<BatchSource>(ctx, s, std::move(in)), 0, { { AggKind::SUM, 1 } }, 10);
    auto out = drain(op);
    std::map<int64_t, int64_t> e;
    for (size_t i = 0; i < k.size(); i++)
        e[k[i]] += v[i];
    auto gk = col_host<int64_t>(ctx, out, 0);
    auto gs = col_host<int64_t>(ctx, out, 1);
    EXPECT(gk.size() == 10);
    auto it = e.begin();
    for (size_t i = 0; i < 10; i++, ++it)
        EXPECT(gk[i] == it->first && gs[i] == it->second);
}

static void test_execution_engine_runs_a_plan(ExecutionContext& ctx)
{
    std::vector<int32_t> a;
    std::vector<int64_t> b;
    std::vector<uint32_t> d;
    Table t = make_table(ctx, 20000, 55, a, b, d);
    // SELECT a, SUM(b), COUNT(*) FROM t WHERE d <= 999 GROUP BY a
    auto scan = std::make_unique<SeqScanOperator>(ctx, t, scan_schema(),
                                                  std::vector<RangePredicate> { { 2, 0, 999 } });
    auto filt = std::make_unique<FilterCompactionOperator>(ctx, scan_schema(), std::move(scan));
    auto agg = std::make_unique<AggregateOperator>(
        ctx, schema_of({ { "a", VELO_BIGINT }, { "s", VELO_BIGINT }, { "c", VELO_BIGINT } }), std::move(filt), 0,
        std::vector<AggregateSpec> { { AggKind::SUM, 1 }, { AggKind::COUNT, 0 } });
    ExecutionEngine engine(ctx);
    auto r = engine.executePlan(std::move(agg));
    EXPECT((bool)r);
    QueryResult& q = r.value();
    std::map<int32_t, std::pair<int64_t, int64_t>> e;
    for (size_t i = 0; i < a.size(); i++)
        if (d[i] <= 999) {
            e[a[i]].first += b[i];
            e[a[i]].second += 1;
        }
    EXPECT(q.getRowCount() == e.size() && engine.getLastExecutionRowCount() == e.size());
    EXPECT(q.schema.getColumnCount() == 3 && engine.getLastExecutionTimeMs() > 0.0);
    auto gk = col_host<int64_t>(ctx, q.batches, 0);
    auto gs = col_host<int64_t>(ctx, q.batches, 1);
    auto gc = col_host<int64_t>(ctx, q.batches, 2);
    size_t i = 0;
    for (auto& kv : e) {
        EXPECT(gk[i] == kv.first && gs[i] == kv.second.first && gc[i] == kv.second.second);
        i++;
    }
    EXPECT(!engine.executePlan(nullptr));
}

// ------------------------------------------------------------------------------------------

struct TestCase {
    const char* name;
    std::function<void(ExecutionContext&)> fn;
};

int main(int argc, char** argv)
{
    std::vector<TestCase> tests = {
        { "order_by_single_column", test_order_by_single_column },
        { "order_by_mixed_directions_and_ties", test_order_by_mixed_directions_and_ties },
        { "order_by_known_answer", test_order_by_known_answer },
        { "sort_carries_nulls", test_sort_carries_nulls },
        { "sort_empty_input", test_sort_empty_input },
        { "scan_filter_compaction", test_scan_filter_compaction },
        { "filter_nothing_and_everything", test_filter_nothing_and_everything },
        { "filter_keeps_nulls_and_uncompacted_columns", test_filter_keeps_nulls_and_uncompacted_columns },
        { "filter_propagates_child_failure", test_filter_propagates_child_failure },
        { "sort_merge_join_cardinality", test_sort_merge_join_cardinality },
        { "hash_join_with_masks", test_hash_join_with_masks },
        { "join_many_to_many", test_join_many_to_many },
        { "join_empty_side", test_join_empty_side },
        { "materialization", test_materialization },
        { "limit_offset", test_limit_offset },
        { "plan_scan_filter_sort_limit", test_plan_scan_filter_sort_limit },
        { "aggregate_sum_count_with_mask", test_aggregate_sum_count_with_mask },
        { "aggregate_bound_and_bigint_keys", test_aggregate_bound_and_bigint_keys },
        { "execution_engine_runs_a_plan", test_execution_engine_runs_a_plan },
    };
    if (argc > 1 && std::strcmp(argv[1], "--list") == 0) {
        for (auto& t : tests)
            std::printf("%s\n", t.name);
        return 0;
    }
    if (argc > 1 && std::strcmp(argv[1], "--no-device") == 0) {
        // without a GPU the context cannot be created: an ExecutionError, no crash
        try {
            ExecutionContext ctx(0);
            std::printf("device present\n");
        } catch (const ExecutionError& e) {
            std::printf("ok no_device_context_error: %s\n", e.what());
        }
        Schema s = schema_of({ { "t.a", VELO_INTEGER }, { "t.$_mask", VELO_BOOLEAN } });
        EXPECT(s.getColumnIndex("$_mask") == 1 && s.getColumnIndex("t.a") == 0 && !s.hasColumn("b"));
        std::printf("ok schema_lookup\n");
        return 0;
    }
    const char* only = argc > 1 ? argv[1] : nullptr;
    ExecutionContext ctx(0);
    int run = 0;
    for (auto& t : tests) {
        if (only && std::strcmp(only, t.name) != 0)
            continue;
        run++;
        try {
            t.fn(ctx);
            std::printf("ok %s\n", t.name);
        } catch (const std::exception& e) {
            std::printf("FAIL %s: %s\n", t.name, e.what());
            g_failures++;
        }
        std::fflush(stdout);
    }
    std::printf("%d run, %d failed\n", run, g_failures);
    return g_failures ? 1 : 0;
}
