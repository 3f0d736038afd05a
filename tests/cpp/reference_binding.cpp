// The reference-side binding of the oblivious operator library: the code a
// VelODB maintainer adds to the reference tree so that its planner's physical
// plans run on this library.  It is written against the reference's own
// headers (namespace velodb: AbstractOperator, UnaryOperator, BinaryOperator,
// AbstractPlanNode, Column, RowBatch, Result, ExecutionError) and calls only
// the C ABI of include/velo_obl.h, in place of the reference's TaskManager
// commands.  tests/test_reference_binding.py compiles it against the
// reference headers wherever the reference tree is present.
//
//   ObliviousSortOperator           replaces SortOperator::next
//                                   (src/operator/sort_operator.cpp:27-120)
//   ObliviousSortMergeJoinOperator  replaces SortMergeJoinOperator::next
//                                   (src/operator/sort_merge_join_operator.cpp:27-257)
//   ObliviousHashJoinOperator       replaces HashJoinOperator::next
//                                   (src/operator/hash_join_operator.cpp:88-393)
//   ObliviousAggregateOperator +    the aggregate the reference plans name
//   AggregatePlanNode               (PlanType::AGGREGATE,
//                                   include/planner/abstract_plan_node.hpp:31)
//                                   but never build; createOperator follows
//                                   SortPlanNode::createOperator
//                                   (src/planner/sort_plan_node.cpp:17-27)
#include "common/exception.hpp"
#include "operator/abstract_operator.hpp"
#include "planner/abstract_plan_node.hpp"
#include "velo_obl.h"

#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace velodb {
namespace velo_binding {

// One command queue per process: the drop-in for the reference's TaskManager
// (the persistent kernel and its command ring).
inline velo_ctx* queue()
{
    static velo_ctx* q = [] {
        velo_config cfg {};
        cfg.device = 0;
        cfg.queue_capacity = 1024;
        velo_ctx* c = nullptr;
        if (velo_init(&cfg, &c) != VELO_OK)
            VELODB_THROW(ExecutionError, std::string("velo_init: ") + velo_last_error_text());
        return c;
    }();
    return q;
}

inline void check(velo_status s, const char* what)
{
    if (s != VELO_OK)
        VELODB_THROW(ExecutionError, std::string(what) + ": " + velo_last_error_text());
}

// submit a command and wait for it (the reference's submitCommand +
// waitCommand pair), bounded at 60 s
inline void run(const velo_cmd& cmd)
{
    uint64_t ticket = 0;
    check(velo_submit(queue(), &cmd, &ticket), "velo_submit");
    check(velo_wait(queue(), ticket, 60'000'000'000ull), "velo_wait");
}

// device memory a Column can adopt (stream-ordered, like cudaMallocAsync)
inline void* alloc(size_t bytes)
{
    void* p = nullptr;
    check(velo_device_alloc(bytes ? bytes : 8, nullptr, &p), "velo_device_alloc");
    return p;
}

inline uint32_t type_of(const Column& c) { return static_cast<uint32_t>(c.getType().getTypeId()); }

// the columns of `src` gathered at the int64 row ids (VELO_OP_PERMUTE)
inline std::vector<Column> gather(const RowBatch& src, const int64_t* d_rowids, size_t n)
{
    std::vector<Column> out;
    for (const Column& c : src.getColumns()) {
        const size_t elem = c.getType().size();
        void* data = alloc(n * elem);
        velo_cmd p;
        std::memset(&p, 0, sizeof p);
        p.opcode = VELO_OP_PERMUTE;
        p.args.permute.d_out = data;
        p.args.permute.d_in = c.getDeviceBuffer();
        p.args.permute.d_indices = d_rowids;
        p.args.permute.n = n;
        p.args.permute.type = type_of(c);
        run(p);
        out.push_back(Column::createFromDeviceBuffers(c.getType().cloneUnique(), data, nullptr, n, n));
    }
    return out;
}

} // namespace velo_binding

// ORDER BY: the reference network, run by the library (same tie order).
class ObliviousSortOperator : public UnaryOperator {
public:
    ObliviousSortOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child,
                          std::vector<size_t> order_indices, std::vector<bool> ascending)
        : UnaryOperator(context, std::move(output_schema), std::move(child))
        , order_(std::move(order_indices))
        , asc_(std::move(ascending))
    {
    }

    Result<RowBatch> next() override;

private:
    std::vector<size_t> order_;
    std::vector<bool> asc_;
    bool done_ = false;
};

// Inner equi-join: PK-FK by the union sort; repeated left keys by the
// many-to-many join (every pair, as the reference's cross product of runs).
class ObliviousSortMergeJoinOperator : public BinaryOperator {
public:
    ObliviousSortMergeJoinOperator(ExecutionContext& context, Schema output_schema,
                                   std::unique_ptr<AbstractOperator> left, std::unique_ptr<AbstractOperator> right,
                                   std::pair<size_t, size_t> keys, bool hashed = false)
        : BinaryOperator(context, std::move(output_schema), std::move(left), std::move(right))
        , keys_(keys)
        , hashed_(hashed)
    {
    }

    Result<RowBatch> next() override;

private:
    std::pair<size_t, size_t> keys_;
    bool hashed_;
    bool done_ = false;
};

class ObliviousHashJoinOperator : public ObliviousSortMergeJoinOperator {
public:
    ObliviousHashJoinOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> left,
                              std::unique_ptr<AbstractOperator> right, std::pair<size_t, size_t> keys)
        : ObliviousSortMergeJoinOperator(context, std::move(output_schema), std::move(left), std::move(right), keys,
                                         true)
    {
    }
};

// GROUP BY one INTEGER/BIGINT key with COUNT and SUM of one BIGINT column.
class ObliviousAggregateOperator : public UnaryOperator {
public:
    ObliviousAggregateOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child,
                               size_t group_column, size_t sum_column, size_t group_bound)
        : UnaryOperator(context, std::move(output_schema), std::move(child))
        , group_(group_column)
        , sum_(sum_column)
        , bound_(group_bound)
    {
    }

    Result<RowBatch> next() override;

private:
    size_t group_, sum_, bound_;
    bool done_ = false;
};

// The plan-node hook the reference names (PlanType::AGGREGATE) without an
// implementation: built by the planner like SortPlanNode, with one child.
class AggregatePlanNode : public AbstractPlanNode {
public:
    AggregatePlanNode(Schema output_schema, size_t group_column, size_t sum_column, size_t group_bound)
        : AbstractPlanNode(PlanType::AGGREGATE, std::move(output_schema))
        , group_(group_column)
        , sum_(sum_column)
        , bound_(group_bound)
    {
    }

    std::unique_ptr<AbstractOperator> createOperator(ExecutionContext& context) const override;

    std::string toString() const override { return "ObliviousAggregate"; }

private:
    size_t group_, sum_, bound_;
};

// ---- operator bodies (out of line, so this translation unit emits them) ----

Result<RowBatch> ObliviousSortOperator::next()
{
    if (done_)
        return Result<RowBatch>::success(RowBatch());
    done_ = true;
    RowBatch in = collectBatches(*child_);
    const size_t n = in.getRowCount();
    if (n == 0)
        return Result<RowBatch>::success(RowBatch());
    in.to(DataLocation::CUDA);
    const size_t cap = velo_next_pow2(n);
    // sort copies of the key columns (capacity next_pow2(n)), then gather
    // every column by the permutation
    std::vector<void*> keys;
    std::vector<uint32_t> types;
    std::vector<uint8_t> asc;
    for (size_t i = 0; i < order_.size(); i++) {
        const Column& c = in.getColumn(order_[i]);
        void* k = velo_binding::alloc(cap * c.getType().size());
        velo_binding::check(velo_copy(k, c.getDeviceBuffer(), n * c.getType().size(), VELO_COPY_D2D, nullptr),
                            "velo_copy");
        keys.push_back(k);
        types.push_back(velo_binding::type_of(c));
        asc.push_back(asc_[i] ? 1 : 0);
    }
    const size_t sb = velo_sort_scratch_bytes(types.data(), (uint32_t)types.size(), n);
    void* scratch = velo_binding::alloc(sb);
    auto* idx = static_cast<int64_t*>(velo_binding::alloc(cap * 8));
    velo_cmd s;
    std::memset(&s, 0, sizeof s);
    s.opcode = VELO_OP_SORT;
    s.args.sort.d_cols = keys.data();
    s.args.sort.types = types.data();
    s.args.sort.ascending = asc.data();
    s.args.sort.n_cols = (uint32_t)keys.size();
    s.args.sort.n = n;
    s.args.sort.capacity = cap;
    s.args.sort.d_indices = idx;
    s.args.sort.d_scratch = scratch;
    s.args.sort.scratch_bytes = sb;
    velo_binding::run(s);
    std::vector<Column> out = velo_binding::gather(in, idx, n);
    for (void* k : keys)
        velo_device_free(k, nullptr);
    velo_device_free(scratch, nullptr);
    velo_device_free(idx, nullptr);
    return Result<RowBatch>::success(buildBatchFromColumns(std::move(out)));
}

Result<RowBatch> ObliviousSortMergeJoinOperator::next()
{
    if (done_)
        return Result<RowBatch>::success(RowBatch());
    done_ = true;
    RowBatch l = collectBatches(*left_child_);
    RowBatch r = collectBatches(*right_child_);
    const size_t bn = l.getRowCount(), pn = r.getRowCount();
    if (bn == 0 || pn == 0)
        return Result<RowBatch>::success(RowBatch());
    l.to(DataLocation::CUDA);
    r.to(DataLocation::CUDA);
    const Column& lk = l.getColumn(keys_.first);
    const Column& rk = r.getColumn(keys_.second);
    const uint32_t kt = velo_binding::type_of(lk);
    size_t bound = pn;
    uint64_t hc[3] = { 0, 0, 0 };
    auto* counts = static_cast<uint64_t*>(velo_binding::alloc(24));
    auto* ob = static_cast<int64_t*>(velo_binding::alloc(bound * 8));
    auto* op = static_cast<int64_t*>(velo_binding::alloc(bound * 8));
    velo_cmd c;
    std::memset(&c, 0, sizeof c);
    size_t sb = hashed_ ? velo_ohash_join_scratch_bytes(bn, pn) : velo_ojoin_scratch_bytes(bn, pn);
    void* scratch = velo_binding::alloc(sb);
    if (hashed_) {
        c.opcode = VELO_OP_OHASH_JOIN;
        c.args.ohash = { lk.getDeviceBuffer(), nullptr, bn, rk.getDeviceBuffer(), nullptr, pn, kt, 0x5EEDull,
                         ob, op, counts, scratch, sb };
    } else {
        c.opcode = VELO_OP_OJOIN_PKFK;
        c.args.ojoin = { lk.getDeviceBuffer(), nullptr, bn, rk.getDeviceBuffer(), nullptr, pn, kt, ob, op,
                         counts, scratch, sb };
    }
    velo_binding::run(c);
    velo_binding::check(velo_copy(hc, counts, 24, VELO_COPY_D2H, nullptr), "velo_copy");
    velo_device_free(scratch, nullptr);
    for (int attempt = 0; (hc[1] || hc[2]) && attempt < 2; attempt++) {
        if (attempt)
            bound = (size_t)hc[0];
        velo_device_free(ob, nullptr);
        velo_device_free(op, nullptr);
        ob = static_cast<int64_t*>(velo_binding::alloc(bound * 8));
        op = static_cast<int64_t*>(velo_binding::alloc(bound * 8));
        sb = velo_ojoin_mn_scratch_bytes(bn, pn, bound);
        scratch = velo_binding::alloc(sb);
        std::memset(&c, 0, sizeof c);
        c.opcode = VELO_OP_OJOIN_MN;
        c.args.ojoin_mn = { lk.getDeviceBuffer(), nullptr, bn, rk.getDeviceBuffer(), nullptr, pn, kt, bound, ob,
                            op, counts, scratch, sb };
        velo_binding::run(c);
        velo_binding::check(velo_copy(hc, counts, 16, VELO_COPY_D2H, nullptr), "velo_copy");
        velo_device_free(scratch, nullptr);
        hc[2] = 0;
    }
    const size_t pairs = (size_t)hc[0] < bound ? (size_t)hc[0] : bound;
    std::vector<Column> out = velo_binding::gather(l, ob, pairs);
    for (Column& col : velo_binding::gather(r, op, pairs))
        out.push_back(std::move(col));
    velo_device_free(ob, nullptr);
    velo_device_free(op, nullptr);
    velo_device_free(counts, nullptr);
    return Result<RowBatch>::success(buildBatchFromColumns(std::move(out)));
}

Result<RowBatch> ObliviousAggregateOperator::next()
{
    if (done_)
        return Result<RowBatch>::success(RowBatch());
    done_ = true;
    RowBatch in = collectBatches(*child_);
    const size_t n = in.getRowCount();
    if (n == 0)
        return Result<RowBatch>::success(RowBatch());
    in.to(DataLocation::CUDA);
    const Column& key = in.getColumn(group_);
    const Column& val = in.getColumn(sum_);
    const size_t bound = bound_ ? (bound_ < n ? bound_ : n) : n;
    auto* ok = static_cast<int64_t*>(velo_binding::alloc(bound * 8));
    auto* os = static_cast<int64_t*>(velo_binding::alloc(bound * 8));
    auto* oc = static_cast<int64_t*>(velo_binding::alloc(bound * 8));
    auto* counts = static_cast<uint64_t*>(velo_binding::alloc(16));
    const size_t sb = velo_ogroupby_scratch_bytes(n);
    void* scratch = velo_binding::alloc(sb);
    const int64_t* sums[1] = { static_cast<const int64_t*>(val.getDeviceBuffer()) };
    int64_t* out_sums[1] = { os };
    velo_binding::check(velo_ogroupby(key.getDeviceBuffer(), velo_binding::type_of(key), sums, 1, 1, nullptr, n,
                                      bound, ok, out_sums, oc, counts, scratch, sb, nullptr),
                        "velo_ogroupby");
    uint64_t hc[2] = { 0, 0 };
    velo_binding::check(velo_copy(hc, counts, 16, VELO_COPY_D2H, nullptr), "velo_copy");
    velo_device_free(scratch, nullptr);
    velo_device_free(counts, nullptr);
    const size_t groups = (size_t)hc[0] < bound ? (size_t)hc[0] : bound;
    std::vector<Column> out;
    out.push_back(Column::createFromDeviceBuffers(DataType::createType(DataTypeId::BIGINT), ok, nullptr, groups,
                                                  bound));
    out.push_back(Column::createFromDeviceBuffers(DataType::createType(DataTypeId::BIGINT), oc, nullptr, groups,
                                                  bound));
    out.push_back(Column::createFromDeviceBuffers(DataType::createType(DataTypeId::BIGINT), os, nullptr, groups,
                                                  bound));
    return Result<RowBatch>::success(buildBatchFromColumns(std::move(out)));
}

std::unique_ptr<AbstractOperator> AggregatePlanNode::createOperator(ExecutionContext& context) const
{
    VELODB_ASSERT_MSG(children_.size() == 1, "AggregatePlanNode must have exactly one child");
    auto child = children_[0]->createOperator(context);
    return std::make_unique<ObliviousAggregateOperator>(context, output_schema_.clone(), std::move(child), group_,
                                                        sum_, bound_);
}

// the binding's classes are complete types the planner can instantiate
static_assert(!std::is_abstract_v<ObliviousSortOperator>);
static_assert(!std::is_abstract_v<ObliviousSortMergeJoinOperator>);
static_assert(!std::is_abstract_v<ObliviousHashJoinOperator>);
static_assert(!std::is_abstract_v<ObliviousAggregateOperator>);
static_assert(!std::is_abstract_v<AggregatePlanNode>);

} // namespace velodb
