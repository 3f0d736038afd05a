// C++ operator layer over the velo_obl C ABI.
//
// The classes keep the shape of the reference's operator plugin API so that a
// physical plan built for the reference maps one to one onto them:
//   AbstractOperator / UnaryOperator / BinaryOperator
//       include/operator/abstract_operator.hpp:18-60 (constructors take the
//       execution context, the output schema and the children; next()
//       returns Result<RowBatch>; an empty batch is the end of the stream;
//       collectBatches() drains a child)
//   SeqScanOperator          include/operator/seq_scan_operator.hpp
//   FilterCompactionOperator include/operator/filter_compaction_operator.hpp
//   SortOperator             include/operator/sort_operator.hpp
//   SortMergeJoinOperator    include/operator/sort_merge_join_operator.hpp
//   HashJoinOperator         include/operator/hash_join_operator.hpp
//   MaterializationOperator  include/operator/materialization_operator.hpp
//   LimitOperator            include/operator/limit_operator.hpp
//   AggregateOperator        the aggregate node the reference plans name
//                            (include/planner/abstract_plan_node.hpp:31) but
//                            do not implement
// Errors inside an operator throw ExecutionError (the reference's
// VELODB_THROW / CHECKED_CALL_THROW); a child's failed Result is returned
// unchanged.  Special columns keep the reference's names: "$_rowid" (BIGINT)
// and "$_mask" (BOOLEAN, one byte per row), optionally prefixed "alias.".
//
// What runs on the device is the oblivious path: the scan's predicate is a
// device mask, FilterCompaction is ORCompact (velo_ocompact_columns), the
// sort is the bitonic network (velo_sort_columns, reference tie order), both
// joins are the oblivious PK-FK union-sort join (velo_ojoin_pkfk) and
// materialization is the oblivious sort-based gather (velo_ogather_u64).
// Columns live in device memory allocated through the C ABI; this layer
// never calls CUDA itself.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "velo_obl.h"

namespace velo_b200 {

// the reference's MAX_BATCH_SIZE (include/common/constants.hpp.in:16)
constexpr size_t MAX_BATCH_SIZE = size_t(1) << 23;

using DataTypeId = velo_type; // same numeric ids as the reference's DataTypeId
size_t type_size(DataTypeId t);

class ExecutionError : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

// throws ExecutionError with the library's error text when st != VELO_OK
void check(velo_status st, const char* what);

template <class T>
class Result {
public:
    static Result success(T v)
    {
        Result r;
        r.ok_ = true;
        r.value_ = std::move(v);
        return r;
    }
    static Result failure(std::string msg)
    {
        Result r;
        r.ok_ = false;
        r.error_ = std::move(msg);
        return r;
    }
    explicit operator bool() const { return ok_; }
    T& value() &
    {
        if (!ok_)
            throw ExecutionError("Result has no value: " + error_);
        return value_;
    }
    T&& value() &&
    {
        if (!ok_)
            throw ExecutionError("Result has no value: " + error_);
        return std::move(value_);
    }
    const std::string& error() const { return error_; }

private:
    bool ok_ = false;
    T value_ {};
    std::string error_;
};

// A command queue (velo_init) on one device: its stream orders every
// allocation, copy and operator launch of the operators built on it.
class ExecutionContext {
public:
    explicit ExecutionContext(int device = 0);
    ~ExecutionContext();
    ExecutionContext(const ExecutionContext&) = delete;
    ExecutionContext& operator=(const ExecutionContext&) = delete;

    void* stream() const { return stream_; }
    velo_ctx* queue() const { return ctx_; }
    // submit one command and wait for it (TaskManager::submitCommand +
    // waitCommand of the reference)
    void run(const velo_cmd& cmd);
    void sync();

private:
    velo_ctx* ctx_ = nullptr;
    void* stream_ = nullptr;
};

// device allocation owned by shared_ptr (freed on the owning context's stream)
std::shared_ptr<void> device_alloc(ExecutionContext& ctx, size_t bytes);

class Column {
public:
    Column() = default;
    Column(ExecutionContext& ctx, DataTypeId type, size_t capacity);

    static Column createFromDeviceBuffers(DataTypeId type, std::shared_ptr<void> data,
                                          std::shared_ptr<void> valid, size_t size, size_t capacity);
    template <class T>
    static Column fromHost(ExecutionContext& ctx, DataTypeId type, const std::vector<T>& values,
                           const std::vector<uint8_t>* valid = nullptr);
    template <class T>
    std::vector<T> toHost(ExecutionContext& ctx) const;
    std::vector<uint8_t> validityToHost(ExecutionContext& ctx) const;

    DataTypeId getType() const { return type_; }
    size_t size() const { return size_; }
    size_t capacity() const { return capacity_; }
    void* rawData() const;
    uint8_t* rawBitmapData() const;
    // a view of rows [begin, end) sharing the buffers
    Column slice(size_t begin, size_t end) const;
    void setSize(size_t n) { size_ = n; }

private:
    DataTypeId type_ = VELO_BIGINT;
    std::shared_ptr<void> data_;
    std::shared_ptr<void> valid_; // one byte per row, 1 = not NULL
    size_t offset_ = 0;
    size_t size_ = 0;
    size_t capacity_ = 0;
};

struct ColumnInfo {
    std::string name;
    DataTypeId type;
};

class Schema {
public:
    Schema() = default;
    explicit Schema(std::vector<ColumnInfo> cols) : cols_(std::move(cols)) { }
    size_t getColumnCount() const { return cols_.size(); }
    const ColumnInfo& getColumnInfo(size_t i) const { return cols_.at(i); }
    // index of `name` or of a column named "<alias>.<name>"; throws if absent
    size_t getColumnIndex(const std::string& name) const;
    bool hasColumn(const std::string& name) const;

private:
    std::vector<ColumnInfo> cols_;
};

class RowBatch {
public:
    RowBatch() = default;
    explicit RowBatch(std::vector<Column> columns);
    void addColumn(Column&& c);
    Column& getColumn(size_t i) { return columns_.at(i); }
    const Column& getColumn(size_t i) const { return columns_.at(i); }
    std::vector<Column>& getColumns() { return columns_; }
    size_t getColumnCount() const { return columns_.size(); }
    size_t getRowCount() const { return num_rows_; }
    void setRowCount(size_t n);
    RowBatch slice(size_t begin, size_t end) const;

private:
    std::vector<Column> columns_;
    size_t num_rows_ = 0;
};

// A device-resident table: the source of scans and of materialization.
struct Table {
    Schema schema;
    std::vector<Column> columns;
    size_t rows = 0;
};

class AbstractOperator {
public:
    AbstractOperator(ExecutionContext& context, Schema output_schema);
    virtual ~AbstractOperator() = default;
    AbstractOperator(const AbstractOperator&) = delete;
    AbstractOperator& operator=(const AbstractOperator&) = delete;
    const Schema& getOutputSchema() const { return output_schema_; }
    virtual Result<RowBatch> next() = 0;
    virtual bool isUnary() const = 0;

protected:
    ExecutionContext& context_;
    Schema output_schema_;
    // all of a child's batches concatenated on the device (throws on a
    // child failure, as the reference's collectBatches does)
    RowBatch collectBatches(AbstractOperator& child);
};

class UnaryOperator : public AbstractOperator {
public:
    UnaryOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child);
    bool isUnary() const override { return true; }

protected:
    std::unique_ptr<AbstractOperator> child_;
};

class BinaryOperator : public AbstractOperator {
public:
    BinaryOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> left_child,
                   std::unique_ptr<AbstractOperator> right_child);
    bool isUnary() const override { return false; }

protected:
    std::unique_ptr<AbstractOperator> left_child_;
    std::unique_ptr<AbstractOperator> right_child_;
};

// lo <= column <= hi (inclusive), conjunctive; column indexes the table
struct RangePredicate {
    size_t column;
    int64_t lo;
    int64_t hi;
};

// Emits the table in MAX_BATCH_SIZE slices followed by "$_rowid" and
// "$_mask" (the predicate evaluated on the device; all ones without one).
class SeqScanOperator : public UnaryOperator {
public:
    SeqScanOperator(ExecutionContext& context, const Table& table, Schema output_schema,
                    std::vector<RangePredicate> predicate = {});
    Result<RowBatch> next() override;

private:
    const Table& table_;
    std::vector<RangePredicate> predicate_;
    size_t current_row_id_ = 0;
};

// Rows whose "$_mask" is set, in input order (ORCompact: the addresses do
// not depend on the mask); compact_columns[i] = false leaves column i as is.
class FilterCompactionOperator : public UnaryOperator {
public:
    FilterCompactionOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child,
                             std::vector<bool> compact_columns = {});
    Result<RowBatch> next() override;

private:
    std::vector<bool> compact_columns_;
};

// ORDER BY over all of the child's rows; emitted in MAX_BATCH_SIZE slices.
class SortOperator : public UnaryOperator {
public:
    SortOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child,
                 std::vector<size_t> order_indices, std::vector<bool> ascending_flags);
    Result<RowBatch> next() override;

private:
    std::vector<size_t> order_indices_;
    std::vector<bool> ascending_flags_;
    bool sorted_ = false;
    RowBatch sorted_batch_;
    size_t current_offset_ = 0;
};

enum class JoinType { INNER, LEFT, RIGHT, FULL, CROSS };

// Inner equi-join, the reference's sort-merge join: the left input is the
// build side.  The output holds the left columns then the right columns, one
// row per matching pair, in key order.  A left side with unique keys takes
// the oblivious PK-FK join (velo_ojoin_pkfk); repeated left keys take the
// oblivious many-to-many join (velo_ojoin_mn), which writes every pair, as
// the reference's cross product of equal-key runs does.
class SortMergeJoinOperator : public BinaryOperator {
public:
    SortMergeJoinOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> left,
                          std::unique_ptr<AbstractOperator> right, std::pair<size_t, size_t> join_key_indices,
                          JoinType join_type = JoinType::INNER);
    Result<RowBatch> next() override;

protected:
    // mask column indices of the build and probe inputs (-1: none); hashed
    // selects the bin-padded hash join, else the union-sort PK-FK join; both
    // hand a build side with repeated keys to the many-to-many join
    Result<RowBatch> join(std::pair<long, long> mask_indices, bool hashed);
    std::pair<size_t, size_t> join_key_indices_;
    JoinType join_type_;
    bool joined_ = false;
    uint64_t hash_seed_ = 0;
};

// The join with the reference's build/probe mask columns (rows whose mask is
// zero do not join), by the oblivious bin-padded hash join
// (velo_ohash_join): both sides hashed into padded bins by a per-operator
// keyed hash, every probe slot compared with every build slot of its bin.
// The reference builds a chained hash table (hash_join_operator.cpp:88-393).
class HashJoinOperator : public SortMergeJoinOperator {
public:
    HashJoinOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> left,
                     std::unique_ptr<AbstractOperator> right, std::pair<size_t, size_t> join_key_indices,
                     std::pair<long, long> mask_indices, JoinType join_type = JoinType::INNER);
    Result<RowBatch> next() override;

private:
    std::pair<long, long> mask_indices_;
};

// Replaces row-id columns by the columns they reference, obliviously: every
// output column c is source_table->columns[source_col_index] gathered at the
// row ids of input column rowid_input_index (NULL where the row id is < 0).
class MaterializationOperator : public UnaryOperator {
public:
    struct ColumnMapping {
        size_t rowid_input_index;
        const Table* source_table;
        size_t source_col_index;
    };
    MaterializationOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child,
                            std::vector<ColumnMapping> mappings);
    Result<RowBatch> next() override;

private:
    std::vector<ColumnMapping> mappings_;
};

enum class AggKind { SUM, COUNT };

struct AggregateSpec {
    AggKind kind;
    size_t column; // input column summed (ignored for COUNT)
};

// GROUP BY one integer key column (INTEGER or BIGINT; BIGINT keys in
// [-2^62, 2^62)) with SUM / COUNT aggregates, oblivious (velo_ogroupby).
// Rows whose "$_mask" is 0 are left out when the input has that column.
// Output: the key as BIGINT, then one BIGINT per aggregate, the groups in key
// order, at most group_bound of them (0 = the number of input rows, i.e. no
// bound).  SUM columns may be any integer type (summed as int64 mod 2^64).
class AggregateOperator : public UnaryOperator {
public:
    AggregateOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child,
                      size_t group_column, std::vector<AggregateSpec> aggregates, size_t group_bound = 0);
    Result<RowBatch> next() override;

private:
    size_t group_column_;
    std::vector<AggregateSpec> aggregates_;
    size_t group_bound_;
    bool done_ = false;
};

class LimitOperator : public UnaryOperator {
public:
    LimitOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child,
                  size_t limit, size_t offset = 0);
    Result<RowBatch> next() override;

private:
    size_t limit_;
    size_t offset_;
    size_t current_count_ = 0;
    size_t skipped_count_ = 0;
};

// The result of a query: the root operator's schema and every batch it
// produced (device-resident).
struct QueryResult {
    Schema schema;
    std::vector<RowBatch> batches;
    size_t rows = 0;
    size_t getRowCount() const { return rows; }
};

// Drives an operator tree to the end of its stream, as the reference's
// ExecutionEngine::executePlan does (src/execution/execution_engine.cpp:
// 118-142).  SQL parsing and planning (executeQuery(sql)) are not part of this
// build: plans arrive as operator trees.
class ExecutionEngine {
public:
    explicit ExecutionEngine(ExecutionContext& context) : context_(context) { }
    Result<QueryResult> executePlan(std::unique_ptr<AbstractOperator> root);
    size_t getLastExecutionRowCount() const { return last_rows_; }
    double getLastExecutionTimeMs() const { return last_ms_; }

private:
    ExecutionContext& context_;
    size_t last_rows_ = 0;
    double last_ms_ = 0.0;
};

// ---- template members --------------------------------------------------

template <class T>
Column Column::fromHost(ExecutionContext& ctx, DataTypeId type, const std::vector<T>& values,
                        const std::vector<uint8_t>* valid)
{
    if (sizeof(T) != type_size(type))
        throw ExecutionError("Column::fromHost: element size does not match the type");
    Column c(ctx, type, values.size());
    check(velo_copy(c.rawData(), values.data(), values.size() * sizeof(T), VELO_COPY_H2D, ctx.stream()),
          "Column::fromHost");
    if (valid)
        check(velo_copy(c.rawBitmapData(), valid->data(), values.size(), VELO_COPY_H2D, ctx.stream()),
              "Column::fromHost");
    c.size_ = values.size();
    ctx.sync();
    return c;
}

template <class T>
std::vector<T> Column::toHost(ExecutionContext& ctx) const
{
    if (sizeof(T) != type_size(type_))
        throw ExecutionError("Column::toHost: element size does not match the type");
    std::vector<T> out(size_);
    check(velo_copy(out.data(), rawData(), size_ * sizeof(T), VELO_COPY_D2H, ctx.stream()), "Column::toHost");
    ctx.sync();
    return out;
}

} // namespace velo_b200
