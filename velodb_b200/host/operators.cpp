// C++ operator layer over the velo_obl C ABI (see include/velo_operator.hpp).
//
// Every device step goes through the C ABI: memory and copies through
// velo_device_alloc / velo_copy, the operators through velo_cmd commands on
// the context's queue (velo_submit + velo_wait, the reference's
// TaskManager::submitCommand + waitCommand) or the column entry points on the
// context's stream.
#include "velo_operator.hpp"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <random>

namespace velo_b200 {

size_t type_size(DataTypeId t)
{
    switch (t) {
    case VELO_BOOLEAN:
    case VELO_TINYINT:
        return 1;
    case VELO_SMALLINT:
        return 2;
    case VELO_INTEGER:
    case VELO_FLOAT:
    case VELO_DATE:
        return 4;
    case VELO_BIGINT:
    case VELO_DOUBLE:
    case VELO_VARCHAR:
        return 8;
    }
    throw ExecutionError("unknown data type id " + std::to_string((int)t));
}

void check(velo_status st, const char* what)
{
    if (st != VELO_OK)
        throw ExecutionError(std::string(what) + ": " + velo_last_error_text());
}

// ---- context -------------------------------------------------------------

ExecutionContext::ExecutionContext(int device)
{
    velo_config cfg { device, 0, 0, 0 };
    check(velo_init(&cfg, &ctx_), "ExecutionContext");
    stream_ = velo_ctx_stream(ctx_);
}

ExecutionContext::~ExecutionContext()
{
    if (ctx_)
        velo_shutdown(ctx_, 60000);
}

void ExecutionContext::run(const velo_cmd& cmd)
{
    uint64_t ticket = 0;
    velo_status st = velo_submit(ctx_, &cmd, &ticket);
    if (st == VELO_OK)
        st = velo_wait(ctx_, ticket, 600ull * 1000 * 1000 * 1000);
    if (st != VELO_OK) {
        char buf[512];
        velo_last_error(ctx_, buf, sizeof buf);
        throw ExecutionError(std::string("command ") + std::to_string(cmd.opcode) + ": " + buf);
    }
}

void ExecutionContext::sync() { check(velo_stream_sync(stream_), "ExecutionContext::sync"); }

std::shared_ptr<void> device_alloc(ExecutionContext& ctx, size_t bytes)
{
    void* p = nullptr;
    check(velo_device_alloc(bytes ? bytes : 1, ctx.stream(), &p), "device_alloc");
    // freed on the legacy stream: safe after the context is gone
    return std::shared_ptr<void>(p, [](void* q) { velo_device_free(q, nullptr); });
}

// ---- columns, schema, batches ---------------------------------------------

Column::Column(ExecutionContext& ctx, DataTypeId type, size_t capacity)
    : type_(type)
    , capacity_(capacity)
{
    data_ = device_alloc(ctx, capacity * type_size(type));
    valid_ = device_alloc(ctx, capacity);
    check(velo_memset(valid_.get(), 1, capacity, ctx.stream()), "Column");
}

Column Column::createFromDeviceBuffers(DataTypeId type, std::shared_ptr<void> data, std::shared_ptr<void> valid,
                                       size_t size, size_t capacity)
{
    Column c;
    c.type_ = type;
    c.data_ = std::move(data);
    c.valid_ = std::move(valid);
    c.size_ = size;
    c.capacity_ = capacity;
    return c;
}

std::vector<uint8_t> Column::validityToHost(ExecutionContext& ctx) const
{
    std::vector<uint8_t> out(size_, 1);
    if (valid_)
        check(velo_copy(out.data(), rawBitmapData(), size_, VELO_COPY_D2H, ctx.stream()), "Column::validityToHost");
    ctx.sync();
    return out;
}

void* Column::rawData() const { return static_cast<char*>(data_.get()) + offset_ * type_size(type_); }

uint8_t* Column::rawBitmapData() const
{
    return valid_ ? static_cast<uint8_t*>(valid_.get()) + offset_ : nullptr;
}

Column Column::slice(size_t begin, size_t end) const
{
    if (begin > end || end > size_)
        throw ExecutionError("Column::slice out of range");
    Column c = *this;
    c.offset_ += begin;
    c.size_ = end - begin;
    c.capacity_ = capacity_ - begin;
    return c;
}

size_t Schema::getColumnIndex(const std::string& name) const
{
    for (size_t i = 0; i < cols_.size(); i++)
        if (cols_[i].name == name)
            return i;
    const std::string suffix = "." + name;
    for (size_t i = 0; i < cols_.size(); i++) {
        const std::string& n = cols_[i].name;
        if (n.size() > suffix.size() && n.compare(n.size() - suffix.size(), suffix.size(), suffix) == 0)
            return i;
    }
    throw ExecutionError("column not found: " + name);
}

bool Schema::hasColumn(const std::string& name) const
{
    try {
        getColumnIndex(name);
        return true;
    } catch (const ExecutionError&) {
        return false;
    }
}

RowBatch::RowBatch(std::vector<Column> columns)
    : columns_(std::move(columns))
    , num_rows_(columns_.empty() ? 0 : columns_.front().size())
{
}

void RowBatch::addColumn(Column&& c)
{
    if (columns_.empty())
        num_rows_ = c.size();
    columns_.push_back(std::move(c));
}

void RowBatch::setRowCount(size_t n)
{
    num_rows_ = n;
    for (auto& c : columns_)
        c.setSize(n);
}

RowBatch RowBatch::slice(size_t begin, size_t end) const
{
    std::vector<Column> cols;
    cols.reserve(columns_.size());
    for (const auto& c : columns_)
        cols.push_back(c.slice(begin, end));
    RowBatch b(std::move(cols));
    b.num_rows_ = end - begin;
    return b;
}

// ---- operator bases --------------------------------------------------------

AbstractOperator::AbstractOperator(ExecutionContext& context, Schema output_schema)
    : context_(context)
    , output_schema_(std::move(output_schema))
{
}

RowBatch AbstractOperator::collectBatches(AbstractOperator& child)
{
    std::vector<RowBatch> parts;
    size_t total = 0;
    for (;;) {
        Result<RowBatch> r = child.next();
        if (!r)
            throw ExecutionError("child operator failed: " + r.error());
        RowBatch b = std::move(r).value();
        if (b.getRowCount() == 0)
            break;
        total += b.getRowCount();
        parts.push_back(std::move(b));
    }
    if (parts.empty())
        return RowBatch();
    if (parts.size() == 1)
        return std::move(parts.front());
    const size_t ncols = parts.front().getColumnCount();
    std::vector<Column> cols;
    for (size_t c = 0; c < ncols; c++) {
        const DataTypeId t = parts.front().getColumn(c).getType();
        const size_t es = type_size(t);
        Column out(context_, t, total);
        size_t at = 0;
        for (auto& p : parts) {
            const Column& src = p.getColumn(c);
            const size_t n = p.getRowCount();
            check(velo_copy(static_cast<char*>(out.rawData()) + at * es, src.rawData(), n * es, VELO_COPY_D2D,
                            context_.stream()),
                  "collectBatches");
            if (src.rawBitmapData())
                check(velo_copy(out.rawBitmapData() + at, src.rawBitmapData(), n, VELO_COPY_D2D, context_.stream()),
                      "collectBatches");
            at += n;
        }
        out.setSize(total);
        cols.push_back(std::move(out));
    }
    context_.sync();
    RowBatch b(std::move(cols));
    b.setRowCount(total);
    return b;
}

UnaryOperator::UnaryOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child)
    : AbstractOperator(context, std::move(output_schema))
    , child_(std::move(child))
{
}

BinaryOperator::BinaryOperator(ExecutionContext& context, Schema output_schema,
                               std::unique_ptr<AbstractOperator> left_child,
                               std::unique_ptr<AbstractOperator> right_child)
    : AbstractOperator(context, std::move(output_schema))
    , left_child_(std::move(left_child))
    , right_child_(std::move(right_child))
{
}

// ---- scan ------------------------------------------------------------------

SeqScanOperator::SeqScanOperator(ExecutionContext& context, const Table& table, Schema output_schema,
                                 std::vector<RangePredicate> predicate)
    : UnaryOperator(context, std::move(output_schema), nullptr)
    , table_(table)
    , predicate_(std::move(predicate))
{
    if (output_schema_.getColumnCount() != table_.columns.size() + 2)
        throw ExecutionError("SeqScanOperator: output schema must be the table's columns, $_rowid, $_mask");
    for (const auto& p : predicate_)
        if (p.column >= table_.columns.size())
            throw ExecutionError("SeqScanOperator: predicate column out of range");
}

Result<RowBatch> SeqScanOperator::next()
{
    if (current_row_id_ >= table_.rows)
        return Result<RowBatch>::success(RowBatch());
    const size_t b = current_row_id_;
    const size_t n = std::min(MAX_BATCH_SIZE, table_.rows - b);
    // the batch owns copies: downstream operators work in place and must
    // never reach the table's buffers
    RowBatch batch;
    for (const auto& c : table_.columns) {
        const Column src = c.slice(b, b + n);
        Column dst(context_, src.getType(), n);
        check(velo_copy(dst.rawData(), src.rawData(), n * type_size(src.getType()), VELO_COPY_D2D,
                        context_.stream()),
              "SeqScan copy");
        if (src.rawBitmapData())
            check(velo_copy(dst.rawBitmapData(), src.rawBitmapData(), n, VELO_COPY_D2D, context_.stream()),
                  "SeqScan copy");
        dst.setSize(n);
        batch.addColumn(std::move(dst));
    }
    Column rowid(context_, VELO_BIGINT, n);
    check(velo_iota_i64(static_cast<int64_t*>(rowid.rawData()), n, (int64_t)b, context_.stream()), "SeqScan rowid");
    rowid.setSize(n);
    Column mask(context_, VELO_BOOLEAN, n);
    uint8_t* m = static_cast<uint8_t*>(mask.rawData());
    if (predicate_.empty())
        check(velo_memset(m, 1, n, context_.stream()), "SeqScan mask");
    for (size_t i = 0; i < predicate_.size(); i++) {
        const Column col = table_.columns[predicate_[i].column].slice(b, b + n);
        check(velo_range_mask(col.rawData(), col.getType(), n, predicate_[i].lo, predicate_[i].hi, m, i > 0 ? 1 : 0,
                              context_.stream()),
              "SeqScan predicate");
    }
    mask.setSize(n);
    batch.addColumn(std::move(rowid));
    batch.addColumn(std::move(mask));
    batch.setRowCount(n);
    context_.sync();
    current_row_id_ += n;
    return Result<RowBatch>::success(std::move(batch));
}

// ---- filter compaction -----------------------------------------------------

FilterCompactionOperator::FilterCompactionOperator(ExecutionContext& context, Schema output_schema,
                                                   std::unique_ptr<AbstractOperator> child,
                                                   std::vector<bool> compact_columns)
    : UnaryOperator(context, std::move(output_schema), std::move(child))
    , compact_columns_(std::move(compact_columns))
{
    if (compact_columns_.empty())
        compact_columns_.assign(output_schema_.getColumnCount(), true);
    if (compact_columns_.size() != output_schema_.getColumnCount())
        throw ExecutionError("FilterCompactionOperator: one compact flag per column");
}

Result<RowBatch> FilterCompactionOperator::next()
{
    Result<RowBatch> r = child_->next();
    if (!r)
        return r;
    RowBatch& batch = r.value();
    const size_t n = batch.getRowCount();
    if (n == 0)
        return r;
    const size_t mask_index = output_schema_.getColumnIndex("$_mask");
    const uint8_t* mask = static_cast<const uint8_t*>(batch.getColumn(mask_index).rawData());
    std::vector<void*> cols;
    std::vector<uint32_t> types;
    std::vector<uint8_t*> valid;
    for (size_t c = 0; c < batch.getColumnCount(); c++) {
        if (!compact_columns_[c])
            continue;
        Column& col = batch.getColumn(c);
        cols.push_back(col.rawData());
        types.push_back(col.getType());
        valid.push_back(col.rawBitmapData());
    }
    const size_t sb = velo_ocompact_columns_scratch_bytes(n);
    std::shared_ptr<void> scratch = device_alloc(context_, sb);
    std::shared_ptr<void> d_count = device_alloc(context_, 8);
    check(velo_ocompact_columns(cols.data(), types.data(), valid.data(), (uint32_t)cols.size(), mask, n,
                                static_cast<uint64_t*>(d_count.get()), scratch.get(), sb, context_.stream()),
          "FilterCompactionOperator");
    uint64_t count = 0;
    check(velo_copy(&count, d_count.get(), 8, VELO_COPY_D2H, context_.stream()), "FilterCompactionOperator");
    context_.sync();
    // the reference reveals the kept row count too
    // (src/operator/filter_compaction_operator.cpp:171-178)
    batch.setRowCount((size_t)count);
    return r;
}

// ---- sort ------------------------------------------------------------------

SortOperator::SortOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child,
                           std::vector<size_t> order_indices, std::vector<bool> ascending_flags)
    : UnaryOperator(context, std::move(output_schema), std::move(child))
    , order_indices_(std::move(order_indices))
    , ascending_flags_(std::move(ascending_flags))
{
    if (order_indices_.empty() || order_indices_.size() > 8 || ascending_flags_.size() != order_indices_.size())
        throw ExecutionError("SortOperator: 1..8 sort columns, one ascending flag each");
}

Result<RowBatch> SortOperator::next()
{
    if (sorted_) {
        const size_t total = sorted_batch_.getRowCount();
        if (current_offset_ >= total)
            return Result<RowBatch>::success(RowBatch());
        const size_t end = std::min(current_offset_ + MAX_BATCH_SIZE, total);
        RowBatch s = sorted_batch_.slice(current_offset_, end);
        current_offset_ = end;
        return Result<RowBatch>::success(std::move(s));
    }
    RowBatch gathered = collectBatches(*child_);
    sorted_ = true;
    if (gathered.getRowCount() == 0)
        return Result<RowBatch>::success(RowBatch());
    const size_t n = gathered.getRowCount();
    const size_t np = velo_next_pow2(n);
    const size_t ncols = gathered.getColumnCount();
    for (size_t i : order_indices_)
        if (i >= ncols)
            return Result<RowBatch>::failure("SortOperator: order index out of range");

    // the sort columns are sorted in place over next_pow2(n) rows: padded copies
    std::vector<Column> keys;
    std::vector<void*> key_ptrs;
    std::vector<uint32_t> key_types;
    std::vector<uint8_t> asc;
    for (size_t k = 0; k < order_indices_.size(); k++) {
        const Column& src = gathered.getColumn(order_indices_[k]);
        Column padded(context_, src.getType(), np);
        check(velo_copy(padded.rawData(), src.rawData(), n * type_size(src.getType()), VELO_COPY_D2D,
                        context_.stream()),
              "SortOperator");
        padded.setSize(n);
        key_ptrs.push_back(padded.rawData());
        key_types.push_back(src.getType());
        asc.push_back(ascending_flags_[k] ? 1 : 0);
        keys.push_back(std::move(padded));
    }
    std::shared_ptr<void> indices = device_alloc(context_, np * 8);
    const size_t sb = velo_sort_scratch_bytes(key_types.data(), (uint32_t)key_types.size(), n);
    std::shared_ptr<void> scratch = device_alloc(context_, sb);
    velo_cmd cmd;
    std::memset(&cmd, 0, sizeof cmd);
    cmd.opcode = VELO_OP_SORT;
    cmd.args.sort.d_cols = key_ptrs.data();
    cmd.args.sort.types = key_types.data();
    cmd.args.sort.ascending = asc.data();
    cmd.args.sort.n_cols = (uint32_t)key_ptrs.size();
    cmd.args.sort.n = n;
    cmd.args.sort.capacity = np;
    cmd.args.sort.d_indices = static_cast<int64_t*>(indices.get());
    cmd.args.sort.d_scratch = scratch.get();
    cmd.args.sort.scratch_bytes = sb;
    context_.sync(); // the padded copies are on the context stream, the command runs after them
    context_.run(cmd);

    // every column's validity and every non-key column's values follow the
    // sort's permutation (OP_PERMUTE, as src/operator/sort_operator.cpp:80-126)
    std::vector<Column> out;
    for (size_t c = 0; c < ncols; c++) {
        const Column& src = gathered.getColumn(c);
        const auto it = std::find(order_indices_.begin(), order_indices_.end(), c);
        Column dst = it != order_indices_.end() ? keys[it - order_indices_.begin()] : Column(context_, src.getType(), n);
        velo_cmd p;
        std::memset(&p, 0, sizeof p);
        p.opcode = VELO_OP_PERMUTE;
        p.args.permute.d_indices = static_cast<const int64_t*>(indices.get());
        p.args.permute.n = n;
        if (it == order_indices_.end()) {
            p.args.permute.d_out = dst.rawData();
            p.args.permute.d_in = src.rawData();
            p.args.permute.type = src.getType();
            context_.run(p);
        }
        if (src.rawBitmapData()) {
            p.args.permute.d_out = dst.rawBitmapData();
            p.args.permute.d_in = src.rawBitmapData();
            p.args.permute.type = VELO_BOOLEAN;
            context_.run(p);
        }
        dst.setSize(n);
        out.push_back(std::move(dst));
    }
    sorted_batch_ = RowBatch(std::move(out));
    sorted_batch_.setRowCount(n);
    current_offset_ = std::min(MAX_BATCH_SIZE, n);
    return Result<RowBatch>::success(sorted_batch_.slice(0, current_offset_));
}

// ---- joins -----------------------------------------------------------------

SortMergeJoinOperator::SortMergeJoinOperator(ExecutionContext& context, Schema output_schema,
                                             std::unique_ptr<AbstractOperator> left,
                                             std::unique_ptr<AbstractOperator> right,
                                             std::pair<size_t, size_t> join_key_indices, JoinType join_type)
    : BinaryOperator(context, std::move(output_schema), std::move(left), std::move(right))
    , join_key_indices_(join_key_indices)
    , join_type_(join_type)
{
}

Result<RowBatch> SortMergeJoinOperator::next()
{
    if (joined_)
        return Result<RowBatch>::success(RowBatch());
    return join({ -1, -1 }, false);
}

Result<RowBatch> SortMergeJoinOperator::join(std::pair<long, long> mask_indices, bool hashed)
{
    joined_ = true;
    if (join_type_ != JoinType::INNER)
        return Result<RowBatch>::failure("only INNER joins are supported");
    RowBatch left = collectBatches(*left_child_);
    if (left.getRowCount() == 0)
        return Result<RowBatch>::success(RowBatch());
    RowBatch right = collectBatches(*right_child_);
    if (right.getRowCount() == 0)
        return Result<RowBatch>::success(RowBatch());
    if (join_key_indices_.first >= left.getColumnCount())
        return Result<RowBatch>::failure("Left join key index out of bounds");
    if (join_key_indices_.second >= right.getColumnCount())
        return Result<RowBatch>::failure("Right join key index out of bounds");
    const Column& lk = left.getColumn(join_key_indices_.first);
    const Column& rk = right.getColumn(join_key_indices_.second);
    if (lk.getType() != rk.getType() || (lk.getType() != VELO_INTEGER && lk.getType() != VELO_BIGINT))
        return Result<RowBatch>::failure("join keys must both be INTEGER or both BIGINT");
    const size_t bn = left.getRowCount(), pn = right.getRowCount();
    const uint8_t* bmask = mask_indices.first >= 0
        ? static_cast<const uint8_t*>(left.getColumn((size_t)mask_indices.first).rawData())
        : nullptr;
    const uint8_t* pmask = mask_indices.second >= 0
        ? static_cast<const uint8_t*>(right.getColumn((size_t)mask_indices.second).rawData())
        : nullptr;
    std::shared_ptr<void> brow = device_alloc(context_, pn * 8), prow = device_alloc(context_, pn * 8);
    std::shared_ptr<void> counts = device_alloc(context_, 24);
    uint64_t hc[3] = { 0, 0, 0 };
    velo_cmd cmd;
    std::memset(&cmd, 0, sizeof cmd);
    if (hashed) {
        // the oblivious bin-padded hash join; a repeated build key or a bin
        // overflow sends the join to the many-to-many sort-merge join below
        const size_t sb = velo_ohash_join_scratch_bytes(bn, pn);
        std::shared_ptr<void> scratch = device_alloc(context_, sb);
        cmd.opcode = VELO_OP_OHASH_JOIN;
        cmd.args.ohash.d_build_keys = lk.rawData();
        cmd.args.ohash.d_build_mask = bmask;
        cmd.args.ohash.build_n = bn;
        cmd.args.ohash.d_probe_keys = rk.rawData();
        cmd.args.ohash.d_probe_mask = pmask;
        cmd.args.ohash.probe_n = pn;
        cmd.args.ohash.key_type = lk.getType();
        cmd.args.ohash.hash_seed = hash_seed_;
        cmd.args.ohash.d_out_build_rowid = static_cast<int64_t*>(brow.get());
        cmd.args.ohash.d_out_probe_rowid = static_cast<int64_t*>(prow.get());
        cmd.args.ohash.d_counts = static_cast<uint64_t*>(counts.get());
        cmd.args.ohash.d_scratch = scratch.get();
        cmd.args.ohash.scratch_bytes = sb;
        context_.run(cmd);
        check(velo_copy(hc, counts.get(), 24, VELO_COPY_D2H, context_.stream()), "join counts");
        context_.sync();
    } else {
        // the oblivious PK-FK join; a repeated build key sends the join to the
        // many-to-many join below
        const size_t sb = velo_ojoin_scratch_bytes(bn, pn);
        std::shared_ptr<void> scratch = device_alloc(context_, sb);
        cmd.opcode = VELO_OP_OJOIN_PKFK;
        cmd.args.ojoin.d_build_keys = lk.rawData();
        cmd.args.ojoin.d_build_mask = bmask;
        cmd.args.ojoin.build_n = bn;
        cmd.args.ojoin.d_probe_keys = rk.rawData();
        cmd.args.ojoin.d_probe_mask = pmask;
        cmd.args.ojoin.probe_n = pn;
        cmd.args.ojoin.key_type = lk.getType();
        cmd.args.ojoin.d_out_build_rowid = static_cast<int64_t*>(brow.get());
        cmd.args.ojoin.d_out_probe_rowid = static_cast<int64_t*>(prow.get());
        cmd.args.ojoin.d_counts = static_cast<uint64_t*>(counts.get());
        cmd.args.ojoin.d_scratch = scratch.get();
        cmd.args.ojoin.scratch_bytes = sb;
        context_.run(cmd);
        check(velo_copy(hc, counts.get(), 16, VELO_COPY_D2H, context_.stream()), "join counts");
        context_.sync();
    }
    if (hc[1] != 0 || hc[2] != 0) {
        // many-to-many: every pair, first bounded by the probe side; a larger
        // pair count (revealed, as the reference's SMJ count step does) sizes
        // a second run
        size_t bound = pn;
        for (int attempt = 0; attempt < 2; attempt++) {
            brow = device_alloc(context_, bound * 8);
            prow = device_alloc(context_, bound * 8);
            const size_t sb = velo_ojoin_mn_scratch_bytes(bn, pn, bound);
            std::shared_ptr<void> scratch = device_alloc(context_, sb);
            std::memset(&cmd, 0, sizeof cmd);
            cmd.opcode = VELO_OP_OJOIN_MN;
            cmd.args.ojoin_mn.d_build_keys = lk.rawData();
            cmd.args.ojoin_mn.d_build_mask = bmask;
            cmd.args.ojoin_mn.build_n = bn;
            cmd.args.ojoin_mn.d_probe_keys = rk.rawData();
            cmd.args.ojoin_mn.d_probe_mask = pmask;
            cmd.args.ojoin_mn.probe_n = pn;
            cmd.args.ojoin_mn.key_type = lk.getType();
            cmd.args.ojoin_mn.max_pairs = bound;
            cmd.args.ojoin_mn.d_out_build_rowid = static_cast<int64_t*>(brow.get());
            cmd.args.ojoin_mn.d_out_probe_rowid = static_cast<int64_t*>(prow.get());
            cmd.args.ojoin_mn.d_counts = static_cast<uint64_t*>(counts.get());
            cmd.args.ojoin_mn.d_scratch = scratch.get();
            cmd.args.ojoin_mn.scratch_bytes = sb;
            context_.run(cmd);
            check(velo_copy(hc, counts.get(), 16, VELO_COPY_D2H, context_.stream()), "join counts");
            context_.sync();
            if (hc[1] == 0)
                break;
            bound = (size_t)hc[0];
        }
    }
    const size_t pairs = (size_t)hc[0];
    std::vector<Column> out;
    auto gather_side = [&](RowBatch& side, const std::shared_ptr<void>& rowids) {
        for (size_t c = 0; c < side.getColumnCount(); c++) {
            const Column& src = side.getColumn(c);
            Column dst(context_, src.getType(), pairs);
            if (pairs) {
                velo_cmd p;
                std::memset(&p, 0, sizeof p);
                p.opcode = VELO_OP_PERMUTE;
                p.args.permute.d_indices = static_cast<const int64_t*>(rowids.get());
                p.args.permute.n = pairs;
                p.args.permute.d_out = dst.rawData();
                p.args.permute.d_in = src.rawData();
                p.args.permute.type = src.getType();
                context_.run(p);
                if (src.rawBitmapData()) {
                    p.args.permute.d_out = dst.rawBitmapData();
                    p.args.permute.d_in = src.rawBitmapData();
                    p.args.permute.type = VELO_BOOLEAN;
                    context_.run(p);
                }
            }
            dst.setSize(pairs);
            out.push_back(std::move(dst));
        }
    };
    gather_side(left, brow);
    gather_side(right, prow);
    RowBatch joined(std::move(out));
    joined.setRowCount(pairs);
    return Result<RowBatch>::success(std::move(joined));
}

HashJoinOperator::HashJoinOperator(ExecutionContext& context, Schema output_schema,
                                   std::unique_ptr<AbstractOperator> left, std::unique_ptr<AbstractOperator> right,
                                   std::pair<size_t, size_t> join_key_indices, std::pair<long, long> mask_indices,
                                   JoinType join_type)
    : SortMergeJoinOperator(context, std::move(output_schema), std::move(left), std::move(right), join_key_indices,
                            join_type)
    , mask_indices_(mask_indices)
{
    // the bin hash is keyed per operator, so bin assignments cannot be
    // chosen ahead by whoever supplies the keys
    std::random_device rd;
    hash_seed_ = ((uint64_t)rd() << 32) ^ (uint64_t)rd();
}

Result<RowBatch> HashJoinOperator::next()
{
    if (joined_)
        return Result<RowBatch>::success(RowBatch());
    return join(mask_indices_, true);
}

// ---- materialization ---------------------------------------------------------

MaterializationOperator::MaterializationOperator(ExecutionContext& context, Schema output_schema,
                                                 std::unique_ptr<AbstractOperator> child,
                                                 std::vector<ColumnMapping> mappings)
    : UnaryOperator(context, std::move(output_schema), std::move(child))
    , mappings_(std::move(mappings))
{
    if (mappings_.size() != output_schema_.getColumnCount())
        throw ExecutionError("MaterializationOperator: one mapping per output column");
    for (const auto& m : mappings_)
        if (!m.source_table || m.source_col_index >= m.source_table->columns.size())
            throw ExecutionError("MaterializationOperator: bad source column");
}

Result<RowBatch> MaterializationOperator::next()
{
    Result<RowBatch> r = child_->next();
    if (!r)
        return r;
    RowBatch& in = r.value();
    const size_t n = in.getRowCount();
    if (n == 0)
        return r;
    RowBatch out;
    for (const auto& m : mappings_) {
        if (m.rowid_input_index >= in.getColumnCount() || in.getColumn(m.rowid_input_index).getType() != VELO_BIGINT)
            return Result<RowBatch>::failure("MaterializationOperator: row-id input must be a BIGINT column");
        const Column& rid = in.getColumn(m.rowid_input_index);
        const Column& src = m.source_table->columns[m.source_col_index];
        const size_t tn = m.source_table->rows;
        Column dst(context_, src.getType(), n);
        const size_t sb = velo_ogather_column_scratch_bytes(tn, n);
        std::shared_ptr<void> scratch = device_alloc(context_, sb);
        check(velo_ogather_column(src.rawData(), src.getType(), src.rawBitmapData(), tn,
                                  static_cast<const int64_t*>(rid.rawData()), n, dst.rawData(), dst.rawBitmapData(),
                                  scratch.get(), sb, context_.stream()),
              "MaterializationOperator");
        context_.sync();
        dst.setSize(n);
        out.addColumn(std::move(dst));
    }
    out.setRowCount(n);
    return Result<RowBatch>::success(std::move(out));
}

// ---- aggregate ----------------------------------------------------------------

AggregateOperator::AggregateOperator(ExecutionContext& context, Schema output_schema,
                                     std::unique_ptr<AbstractOperator> child, size_t group_column,
                                     std::vector<AggregateSpec> aggregates, size_t group_bound)
    : UnaryOperator(context, std::move(output_schema), std::move(child))
    , group_column_(group_column)
    , aggregates_(std::move(aggregates))
    , group_bound_(group_bound)
{
    if (aggregates_.empty())
        throw ExecutionError("AggregateOperator: at least one aggregate");
    if (output_schema_.getColumnCount() != 1 + aggregates_.size())
        throw ExecutionError("AggregateOperator: output schema must be the key and one column per aggregate");
}

Result<RowBatch> AggregateOperator::next()
{
    if (done_)
        return Result<RowBatch>::success(RowBatch());
    done_ = true;
    RowBatch in = collectBatches(*child_);
    const size_t n = in.getRowCount();
    if (n == 0)
        return Result<RowBatch>::success(RowBatch());
    if (group_column_ >= in.getColumnCount())
        return Result<RowBatch>::failure("AggregateOperator: group column out of range");
    const Column& key = in.getColumn(group_column_);
    if (key.getType() != VELO_INTEGER && key.getType() != VELO_BIGINT)
        return Result<RowBatch>::failure("AggregateOperator: the group key must be INTEGER or BIGINT");
    const size_t bound = group_bound_ ? std::min(group_bound_, n) : n;
    // "$_mask" of the input, when there is one
    const uint8_t* mask = nullptr;
    for (size_t c = 0; c < in.getColumnCount() && c < child_->getOutputSchema().getColumnCount(); c++) {
        const std::string& nm = child_->getOutputSchema().getColumnInfo(c).name;
        if (nm == "$_mask" || (nm.size() > 7 && nm.compare(nm.size() - 7, 7, ".$_mask") == 0))
            mask = static_cast<const uint8_t*>(in.getColumn(c).rawData());
    }
    // SUM operands as int64 columns
    std::vector<std::shared_ptr<void>> wide(aggregates_.size());
    for (size_t a = 0; a < aggregates_.size(); a++) {
        if (aggregates_[a].kind != AggKind::SUM)
            continue;
        if (aggregates_[a].column >= in.getColumnCount())
            return Result<RowBatch>::failure("AggregateOperator: SUM column out of range");
        const Column& c = in.getColumn(aggregates_[a].column);
        wide[a] = device_alloc(context_, n * 8);
        check(velo_widen_i64(c.rawData(), c.getType(), n, static_cast<int64_t*>(wide[a].get()), context_.stream()),
              "AggregateOperator");
    }
    std::vector<Column> out;
    out.emplace_back(context_, VELO_BIGINT, bound);
    for (size_t a = 0; a < aggregates_.size(); a++)
        out.emplace_back(context_, VELO_BIGINT, bound);
    const size_t sb = velo_ogroupby_scratch_bytes(n);
    std::shared_ptr<void> scratch = device_alloc(context_, sb);
    std::shared_ptr<void> counts = device_alloc(context_, 16);
    std::shared_ptr<void> keys_tmp = device_alloc(context_, bound * 8);
    // one or two aggregates per call: the groups (and their order) are the
    // same in every call, so the key column is written by the first call only
    size_t a = 0;
    bool first = true;
    while (a < aggregates_.size()) {
        std::vector<size_t> take;
        bool with_count = false;
        std::vector<const int64_t*> sums;
        std::vector<int64_t*> outs;
        int64_t* out_count = nullptr;
        while (a < aggregates_.size() && take.size() < 2) {
            if (aggregates_[a].kind == AggKind::COUNT) {
                if (with_count)
                    break; // a second COUNT goes to the next call
                with_count = true;
                out_count = static_cast<int64_t*>(out[1 + a].rawData());
            } else {
                sums.push_back(static_cast<const int64_t*>(wide[a].get()));
                outs.push_back(static_cast<int64_t*>(out[1 + a].rawData()));
            }
            take.push_back(a);
            a++;
        }
        int64_t* keys_out = first ? static_cast<int64_t*>(out[0].rawData()) : static_cast<int64_t*>(keys_tmp.get());
        check(velo_ogroupby(key.rawData(), key.getType(), sums.data(), (uint32_t)sums.size(), with_count ? 1u : 0u,
                            mask, n, bound, keys_out, outs.data(), out_count, static_cast<uint64_t*>(counts.get()),
                            scratch.get(), sb, context_.stream()),
              "AggregateOperator");
        first = false;
    }
    uint64_t hc[2] = { 0, 0 };
    check(velo_copy(hc, counts.get(), 16, VELO_COPY_D2H, context_.stream()), "AggregateOperator");
    context_.sync();
    const size_t rows = std::min<size_t>((size_t)hc[0], bound);
    RowBatch batch(std::move(out));
    batch.setRowCount(rows);
    if (rows == 0)
        return Result<RowBatch>::success(RowBatch());
    return Result<RowBatch>::success(std::move(batch));
}

// ---- limit -----------------------------------------------------------------

LimitOperator::LimitOperator(ExecutionContext& context, Schema output_schema, std::unique_ptr<AbstractOperator> child,
                             size_t limit, size_t offset)
    : UnaryOperator(context, std::move(output_schema), std::move(child))
    , limit_(limit)
    , offset_(offset)
{
}

Result<RowBatch> LimitOperator::next()
{
    for (;;) {
        if (current_count_ >= limit_)
            return Result<RowBatch>::success(RowBatch());
        Result<RowBatch> r = child_->next();
        if (!r)
            return r;
        RowBatch& b = r.value();
        const size_t rows = b.getRowCount();
        if (rows == 0)
            return r;
        size_t skip = 0;
        if (skipped_count_ < offset_) {
            skip = std::min(offset_ - skipped_count_, rows);
            skipped_count_ += skip;
        }
        size_t take = rows - skip;
        if (current_count_ + take > limit_)
            take = limit_ - current_count_;
        if (take == 0)
            continue; // the whole batch was skipped by the offset
        current_count_ += take;
        return Result<RowBatch>::success(b.slice(skip, skip + take));
    }
}

// ---- execution engine ---------------------------------------------------------

Result<QueryResult> ExecutionEngine::executePlan(std::unique_ptr<AbstractOperator> root)
{
    if (!root)
        return Result<QueryResult>::failure("Cannot execute null plan");
    const auto t0 = std::chrono::steady_clock::now();
    QueryResult res;
    res.schema = root->getOutputSchema();
    for (;;) {
        Result<RowBatch> r = root->next();
        if (!r)
            return Result<QueryResult>::failure(r.error());
        RowBatch b = std::move(r).value();
        if (b.getRowCount() == 0)
            break;
        res.rows += b.getRowCount();
        res.batches.push_back(std::move(b));
    }
    context_.sync();
    last_rows_ = res.rows;
    last_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return Result<QueryResult>::success(std::move(res));
}

} // namespace velo_b200
