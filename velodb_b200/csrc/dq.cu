// Host side of the persistent command queue: planning of each command into a
// job (the same pipeline steps, scratch layouts and validation as the direct
// entry points), the host-mapped ring, launch and relaunch of the consumer
// kernel, and completion polling.  Job format and consumer: dq.cuh,
// dq_kernel.cu.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

#include "dq.cuh"
#include "dq_host.hpp"
#include "net_host.cuh"

namespace velo {

velo_status dq_launch(const DqParams& a, bool fresh, cudaStream_t stream, int* grid_out);

size_t compact_scratch_for(size_t capacity, int lt);

// ---- plans --------------------------------------------------------------------

DqPlan::DqPlan() : job_(new DqJob)
{
    std::memset(&job_->h, 0, sizeof(job_->h));
}

DqPlan::~DqPlan()
{
    delete job_;
}

uint32_t DqPlan::steps() const
{
    return job_->h.nsteps;
}

namespace {

// appends steps and argument blocks to a plan; a job that outgrows the limits
// is marked, and refused when it is published
class B {
public:
    explicit B(DqPlan& p) : p_(p), j_(p.job()) {}
    template <class A>
    uint32_t arg(const A& a)
    {
        static_assert(sizeof(A) <= (size_t)DQ_STEP_ARG_MAX, "argument block larger than the staging area");
        static_assert(std::is_trivially_copyable<A>::value, "argument blocks are plain data");
        const uint32_t off = (uint32_t)align_up(j_.h.arg_bytes, 16);
        if (off + sizeof(A) > (size_t)DQ_ARG_BYTES) {
            fail();
            return 0;
        }
        std::memcpy(j_.args + off, &a, sizeof(A));
        j_.h.arg_bytes = off + (uint32_t)sizeof(A);
        return off;
    }
    void step(uint32_t kind, uint64_t ntiles, uint32_t arg, NetPass pass = NetPass {})
    {
        const uint64_t items = j_.h.nitems;
        if (j_.h.nsteps >= (uint32_t)DQ_MAX_STEPS || ntiles == 0 || ntiles > DQ_MAX_ITEMS_PER_STEP
            || items + ntiles > 0xFFFFFFFFull) {
            fail();
            return;
        }
        j_.steps[j_.h.nsteps++] = DqStep { kind, (uint32_t)ntiles, (uint32_t)items, arg, pass };
        j_.h.nitems = (uint32_t)(items + ntiles);
    }
    // network passes over 2^g.logN rows in 2^lt-row tiles
    template <class R>
    void net(uint32_t kind, const typename R::Cols& c, const NetGeom& g, const uint32_t* prefix,
             const std::vector<NetPass>& passes, int lt)
    {
        DqNetArgs<R> a;
        std::memset(&a, 0, sizeof(a));
        a.c = c;
        a.g = g;
        a.prefix = prefix;
        const uint32_t off = arg(a);
        const uint64_t nt = g.logN > lt ? 1ull << (g.logN - lt) : 1ull;
        for (const NetPass& p : passes)
            step(kind, nt, off, p);
    }
    template <class R>
    void count(uint32_t kind, const typename R::Cols& c, size_t n, int lt, uint32_t* counts, uint64_t ntiles)
    {
        DqCountArgs<R> a;
        std::memset(&a, 0, sizeof(a));
        a.c = c;
        a.n = n;
        a.lt = lt;
        a.counts = counts;
        step(kind, ntiles, arg(a));
    }
    void scan(const uint32_t* counts, uint64_t ntiles, uint32_t* prefix, uint64_t* d_count)
    {
        DqScanArgs a {};
        a.counts = counts;
        a.prefix = prefix;
        a.d_count = d_count;
        a.ntiles = (int)ntiles;
        step(DQ_K_SCAN_TILES, 1, arg(a));
    }
    // an element-wise step over n elements (at least one item)
    void elem(uint32_t kind, const DqElemArgs& e, size_t n)
    {
        const uint64_t items = (n + DQ_ELEM_ITEM - 1) / DQ_ELEM_ITEM;
        step(kind, items ? items : 1, arg(e));
    }
    void fail() { p_.overflow(); }

private:
    DqPlan& p_;
    DqJob& j_;
};

DqElemArgs elem_args()
{
    DqElemArgs e;
    std::memset(&e, 0, sizeof(e));
    return e;
}

void set_words(B& b, uint64_t* out, uint64_t v, size_t n)
{
    DqElemArgs e = elem_args();
    e.out = out;
    e.key = v;
    e.n = n;
    b.elem(DQ_K_SET_WORDS, e, n);
}

} // namespace

void dq_plan_range_mask_i32(DqPlan& p, const int32_t* c, size_t n, int32_t lo, int32_t hi, uint8_t* m)
{
    B b(p);
    DqElemArgs e = elem_args();
    e.in = c;
    e.n = n;
    e.lo = lo;
    e.hi = hi;
    e.out = m;
    b.elem(DQ_K_RANGE_MASK_I32, e, n);
}

void dq_plan_range_mask_i64(DqPlan& p, const int64_t* c, size_t n, int64_t lo, int64_t hi, uint8_t* m)
{
    B b(p);
    DqElemArgs e = elem_args();
    e.in = c;
    e.n = n;
    e.lo = lo;
    e.hi = hi;
    e.out = m;
    b.elem(DQ_K_RANGE_MASK_I64, e, n);
}

void dq_plan_rowid_keys(DqPlan& p, const int64_t* rowid, size_t n, int64_t offset, int64_t* key, uint8_t* m)
{
    B b(p);
    DqElemArgs e = elem_args();
    e.in = rowid;
    e.n = n;
    e.lo = offset;
    e.out = key;
    e.idx = m;
    b.elem(DQ_K_ROWID_KEYS, e, n);
}

void dq_plan_rowid_rids(DqPlan& p, const int64_t* rowid, size_t n, uint32_t missing, uint32_t* rid)
{
    B b(p);
    DqElemArgs e = elem_args();
    e.in = rowid;
    e.n = n;
    e.value = missing;
    e.out = rid;
    b.elem(DQ_K_ROWID_RIDS, e, n);
}

void dq_plan_fill_u8(DqPlan& p, uint8_t* out, uint8_t v, size_t n)
{
    B b(p);
    DqElemArgs e = elem_args();
    e.out = out;
    e.value = v;
    e.n = n;
    b.elem(DQ_K_FILL_U8, e, n);
}

void dq_plan_set_words(DqPlan& p, uint64_t* out, uint64_t v, size_t n)
{
    B b(p);
    set_words(b, out, v, n);
}

void dq_plan_sum_u64(DqPlan& p, const uint64_t* v, size_t n, unsigned long long* out)
{
    B b(p);
    DqElemArgs e = elem_args();
    e.in = v;
    e.n = n;
    e.out = out;
    b.elem(DQ_K_SUM_U64, e, n);
}

void dq_plan_copy_words(DqPlan& p, const uint64_t* src, uint64_t* dst, uint32_t words)
{
    B b(p);
    DqCopyArgs a {};
    a.src = src;
    a.dst = dst;
    a.words = words;
    b.step(DQ_K_COPY_WORDS, 1, b.arg(a));
}

// ---- the oblivious pipelines ----------------------------------------------------

static velo_status plan_osort_kp(B& b, uint64_t* k, uint32_t* pay, size_t n, size_t capacity)
{
    if (n == 0)
        return VELO_OK;
    if (!k || !pay)
        return einval("velo_osort_kp: null buffer");
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);
    if (logN > MAX_LOGN)
        return einval("velo_osort_kp: n too large");
    if (capacity < np)
        return einval("velo_osort_kp: capacity must be >= next_pow2(n)");
    if (np == 1)
        return VELO_OK;
    std::vector<NetPass> passes;
    plan_sort(logN, DQ_LT, DQ_LT - 5, passes);
    b.net<RowKP>(DQ_K_SORT_KP, RowKP::Cols { k, pay }, NetGeom { n, logN, 0 }, nullptr, passes, DQ_LT);
    return VELO_OK;
}

static velo_status plan_ocompact_kpm(B& b, uint64_t* k, uint32_t* pay, uint8_t* m, size_t n, size_t capacity,
                                     uint64_t* d_count, void* d_scratch, size_t scratch_bytes)
{
    if (n == 0) {
        if (d_count)
            set_words(b, d_count, 0, 1);
        return VELO_OK;
    }
    if (!k || !pay || !m)
        return einval("velo_ocompact_kpm: null buffer");
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);
    if (logN > MAX_LOGN)
        return einval("velo_ocompact_kpm: n too large");
    if (capacity < np)
        return einval("velo_ocompact_kpm: capacity must be >= next_pow2(n)");
    const size_t need = compact_scratch_for(np, DQ_LT);
    if (!d_scratch || scratch_bytes < need) {
        set_error("velo_ocompact_kpm: scratch must hold velo_compact_scratch_bytes(capacity, NULL) bytes");
        return VELO_ENOMEM;
    }
    const uint64_t ntiles = logN > DQ_LT ? 1ull << (logN - DQ_LT) : 1;
    uint32_t* counts = static_cast<uint32_t*>(d_scratch);
    uint32_t* prefix = reinterpret_cast<uint32_t*>(static_cast<char*>(d_scratch) + align_up(ntiles * 4, 256));
    const RowKPM::Cols c { k, pay, m };
    b.count<RowKPM>(DQ_K_COUNT_KPM, c, n, DQ_LT, counts, ntiles);
    b.scan(counts, ntiles, prefix, d_count);
    std::vector<NetPass> passes;
    plan_compact(logN, DQ_LT, DQ_LT - 5, passes);
    b.net<RowKPM>(DQ_K_COMPACT_KPM, c, NetGeom { n, logN, 0 }, prefix, passes, DQ_LT);
    return VELO_OK;
}

velo_status dq_plan_filter_groupby(DqPlan& p, const velo_lineitem* cols, size_t n, const velo_lineitem_pred* pred,
                                   uint32_t group_bound, int64_t* d_out, uint64_t* d_counts, void* d_scratch,
                                   size_t scratch_bytes)
{
    B b(p);
    if (!cols || !pred || !d_out || !d_counts)
        return einval("velo_filter_groupby: null argument");
    if (group_bound == 0 || group_bound > SEG_MAX_G)
        return einval("velo_filter_groupby: group_bound must be 1..16");
    if (n == 0 || next_pow2(n) > ((size_t)1 << MAX_LOGN))
        return einval("velo_filter_groupby: n must be 1..2^31");
    if (!cols->qty || !cols->price || !cols->disc || !cols->tax || !cols->shipdate || !cols->flag1 || !cols->flag2)
        return einval("velo_filter_groupby: null column");
    const LiScratch s = li_layout(static_cast<char*>(d_scratch), n, group_bound);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_filter_groupby: scratch must hold velo_filter_groupby_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    const LiCols c { cols->qty, cols->price, cols->disc, cols->tax, cols->shipdate, cols->flag1, cols->flag2 };
    const LiParams prm { pred->qty_lo, pred->disc_lo, band_bits(pred->qty_lo, pred->qty_hi), 0 };
    const int W = prm.qbits + band_bits(pred->disc_lo, pred->disc_hi) <= (uint32_t)LI_FIELD_BITS ? 2 : 3;
    // two-word records in 4096-row tiles, three-word records in 2048-row tiles
    const int lt = W == 2 ? DQ_LT : DQ_LT3;
    const int lmax = lt - 4 < 8 ? lt - 4 : 8;
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);
    // 1. predicate + pack, per-tile pass counts, their scan
    DqLiPackArgs pk;
    std::memset(&pk, 0, sizeof(pk));
    pk.c = c;
    pk.p = *pred;
    pk.prm = prm;
    pk.n = n;
    pk.n_rec = s.n_rec;
    pk.lt = lt;
    for (int i = 0; i < 3; i++)
        pk.w[i] = s.w[i];
    pk.counts = s.counts;
    b.step(W == 2 ? DQ_K_LI_PACK2 : DQ_K_LI_PACK3, s.n_rec >> lt, b.arg(pk));
    const uint64_t ntiles_np = logN > lt ? 1ull << (logN - lt) : 1;
    b.scan(s.counts, ntiles_np, s.prefix, s.d_rows);
    // 2. ORCompact and 3. sort of the next_pow2(n) records
    std::vector<NetPass> cp, sp;
    plan_compact(logN, lt, lmax, cp);
    plan_sort(logN, lt, lmax, sp);
    const NetGeom g { np, logN, 0 };
    if (W == 2) {
        using R = LiTypes<2>::Rec;
        R::Cols rc;
        std::memset(&rc, 0, sizeof(rc));
        for (int i = 0; i < 2; i++) {
            rc.w[i] = s.w[i];
            rc.pad[i] = ~0ull;
        }
        rc.mask[0] = LI_KEYMASK;
        rc.mark_bit = 63;
        rc.mark_inv = 1;
        rc.mark_word = 0;
        b.net<R>(DQ_K_COMPACT_LI2, rc, g, s.prefix, cp, lt);
        if (logN > 0)
            b.net<R>(DQ_K_SORT_LI2, rc, g, nullptr, sp, lt);
    } else {
        using R = LiTypes<3>::Rec;
        R::Cols rc;
        std::memset(&rc, 0, sizeof(rc));
        for (int i = 0; i < 3; i++) {
            rc.w[i] = s.w[i];
            rc.pad[i] = ~0ull;
        }
        rc.mask[0] = LI_KEYMASK;
        rc.mark_bit = 63;
        rc.mark_inv = 1;
        rc.mark_word = 0;
        b.net<R>(DQ_K_COMPACT_LI3, rc, g, s.prefix, cp, lt);
        if (logN > 0)
            b.net<R>(DQ_K_SORT_LI3, rc, g, nullptr, sp, lt);
    }
    // 4. segmented sums with the public output bound
    size_t nseg = np < (size_t)SEG_TS ? (size_t)SEG_TS : np;
    DqSegArgs sg;
    std::memset(&sg, 0, sizeof(sg));
    for (int i = 0; i < 3; i++)
        sg.w[i] = s.w[i];
    sg.aggs = s.aggs;
    sg.runs = s.runs;
    sg.carry = s.carry;
    sg.tail_prefix = s.tail_prefix;
    sg.n_groups = s.n_groups;
    sg.tile_out = s.tile_out;
    sg.out = d_out;
    sg.d_rows = s.d_rows;
    sg.d_counts = d_counts;
    sg.prm = prm;
    sg.ntiles = (int)(nseg / SEG_TS);
    sg.G = (int)group_bound;
    const uint32_t sa = b.arg(sg);
    b.step(W == 2 ? DQ_K_SEG_SUMMARY2 : DQ_K_SEG_SUMMARY3, (uint64_t)sg.ntiles, sa);
    b.step(W == 2 ? DQ_K_SEG_CARRIES2 : DQ_K_SEG_CARRIES3, 1, sa);
    b.step(W == 2 ? DQ_K_SEG_EMIT2 : DQ_K_SEG_EMIT3, (uint64_t)sg.ntiles, sa);
    b.step(DQ_K_SEG_FINISH, (uint64_t)group_bound * (1 + LI_V), sa);
    return VELO_OK;
}

velo_status dq_plan_join_topk(DqPlan& p, const velo_join_tables* t, const velo_join_pred* pred, uint32_t k,
                              int64_t* d_out, uint64_t* d_counts, void* d_scratch, size_t scratch_bytes)
{
    B b(p);
    if (!t || !pred || !d_out || !d_counts)
        return einval("velo_join_groupby_topk: null argument");
    if (!t->dim_key || !t->dim_date || !t->fact_fk || !t->fact_price || t->n_dim == 0)
        return einval("velo_join_groupby_topk: null column or empty dimension table");
    if (k == 0 || k > 1024)
        return einval("velo_join_groupby_topk: k must be 1..1024");
    if (t->n_dim + t->n_fact > ((size_t)1 << MAX_LOGN))
        return einval("velo_join_groupby_topk: tables too large");
    const JoinScratch s = join_layout(static_cast<char*>(d_scratch), t->n_dim, t->n_fact);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_join_groupby_topk: scratch must hold velo_join_groupby_topk_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    const int logR = ilog2_floor(s.n_rec);
    const int logU = ilog2_floor(next_pow2(t->n_dim + t->n_fact));
    // 1. pack
    DqJoinPackArgs pk {};
    pk.dk = t->dim_key;
    pk.dd = t->dim_date;
    pk.ff = t->fact_fk;
    pk.fp = t->fact_price;
    pk.nd = t->n_dim;
    pk.nf = t->n_fact;
    pk.n_rec = s.n_rec;
    pk.date_hi = pred->date_hi;
    pk.price_hi = pred->price_hi;
    pk.w0 = s.u[0];
    pk.w1 = s.u[1];
    b.step(DQ_K_JOIN_PACK, (s.n_rec + DQ_ELEM_ITEM - 1) / DQ_ELEM_ITEM, b.arg(pk));
    JRec::Cols uc;
    std::memset(&uc, 0, sizeof(uc));
    uc.w[0] = s.u[0];
    uc.w[1] = s.u[1];
    uc.mask[0] = J_KEYTAG;
    uc.pad[0] = uc.pad[1] = ~0ull;
    uc.mark_bit = 29;
    uc.mark_inv = 0;
    uc.mark_word = 0;
    // 2. sort the union on (key, tag)
    if (logU > 0) {
        std::vector<NetPass> sp;
        plan_sort(logU, DQ_LT, J_LMAX, sp);
        b.net<JRec>(DQ_K_SORT_JREC, uc, NetGeom { (size_t)1 << logU, logU, 0 }, nullptr, sp, DQ_LT);
    }
    // 3. forward fill of the dimension side
    DqJFillArgs fa {};
    fa.w0 = s.u[0];
    fa.tile_last = s.tile_last;
    fa.carry = s.fcarry;
    fa.ntiles = (int)(s.n_rec / FILL_TS);
    const uint32_t fo = b.arg(fa);
    b.step(DQ_K_JFILL_SUMMARY, (uint64_t)fa.ntiles, fo);
    b.step(DQ_K_JFILL_CARRIES, 1, fo);
    b.step(DQ_K_JFILL_APPLY, (uint64_t)fa.ntiles, fo);
    // 4. ORCompact of the joined fact rows
    const uint64_t ntc = logR > DQ_LT ? 1ull << (logR - DQ_LT) : 1;
    b.count<JRec>(DQ_K_COUNT_JREC, uc, s.n_rec, DQ_LT, s.counts, ntc);
    b.scan(s.counts, ntc, s.prefix, s.n_joined);
    std::vector<NetPass> cp;
    plan_compact(logR, DQ_LT, J_LMAX, cp);
    b.net<JRec>(DQ_K_COMPACT_JREC, uc, NetGeom { s.n_rec, logR, 0 }, s.prefix, cp, DQ_LT);
    // 5. group-by fk fused with the first top-k round
    const int nts = (int)(s.n_rec / SEG_TS);
    const int cand = k <= (uint32_t)J_TOPK_MIN ? J_TOPK_MIN : (int)next_pow2(k);
    DqJSegArgs ja;
    std::memset(&ja, 0, sizeof(ja));
    ja.c = uc;
    ja.aggs = s.aggs;
    ja.runs = s.runs;
    ja.carry = s.carry;
    ja.tail_prefix = s.tail_prefix;
    ja.n_groups = s.n_groups;
    ja.out0 = s.cand[0];
    ja.out1 = s.cand[1];
    ja.ntiles = nts;
    ja.cand = cand;
    const uint32_t jo = b.arg(ja);
    b.step(DQ_K_JSEG_SUMMARY, (uint64_t)nts, jo);
    b.step(DQ_K_JSEG_CARRIES, 1, jo);
    b.step(DQ_K_JSEG_EMIT_TOPK, (uint64_t)nts, jo);
    // 6. top-k rounds over blocks of candidates (the union area is free now)
    uint64_t* cur[2] = { s.cand[0], s.cand[1] };
    uint64_t* nxt[2] = { s.u[0], s.u[1] };
    size_t n_c = (size_t)nts * cand;
    while (n_c > (size_t)cand) {
        const int rn = n_c < (size_t)TK_RED_ROWS ? (int)n_c : TK_RED_ROWS;
        const size_t blocks = n_c / rn;
        DqTopkArgs ta {};
        ta.in0 = cur[0];
        ta.in1 = cur[1];
        ta.out0 = nxt[0];
        ta.out1 = nxt[1];
        ta.rn = rn;
        ta.c = cand;
        b.step(DQ_K_TOPK_REDUCE, blocks, b.arg(ta));
        n_c = blocks * cand;
        std::swap(cur[0], nxt[0]);
        std::swap(cur[1], nxt[1]);
    }
    DqTopkArgs to {};
    to.in0 = cur[0];
    to.in1 = cur[1];
    to.k = k;
    to.out = d_out;
    to.n_groups = s.n_groups;
    to.n_joined = s.n_joined;
    to.d_counts = d_counts;
    b.step(DQ_K_TOPK_OUT, 1, b.arg(to));
    return VELO_OK;
}

// forward fill over a sorted union of 3-word records (fill.F = JoinFill or GatherFill)
static void plan_union_fill(B& b, uint32_t sum_kind, uint32_t apply_kind, const UnionScratch& s, size_t rows,
                            unsigned long long* d_stat)
{
    DqUFillArgs fa {};
    fa.w0 = s.w[0];
    fa.w1 = s.w[1];
    fa.w2 = s.w[2];
    fa.tl = s.tl;
    fa.carry = s.carry;
    fa.d_stat = d_stat;
    fa.ntiles = (int)(rows / FL_TS);
    const uint32_t off = b.arg(fa);
    b.step(sum_kind, (uint64_t)fa.ntiles, off);
    b.step(DQ_K_UFILL_SCAN, 1, off);
    b.step(apply_kind, (uint64_t)fa.ntiles, off);
}

velo_status dq_plan_ojoin_pkfk(DqPlan& p, const void* d_build_keys, const uint8_t* d_build_mask, size_t build_n,
                               const void* d_probe_keys, const uint8_t* d_probe_mask, size_t probe_n,
                               uint32_t key_type, int64_t* d_out_build_rowid, int64_t* d_out_probe_rowid,
                               uint64_t* d_counts, void* d_scratch, size_t scratch_bytes)
{
    B b(p);
    if (!d_counts)
        return einval("velo_ojoin_pkfk: null counts");
    if (key_type != VELO_INTEGER && key_type != VELO_BIGINT)
        return einval("velo_ojoin_pkfk: join keys must be INTEGER or BIGINT");
    if (probe_n == 0 || build_n == 0) {
        set_words(b, d_counts, 0, 2);
        if (probe_n) {
            set_words(b, reinterpret_cast<uint64_t*>(d_out_build_rowid), ~0ull, probe_n);
            set_words(b, reinterpret_cast<uint64_t*>(d_out_probe_rowid), ~0ull, probe_n);
        }
        return VELO_OK;
    }
    if (!d_build_keys || !d_probe_keys || !d_out_build_rowid || !d_out_probe_rowid)
        return einval("velo_ojoin_pkfk: null buffer");
    const size_t rows = union_rows(build_n + probe_n);
    const int logR = ilog2_floor(rows);
    if (logR > MAX_LOGN)
        return einval("velo_ojoin_pkfk: too large");
    const UnionScratch s = union_layout(static_cast<char*>(d_scratch), rows);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_ojoin_pkfk: scratch must hold velo_ojoin_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    set_words(b, reinterpret_cast<uint64_t*>(s.stat), 0, 1);
    DqOJoinArgs oa {};
    oa.bk = d_build_keys;
    oa.pk = d_probe_keys;
    oa.bm = d_build_mask;
    oa.pm = d_probe_mask;
    oa.bn = build_n;
    oa.pn = probe_n;
    oa.rows = rows;
    oa.key64 = key_type == VELO_BIGINT;
    oa.w0 = s.w[0];
    oa.w1 = s.w[1];
    oa.w2 = s.w[2];
    oa.ob = d_out_build_rowid;
    oa.op = d_out_probe_rowid;
    oa.n_joined = s.n_marked;
    oa.dups = s.stat;
    oa.d_counts = d_counts;
    const uint32_t oo = b.arg(oa);
    b.step(DQ_K_OJOIN_PACK, (rows + DQ_ELEM_ITEM - 1) / DQ_ELEM_ITEM, oo);
    Rec3K2::Cols c;
    std::memset(&c, 0, sizeof(c));
    for (int i = 0; i < 3; i++) {
        c.w[i] = s.w[i];
        c.pad[i] = ~0ull;
    }
    c.mask[0] = ~0ull;
    c.mask[1] = OJ_TAG;
    c.mark_word = 1;
    c.mark_bit = 61;
    c.mark_inv = 0;
    const NetGeom g { rows, logR, 0 };
    std::vector<NetPass> sp, cp;
    plan_sort(logR, DQ_LT3, DQ_LT3 - 5, sp);
    b.net<Rec3K2>(DQ_K_SORT_REC3K2, c, g, nullptr, sp, DQ_LT3);
    plan_union_fill(b, DQ_K_UFILL_SUM_JOIN, DQ_K_UFILL_APPLY_JOIN, s, rows, s.stat);
    const uint64_t nct = rows >> DQ_LT3;
    b.count<Rec3K2>(DQ_K_COUNT_REC3K2, c, rows, DQ_LT3, s.counts, nct);
    b.scan(s.counts, nct, s.prefix, s.n_marked);
    plan_compact(logR, DQ_LT3, DQ_LT3 - 5, cp);
    b.net<Rec3K2>(DQ_K_COMPACT_REC3K2, c, g, s.prefix, cp, DQ_LT3);
    b.step(DQ_K_OJOIN_OUT, (probe_n + DQ_ELEM_ITEM - 1) / DQ_ELEM_ITEM, oo);
    b.step(DQ_K_JOIN_COUNTS, 1, oo);
    return VELO_OK;
}

velo_status dq_plan_ogather(DqPlan& p, const uint64_t* d_table, size_t table_n, const uint32_t* d_rids, size_t n_req,
                            uint64_t* d_out, void* d_scratch, size_t scratch_bytes)
{
    B b(p);
    if (n_req == 0)
        return VELO_OK;
    if (!d_table || !d_rids || !d_out)
        return einval("velo_ogather_u64: null buffer");
    if (table_n >= 0xFFFFFFFFull || n_req >= 0xFFFFFFFFull)
        return einval("velo_ogather_u64: sizes must fit 32 bits");
    const size_t rows = union_rows(table_n + n_req);
    const int logR = ilog2_floor(rows);
    if (logR > MAX_LOGN)
        return einval("velo_ogather_u64: too large");
    const UnionScratch s = union_layout(static_cast<char*>(d_scratch), rows);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_ogather_u64: scratch must hold velo_ogather_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    DqOGatherArgs ga {};
    ga.table = d_table;
    ga.rids = d_rids;
    ga.tn = table_n;
    ga.rn = n_req;
    ga.rows = rows;
    ga.w0 = s.w[0];
    ga.w1 = s.w[1];
    ga.w2 = s.w[2];
    ga.out = d_out;
    const uint32_t go = b.arg(ga);
    b.step(DQ_K_OGATHER_PACK, (rows + DQ_ELEM_ITEM - 1) / DQ_ELEM_ITEM, go);
    Rec3::Cols c;
    std::memset(&c, 0, sizeof(c));
    for (int i = 0; i < 3; i++) {
        c.w[i] = s.w[i];
        c.pad[i] = ~0ull;
    }
    c.mask[0] = 0xFFFFFFFF80000000ull;
    c.mark_bit = 0;
    c.mark_inv = 0;
    c.mark_word = 0;
    const NetGeom g { rows, logR, 0 };
    std::vector<NetPass> sp;
    plan_sort(logR, DQ_LT3, DQ_LT3 - 5, sp);
    b.net<Rec3>(DQ_K_SORT_REC3, c, g, nullptr, sp, DQ_LT3);
    plan_union_fill(b, DQ_K_UFILL_SUM_GATHER, DQ_K_UFILL_APPLY_GATHER, s, rows, nullptr);
    c.mask[0] = ~0ull;
    b.net<Rec3>(DQ_K_SORT_REC3, c, g, nullptr, sp, DQ_LT3);
    b.step(DQ_K_OGATHER_OUT, (n_req + DQ_ELEM_ITEM - 1) / DQ_ELEM_ITEM, go);
    return VELO_OK;
}

// ---- the reference command set ---------------------------------------------------

static velo_status plan_elementwise(B& b, const velo_cmd& m)
{
    const auto& a = m.args;
    DqElemArgs e = elem_args();
    switch (m.opcode) {
    case VELO_OP_PERMUTE: {
        if (a.permute.n == 0)
            return VELO_OK;
        if (!a.permute.d_out || !a.permute.d_in || !a.permute.d_indices)
            return einval("velo_permute: null buffer");
        const int bytes = type_bytes(a.permute.type);
        if (bytes == 0)
            return einval("velo_permute: unsupported type");
        e.out = a.permute.d_out;
        e.in = a.permute.d_in;
        e.idx = a.permute.d_indices;
        e.n = a.permute.n;
        e.bytes = (uint32_t)bytes;
        b.elem(DQ_K_PERMUTE, e, e.n);
        return VELO_OK;
    }
    case VELO_OP_GATHER: {
        if (a.gather.n == 0)
            return VELO_OK;
        if (!a.gather.d_out || !a.gather.d_in || !a.gather.d_indices)
            return einval("velo_gather: null buffer");
        const int bytes = type_bytes(a.gather.type);
        if (bytes == 0)
            return einval("velo_gather: unsupported type");
        e.out = a.gather.d_out;
        e.in = a.gather.d_in;
        e.idx = a.gather.d_indices;
        e.mask = a.gather.d_mask;
        e.n = a.gather.n;
        e.bytes = (uint32_t)bytes;
        b.elem(DQ_K_GATHER, e, e.n);
        return VELO_OK;
    }
    case VELO_OP_COMPARE_EQ: {
        if (a.compare_eq.n == 0)
            return VELO_OK;
        if (!a.compare_eq.d_left || !a.compare_eq.d_right || !a.compare_eq.d_out_mask)
            return einval("velo_compare_eq: null buffer");
        e.in = a.compare_eq.d_left;
        e.in2 = a.compare_eq.d_right;
        e.out = a.compare_eq.d_out_mask;
        e.n = a.compare_eq.n;
        e.value = a.compare_eq.type;
        b.elem(DQ_K_COMPARE_EQ, e, e.n);
        return VELO_OK;
    }
    case VELO_OP_COMPOSE_POSITION_MAP: {
        if (a.compose.n == 0)
            return VELO_OK;
        if (!a.compose.d_old || !a.compose.d_sigma || !a.compose.d_new)
            return einval("velo_compose_position_map: null buffer");
        e.in = a.compose.d_old;
        e.idx = a.compose.d_sigma;
        e.out = a.compose.d_new;
        e.n = a.compose.n;
        b.elem(DQ_K_COMPOSE, e, e.n);
        return VELO_OK;
    }
    case VELO_OP_ENRICH_POSITIONS: {
        if (a.enrich.n == 0)
            return VELO_OK;
        if (!a.enrich.d_record_ids || !a.enrich.d_map || !a.enrich.d_out)
            return einval("velo_enrich_positions: null buffer");
        e.in = a.enrich.d_map;
        e.idx = a.enrich.d_record_ids;
        e.out = a.enrich.d_out;
        e.n = a.enrich.n;
        b.elem(DQ_K_COMPOSE, e, e.n);
        return VELO_OK;
    }
    case VELO_OP_SCATTER: {
        if (!a.scatter.d_count)
            return einval("velo_scatter: null count");
        const size_t n = a.scatter.n;
        if (n == 0) {
            set_words(b, a.scatter.d_count, 0, 1);
            return VELO_OK;
        }
        if (!a.scatter.d_mask || !a.scatter.d_out_indices)
            return einval("velo_scatter: null buffer");
        if (!a.scatter.d_scratch || a.scatter.scratch_bytes < velo_scatter_scratch_bytes(n)) {
            set_error("velo_scatter: scratch must hold velo_scatter_scratch_bytes(n) bytes");
            return VELO_ENOMEM;
        }
        const size_t nt = (n + (1 << SC_LT) - 1) >> SC_LT;
        uint32_t* counts = static_cast<uint32_t*>(a.scatter.d_scratch);
        uint32_t* prefix = reinterpret_cast<uint32_t*>(static_cast<char*>(a.scatter.d_scratch) + align_up(nt * 4, 256));
        e.mask = a.scatter.d_mask;
        e.n = n;
        e.out = counts;
        b.step(DQ_K_SCATTER_COUNT, nt, b.arg(e));
        b.scan(counts, nt, prefix, a.scatter.d_count);
        DqElemArgs w = elem_args();
        w.mask = a.scatter.d_mask;
        w.n = n;
        w.in = prefix;
        w.out = a.scatter.d_out_indices;
        b.step(DQ_K_SCATTER_WRITE, nt, b.arg(w));
        return VELO_OK;
    }
    default:
        return VELO_ENOTSUP;
    }
}

velo_status dq_plan_cmd(DqPlan& p, const velo_cmd& m)
{
    B b(p);
    const auto& a = m.args;
    switch (m.opcode) {
    case VELO_OP_NOP:
        return VELO_OK;
    case VELO_OP_PERMUTE:
    case VELO_OP_GATHER:
    case VELO_OP_COMPARE_EQ:
    case VELO_OP_COMPOSE_POSITION_MAP:
    case VELO_OP_ENRICH_POSITIONS:
    case VELO_OP_SCATTER:
        return plan_elementwise(b, m);
    case VELO_OP_OSORT_KP:
        return plan_osort_kp(b, a.osort_kp.d_keys, a.osort_kp.d_payload, a.osort_kp.n, a.osort_kp.capacity);
    case VELO_OP_OCOMPACT_KPM:
        return plan_ocompact_kpm(b, a.ocompact_kpm.d_keys, a.ocompact_kpm.d_payload, a.ocompact_kpm.d_marks,
                                 a.ocompact_kpm.n, a.ocompact_kpm.capacity, a.ocompact_kpm.d_count,
                                 a.ocompact_kpm.d_scratch, a.ocompact_kpm.scratch_bytes);
    case VELO_OP_OSHUFFLE: {
        const auto& s = a.oshuffle;
        if (s.n == 0)
            return VELO_OK;
        if (!s.d_map)
            return einval("velo_oshuffle_position_map: null map");
        const size_t np = next_pow2(s.n);
        if (np > ((size_t)1 << MAX_LOGN))
            return einval("velo_oshuffle_position_map: n too large");
        if (!s.d_scratch || s.scratch_bytes < velo_oshuffle_scratch_bytes(s.n)) {
            set_error("velo_oshuffle_position_map: scratch must hold velo_oshuffle_scratch_bytes(n) bytes");
            return VELO_ENOMEM;
        }
        uint64_t* k = static_cast<uint64_t*>(s.d_scratch);
        uint32_t* pay = reinterpret_cast<uint32_t*>(static_cast<char*>(s.d_scratch) + align_up(np * 8, 256));
        DqElemArgs e = elem_args();
        e.in = s.d_map;
        e.n = s.n;
        e.np = np;
        e.counter = s.counter;
        e.key = s.key;
        e.out = k;
        e.idx = pay;
        b.elem(DQ_K_SHUFFLE_PACK, e, np);
        velo_status rc = plan_osort_kp(b, k, pay, np, np);
        if (rc != VELO_OK)
            return rc;
        DqElemArgs c = elem_args();
        c.out = s.d_map;
        c.in = pay;
        c.n = s.n;
        b.elem(DQ_K_COPY_U32, c, s.n);
        return VELO_OK;
    }
    case VELO_OP_OJOIN_PKFK: {
        const auto& j = a.ojoin;
        return dq_plan_ojoin_pkfk(p, j.d_build_keys, j.d_build_mask, j.build_n, j.d_probe_keys, j.d_probe_mask,
                                  j.probe_n, j.key_type, j.d_out_build_rowid, j.d_out_probe_rowid, j.d_counts,
                                  j.d_scratch, j.scratch_bytes);
    }
    case VELO_OP_OGATHER: {
        const auto& g = a.ogather;
        return dq_plan_ogather(p, g.d_table, g.table_n, g.d_rids, g.n_req, g.d_out, g.d_scratch, g.scratch_bytes);
    }
    case VELO_OP_FILTER_GROUPBY: {
        const auto& f = a.filter_groupby;
        if (m.flags & VELO_REVEAL_COUNT)
            return einval("persistent queue: VELO_REVEAL_COUNT synchronises; call velo_filter_groupby directly");
        return dq_plan_filter_groupby(p, f.cols, f.n, f.pred, f.group_bound, f.d_out, f.d_counts, f.d_scratch,
                                      f.scratch_bytes);
    }
    case VELO_OP_JOIN_GROUPBY_TOPK: {
        const auto& j = a.join_topk;
        return dq_plan_join_topk(p, j.tables, j.pred, j.k, j.d_out, j.d_counts, j.d_scratch, j.scratch_bytes);
    }
    default:
        set_error("persistent queue: this opcode runs on the stream queue only (velo_init without "
                  "VELO_QUEUE_PERSISTENT)");
        return VELO_ENOTSUP;
    }
}

// ---- the queue ------------------------------------------------------------------

struct DqEngine {
    int device = 0;
    cudaStream_t stream = nullptr;
    DqState* d_st = nullptr;
    DqJob* d_table = nullptr;
    char* h_mem = nullptr; // pinned, mapped: control words, then the ring
    DqHostCtl* ctl = nullptr;
    DqJob* ring = nullptr;
    DqParams prm {};
    std::mutex mu;
    uint64_t next_seq = 1;     // seq of the next publication
    uint64_t retired_below = 1; // every job below is complete and its status recorded
    std::deque<std::pair<uint64_t, int>> failed; // retired jobs whose status was an error
    bool launched = false;
    uint64_t launches = 0;
};

namespace {

volatile DqHostCtl* vctl(DqEngine* e)
{
    return const_cast<volatile DqHostCtl*>(e->ctl);
}

// record completed jobs in order (mu held)
void retire(DqEngine* e)
{
    volatile DqHostCtl* c = vctl(e);
    while (e->retired_below < e->next_seq) {
        const int hs = (int)((e->retired_below - 1) % DQ_HOST_RING);
        if (c->done_seq[hs] != e->retired_below)
            break;
        std::atomic_thread_fence(std::memory_order_acquire);
        const int st = c->status[hs];
        if (st != VELO_OK) {
            e->failed.emplace_back(e->retired_below, st);
            if (e->failed.size() > 4096)
                e->failed.pop_front();
        }
        e->retired_below++;
    }
}

// (re)launch the consumer when it is not running and a job is pending (mu
// held).  The consumer writes the number of the launch that decided to exit
// into the control words, so no CUDA call is needed to see that it left; a
// relaunch queues behind the leaving grid on the same stream.
velo_status ensure_running(DqEngine* e)
{
    if (vctl(e)->fault)
        return VELO_OK;
    if (!e->launched) {
        int grid = 0;
        VELO_CUDA_TRY(cudaSetDevice(e->device), "cudaSetDevice");
        velo_status rc = dq_launch(e->prm, true, e->stream, &grid);
        if (rc != VELO_OK)
            return rc;
        e->launched = true;
        e->launches++;
        return VELO_OK;
    }
    if (vctl(e)->exited_launch != e->launches)
        return VELO_OK; // the current launch is running
    retire(e);
    if (e->retired_below >= e->next_seq)
        return VELO_OK; // nothing pending
    VELO_CUDA_TRY(cudaSetDevice(e->device), "cudaSetDevice");
    velo_status rc = dq_launch(e->prm, false, e->stream, nullptr);
    if (rc == VELO_OK)
        e->launches++;
    return rc;
}

} // namespace

velo_status dq_create(int device, uint32_t idle_us, DqEngine** out)
{
    if (!out)
        return einval("persistent queue: null output");
    *out = nullptr;
    std::unique_ptr<DqEngine> e(new DqEngine());
    e->device = device;
    VELO_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    VELO_CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaError_t err = cudaMalloc(&e->d_st, sizeof(DqState));
    if (err == cudaSuccess)
        err = cudaMalloc(&e->d_table, sizeof(DqJob) * DQ_DEV_RING);
    const size_t ctl_bytes = align_up(sizeof(DqHostCtl), 256);
    if (err == cudaSuccess)
        err = cudaHostAlloc(&e->h_mem, ctl_bytes + sizeof(DqJob) * DQ_HOST_RING, cudaHostAllocMapped);
    if (err != cudaSuccess) {
        if (e->d_st)
            cudaFree(e->d_st);
        if (e->d_table)
            cudaFree(e->d_table);
        cudaStreamDestroy(e->stream);
        return cuda_fail(err, "persistent queue allocation");
    }
    std::memset(e->h_mem, 0, ctl_bytes + sizeof(DqJob) * DQ_HOST_RING);
    e->ctl = reinterpret_cast<DqHostCtl*>(e->h_mem);
    e->ring = reinterpret_cast<DqJob*>(e->h_mem + ctl_bytes);
    void* d_h = nullptr;
    VELO_CUDA_TRY(cudaHostGetDevicePointer(&d_h, e->h_mem, 0), "cudaHostGetDevicePointer");
    e->prm.st = e->d_st;
    e->prm.table = e->d_table;
    e->prm.ctl = reinterpret_cast<DqHostCtl*>(d_h);
    e->prm.ring = reinterpret_cast<const DqJob*>(static_cast<char*>(d_h) + ctl_bytes);
    e->prm.wait_ns = 10ull * 1000 * 1000 * 1000;
    e->prm.idle_ns = (uint64_t)(idle_us ? idle_us : 1000) * 1000;
    *out = e.release();
    return VELO_OK;
}

velo_status dq_publish(DqEngine* e, DqPlan& p, uint64_t after, uint64_t* seq_out)
{
    if (!e)
        return einval("persistent queue: null queue");
    DqJob& j = p.job();
    if (!p.ok())
        return einval("persistent queue: the command needs more steps or argument space than one job holds");
    B b(p);
    if (j.h.nsteps == 0)
        b.step(DQ_K_NOP, 1, 0); // an empty command still completes as a job
    std::lock_guard<std::mutex> lock(e->mu);
    if (vctl(e)->fault) {
        set_error("persistent queue: the consumer stopped on an inconsistent job table");
        return VELO_ECUDA;
    }
    const uint64_t seq = e->next_seq;
    const int hs = (int)((seq - 1) % DQ_HOST_RING);
    // back-pressure: the ring slot's previous job must be complete (bounded)
    const auto t0 = std::chrono::steady_clock::now();
    while (seq > (uint64_t)DQ_HOST_RING && e->retired_below <= seq - DQ_HOST_RING) {
        velo_status rc = ensure_running(e);
        if (rc != VELO_OK)
            return rc;
        retire(e);
        if (e->retired_below > seq - DQ_HOST_RING)
            break;
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(10)) {
            set_error("persistent queue: ring full and nothing completed for 10 s");
            return VELO_ETIMEDOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    j.h.seq = seq;
    j.h.after = after;
    DqJob* dst = e->ring + hs;
    std::memcpy(&dst->h, &j.h, sizeof(DqJobHdr));
    std::memcpy(dst->steps, j.steps, sizeof(DqStep) * j.h.nsteps);
    std::memcpy(dst->args, j.args, j.h.arg_bytes);
    std::atomic_thread_fence(std::memory_order_seq_cst);
    vctl(e)->head = seq;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    e->next_seq = seq + 1;
    if (seq_out)
        *seq_out = seq;
    return ensure_running(e);
}

bool dq_poll(DqEngine* e, uint64_t seq, velo_status* status)
{
    std::lock_guard<std::mutex> lock(e->mu);
    if (seq >= e->retired_below && seq < e->next_seq) {
        // jobs complete out of order: read the job's own ring slot, which is
        // not reused before the job is retired
        const int hs = (int)((seq - 1) % DQ_HOST_RING);
        if (vctl(e)->done_seq[hs] == seq) {
            std::atomic_thread_fence(std::memory_order_acquire);
            if (status)
                *status = (velo_status)vctl(e)->status[hs];
            return true;
        }
    }
    retire(e);
    if (seq < e->retired_below) {
        velo_status st = VELO_OK;
        for (const auto& f : e->failed)
            if (f.first == seq)
                st = (velo_status)f.second;
        if (status)
            *status = st;
        return true;
    }
    if (vctl(e)->fault) {
        if (status)
            *status = VELO_ECUDA;
        return true;
    }
    const velo_status rc = ensure_running(e);
    if (rc != VELO_OK) {
        if (status)
            *status = rc;
        return true;
    }
    return false;
}

velo_status dq_wait(DqEngine* e, uint64_t seq, uint64_t timeout_ns)
{
    if (!e)
        return einval("persistent queue: null queue");
    {
        std::lock_guard<std::mutex> lock(e->mu);
        if (seq == 0 || seq >= e->next_seq)
            return einval("velo_wait: unknown ticket");
    }
    const auto t0 = std::chrono::steady_clock::now();
    int spins = 0;
    for (;;) {
        velo_status st = VELO_OK;
        if (dq_poll(e, seq, &st)) {
            if (st == VELO_ETIMEDOUT)
                set_error("velo_wait: a device-side wait of the job ran out of time");
            else if (st == VELO_ECUDA)
                set_error("velo_wait: the persistent queue stopped on an inconsistent job table");
            else if (st != VELO_OK)
                set_error("velo_wait: the job failed");
            return st;
        }
        if ((uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0)
                .count()
            > timeout_ns) {
            set_error("velo_wait: ticket not complete at the time limit");
            return VELO_ETIMEDOUT;
        }
        if (spins++ < 2000)
            std::this_thread::yield();
        else
            std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

velo_status dq_destroy(DqEngine* e, uint32_t timeout_ms)
{
    if (!e)
        return VELO_OK;
    {
        std::lock_guard<std::mutex> lock(e->mu);
        vctl(e)->stop = 1;
        std::atomic_thread_fence(std::memory_order_seq_cst);
    }
    const auto t0 = std::chrono::steady_clock::now();
    velo_status rc = VELO_OK;
    for (;;) {
        {
            std::lock_guard<std::mutex> lock(e->mu);
            // pending jobs need a running consumer to finish
            rc = ensure_running(e);
            if (rc != VELO_OK)
                break;
            const cudaError_t q = cudaStreamQuery(e->stream);
            retire(e);
            if (q == cudaSuccess && e->retired_below >= e->next_seq)
                break;
            if (q != cudaSuccess && q != cudaErrorNotReady) {
                rc = cuda_fail(q, "velo_shutdown");
                break;
            }
            if (vctl(e)->fault && q == cudaSuccess)
                break;
        }
        if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms)) {
            set_error("velo_shutdown: persistent queue still running at the time limit");
            rc = VELO_ETIMEDOUT;
            break;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    if (rc == VELO_OK) {
        cudaFree(e->d_st);
        cudaFree(e->d_table);
        cudaFreeHost(e->h_mem);
        cudaStreamDestroy(e->stream);
        delete e;
    }
    // on a timeout the queue's memory stays allocated: the consumer may still
    // read it
    return rc;
}

void* dq_stream(DqEngine* e)
{
    return e ? (void*)e->stream : nullptr;
}

uint64_t dq_launches(DqEngine* e)
{
    if (!e)
        return 0;
    std::lock_guard<std::mutex> lock(e->mu);
    return e->launches;
}

} // namespace velo
