// Serving layer: a request loop with continuous admission over resident
// tables.
//
// Queries arrive at any time (velo_server_submit, thread-safe).  A scheduler
// thread admits them in arrival order as soon as an execution slot (a CUDA
// stream) is free AND the query's device scratch fits in the HBM budget --
// one arena allocated once at start, carved per query by a first-fit
// allocator, never cudaMalloc on the request path.  Admitted queries run
// concurrently on their own streams, so their kernels overlap on the device;
// when a query's completion event fires, its scratch and slot are released
// and the next waiting query is admitted.  Every wait is bounded.  Tables
// stay resident on the device for the server's lifetime.
//
// With VELO_SERVE_PERSISTENT the admitted queries run as jobs of one
// persistent command queue (dq.cu) instead of on per-slot streams: each query
// is planned into one job whose last steps copy its result words into the
// slot's mapped host buffer, and the loop polls the jobs' completion words.
//
// The reference has no serving layer: ExecutionEngine::executeQuery runs one
// query at a time on the caller's thread (src/execution/execution_engine.cpp:
// 67-142) and the persistent kernel serialises all commands.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.hpp"
#include "dq_host.hpp"
#include "ops.cuh"

namespace velo {

// ---- small kernels used by the three-way join chain (bodies in ops.cuh) ------

__global__ void k_range_mask_i32(const int32_t* c, size_t n, int32_t lo, int32_t hi, uint8_t* m)
{
    range_mask_body(c, n, lo, hi, m, blockIdx.x, gridDim.x);
}

__global__ void k_range_mask_i64(const int64_t* c, size_t n, int64_t lo, int64_t hi, uint8_t* m)
{
    range_mask_body(c, n, lo, hi, m, blockIdx.x, gridDim.x);
}

__global__ void k_rowid_keys(const int64_t* rowid, size_t n, int64_t offset, int64_t* key, uint8_t* m)
{
    rowid_keys_body(rowid, n, offset, key, m, blockIdx.x, gridDim.x);
}

__global__ void k_rowid_rids(const int64_t* rowid, size_t n, uint32_t missing, uint32_t* rid)
{
    rowid_rids_body(rowid, n, missing, rid, blockIdx.x, gridDim.x);
}

__global__ void k_sum_u64(const uint64_t* v, size_t n, unsigned long long* out)
{
    __shared__ unsigned long long s[32];
    sum_u64_body(v, n, out, blockIdx.x, gridDim.x, s);
}

static unsigned grid_n(size_t n)
{
    const size_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 8 ? (b ? b : 1) : 148 * 8);
}

// ---- first-fit arena -------------------------------------------------------

class Arena {
public:
    velo_status init(size_t bytes)
    {
        VELO_CUDA_TRY(cudaMalloc(&base_, bytes), "cudaMalloc(serving arena)");
        size_ = bytes;
        free_[0] = bytes;
        return VELO_OK;
    }
    ~Arena()
    {
        if (base_)
            cudaFree(base_);
    }
    // returns nullptr when no hole is large enough
    char* alloc(size_t bytes)
    {
        bytes = align_up(bytes ? bytes : 1, 256);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                const size_t off = it->first, rem = it->second - bytes;
                free_.erase(it);
                if (rem)
                    free_[off + bytes] = rem;
                used_[off] = bytes;
                in_use_ += bytes;
                return base_ + off;
            }
        }
        return nullptr;
    }
    void release(char* p)
    {
        const size_t off = (size_t)(p - base_);
        auto u = used_.find(off);
        if (u == used_.end())
            return;
        size_t start = off, len = u->second;
        in_use_ -= len;
        used_.erase(u);
        auto next = free_.lower_bound(start);
        if (next != free_.end() && next->first == start + len) {
            len += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == start) {
                start = prev->first;
                len += prev->second;
                free_.erase(prev);
            }
        }
        free_[start] = len;
    }
    size_t size() const { return size_; }
    size_t in_use() const { return in_use_; }

private:
    char* base_ = nullptr;
    size_t size_ = 0, in_use_ = 0;
    std::map<size_t, size_t> free_; // offset -> length
    std::map<size_t, size_t> used_;
};

using Clock = std::chrono::steady_clock;

struct Query {
    uint64_t id;
    velo_query q;
    Clock::time_point submit, start, end;
    int slot = -1;
    char* scratch = nullptr;
    size_t need = 0;
    velo_query_result res {};
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    int64_t* h_out = nullptr; // pinned, mapped result staging: 96 int64 + 2 u64
    int64_t* d_out_h = nullptr; // device address of h_out
    uint64_t job = 0;           // persistent mode: the query's job
    Query* q = nullptr;
};

} // namespace velo

using namespace velo;

struct velo_server {
    velo_server_config cfg {};
    velo_served_tables t {};
    Arena arena;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Query*> pending;
    std::unordered_map<uint64_t, Query*> all;
    uint64_t next_id = 1;
    std::atomic<bool> stop { false };
    std::thread loop;
    Clock::time_point t0 = Clock::now();
    uint64_t admitted = 0, completed = 0, peak_inflight = 0;
    size_t peak_arena = 0;
    velo::DqEngine* dq = nullptr; // VELO_SERVE_PERSISTENT
};

namespace velo {

static double ms_since(const velo_server* s, Clock::time_point t)
{
    return std::chrono::duration<double, std::milli>(t - s->t0).count();
}

// device scratch a query needs (all of it comes from the arena)
static size_t query_need(const velo_server* s, const velo_query& q)
{
    const size_t out = 4096;
    switch (q.shape) {
    case VELO_Q_FILTER_GROUPBY:
        return velo_filter_groupby_scratch_bytes(q.n, 8) + out;
    case VELO_Q_JOIN_TOPK:
        return velo_join_groupby_topk_scratch_bytes(q.dim_n, q.n) + out;
    case VELO_Q_JOIN3: {
        const size_t j1 = velo_ojoin_scratch_bytes(q.dim_n, q.n);
        const size_t j2 = velo_ojoin_scratch_bytes(q.n, q.f2_n);
        const size_t g = velo_ogather_scratch_bytes(q.f2_n, q.f2_n);
        const size_t mid = align_up(q.dim_n, 256) + align_up(q.n, 256) + 2 * align_up(q.n * 8, 256) // masks, J1
                           + align_up(q.n * 8, 256) + align_up(q.n, 256) + align_up(q.f2_n, 256)       // keys, masks
                           + 2 * align_up(q.f2_n * 8, 256) + align_up(q.f2_n * 4, 256)                  // J2, rids
                           + align_up(q.f2_n * 8, 256);                                                  // gathered
        size_t mx = j1 > j2 ? j1 : j2;
        mx = mx > g ? mx : g;
        return mid + mx + out;
    }
    default:
        return 0;
    }
}

static bool query_valid(const velo_server* s, const velo_query& q)
{
    const velo_served_tables& t = s->t;
    switch (q.shape) {
    case VELO_Q_FILTER_GROUPBY:
        return q.n > 0 && q.offset + q.n <= t.fact_n;
    case VELO_Q_JOIN_TOPK:
        return q.n > 0 && q.dim_n > 0 && q.offset + q.n <= t.fact_n && q.dim_offset + q.dim_n <= t.dim_n;
    case VELO_Q_JOIN3:
        return q.n > 0 && q.dim_n > 0 && q.f2_n > 0 && q.offset + q.n <= t.fact_n && q.dim_offset + q.dim_n <= t.dim_n
            && q.f2_offset + q.f2_n <= t.fact2_n && q.f2_n < 0xFFFFFFFFull;
    default:
        return false;
    }
}

// plans a query's whole pipeline as one job of the persistent queue; its
// last steps copy the result words into the slot's mapped host buffer
static velo_status launch_query_dq(velo_server* s, Query* qq, Slot& sl)
{
    const velo_query& q = qq->q;
    const velo_served_tables& t = s->t;
    char* p = qq->scratch;
    std::memset(sl.h_out, 0, 100 * sizeof(int64_t));
    auto take = [&](size_t b) {
        char* r = p;
        p += align_up(b ? b : 1, 256);
        return r;
    };
    int64_t* d_out = reinterpret_cast<int64_t*>(take(96 * 8));
    uint64_t* d_counts = reinterpret_cast<uint64_t*>(take(16));
    DqPlan plan;
    velo_status rc = VELO_OK;
    uint32_t out_words = 0;
    if (q.shape == VELO_Q_FILTER_GROUPBY) {
        velo_lineitem c = t.fact;
        c.qty += q.offset;
        c.price += q.offset;
        c.disc += q.offset;
        c.tax += q.offset;
        c.shipdate += q.offset;
        c.flag1 += q.offset;
        c.flag2 += q.offset;
        const size_t nb = velo_filter_groupby_scratch_bytes(q.n, 8);
        rc = dq_plan_filter_groupby(plan, &c, q.n, &q.pred, 8, d_out, d_counts, take(nb), nb);
        out_words = 8 * 6;
    } else if (q.shape == VELO_Q_JOIN_TOPK) {
        velo_join_tables jt { t.dim_key32 + q.dim_offset, t.dim_date + q.dim_offset, q.dim_n,
                              t.fact_fk32 + q.offset, t.fact.price + q.offset, q.n };
        const size_t nb = velo_join_groupby_topk_scratch_bytes(q.dim_n, q.n);
        rc = dq_plan_join_topk(plan, &jt, &q.jpred, 10, d_out, d_counts, take(nb), nb);
        out_words = 10 * 3;
    } else {
        // three-way chain dim <- fact <- fact2, as on the stream path
        uint8_t* dmask = reinterpret_cast<uint8_t*>(take(q.dim_n));
        uint8_t* fmask = reinterpret_cast<uint8_t*>(take(q.n));
        int64_t* j1b = reinterpret_cast<int64_t*>(take(q.n * 8));
        int64_t* j1p = reinterpret_cast<int64_t*>(take(q.n * 8));
        int64_t* fkey = reinterpret_cast<int64_t*>(take(q.n * 8));
        uint8_t* fkmask = reinterpret_cast<uint8_t*>(take(q.n));
        uint8_t* f2mask = reinterpret_cast<uint8_t*>(take(q.f2_n));
        int64_t* j2b = reinterpret_cast<int64_t*>(take(q.f2_n * 8));
        int64_t* j2p = reinterpret_cast<int64_t*>(take(q.f2_n * 8));
        uint32_t* rids = reinterpret_cast<uint32_t*>(take(q.f2_n * 4));
        uint64_t* vals = reinterpret_cast<uint64_t*>(take(q.f2_n * 8));
        const size_t j1n = velo_ojoin_scratch_bytes(q.dim_n, q.n), j2n = velo_ojoin_scratch_bytes(q.n, q.f2_n),
                     gn = velo_ogather_scratch_bytes(q.f2_n, q.f2_n);
        size_t mx = j1n > j2n ? j1n : j2n;
        mx = mx > gn ? mx : gn;
        char* sc = take(mx);
        dq_plan_range_mask_i32(plan, t.dim_date + q.dim_offset, q.dim_n, INT32_MIN, q.jpred.date_hi - 1, dmask);
        dq_plan_range_mask_i64(plan, t.fact.price + q.offset, q.n, INT64_MIN, q.jpred.price_hi - 1, fmask);
        rc = dq_plan_ojoin_pkfk(plan, t.dim_key + q.dim_offset, dmask, q.dim_n, t.fact_fk + q.offset, fmask, q.n,
                                VELO_BIGINT, j1b, j1p, d_counts, sc, mx);
        if (rc == VELO_OK) {
            dq_plan_rowid_keys(plan, j1p, q.n, (int64_t)q.offset, fkey, fkmask);
            dq_plan_fill_u8(plan, f2mask, 1, q.f2_n);
            rc = dq_plan_ojoin_pkfk(plan, fkey, fkmask, q.n, t.fact2_fk + q.f2_offset, f2mask, q.f2_n, VELO_BIGINT,
                                    j2b, j2p, d_counts, sc, mx);
        }
        if (rc == VELO_OK) {
            dq_plan_rowid_rids(plan, j2p, q.f2_n, (uint32_t)q.f2_n, rids);
            rc = dq_plan_ogather(plan, reinterpret_cast<const uint64_t*>(t.fact2_price + q.f2_offset), q.f2_n, rids,
                                 q.f2_n, vals, sc, mx);
        }
        if (rc == VELO_OK) {
            dq_plan_set_words(plan, reinterpret_cast<uint64_t*>(d_out), 0, 1);
            dq_plan_sum_u64(plan, vals, q.f2_n, reinterpret_cast<unsigned long long*>(d_out));
        }
        out_words = 1;
    }
    if (rc != VELO_OK)
        return rc;
    dq_plan_copy_words(plan, reinterpret_cast<const uint64_t*>(d_out), reinterpret_cast<uint64_t*>(sl.d_out_h),
                       out_words);
    dq_plan_copy_words(plan, d_counts, reinterpret_cast<uint64_t*>(sl.d_out_h + 96), 2);
    return dq_publish(s->dq, plan, 0, &sl.job);
}

// enqueues a query's whole pipeline on its slot's stream
static velo_status launch_query(velo_server* s, Query* qq, Slot& sl)
{
    if (s->dq)
        return launch_query_dq(s, qq, sl);
    const velo_query& q = qq->q;
    const velo_served_tables& t = s->t;
    cudaStream_t st = sl.stream;
    char* p = qq->scratch;
    // the slot's staging buffer is idle (its last copy completed before the
    // slot was released): clear it so words a shape does not write read 0
    std::memset(sl.h_out, 0, 100 * sizeof(int64_t));
    auto take = [&](size_t b) {
        char* r = p;
        p += align_up(b ? b : 1, 256);
        return r;
    };
    int64_t* d_out = reinterpret_cast<int64_t*>(take(96 * 8));
    uint64_t* d_counts = reinterpret_cast<uint64_t*>(take(16));
    velo_status rc = VELO_OK;
    size_t out_words = 0;
    if (q.shape == VELO_Q_FILTER_GROUPBY) {
        velo_lineitem c = t.fact;
        c.qty += q.offset;
        c.price += q.offset;
        c.disc += q.offset;
        c.tax += q.offset;
        c.shipdate += q.offset;
        c.flag1 += q.offset;
        c.flag2 += q.offset;
        const size_t nb = velo_filter_groupby_scratch_bytes(q.n, 8);
        rc = velo_filter_groupby(&c, q.n, &q.pred, 8, 0, d_out, d_counts, take(nb), nb, st);
        out_words = 8 * 6;
    } else if (q.shape == VELO_Q_JOIN_TOPK) {
        velo_join_tables jt { t.dim_key32 + q.dim_offset, t.dim_date + q.dim_offset, q.dim_n,
                              t.fact_fk32 + q.offset, t.fact.price + q.offset, q.n };
        const size_t nb = velo_join_groupby_topk_scratch_bytes(q.dim_n, q.n);
        rc = velo_join_groupby_topk(&jt, &q.jpred, 10, d_out, d_counts, take(nb), nb, st);
        out_words = 10 * 3;
    } else {
        // three-way chain: dim <- fact <- fact2
        uint8_t* dmask = reinterpret_cast<uint8_t*>(take(q.dim_n));
        uint8_t* fmask = reinterpret_cast<uint8_t*>(take(q.n));
        int64_t* j1b = reinterpret_cast<int64_t*>(take(q.n * 8));
        int64_t* j1p = reinterpret_cast<int64_t*>(take(q.n * 8));
        int64_t* fkey = reinterpret_cast<int64_t*>(take(q.n * 8));
        uint8_t* fkmask = reinterpret_cast<uint8_t*>(take(q.n));
        uint8_t* f2mask = reinterpret_cast<uint8_t*>(take(q.f2_n));
        int64_t* j2b = reinterpret_cast<int64_t*>(take(q.f2_n * 8));
        int64_t* j2p = reinterpret_cast<int64_t*>(take(q.f2_n * 8));
        uint32_t* rids = reinterpret_cast<uint32_t*>(take(q.f2_n * 4));
        uint64_t* vals = reinterpret_cast<uint64_t*>(take(q.f2_n * 8));
        const size_t j1n = velo_ojoin_scratch_bytes(q.dim_n, q.n), j2n = velo_ojoin_scratch_bytes(q.n, q.f2_n),
                     gn = velo_ogather_scratch_bytes(q.f2_n, q.f2_n);
        size_t mx = j1n > j2n ? j1n : j2n;
        mx = mx > gn ? mx : gn;
        char* sc = take(mx);
        k_range_mask_i32<<<grid_n(q.dim_n), 256, 0, st>>>(t.dim_date + q.dim_offset, q.dim_n, INT32_MIN,
                                                           q.jpred.date_hi - 1, dmask);
        k_range_mask_i64<<<grid_n(q.n), 256, 0, st>>>(t.fact.price + q.offset, q.n, INT64_MIN, q.jpred.price_hi - 1,
                                                       fmask);
        rc = velo_ojoin_pkfk(t.dim_key + q.dim_offset, dmask, q.dim_n, t.fact_fk + q.offset, fmask, q.n, VELO_BIGINT,
                             j1b, j1p, d_counts, sc, mx, st);
        if (rc == VELO_OK) {
            // fact rows of the first join become the build side (key = global fact row id)
            k_rowid_keys<<<grid_n(q.n), 256, 0, st>>>(j1p, q.n, (int64_t)q.offset, fkey, fkmask);
            cudaMemsetAsync(f2mask, 1, q.f2_n, st);
            rc = velo_ojoin_pkfk(fkey, fkmask, q.n, t.fact2_fk + q.f2_offset, f2mask, q.f2_n, VELO_BIGINT, j2b, j2p,
                                 d_counts, sc, mx, st);
        }
        if (rc == VELO_OK) {
            // sum of fact2.price over the joined fact2 rows, gathered obliviously
            k_rowid_rids<<<grid_n(q.f2_n), 256, 0, st>>>(j2p, q.f2_n, (uint32_t)q.f2_n, rids);
            rc = velo_ogather_u64(reinterpret_cast<const uint64_t*>(t.fact2_price + q.f2_offset), q.f2_n, rids, q.f2_n,
                                  vals, sc, mx, st);
        }
        if (rc == VELO_OK) {
            cudaMemsetAsync(d_out, 0, 8, st);
            k_sum_u64<<<grid_n(q.f2_n), 256, 0, st>>>(vals, q.f2_n, reinterpret_cast<unsigned long long*>(d_out));
            VELO_CUDA_TRY(cudaGetLastError(), "join3 kernels");
        }
        out_words = 1;
    }
    if (rc != VELO_OK)
        return rc;
    VELO_CUDA_TRY(cudaMemcpyAsync(sl.h_out, d_out, out_words * 8, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    VELO_CUDA_TRY(cudaMemcpyAsync(sl.h_out + 96, d_counts, 16, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    VELO_CUDA_TRY(cudaEventRecord(sl.done, st), "cudaEventRecord");
    return VELO_OK;
}

static void finish(velo_server* s, Query* q, int status)
{
    Slot& sl = s->slots[q->slot];
    q->end = Clock::now();
    q->res.status = status;
    if (status == VELO_OK) {
        std::memcpy(q->res.out, sl.h_out, sizeof(q->res.out));
        std::memcpy(q->res.counts, sl.h_out + 96, sizeof(q->res.counts));
    }
    q->res.submit_ms = ms_since(s, q->submit);
    q->res.start_ms = ms_since(s, q->start);
    q->res.end_ms = ms_since(s, q->end);
    s->arena.release(q->scratch);
    q->scratch = nullptr;
    sl.q = nullptr;
    q->slot = -1;
    s->completed++;
}

static void serve(velo_server* s)
{
    cudaSetDevice(s->cfg.device);
    while (true) {
        bool idle = true;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            // completions
            for (size_t i = 0; i < s->slots.size(); i++) {
                Slot& sl = s->slots[i];
                if (!sl.q)
                    continue;
                if (s->dq) {
                    velo_status st = VELO_OK;
                    if (!dq_poll(s->dq, sl.job, &st))
                        continue;
                    finish(s, sl.q, st);
                    idle = false;
                    s->cv.notify_all();
                    continue;
                }
                const cudaError_t e = cudaEventQuery(sl.done);
                if (e == cudaErrorNotReady)
                    continue;
                finish(s, sl.q, e == cudaSuccess ? VELO_OK : VELO_ECUDA);
                idle = false;
                s->cv.notify_all();
            }
            // admission: arrival order, as long as a slot and arena space exist
            while (!s->pending.empty()) {
                int free_slot = -1;
                for (size_t i = 0; i < s->slots.size(); i++)
                    if (!s->slots[i].q) {
                        free_slot = (int)i;
                        break;
                    }
                if (free_slot < 0)
                    break;
                Query* q = s->pending.front();
                char* mem = s->arena.alloc(q->need);
                if (!mem)
                    break;
                s->pending.pop_front();
                q->scratch = mem;
                q->slot = free_slot;
                q->start = Clock::now();
                Slot& sl = s->slots[free_slot];
                sl.q = q;
                s->admitted++;
                size_t inflight = 0;
                for (auto& x : s->slots)
                    inflight += x.q ? 1 : 0;
                s->peak_inflight = inflight > s->peak_inflight ? inflight : s->peak_inflight;
                s->peak_arena = s->arena.in_use() > s->peak_arena ? s->arena.in_use() : s->peak_arena;
                const velo_status rc = launch_query(s, q, sl);
                if (rc != VELO_OK) {
                    if (!s->dq)
                        cudaStreamSynchronize(sl.stream);
                    finish(s, q, rc);
                    s->cv.notify_all();
                }
                idle = false;
            }
            if (s->stop.load() && s->pending.empty()) {
                bool any = false;
                for (auto& x : s->slots)
                    any |= x.q != nullptr;
                if (!any)
                    return;
            }
        }
        if (idle)
            std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

} // namespace velo

extern "C" velo_status velo_server_create(const velo_server_config* cfg, const velo_served_tables* tables,
                                          velo_server** out)
{
    if (!cfg || !tables || !out)
        return einval("velo_server_create: null argument");
    *out = nullptr;
    if (cfg->slots == 0 || cfg->slots > 64 || cfg->hbm_budget_bytes == 0)
        return einval("velo_server_create: 1..64 slots and a nonzero HBM budget required");
    velo_server* s = new velo_server();
    s->cfg = *cfg;
    s->t = *tables;
    velo_status rc = VELO_OK;
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess)
        rc = cuda_fail(e, "cudaSetDevice");
    if (rc == VELO_OK)
        rc = s->arena.init(cfg->hbm_budget_bytes);
    if (rc == VELO_OK && (cfg->flags & VELO_SERVE_PERSISTENT))
        rc = dq_create(cfg->device, cfg->idle_us, &s->dq);
    s->slots.resize(cfg->slots);
    for (auto& sl : s->slots) {
        if (rc != VELO_OK)
            break;
        if ((e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaHostAlloc(&sl.h_out, 100 * 8, cudaHostAllocMapped)) != cudaSuccess ||
            (e = cudaHostGetDevicePointer((void**)&sl.d_out_h, sl.h_out, 0)) != cudaSuccess)
            rc = cuda_fail(e, "velo_server_create");
    }
    if (rc != VELO_OK) {
        if (s->dq)
            dq_destroy(s->dq, 10000);
        for (auto& sl : s->slots) {
            if (sl.stream)
                cudaStreamDestroy(sl.stream);
            if (sl.done)
                cudaEventDestroy(sl.done);
            if (sl.h_out)
                cudaFreeHost(sl.h_out);
        }
        delete s;
        return rc;
    }
    s->loop = std::thread(serve, s);
    *out = s;
    return VELO_OK;
}

extern "C" velo_status velo_server_submit(velo_server* s, const velo_query* q, uint64_t* qid)
{
    if (!s || !q)
        return einval("velo_server_submit: null argument");
    if (!query_valid(s, *q))
        return einval("velo_server_submit: query shape or table slice out of range");
    Query* x = new Query();
    x->q = *q;
    x->need = query_need(s, *q);
    if (x->need > s->arena.size()) {
        delete x;
        set_error("velo_server_submit: query needs more device memory than the whole HBM budget");
        return VELO_ENOMEM;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop.load()) {
        delete x;
        return einval("velo_server_submit: server is stopping");
    }
    x->id = s->next_id++;
    x->submit = Clock::now();
    x->res.qid = x->id;
    x->res.shape = q->shape;
    s->all[x->id] = x;
    s->pending.push_back(x);
    if (qid)
        *qid = x->id;
    return VELO_OK;
}

extern "C" velo_status velo_server_wait(velo_server* s, uint64_t qid, uint64_t timeout_ns, velo_query_result* out)
{
    if (!s)
        return einval("velo_server_wait: null server");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->all.find(qid);
    if (it == s->all.end())
        return einval("velo_server_wait: unknown query (or already collected)");
    Query* q = it->second;
    const bool ok = s->cv.wait_for(lock, std::chrono::nanoseconds(timeout_ns),
                                   [&] { return q->res.end_ms > 0.0 || q->end != Clock::time_point {}; });
    if (!ok) {
        set_error("velo_server_wait: query not complete at the time limit");
        return VELO_ETIMEDOUT;
    }
    if (out)
        *out = q->res;
    s->all.erase(it);
    const velo_status st = q->res.status;
    delete q;
    return st;
}

extern "C" velo_status velo_server_stats(velo_server* s, velo_server_stats_t* out)
{
    if (!s || !out)
        return einval("velo_server_stats: null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    out->admitted = s->admitted;
    out->completed = s->completed;
    out->pending = s->pending.size();
    out->peak_inflight = s->peak_inflight;
    out->arena_bytes = s->arena.size();
    out->peak_arena_bytes = s->peak_arena;
    return VELO_OK;
}

extern "C" velo_status velo_server_destroy(velo_server* s, uint32_t timeout_ms)
{
    if (!s)
        return VELO_OK;
    s->stop.store(true);
    // the loop exits once nothing is pending or running; bounded join
    const auto t0 = Clock::now();
    velo_status rc = VELO_OK;
    while (true) {
        {
            std::lock_guard<std::mutex> lock(s->mu);
            bool any = !s->pending.empty();
            for (auto& x : s->slots)
                any |= x.q != nullptr;
            if (!any)
                break;
        }
        if (Clock::now() - t0 > std::chrono::milliseconds(timeout_ms)) {
            set_error("velo_server_destroy: queries still running at the time limit");
            rc = VELO_ETIMEDOUT;
            break;
        }
        std::this_thread::sleep_for(std::chrono::milliseconds(1));
    }
    if (rc != VELO_OK) {
        // leave the loop running on purpose: it still owns in-flight work
        s->loop.detach();
        return rc;
    }
    s->loop.join();
    if (s->dq) {
        rc = dq_destroy(s->dq, timeout_ms);
        if (rc != VELO_OK)
            return rc; // the queue keeps its memory; the server object stays
        s->dq = nullptr;
    }
    for (auto& kv : s->all)
        delete kv.second;
    for (auto& sl : s->slots) {
        cudaStreamSynchronize(sl.stream);
        cudaStreamDestroy(sl.stream);
        cudaEventDestroy(sl.done);
        cudaFreeHost(sl.h_out);
    }
    delete s;
    return VELO_OK;
}
