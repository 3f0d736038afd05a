// Command queue: velo_init / velo_submit / velo_batch_submit / velo_wait /
// velo_shutdown, over a CUDA stream (default) or over the persistent device
// consumer (VELO_QUEUE_PERSISTENT, dq.cu / dq_kernel.cu).
//
// The reference's TaskManager keeps one cooperative persistent kernel polling
// a host-mapped ring and runs commands strictly one at a time with a
// grid.sync() between them (src/cuda/task_manager.cu:26-78,
// src/cuda/persistent_kernel.cu:76-124); its host waits spin with no limit
// (src/cuda/commands.cpp:69-91).  Here a context owns a non-blocking stream;
// a submitted command is dispatched to its oblivious kernels on that stream
// and completes when its ticket's event does.  Batches of sorts and
// compactions go to the persistent scheduler as one launch.  Every host wait
// is bounded and nothing spins on the device while the queue is idle.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.hpp"
#include "dq_host.hpp"

struct velo_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t capacity = 1024;
    std::mutex mu;
    uint64_t next_ticket = 1;
    std::deque<std::pair<uint64_t, cudaEvent_t>> inflight; // (ticket, event), oldest first
    std::vector<cudaEvent_t> free_events;
    uint64_t completed_below = 1; // every ticket < this is known complete
    std::deque<std::pair<uint64_t, velo_batch*>> plans; // batch plans kept alive until their ticket completes
    std::deque<uint64_t> failed;                        // tickets whose batch reported a device wait timeout
    std::string last_error;
    velo::DqEngine* dq = nullptr; // VELO_QUEUE_PERSISTENT: tickets are job numbers of this queue
    uint64_t dq_last = 0;         // the last job published
};

namespace {

velo_status ctx_fail(velo_ctx* c, velo_status rc)
{
    if (rc != VELO_OK)
        c->last_error = velo_last_error_text();
    return rc;
}

// dispatches one command on the context stream
velo_status dispatch(velo_ctx* c, const velo_cmd& m)
{
    void* st = (void*)c->stream;
    const auto& a = m.args;
    switch (m.opcode) {
    case VELO_OP_NOP:
        return VELO_OK;
    case VELO_OP_PERMUTE:
        return velo_permute(a.permute.d_out, a.permute.d_in, a.permute.d_indices, a.permute.n, a.permute.type, st);
    case VELO_OP_SCATTER:
        return velo_scatter(a.scatter.d_mask, a.scatter.n, a.scatter.d_out_indices, a.scatter.d_count,
                            a.scatter.d_scratch, a.scatter.scratch_bytes, st);
    case VELO_OP_GATHER:
        return velo_gather(a.gather.d_out, a.gather.d_in, a.gather.d_indices, a.gather.d_mask, a.gather.n,
                           a.gather.type, st);
    case VELO_OP_SORT:
        return velo_sort_columns(a.sort.d_cols, a.sort.types, a.sort.ascending, a.sort.n_cols, a.sort.n,
                                 a.sort.capacity, a.sort.d_indices, a.sort.d_scratch, a.sort.scratch_bytes, st);
    case VELO_OP_COMPARE_EQ:
        return velo_compare_eq(a.compare_eq.d_left, a.compare_eq.d_right, a.compare_eq.d_out_mask, a.compare_eq.n,
                               a.compare_eq.type, st);
    case VELO_OP_COMPOSE_POSITION_MAP:
        return velo_compose_position_map(a.compose.d_old, a.compose.d_sigma, a.compose.d_new, a.compose.n, st);
    case VELO_OP_ENRICH_POSITIONS:
        return velo_enrich_positions(a.enrich.d_record_ids, a.enrich.d_map, a.enrich.d_out, a.enrich.n, st);
    case VELO_OP_OSORT_KP:
        return velo_osort_kp(a.osort_kp.d_keys, a.osort_kp.d_payload, a.osort_kp.n, a.osort_kp.capacity, nullptr, st);
    case VELO_OP_OCOMPACT_KPM:
        return velo_ocompact_kpm(a.ocompact_kpm.d_keys, a.ocompact_kpm.d_payload, a.ocompact_kpm.d_marks,
                                 a.ocompact_kpm.n, a.ocompact_kpm.capacity, a.ocompact_kpm.d_count,
                                 a.ocompact_kpm.d_scratch, a.ocompact_kpm.scratch_bytes, nullptr, st);
    case VELO_OP_OSORT_RECORDS:
        return velo_osort_records(a.osort_records.d_words, a.osort_records.n_words, a.osort_records.key_mask,
                                  a.osort_records.n, a.osort_records.capacity, m.flags, nullptr, st);
    case VELO_OP_OJOIN_PKFK:
        return velo_ojoin_pkfk(a.ojoin.d_build_keys, a.ojoin.d_build_mask, a.ojoin.build_n, a.ojoin.d_probe_keys,
                               a.ojoin.d_probe_mask, a.ojoin.probe_n, a.ojoin.key_type, a.ojoin.d_out_build_rowid,
                               a.ojoin.d_out_probe_rowid, a.ojoin.d_counts, a.ojoin.d_scratch, a.ojoin.scratch_bytes,
                               st);
    case VELO_OP_OJOIN_MN:
        return velo_ojoin_mn(a.ojoin_mn.d_build_keys, a.ojoin_mn.d_build_mask, a.ojoin_mn.build_n,
                             a.ojoin_mn.d_probe_keys, a.ojoin_mn.d_probe_mask, a.ojoin_mn.probe_n, a.ojoin_mn.key_type,
                             a.ojoin_mn.max_pairs, a.ojoin_mn.d_out_build_rowid, a.ojoin_mn.d_out_probe_rowid,
                             a.ojoin_mn.d_counts, a.ojoin_mn.d_scratch, a.ojoin_mn.scratch_bytes, st);
    case VELO_OP_OHASH_JOIN:
        return velo_ohash_join(a.ohash.d_build_keys, a.ohash.d_build_mask, a.ohash.build_n, a.ohash.d_probe_keys,
                               a.ohash.d_probe_mask, a.ohash.probe_n, a.ohash.key_type, a.ohash.hash_seed,
                               a.ohash.d_out_build_rowid, a.ohash.d_out_probe_rowid, a.ohash.d_counts,
                               a.ohash.d_scratch, a.ohash.scratch_bytes, st);
    case VELO_OP_OGATHER:
        return velo_ogather_u64(a.ogather.d_table, a.ogather.table_n, a.ogather.d_rids, a.ogather.n_req,
                                a.ogather.d_out, a.ogather.d_scratch, a.ogather.scratch_bytes, st);
    case VELO_OP_OSHUFFLE:
        return velo_oshuffle_position_map(a.oshuffle.d_map, a.oshuffle.n, a.oshuffle.key, a.oshuffle.counter,
                                          a.oshuffle.d_scratch, a.oshuffle.scratch_bytes, st);
    case VELO_OP_FILTER_GROUPBY:
        if (m.flags & VELO_REVEAL_COUNT)
            return velo::einval("velo_submit: VELO_REVEAL_COUNT synchronises; call velo_filter_groupby directly");
        return velo_filter_groupby(a.filter_groupby.cols, a.filter_groupby.n, a.filter_groupby.pred,
                                   a.filter_groupby.group_bound, 0, a.filter_groupby.d_out, a.filter_groupby.d_counts,
                                   a.filter_groupby.d_scratch, a.filter_groupby.scratch_bytes, st);
    case VELO_OP_JOIN_GROUPBY_TOPK:
        return velo_join_groupby_topk(a.join_topk.tables, a.join_topk.pred, a.join_topk.k, a.join_topk.d_out,
                                      a.join_topk.d_counts, a.join_topk.d_scratch, a.join_topk.scratch_bytes, st);
    default:
        return velo::einval("velo_submit: unknown opcode");
    }
}

// retire completed tickets from the front of the in-flight list (mu held)
void retire(velo_ctx* c)
{
    while (!c->inflight.empty()) {
        const auto& f = c->inflight.front();
        if (cudaEventQuery(f.second) != cudaSuccess)
            break;
        c->completed_below = f.first + 1;
        c->free_events.push_back(f.second);
        c->inflight.pop_front();
    }
    while (!c->plans.empty() && c->plans.front().first < c->completed_below) {
        velo_batch* b = c->plans.front().second;
        // the ticket is complete, so the status word is final: read it on the
        // legacy stream, which never waits for this non-blocking stream
        if (velo_batch_status(b, nullptr) != VELO_OK) {
            c->failed.push_back(c->plans.front().first);
            c->last_error = velo_last_error_text();
        }
        velo_batch_destroy(b);
        c->plans.pop_front();
    }
}

velo_status record_ticket(velo_ctx* c, uint64_t* ticket)
{
    // bounded back-pressure: wait (at most 10 s) while the ring is full
    const auto t0 = std::chrono::steady_clock::now();
    while (c->inflight.size() >= c->capacity) {
        retire(c);
        if (c->inflight.size() < c->capacity)
            break;
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(10)) {
            velo::set_error("velo_submit: queue full and nothing completed for 10 s");
            return VELO_ETIMEDOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    cudaEvent_t ev;
    if (!c->free_events.empty()) {
        ev = c->free_events.back();
        c->free_events.pop_back();
    } else {
        VELO_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
    }
    VELO_CUDA_TRY(cudaEventRecord(ev, c->stream), "cudaEventRecord");
    const uint64_t t = c->next_ticket++;
    c->inflight.emplace_back(t, ev);
    if (ticket)
        *ticket = t;
    return VELO_OK;
}

} // namespace

extern "C" velo_status velo_init(const velo_config* config, velo_ctx** out)
{
    if (!out)
        return velo::einval("velo_init: null output");
    *out = nullptr;
    velo_ctx* c = new velo_ctx();
    c->device = config ? config->device : 0;
    c->capacity = (config && config->queue_capacity) ? config->queue_capacity : 1024;
    if (config && (config->flags & VELO_QUEUE_PERSISTENT)) {
        const velo_status rc = velo::dq_create(c->device, config->idle_us, &c->dq);
        if (rc != VELO_OK) {
            delete c;
            return rc;
        }
        c->stream = (cudaStream_t)velo::dq_stream(c->dq);
        *out = c;
        return VELO_OK;
    }
    cudaError_t err = cudaSetDevice(c->device);
    if (err == cudaSuccess)
        err = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        delete c;
        return velo::cuda_fail(err, "velo_init");
    }
    *out = c;
    return VELO_OK;
}

extern "C" velo_status velo_shutdown(velo_ctx* c, uint32_t timeout_ms)
{
    if (!c)
        return VELO_OK;
    if (c->dq) {
        const velo_status rq = velo::dq_destroy(c->dq, timeout_ms);
        delete c;
        return rq;
    }
    velo_status rc = VELO_OK;
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t q = cudaStreamQuery(c->stream);
        if (q == cudaSuccess)
            break;
        if (q != cudaErrorNotReady) {
            rc = velo::cuda_fail(q, "velo_shutdown");
            break;
        }
        if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms)) {
            velo::set_error("velo_shutdown: commands still running at the time limit");
            rc = VELO_ETIMEDOUT;
            break;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    if (rc == VELO_OK) {
        for (auto& pl : c->plans)
            velo_batch_destroy(pl.second);
        for (auto& f : c->inflight)
            cudaEventDestroy(f.second);
        for (auto e : c->free_events)
            cudaEventDestroy(e);
        cudaStreamDestroy(c->stream);
    }
    // on a timeout the stream and events are left to the CUDA context (work
    // may still reference them); the host object is released either way
    delete c;
    return rc;
}

extern "C" velo_status velo_submit(velo_ctx* c, const velo_cmd* cmd, uint64_t* ticket)
{
    if (!c || !cmd)
        return velo::einval("velo_submit: null argument");
    std::lock_guard<std::mutex> lock(c->mu);
    if (c->dq) {
        velo::DqPlan plan;
        velo_status rc = velo::dq_plan_cmd(plan, *cmd);
        uint64_t seq = 0;
        if (rc == VELO_OK)
            rc = velo::dq_publish(c->dq, plan, (cmd->flags & VELO_CMD_UNORDERED) ? 0 : c->dq_last, &seq);
        if (rc != VELO_OK)
            return ctx_fail(c, rc);
        c->dq_last = seq;
        if (ticket)
            *ticket = seq;
        return VELO_OK;
    }
    velo_status rc = dispatch(c, *cmd);
    if (rc != VELO_OK)
        return ctx_fail(c, rc);
    return ctx_fail(c, record_ticket(c, ticket));
}

extern "C" velo_status velo_batch_submit(velo_ctx* c, const velo_cmd* cmds, size_t n, uint64_t* tickets)
{
    if (!c || (!cmds && n))
        return velo::einval("velo_batch_submit: null argument");
    std::lock_guard<std::mutex> lock(c->mu);
    if (c->dq) {
        // every command a job of its own, ordered after what came before the
        // batch and unordered among the batch
        const uint64_t after = c->dq_last;
        uint64_t last = after;
        for (size_t i = 0; i < n; i++) {
            velo::DqPlan plan;
            velo_status rc = velo::dq_plan_cmd(plan, cmds[i]);
            uint64_t seq = 0;
            if (rc == VELO_OK)
                rc = velo::dq_publish(c->dq, plan, after, &seq);
            if (rc != VELO_OK) {
                c->dq_last = last;
                return ctx_fail(c, rc);
            }
            last = seq;
            if (tickets)
                tickets[i] = seq;
        }
        c->dq_last = last;
        return VELO_OK;
    }
    std::vector<velo_batch_item> items;
    std::vector<size_t> others;
    for (size_t i = 0; i < n; i++) {
        const velo_cmd& m = cmds[i];
        if (m.opcode == VELO_OP_OSORT_KP) {
            velo_batch_item it {};
            it.kind = VELO_ITEM_SORT_KP;
            it.d_keys = m.args.osort_kp.d_keys;
            it.d_payload = m.args.osort_kp.d_payload;
            it.n = m.args.osort_kp.n;
            it.capacity = m.args.osort_kp.capacity;
            items.push_back(it);
        } else if (m.opcode == VELO_OP_OCOMPACT_KPM) {
            velo_batch_item it {};
            it.kind = VELO_ITEM_COMPACT_KPM;
            it.d_keys = m.args.ocompact_kpm.d_keys;
            it.d_payload = m.args.ocompact_kpm.d_payload;
            it.d_marks = m.args.ocompact_kpm.d_marks;
            it.n = m.args.ocompact_kpm.n;
            it.capacity = m.args.ocompact_kpm.capacity;
            it.d_count = m.args.ocompact_kpm.d_count;
            items.push_back(it);
        } else {
            others.push_back(i);
        }
    }
    velo_status rc = VELO_OK;
    velo_batch* b = nullptr;
    if (!items.empty()) {
        rc = velo_batch_create(items.data(), items.size(), nullptr, &b);
        if (rc == VELO_OK)
            rc = velo_batch_launch(b, (void*)c->stream);
        if (rc != VELO_OK) {
            if (b) {
                cudaStreamSynchronize(c->stream);
                velo_batch_destroy(b);
            }
            return ctx_fail(c, rc);
        }
    }
    for (size_t i : others) {
        rc = dispatch(c, cmds[i]);
        if (rc != VELO_OK)
            break;
    }
    uint64_t t = 0;
    const velo_status rt = record_ticket(c, &t);
    if (b) {
        if (rt == VELO_OK) {
            // the plan's device memory must outlive the launch: it is freed
            // when the ticket retires
            c->plans.emplace_back(t, b);
        } else {
            cudaStreamSynchronize(c->stream);
            velo_batch_destroy(b);
        }
    }
    if (rc != VELO_OK)
        return ctx_fail(c, rc);
    if (rt != VELO_OK)
        return ctx_fail(c, rt);
    for (size_t i = 0; i < n; i++)
        if (tickets)
            tickets[i] = t;
    return VELO_OK;
}

extern "C" velo_status velo_wait(velo_ctx* c, uint64_t ticket, uint64_t timeout_ns)
{
    if (!c)
        return velo::einval("velo_wait: null context");
    if (c->dq) {
        const velo_status rc = velo::dq_wait(c->dq, ticket, timeout_ns);
        if (rc != VELO_OK) {
            std::lock_guard<std::mutex> lock(c->mu);
            ctx_fail(c, rc);
        }
        return rc;
    }
    const auto t0 = std::chrono::steady_clock::now();
    int spins = 0;
    for (;;) {
        {
            std::lock_guard<std::mutex> lock(c->mu);
            if (ticket >= c->next_ticket)
                return ctx_fail(c, velo::einval("velo_wait: unknown ticket"));
            retire(c);
            if (ticket < c->completed_below) {
                for (uint64_t f : c->failed)
                    if (f == ticket) {
                        velo::set_error("velo_wait: a device-side wait of the ticket's batch ran out of time");
                        return ctx_fail(c, VELO_ETIMEDOUT);
                    }
                return VELO_OK;
            }
            cudaError_t q = cudaStreamQuery(c->stream);
            if (q != cudaSuccess && q != cudaErrorNotReady)
                return ctx_fail(c, velo::cuda_fail(q, "velo_wait"));
        }
        if ((uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0)
                .count()
            > timeout_ns) {
            std::lock_guard<std::mutex> lock(c->mu);
            velo::set_error("velo_wait: ticket not complete at the time limit");
            return ctx_fail(c, VELO_ETIMEDOUT);
        }
        if (spins++ < 2000)
            std::this_thread::yield();
        else
            std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

extern "C" velo_status velo_last_error(velo_ctx* c, char* buf, size_t len)
{
    if (!buf || len == 0)
        return velo::einval("velo_last_error: empty buffer");
    std::string s;
    if (c) {
        std::lock_guard<std::mutex> lock(c->mu);
        s = c->last_error;
    } else {
        s = velo_last_error_text();
    }
    const size_t k = s.size() < len - 1 ? s.size() : len - 1;
    std::memcpy(buf, s.data(), k);
    buf[k] = '\0';
    return VELO_OK;
}

extern "C" size_t velo_cmd_size(void)
{
    return sizeof(velo_cmd);
}

extern "C" void* velo_ctx_stream(velo_ctx* c)
{
    return c ? (void*)c->stream : nullptr;
}

extern "C" uint64_t velo_ctx_launches(velo_ctx* c)
{
    return (c && c->dq) ? velo::dq_launches(c->dq) : 0;
}
