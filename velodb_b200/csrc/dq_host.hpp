// Host interface of the persistent command queue (dq.cu) for the command
// queue (queue.cpp) and the serving layer (server.cu).
#pragma once

#include <cstddef>
#include <cstdint>

#include "velo_obl.h"

namespace velo {

struct DqEngine;
struct DqJob;

// A job under construction: commands are appended in order, each as the
// steps of its pipeline; one job may hold several commands (they run one
// after another inside the job).
class DqPlan {
public:
    DqPlan();
    ~DqPlan();
    DqPlan(const DqPlan&) = delete;
    DqPlan& operator=(const DqPlan&) = delete;
    DqJob& job() { return *job_; }
    // steps so far and whether every append fitted the job limits
    uint32_t steps() const;
    bool ok() const { return !overflow_; }
    // an append did not fit (too many steps, items or argument bytes)
    void overflow() { overflow_ = true; }

private:
    DqJob* job_;
    bool overflow_ = false;
};

// appends one command of the command set; VELO_ENOTSUP for commands the
// persistent queue does not run
velo_status dq_plan_cmd(DqPlan& p, const velo_cmd& cmd);
// the served query shapes' pipelines (pointers as the direct entry points)
velo_status dq_plan_filter_groupby(DqPlan& p, const velo_lineitem* cols, size_t n, const velo_lineitem_pred* pred,
                                   uint32_t group_bound, int64_t* d_out, uint64_t* d_counts, void* d_scratch,
                                   size_t scratch_bytes);
velo_status dq_plan_join_topk(DqPlan& p, const velo_join_tables* t, const velo_join_pred* pred, uint32_t k,
                              int64_t* d_out, uint64_t* d_counts, void* d_scratch, size_t scratch_bytes);
velo_status dq_plan_ojoin_pkfk(DqPlan& p, const void* d_build_keys, const uint8_t* d_build_mask, size_t build_n,
                               const void* d_probe_keys, const uint8_t* d_probe_mask, size_t probe_n,
                               uint32_t key_type, int64_t* d_out_build_rowid, int64_t* d_out_probe_rowid,
                               uint64_t* d_counts, void* d_scratch, size_t scratch_bytes);
velo_status dq_plan_ogather(DqPlan& p, const uint64_t* d_table, size_t table_n, const uint32_t* d_rids, size_t n_req,
                            uint64_t* d_out, void* d_scratch, size_t scratch_bytes);
// small steps of the served three-way chain
void dq_plan_range_mask_i32(DqPlan& p, const int32_t* c, size_t n, int32_t lo, int32_t hi, uint8_t* m);
void dq_plan_range_mask_i64(DqPlan& p, const int64_t* c, size_t n, int64_t lo, int64_t hi, uint8_t* m);
void dq_plan_rowid_keys(DqPlan& p, const int64_t* rowid, size_t n, int64_t offset, int64_t* key, uint8_t* m);
void dq_plan_rowid_rids(DqPlan& p, const int64_t* rowid, size_t n, uint32_t missing, uint32_t* rid);
void dq_plan_fill_u8(DqPlan& p, uint8_t* out, uint8_t v, size_t n);
void dq_plan_set_words(DqPlan& p, uint64_t* out, uint64_t v, size_t n);
void dq_plan_sum_u64(DqPlan& p, const uint64_t* v, size_t n, unsigned long long* out);
// copies `words` u64 from device memory to `dst` (device memory, or the
// device address of mapped host memory)
void dq_plan_copy_words(DqPlan& p, const uint64_t* src, uint64_t* dst, uint32_t words);

// The consumer kernel exits after idle_us microseconds without work
// (0: 1000) and is relaunched by the next publication or wait.
velo_status dq_create(int device, uint32_t idle_us, DqEngine** out);
// Waits (bounded) for every published job and the consumer's exit, then
// frees the queue; VELO_ETIMEDOUT leaves the device memory allocated.
velo_status dq_destroy(DqEngine* e, uint32_t timeout_ms);
// Publishes the plan as one job.  after = 0: no ordering; otherwise the job
// starts once every job with seq <= after is complete.  Waits (bounded) for a
// free ring slot.
velo_status dq_publish(DqEngine* e, DqPlan& p, uint64_t after, uint64_t* seq);
// true once job `seq` is complete; *status = its status
bool dq_poll(DqEngine* e, uint64_t seq, velo_status* status);
velo_status dq_wait(DqEngine* e, uint64_t seq, uint64_t timeout_ns);
// the stream the consumer runs on
void* dq_stream(DqEngine* e);
// consumer launches so far (first launch and relaunches after idle exits)
uint64_t dq_launches(DqEngine* e);

} // namespace velo
