// Batches of independent oblivious sorts and compactions run by the
// persistent scheduler (sched.cuh): batch planning, launch, autotuning.
#include <chrono>
#include <vector>

#include "net_host.cuh"
#include "sched.cuh"

namespace velo {

// the autotuner's search space: tile 2^11..2^13 rows x 256/512/1024 threads
#define VELO_FOR_SCHED_TUNES(X)                                                                                        \
    X(8, 3)                                                                                                            \
    X(9, 2)                                                                                                            \
    X(10, 1)                                                                                                           \
    X(8, 4)                                                                                                            \
    X(9, 3)                                                                                                            \
    X(10, 2)                                                                                                           \
    X(8, 5)                                                                                                            \
    X(9, 4)                                                                                                            \
    X(10, 3)

template <int LOG_NT, int LOG_E>
velo_status sched_launch(const SchedArgs& a, int sms, cudaStream_t st);

} // namespace velo

struct velo_batch {
    int log_nt = 9, log_e = 4;
    std::vector<velo::SchedStep> steps;
    std::vector<velo::SchedInst> insts;
    std::vector<uint64_t*> zero_counts; // d_count of empty compactions
    void* dmem = nullptr;               // steps | insts | done | next | status | compaction scratch
    velo::SchedStep* d_steps = nullptr;
    velo::SchedInst* d_insts = nullptr;
    uint32_t* d_item_step = nullptr;
    uint32_t* d_done = nullptr;
    unsigned long long* d_next = nullptr;
    int* d_status = nullptr;
    uint64_t total_items = 0;
    uint64_t timeout_ns = 2000000000ull;
    size_t counter_bytes = 0; // done + next + status, cleared before every launch
    int sms = 148;
    int device = 0;
};

using namespace velo;

static velo_status batch_plan(velo_batch* b, const velo_batch_item* items, size_t n_items)
{
    const int lt = b->log_nt + b->log_e;
    const int lmax = lt - 5 < 8 ? lt - 5 : 8;
    std::vector<std::vector<std::pair<uint32_t, NetPass>>> per(n_items); // (kind, pass) per instance
    std::vector<std::vector<uint32_t>> tiles(n_items);
    size_t scratch_u32 = 0;
    b->insts.resize(n_items);
    for (size_t i = 0; i < n_items; i++) {
        const velo_batch_item& it = items[i];
        SchedInst& in = b->insts[i];
        in = SchedInst {};
        if (it.kind != VELO_ITEM_SORT_KP && it.kind != VELO_ITEM_COMPACT_KPM)
            return einval("velo_batch_create: unknown item kind");
        in.k = it.d_keys;
        in.p = it.d_payload;
        in.m = it.d_marks;
        in.d_count = it.d_count;
        in.n = it.n;
        if (it.n == 0) {
            if (it.kind == VELO_ITEM_COMPACT_KPM && it.d_count)
                b->zero_counts.push_back(it.d_count);
            continue;
        }
        if (!it.d_keys || !it.d_payload || (it.kind == VELO_ITEM_COMPACT_KPM && !it.d_marks))
            return einval("velo_batch_create: null buffer");
        const size_t np = next_pow2(it.n);
        if (np > ((size_t)1 << MAX_LOGN) || it.capacity < np)
            return einval("velo_batch_create: capacity must be >= next_pow2(n)");
        in.logN = ilog2_floor(np);
        const int ntiles = in.logN > lt ? 1 << (in.logN - lt) : 1;
        in.ntiles = ntiles;
        std::vector<NetPass> passes;
        if (it.kind == VELO_ITEM_SORT_KP) {
            if (np > 1)
                plan_sort(in.logN, lt, lmax, passes);
            for (auto& p : passes) {
                per[i].push_back({ STEP_SORT_PASS, p });
                tiles[i].push_back((uint32_t)ntiles);
            }
        } else {
            per[i].push_back({ STEP_COMPACT_COUNT, NetPass {} });
            tiles[i].push_back((uint32_t)ntiles);
            per[i].push_back({ STEP_COMPACT_SCAN, NetPass {} });
            tiles[i].push_back(1);
            plan_compact(in.logN, lt, lmax, passes);
            for (auto& p : passes) {
                per[i].push_back({ STEP_COMPACT_PASS, p });
                tiles[i].push_back((uint32_t)ntiles);
            }
            scratch_u32 += (size_t)2 * ntiles + 1 + 64; // counts + prefix, 256-byte aligned below
        }
    }
    // round-robin interleave by pass index
    size_t max_steps = 0;
    for (auto& v : per)
        max_steps = v.size() > max_steps ? v.size() : max_steps;
    std::vector<uint32_t> dep(n_items, 0);
    uint64_t item = 0;
    for (size_t r = 0; r < max_steps; r++) {
        for (size_t i = 0; i < n_items; i++) {
            if (r >= per[i].size())
                continue;
            SchedStep s {};
            s.item_begin = item;
            s.inst = (uint32_t)i;
            s.kind = per[i][r].first;
            s.pass = per[i][r].second;
            s.ntiles = tiles[i][r];
            s.dep = dep[i];
            dep[i] += s.ntiles;
            item += s.ntiles;
            b->steps.push_back(s);
        }
    }
    b->total_items = item;
    if (b->steps.size() > 0xFFFFFFFFull)
        return einval("velo_batch_create: too many steps");
    // step of every item, so a claim costs one load
    std::vector<uint32_t> item_step((size_t)item);
    for (size_t s = 0; s < b->steps.size(); s++)
        for (uint32_t t = 0; t < b->steps[s].ntiles; t++)
            item_step[(size_t)b->steps[s].item_begin + t] = (uint32_t)s;
    // device memory: steps | insts | item steps | compaction scratch | done | next | status
    const size_t steps_b = align_up(b->steps.size() * sizeof(SchedStep) + 1, 256);
    const size_t items_b = align_up(item_step.size() * 4 + 1, 256);
    const size_t insts_b = align_up(b->insts.size() * sizeof(SchedInst) + 1, 256);
    const size_t scr_b = align_up(scratch_u32 * 4 + 256 * n_items + 1, 256);
    const size_t done_b = align_up(n_items * 4 + 1, 256);
    b->counter_bytes = done_b + 256;
    VELO_CUDA_TRY(cudaMalloc(&b->dmem, steps_b + insts_b + items_b + scr_b + b->counter_bytes),
                  "cudaMalloc(batch)");
    char* base = static_cast<char*>(b->dmem);
    b->d_steps = reinterpret_cast<SchedStep*>(base);
    b->d_insts = reinterpret_cast<SchedInst*>(base + steps_b);
    b->d_item_step = reinterpret_cast<uint32_t*>(base + steps_b + insts_b);
    char* scr = base + steps_b + insts_b + items_b;
    b->d_done = reinterpret_cast<uint32_t*>(scr + scr_b);
    b->d_next = reinterpret_cast<unsigned long long*>(scr + scr_b + done_b);
    b->d_status = reinterpret_cast<int*>(scr + scr_b + done_b + 64);
    size_t off = 0;
    for (size_t i = 0; i < n_items; i++) {
        if (items[i].kind != VELO_ITEM_COMPACT_KPM || items[i].n == 0)
            continue;
        SchedInst& in = b->insts[i];
        in.counts = reinterpret_cast<uint32_t*>(scr + off);
        off += align_up((size_t)in.ntiles * 4, 256);
        in.prefix = reinterpret_cast<uint32_t*>(scr + off);
        off += align_up(((size_t)in.ntiles + 1) * 4, 256);
    }
    VELO_CUDA_TRY(cudaMemcpy(b->d_steps, b->steps.data(), b->steps.size() * sizeof(SchedStep),
                             cudaMemcpyHostToDevice),
                  "cudaMemcpy(steps)");
    VELO_CUDA_TRY(cudaMemcpy(b->d_insts, b->insts.data(), b->insts.size() * sizeof(SchedInst),
                             cudaMemcpyHostToDevice),
                  "cudaMemcpy(insts)");
    if (!item_step.empty())
        VELO_CUDA_TRY(cudaMemcpy(b->d_item_step, item_step.data(), item_step.size() * 4, cudaMemcpyHostToDevice),
                      "cudaMemcpy(item steps)");
    return VELO_OK;
}

extern "C" velo_status velo_batch_create(const velo_batch_item* items, size_t n_items, const velo_tune* tune,
                                         velo_batch** out)
{
    if (!out || (!items && n_items))
        return einval("velo_batch_create: null argument");
    *out = nullptr;
    // default tile: 4096 rows of 256 threads, the autotuner's pick on the
    // 512-instance mix of 2^10..2^22 rows (35.4 ms against 39.5 ms for
    // 8192 rows of 512 threads)
    int log_nt = 8, log_e = 4;
    velo_status rc = resolve_tune(tune, 8, 4, &log_nt, &log_e);
    if (rc != VELO_OK)
        return rc;
    bool ok = false;
#define X(a, c)                                                                                                        \
    ok |= (log_nt == a && log_e == c);
    VELO_FOR_SCHED_TUNES(X)
#undef X
    if (!ok)
        return einval("velo_batch_create: tile configuration outside the batched search space");
    velo_batch* b = new velo_batch();
    b->log_nt = log_nt;
    b->log_e = log_e;
    cudaGetDevice(&b->device);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    rc = batch_plan(b, items, n_items);
    if (rc != VELO_OK) {
        velo_batch_destroy(b);
        return rc;
    }
    *out = b;
    return VELO_OK;
}

extern "C" void velo_batch_destroy(velo_batch* b)
{
    if (!b)
        return;
    if (b->dmem)
        cudaFree(b->dmem);
    delete b;
}

extern "C" velo_status velo_batch_launch(velo_batch* b, void* stream)
{
    if (!b)
        return einval("velo_batch_launch: null batch");
    cudaStream_t st = (cudaStream_t)stream;
    for (uint64_t* p : b->zero_counts)
        VELO_CUDA_TRY(cudaMemsetAsync(p, 0, sizeof(uint64_t), st), "cudaMemsetAsync");
    if (b->total_items == 0)
        return VELO_OK;
    VELO_CUDA_TRY(cudaMemsetAsync(b->d_done, 0, b->counter_bytes, st), "cudaMemsetAsync(counters)");
    SchedArgs a;
    a.steps = b->d_steps;
    a.insts = b->d_insts;
    a.item_step = b->d_item_step;
    a.done = b->d_done;
    a.next_item = b->d_next;
    a.status = b->d_status;
    a.total_items = b->total_items;
    a.timeout_ns = b->timeout_ns;
    a.nsteps = (int)b->steps.size();
#define X(x, y)                                                                                                        \
    if (b->log_nt == x && b->log_e == y)                                                                               \
        return sched_launch<x, y>(a, b->sms, st);
    VELO_FOR_SCHED_TUNES(X)
#undef X
    return einval("velo_batch_launch: bad configuration");
}

extern "C" velo_status velo_batch_status(velo_batch* b, void* stream)
{
    if (!b)
        return einval("velo_batch_status: null batch");
    int h = 0;
    cudaStream_t st = (cudaStream_t)stream;
    if (b->total_items) {
        VELO_CUDA_TRY(cudaMemcpyAsync(&h, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    }
    VELO_CUDA_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    if (h != 0) {
        set_error("velo_batch: a scheduler wait ran out of time");
        return h;
    }
    return VELO_OK;
}

extern "C" velo_status velo_batch_set_timeout(velo_batch* b, uint64_t timeout_ns)
{
    if (!b || timeout_ns == 0)
        return einval("velo_batch_set_timeout: null batch or zero limit");
    b->timeout_ns = timeout_ns;
    return VELO_OK;
}

extern "C" velo_status velo_batch_inject_unmet_wait(velo_batch* b, uint32_t item)
{
    if (!b || item >= b->insts.size())
        return einval("velo_batch_inject_unmet_wait: bad batch or item");
    for (size_t i = 0; i < b->steps.size(); i++) {
        if (b->steps[i].inst == item) {
            SchedStep s = b->steps[i];
            s.dep = 0xFFFFFFFFu; // a completion count that is never reached
            VELO_CUDA_TRY(cudaMemcpy(b->d_steps + i, &s, sizeof(SchedStep), cudaMemcpyHostToDevice),
                          "cudaMemcpy(step)");
            return VELO_OK;
        }
    }
    return einval("velo_batch_inject_unmet_wait: command has no work items");
}

extern "C" velo_status velo_batch_autotune(const velo_batch_item* items, size_t n_items, uint32_t reps,
                                           velo_tune* best, float* ms_out, void* stream)
{
    // The networks are data-oblivious, so every candidate does the same work
    // on any data and timing on the live buffers is representative;
    // re-running keeps sorted outputs and compactions' marked prefixes.
    if (!best)
        return einval("velo_batch_autotune: null output");
    cudaStream_t st = (cudaStream_t)stream;
    const int cand[][2] = {
#define X(a, c) { a, c },
        VELO_FOR_SCHED_TUNES(X)
#undef X
    };
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    VELO_CUDA_TRY(cudaEventCreate(&e0), "cudaEventCreate");
    VELO_CUDA_TRY(cudaEventCreate(&e1), "cudaEventCreate");
    velo_status rc = VELO_OK;
    for (size_t c = 0; c < sizeof(cand) / sizeof(cand[0]); c++) {
        velo_tune t { (uint32_t)(cand[c][0] + cand[c][1]), 1u << cand[c][0] };
        velo_batch* b = nullptr;
        rc = velo_batch_create(items, n_items, &t, &b);
        if (rc != VELO_OK)
            break;
        rc = velo_batch_launch(b, st); // warm-up
        float total = 0.f;
        for (uint32_t r = 0; r < (reps ? reps : 1) && rc == VELO_OK; r++) {
            cudaEventRecord(e0, st);
            rc = velo_batch_launch(b, st);
            cudaEventRecord(e1, st);
            if (rc == VELO_OK && cudaEventSynchronize(e1) == cudaSuccess) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                total += ms;
            }
        }
        if (rc == VELO_OK)
            rc = velo_batch_status(b, st);
        velo_batch_destroy(b);
        if (rc != VELO_OK)
            break;
        const float ms = total / (float)(reps ? reps : 1);
        if (ms_out)
            ms_out[c] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            *best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}
