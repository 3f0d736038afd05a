// Host-side helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "velo_obl.h"

namespace velo {

void set_error(const std::string& msg);

inline velo_status cuda_fail(cudaError_t err, const char* what)
{
    set_error(std::string(what) + ": " + cudaGetErrorString(err));
    return VELO_ECUDA;
}

inline velo_status einval(const std::string& msg)
{
    set_error(msg);
    return VELO_EINVAL;
}

inline int ilog2_floor(size_t x)
{
    int l = -1;
    while (x) {
        l++;
        x >>= 1;
    }
    return l;
}

inline size_t next_pow2(size_t x)
{
    if (x <= 1)
        return 1;
    x--;
    x |= x >> 1;
    x |= x >> 2;
    x |= x >> 4;
    x |= x >> 8;
    x |= x >> 16;
    x |= x >> 32;
    return x + 1;
}

// bytes of one value of a velo_type (0: not a fixed-width type)
inline int type_bytes(uint32_t t)
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
    default:
        return 0;
    }
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Largest supported padded size: the mark prefix counts are u32.
constexpr int MAX_LOGN = 31;

// Stage timing (velo_set_stage_timing): events around the stages of one
// pipeline call on its stream, results stored for the calling thread.
bool stage_timing_on();
void store_stage_times(const float* ms, int n);

// Pass timing (velo_set_pass_timing): while on, launch_net records an event
// after each network pass and appends (kind, log2 rows, row bytes, ms) of
// every pass to the calling thread's list.
bool pass_timing_on();
// merge passes with bulk-copy prefetch (velo_set_merge_pipeline)
bool merge_pipe_on();
void store_pass_time(int kind, int log_n, int row_bytes, float ms);

class StageTimer {
public:
    static constexpr int MAX_STAGES = 8;
    explicit StageTimer(cudaStream_t st) : st_(st), on_(stage_timing_on())
    {
        if (!on_)
            return;
        for (int i = 0; i <= MAX_STAGES; i++)
            if (cudaEventCreate(&ev_[i]) != cudaSuccess)
                on_ = false;
        if (on_)
            cudaEventRecord(ev_[0], st_);
    }
    // the stage that started at the previous mark ends here
    void mark()
    {
        if (on_ && n_ < MAX_STAGES)
            cudaEventRecord(ev_[++n_], st_);
    }
    // synchronize on the last event and store the stage durations
    void finish()
    {
        if (!on_ || n_ == 0)
            return;
        float ms[MAX_STAGES] = {};
        if (cudaEventSynchronize(ev_[n_]) == cudaSuccess)
            for (int i = 0; i < n_; i++)
                cudaEventElapsedTime(&ms[i], ev_[i], ev_[i + 1]);
        store_stage_times(ms, n_);
    }
    ~StageTimer()
    {
        if (on_)
            for (int i = 0; i <= MAX_STAGES; i++)
                if (ev_[i])
                    cudaEventDestroy(ev_[i]);
    }

private:
    cudaStream_t st_;
    bool on_;
    int n_ = 0;
    cudaEvent_t ev_[MAX_STAGES + 1] = {};
};

} // namespace velo

#define VELO_CUDA_TRY(call, what)                                                                                      \
    do {                                                                                                               \
        cudaError_t err__ = (call);                                                                                    \
        if (err__ != cudaSuccess)                                                                                      \
            return ::velo::cuda_fail(err__, what);                                                                     \
    } while (0)
