// Persistent scheduler for batches of independent oblivious sorts and
// compactions (the batched form of the command queue).
//
// The reference runs every command on one cooperative persistent grid and
// separates commands by grid.sync(), so one command occupies the whole GPU at
// a time (src/cuda/persistent_kernel.cu:76-124).  Here a batch of commands is
// flattened into work items (instance, pass, tile), ordered round-robin by
// pass index across instances, and one persistent launch runs them all:
// every CTA repeatedly claims the next item with an atomic counter, waits
// until the item's instance has finished its previous pass (a per-instance
// count of completed tiles), runs the tile, and publishes its completion.
// Small instances fill the SMs that large ones leave idle, and no pass of one
// instance waits for any other instance.
//
// Deadlock freedom: items are claimed in increasing order and an item only
// waits for items of earlier passes of its own instance, which precede it in
// the order and are therefore held by running CTAs.  Every wait is still
// bounded by a time limit; on expiry the CTA records VELO_ETIMEDOUT in the
// status word, marks its item done and carries on, so the launch always
// terminates and the host reads the error.
#pragma once

#include "network.cuh"

namespace velo {

enum StepKind : uint32_t {
    STEP_SORT_PASS = 1,     // bitonic pass of a (key, payload) sort
    STEP_COMPACT_COUNT = 2, // per-tile mark counts of a compaction
    STEP_COMPACT_SCAN = 3,  // exclusive scan of the tile counts (one tile)
    STEP_COMPACT_PASS = 4,  // ORCompact pass
};

struct SchedStep {
    uint64_t item_begin; // global index of the step's first item
    uint32_t inst;       // instance
    uint32_t kind;       // StepKind
    uint32_t ntiles;     // items of the step
    uint32_t dep;        // completed tiles of the instance needed first
    NetPass pass;
};

struct SchedInst {
    uint64_t* k;
    uint32_t* p;
    uint8_t* m;
    uint64_t* d_count;
    uint32_t* counts; // compaction: per-tile counts, then exclusive prefix
    uint32_t* prefix;
    size_t n;
    int logN;
    int ntiles;
};

struct SchedArgs {
    const SchedStep* steps;
    const SchedInst* insts;
    const uint32_t* item_step; // step of every item (built with the plan)
    uint32_t* done;
    unsigned long long* next_item;
    int* status;
    uint64_t total_items;
    uint64_t timeout_ns;
    int nsteps;
};

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int LOG_NT, int LOG_E>
struct Sched {
    using NS = Net<RowKP, LOG_NT, LOG_E>;
    using NC = Net<RowKPM, LOG_NT, LOG_E>;
    static constexpr int LT = LOG_NT + LOG_E;
    static constexpr size_t SMEM = NS::smem_bytes_sort() > NC::smem_bytes_compact() ? NS::smem_bytes_sort()
                                                                                       : NC::smem_bytes_compact();

    // Thread 0 claims the next item while the CTA still works on the current
    // one, so the claim, the step lookup and the dependency poll overlap the
    // tile work of the item before.  A CTA holds at most one claimed item
    // besides the one it runs; the smallest unfinished claimed item is always
    // one that a CTA runs, so the launch cannot deadlock.
    __device__ static void run(const SchedArgs& a, char* sm)
    {
        __shared__ unsigned long long s_item, s_next;
        __shared__ SchedStep s_st;
        __shared__ SchedInst s_in;
        __shared__ uint32_t s_tmp[33];
        if (threadIdx.x == 0)
            s_next = atomicAdd(a.next_item, 1ull);
        for (;;) {
            if (threadIdx.x == 0) {
                const unsigned long long x = s_next;
                s_item = x;
                if (x < a.total_items) {
                    s_next = atomicAdd(a.next_item, 1ull);
                    const SchedStep st = a.steps[__ldg(a.item_step + x)];
                    s_st = st;
                    s_in = a.insts[st.inst];
                    // bounded wait for the instance's previous passes
                    const uint64_t t0 = globaltimer_ns();
                    uint32_t spins = 0;
                    while (*((volatile uint32_t*)(a.done + st.inst)) < st.dep) {
                        if (globaltimer_ns() - t0 > a.timeout_ns) {
                            atomicExch(a.status, (int)VELO_ETIMEDOUT);
                            break;
                        }
                        __nanosleep(spins < 64 ? 32 : 256);
                        spins++;
                    }
                    __threadfence();
                }
            }
            __syncthreads();
            const unsigned long long item = s_item;
            if (item >= a.total_items)
                return;
            const SchedStep st = s_st;
            const SchedInst in = s_in;
            VELO_TRACE_WORK(item);
            const int tile = (int)(item - st.item_begin);
            NetGeom g { in.n, in.logN, 0 };
            switch (st.kind) {
            case STEP_SORT_PASS: {
                RowKP::Cols c { in.k, in.p };
                NS::template run<true>(c, g, st.pass, nullptr, tile, sm);
                break;
            }
            case STEP_COMPACT_COUNT: {
                RowKPM::Cols c { in.k, in.p, in.m };
                count_tile<RowKPM>(c, in.n, LT, tile, in.counts, s_tmp);
                break;
            }
            case STEP_COMPACT_SCAN:
                scan_tiles(in.counts, in.ntiles, in.prefix, in.d_count, s_tmp);
                break;
            case STEP_COMPACT_PASS: {
                RowKPM::Cols c { in.k, in.p, in.m };
                NC::template run<false>(c, g, st.pass, in.prefix, tile, sm);
                break;
            }
            default:
                break;
            }
            // the CTA's stores, then one gpu-scope fence and the completion
            // count (bar.sync orders every thread's stores before thread 0's
            // fence, which releases them with the count)
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(a.done + st.inst, 1u);
            }
        }
    }
};

template <int LOG_NT, int LOG_E>
__global__ void __launch_bounds__(1 << LOG_NT) k_sched(SchedArgs a)
{
    extern __shared__ __align__(16) char sm[];
    VELO_TRACE_KERNEL(TS_K_SCHED);
    Sched<LOG_NT, LOG_E>::run(a, sm);
}

} // namespace velo
