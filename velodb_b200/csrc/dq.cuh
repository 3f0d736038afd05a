// Persistent command queue: the job format shared by the host planner
// (dq.cu) and the device consumer (dq_kernel.cu).
//
// The reference's TaskManager runs ONE cooperative persistent kernel that
// polls a host-mapped command ring and executes one command at a time, the
// whole grid on it, separated by grid.sync() (src/cuda/persistent_kernel.cu:
// 76-124, src/cuda/commands.cpp:47-91).  Here the host plans every command
// into a job -- a list of steps, each step one pass of the oblivious pipeline
// split into tile-sized work items -- and writes it into a host-mapped ring.
// A persistent kernel (one CTA per SM slot) ingests published jobs into a
// device-side job table.  Each job has one open step at a time; every CTA
// takes a ready item of the oldest open job that has one, runs it and counts
// it done, and the step's last item opens the next step.  Many jobs run at
// once, and an item never waits for another.  The kernel exits by itself
// once nothing is left to do for a short idle time, and the host relaunches
// it when new jobs arrive.
#pragma once

#include <cstdint>

#include "groupby.cuh"
#include "join.cuh"
#include "ops.cuh"

namespace velo {

constexpr int DQ_THREADS = 256;
constexpr int DQ_HOST_RING = 64;    // jobs published and not yet retired
constexpr int DQ_DEV_RING = 256;    // device job table slots (a multiple of the host ring)
constexpr int DQ_MAX_STEPS = 384;   // passes of one job
constexpr int DQ_ARG_BYTES = 8192;  // argument blocks of one job
constexpr int DQ_STEP_ARG_MAX = 512; // largest argument block of one step (staged in shared memory)
// tile of the three-word record networks (256 threads x 8 rows); every other
// network runs 4096-row tiles (256 threads x 16 rows)
constexpr int DQ_LT3 = 11;
constexpr int DQ_LT = 12;
// rows an element-wise item covers
constexpr int DQ_ELEM_ITEM = DQ_THREADS * 16;

enum DqKind : uint32_t {
    DQ_K_NOP = 0,
    // network passes (tile = item)
    DQ_K_SORT_KP,
    DQ_K_COMPACT_KPM,
    DQ_K_SORT_LI2,
    DQ_K_COMPACT_LI2,
    DQ_K_SORT_LI3,
    DQ_K_COMPACT_LI3,
    DQ_K_SORT_JREC,
    DQ_K_COMPACT_JREC,
    DQ_K_SORT_REC3,
    DQ_K_SORT_REC3K2,
    DQ_K_COMPACT_REC3K2,
    // mark counts of network tiles, and their scan (one item)
    DQ_K_COUNT_KPM,
    DQ_K_COUNT_JREC,
    DQ_K_COUNT_REC3K2,
    DQ_K_SCAN_TILES,
    // filter + group-by
    DQ_K_LI_PACK2,
    DQ_K_LI_PACK3,
    DQ_K_SEG_SUMMARY2,
    DQ_K_SEG_SUMMARY3,
    DQ_K_SEG_CARRIES2,
    DQ_K_SEG_CARRIES3,
    DQ_K_SEG_EMIT2,
    DQ_K_SEG_EMIT3,
    DQ_K_SEG_FINISH,
    // join + group-by + top-k
    DQ_K_JOIN_PACK,
    DQ_K_JFILL_SUMMARY,
    DQ_K_JFILL_CARRIES,
    DQ_K_JFILL_APPLY,
    DQ_K_JSEG_SUMMARY,
    DQ_K_JSEG_CARRIES,
    DQ_K_JSEG_EMIT_TOPK,
    DQ_K_TOPK_REDUCE,
    DQ_K_TOPK_OUT,
    // union-sort operators (PK-FK join, oblivious gather)
    DQ_K_UFILL_SUM_JOIN,
    DQ_K_UFILL_SUM_GATHER,
    DQ_K_UFILL_SCAN,
    DQ_K_UFILL_APPLY_JOIN,
    DQ_K_UFILL_APPLY_GATHER,
    DQ_K_OJOIN_PACK,
    DQ_K_OJOIN_OUT,
    DQ_K_JOIN_COUNTS,
    DQ_K_OGATHER_PACK,
    DQ_K_OGATHER_OUT,
    // element-wise operators of the reference command set
    DQ_K_PERMUTE,
    DQ_K_GATHER,
    DQ_K_COMPARE_EQ,
    DQ_K_COMPOSE,
    DQ_K_FILL_U8,
    DQ_K_SCATTER_COUNT,
    DQ_K_SCATTER_WRITE,
    DQ_K_SHUFFLE_PACK,
    DQ_K_COPY_U32,
    // small steps of the served three-way join chain and of result delivery
    DQ_K_RANGE_MASK_I32,
    DQ_K_RANGE_MASK_I64,
    DQ_K_ROWID_KEYS,
    DQ_K_ROWID_RIDS,
    DQ_K_SUM_U64,
    DQ_K_SET_WORDS,
    DQ_K_COPY_WORDS,
    DQ_K_COUNT_KINDS
};

// one step: `ntiles` items, numbered from `begin` within the job (copied
// as two 16-byte words)
struct alignas(16) DqStep {
    uint32_t kind;
    uint32_t ntiles;
    uint32_t begin;
    uint32_t arg; // byte offset of the step's argument block in the job
    NetPass pass; // network passes only
};
static_assert(sizeof(DqStep) == 32, "32-byte steps");

struct alignas(16) DqJobHdr {
    uint64_t seq;   // 1, 2, ... in publication order
    uint64_t after; // every job with seq <= after completes before this one starts (0: none)
    uint32_t nsteps;
    uint32_t nitems;
    uint32_t arg_bytes;
    uint32_t pad_[9];
};
static_assert(sizeof(DqJobHdr) == 64, "64-byte header");

struct DqJob {
    DqJobHdr h;
    DqStep steps[DQ_MAX_STEPS];
    // argument blocks; the consumer stages DQ_STEP_ARG_MAX bytes from each
    // block's start, so the array has that much slack past DQ_ARG_BYTES
    alignas(16) unsigned char args[DQ_ARG_BYTES + DQ_STEP_ARG_MAX];
};

// ---- argument blocks ---------------------------------------------------------

template <class R>
struct DqNetArgs {
    typename R::Cols c;
    NetGeom g;
    const uint32_t* prefix;
};

template <class R>
struct DqCountArgs {
    typename R::Cols c;
    size_t n;
    int lt;
    uint32_t* counts;
};

struct DqScanArgs {
    const uint32_t* counts;
    uint32_t* prefix;
    uint64_t* d_count;
    int ntiles;
};

struct DqLiPackArgs {
    LiCols c;
    velo_lineitem_pred p;
    LiParams prm;
    size_t n, n_rec;
    int lt;
    uint64_t* w[3];
    uint32_t* counts;
};

struct DqSegArgs {
    uint64_t* w[3];
    SegTileAgg* aggs;
    int64_t* runs;
    int64_t* carry;
    uint32_t* tail_prefix;
    uint64_t* n_groups;
    int64_t* tile_out;
    int64_t* out;
    const uint64_t* d_rows;
    uint64_t* d_counts;
    LiParams prm;
    int ntiles;
    int G;
};

struct DqJoinPackArgs {
    const int32_t *dk, *dd, *ff;
    const int64_t* fp;
    size_t nd, nf, n_rec;
    int32_t date_hi;
    int64_t price_hi;
    uint64_t *w0, *w1;
};

struct DqJFillArgs {
    uint64_t* w0;
    DimCarry* tile_last;
    DimCarry* carry;
    int ntiles;
};

struct DqJSegArgs {
    JRec::Cols c;
    SegTileAgg* aggs;
    int64_t* runs;
    int64_t* carry;
    uint32_t* tail_prefix;
    uint64_t* n_groups;
    uint64_t *out0, *out1;
    int ntiles;
    int cand;
};

struct DqTopkArgs {
    const uint64_t *in0, *in1;
    uint64_t *out0, *out1;
    int rn;
    int c;
    // final step
    size_t k;
    int64_t* out;
    const uint64_t* n_groups;
    const uint64_t* n_joined;
    uint64_t* d_counts;
};

struct DqUFillArgs {
    uint64_t *w0, *w1, *w2;
    FillCarry* tl;
    FillCarry* carry;
    unsigned long long* d_stat;
    int ntiles;
};

struct DqOJoinArgs {
    const void *bk, *pk;
    const uint8_t *bm, *pm;
    size_t bn, pn, rows;
    int key64;
    uint64_t *w0, *w1, *w2;
    int64_t *ob, *op;
    const uint64_t* n_joined;
    const unsigned long long* dups;
    uint64_t* d_counts;
};

struct DqOGatherArgs {
    const uint64_t* table;
    const uint32_t* rids;
    size_t tn, rn, rows;
    uint64_t *w0, *w1, *w2;
    uint64_t* out;
};

// element-wise steps: n elements of `bytes` bytes (permute, gather,
// compare_eq), or the operator's own meaning of the fields
struct DqElemArgs {
    void* out;
    const void* in;
    const void* idx;
    const uint8_t* mask;
    const void* in2;
    size_t n;
    size_t np;
    uint64_t key, counter;
    int64_t lo, hi;
    uint32_t bytes;
    uint32_t value;
};

struct DqCopyArgs {
    const uint64_t* src;
    uint64_t* dst; // device address of host-mapped memory (or device memory)
    uint32_t words;
};

// ---- device-side state ---------------------------------------------------------

// A job's slot in the device job table.  Only the job's current step is
// open for claims: `claim` packs the step, its item count and the items
// handed out so far, and a CTA takes item k by a compare-and-swap of k -> k+1.
// The CTA that completes the step's last item opens the next step (or marks
// the job complete with step DQ_STEP_DONE), so no CTA ever waits on an item
// dependency: it only takes items that are ready.
constexpr unsigned long long DQ_STEP_DONE = 0xFFFFull;
__host__ __device__ constexpr unsigned long long dq_claim_word(unsigned long long step, unsigned long long ntiles)
{
    return (step << 48) | (ntiles << 24);
}
constexpr uint64_t DQ_MAX_ITEMS_PER_STEP = (1ull << 24) - 1;

// one 128-byte line per slot: every CTA adds to the claim and done words of
// the open jobs, which must not share lines with each other or with the
// queue-wide words below
struct alignas(128) DqSlot {
    unsigned long long claim; // [63:48] step | [47:24] items of the step | [23:0] items handed out
    unsigned long long seq;   // job held by the slot (0: none yet)
    unsigned int done;        // completed items of the current step
    int status;               // VELO_OK, or the first error of the job
    unsigned int nsteps;
    unsigned int pad_;
};

struct DqState {
    // read by every idle CTA: one line of their own
    alignas(128) unsigned long long ingested; // jobs ingested (seqs 1..ingested)
    unsigned long long complete_below;        // every job with seq < complete_below is complete
    int exiting;                              // the grid is leaving; no more ingests
    unsigned int host_stop;                   // device copy of the host's stop word
    // the host-ring poller's words
    alignas(128) unsigned long long last_poll; // %globaltimer of the last read of the host ring
    unsigned long long launches;
    int lock; // held while a CTA ingests or decides to exit
    DqSlot slot[DQ_DEV_RING];
};

// host-mapped words: the host writes head/stop, the device the rest
struct DqHostCtl {
    unsigned long long head;            // jobs published
    unsigned int stop;                  // leave as soon as every published job is done
    unsigned int pad_;
    unsigned long long done_seq[DQ_HOST_RING]; // seq of the last job completed in each ring slot
    int status[DQ_HOST_RING];
    int fault; // set when the consumer stopped on an inconsistent job table
    int pad2_;
    unsigned long long exited_launch; // the consumer launch that decided to exit (launches count from 1)
};

struct DqParams {
    DqState* st;
    DqJob* table;        // device job table (DQ_DEV_RING slots)
    const DqJob* ring;   // host-mapped ring (DQ_HOST_RING slots)
    DqHostCtl* ctl;      // host-mapped control words
    uint64_t wait_ns;    // limit of one dependency wait
    uint64_t idle_ns;    // idle time after which the grid exits
};

} // namespace velo
