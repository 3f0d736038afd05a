// Oblivious segmented aggregation over key-sorted records with a small public
// output bound G (group-by tail of the filter + group-by pipeline).
//
// The algorithm is the segmented-sum group-by of the reference's oblivious
// aggregation (obliviator/operator_2/enclave/scalable_oblivious_join.c:221-262:
// forward segmented sum, group boundaries, compaction of one row per group),
// organised for the GPU in three passes over tiles of TS sorted rows:
//   A  per tile: first/last key, sum of the trailing key run, number of
//      complete groups ending inside the tile
//   B  one CTA: carries between tiles (segmented scan over tiles) and the
//      exclusive group-count prefix
//   C  per tile: in-tile segmented scan + carry; the last row of each valid
//      group carries the group total; the group with rank r (its position in
//      key order) is accumulated into output slot r by masked sums over all
//      G slots -- every row touches every slot, so addresses never depend on
//      the data
//   D  one CTA: slot-wise sum of the per-tile slot vectors.
// Rows whose "valid" flag is clear form their own key runs (the flag is part
// of the key) and never produce output.
#pragma once

#include <cstdint>
#include <type_traits>

#include "trace.cuh"

namespace velo {

constexpr int SEG_TS = 1024;     // rows per tile
constexpr int SEG_THREADS = 256; // 4 contiguous rows per thread
constexpr int SEG_RPT = SEG_TS / SEG_THREADS;
constexpr int SEG_MAX_G = 16;
// smem row slot with one pad word per 4 rows, so that the 4 contiguous rows
// of each of 16 neighbouring threads (8-byte words, a half-warp a shared
// memory wavefront) fall in different banks: thread t's row r at 5t + r
__device__ __forceinline__ int seg_slot(int i) { return i + (i >> 2); }
constexpr int SEG_TS_PAD = SEG_TS + SEG_TS / 4;
static_assert(SEG_RPT == 4, "seg_slot pads after each thread's 4 rows");

struct SegTileAgg {
    uint64_t head_key;
    uint64_t tail_key;
    uint32_t uniform;    // whole tile is one key run
    uint32_t tails;      // valid groups ending inside the tile (excluding its last row)
    uint32_t tail_valid; // the tile's last row is valid
    uint32_t pad_;
};

// Block-wide inclusive segmented scan (flag = "a new run starts at this
// thread's first row"; the operator resets at flags).  V int64 values.  Warp
// shuffles scan each warp; the warps' totals go through shared memory
// (sm_vals[i * 32 + warp], sm_flags[warp]) and each thread adds the carry
// of the warps before its own.  Ends with a barrier, so the caller may reuse
// sm_vals at once.
template <int V>
__device__ __forceinline__ void block_seg_scan(bool& flag, int64_t (&x)[V], int64_t* sm_vals, uint32_t* sm_flags)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool f = flag;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int64_t y[V];
#pragma unroll
        for (int i = 0; i < V; i++)
            y[i] = __shfl_up_sync(0xFFFFFFFFu, x[i], off);
        const bool fy = __shfl_up_sync(0xFFFFFFFFu, f ? 1 : 0, off) != 0;
        if (lane >= off) {
#pragma unroll
            for (int i = 0; i < V; i++)
                x[i] = f ? x[i] : x[i] + y[i];
            f = f | fy;
        }
    }
    __syncthreads(); // the caller may still read sm_vals
    if (lane == 31) {
#pragma unroll
        for (int i = 0; i < V; i++)
            sm_vals[i * 32 + warp] = x[i];
        sm_flags[warp] = f ? 1u : 0u;
    }
    __syncthreads();
    // the inclusive value at the end of the previous warp (the warp index is
    // public, so the loop bound is too)
    int64_t c[V];
#pragma unroll
    for (int i = 0; i < V; i++)
        c[i] = 0;
    bool cf = false;
    for (int w = 0; w < warp; w++) {
        const bool fw = sm_flags[w] != 0;
#pragma unroll
        for (int i = 0; i < V; i++)
            c[i] = fw ? sm_vals[i * 32 + w] : c[i] + sm_vals[i * 32 + w];
        cf = cf | fw;
    }
#pragma unroll
    for (int i = 0; i < V; i++)
        x[i] = f ? x[i] : x[i] + c[i];
    flag = f | cf;
    __syncthreads();
}

__device__ __forceinline__ uint32_t block_sum_u32(uint32_t x, uint32_t* tmp)
{
    for (int o = 16; o > 0; o >>= 1)
        x += __shfl_xor_sync(0xffffffffu, x, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
        tmp[threadIdx.x >> 5] = x;
    __syncthreads();
    uint32_t s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
        s += tmp[w];
    return s;
}

__device__ __forceinline__ int64_t warp_sum_i64(int64_t x)
{
    for (int o = 16; o > 0; o >>= 1)
        x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Warp reduce-scatter of 16 int64 values a lane: four halving steps over
// lane bits 4..1 (each lane keeps the half its lane bit selects and adds the
// partner's copy of it) and one add across lane bit 0; afterwards a[0] of
// lane L is the warp sum of value L >> 1.
__device__ __forceinline__ void warp_reduce_scatter16(int64_t (&a)[16], int lane)
{
#pragma unroll
    for (int step = 0; step < 4; step++) {
        const int o = 16 >> step;
        const int h = 8 >> step; // current length / 2
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int k = 0; k < h; k++) {
            const int64_t keep = up ? a[h + k] : a[k];
            const int64_t send = up ? a[k] : a[h + k];
            a[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    a[0] += __shfl_xor_sync(0xffffffffu, a[0], 1);
}

// Group records with a separate flag word (Agg::FLAG_WORD = true): o0 = the
// whole 64-bit out_bits(key), o1 = [63] not the last row of a valid group,
// then the sums; otherwise the flag shares word 0 with a key of at most 63 bits.
template <class A, class = void>
struct SegFlagWord {
    static constexpr bool value = false;
};
template <class A>
struct SegFlagWord<A, std::void_t<decltype(A::FLAG_WORD)>> {
    static constexpr bool value = A::FLAG_WORD;
};

// Agg: static constexpr int W (record words), V (values); struct Params
//      (public decoding parameters passed to every pass);
//      static uint64_t key(const uint64_t* w)      -- run key (includes validity)
//      static bool valid(const uint64_t* w)
//      static void values(const uint64_t* w, int64_t (&v)[V], const Params&)  -- zero when invalid
//      static int64_t out_key_from(uint64_t key)
template <class Agg>
struct SegAgg {
    static constexpr int W = Agg::W;
    static constexpr int V = Agg::V;
    // group record words of emit_rows: key (and flag), then the V sums
    static constexpr int FW = SegFlagWord<Agg>::value ? 1 : 0;
    static constexpr int OW = 1 + FW + V;
    // the tile area holds the W input words, later the OW output words
    static constexpr int TW = W > OW ? W : OW;
    using Params = typename Agg::Params;
    // emit_rows stages 1+V output words in the tile area; the other passes
    // only the W input words (smaller footprint, more CTAs per SM)
    static constexpr size_t SMEM = (size_t)SEG_TS_PAD * TW * 8 + (size_t)V * SEG_THREADS * 8 + SEG_THREADS * 4 + 256;
    static constexpr size_t SMEM_IN = (size_t)SEG_TS_PAD * W * 8 + (size_t)V * SEG_THREADS * 8 + SEG_THREADS * 4 + 256;
    static_assert((size_t)SEG_MAX_G * (1 + V) * 8 * 8 <= (size_t)SEG_TS_PAD * W * 8, "emit reduction fits the tile area");

    // stage the tile's records in smem (coalesced), then thread t owns rows
    // [t*RPT, t*RPT + RPT)
    __device__ static void load_tile(uint64_t* const* words, size_t base, uint64_t* sw)
    {
        for (int i = threadIdx.x; i < SEG_TS; i += SEG_THREADS) {
            VELO_TRACE_AT(TS_SEG_LOAD, words[0] + base + i);
#pragma unroll
            for (int x = 0; x < W; x++)
                sw[x * SEG_TS_PAD + seg_slot(i)] = words[x][base + i];
        }
        __syncthreads();
    }

    __device__ static void row(const uint64_t* sw, int i, uint64_t (&w)[W])
    {
#pragma unroll
        for (int x = 0; x < W; x++)
            w[x] = sw[x * SEG_TS_PAD + seg_slot(i)];
    }

    // pass A
    __device__ static void tile_summary(uint64_t* const* words, int tile, SegTileAgg* aggs, int64_t* tail_runs,
                                        const Params& prm, char* smem)
    {
        uint64_t* sw = reinterpret_cast<uint64_t*>(smem);
        uint32_t* tmp = reinterpret_cast<uint32_t*>(smem + (size_t)SEG_TS_PAD * W * 8);
        int64_t* red = reinterpret_cast<int64_t*>(smem + (size_t)SEG_TS_PAD * W * 8 + 256);
        const size_t base = (size_t)tile * SEG_TS;
        load_tile(words, base, sw);
        uint64_t wl[W];
        row(sw, SEG_TS - 1, wl);
        const uint64_t tail_key = Agg::key(wl);
        int64_t run[V];
#pragma unroll
        for (int i = 0; i < V; i++)
            run[i] = 0;
        uint32_t tails = 0;
        const int r0 = threadIdx.x * SEG_RPT;
#pragma unroll
        for (int r = 0; r < SEG_RPT; r++) {
            uint64_t w[W], wn[W];
            row(sw, r0 + r, w);
            const int nxt = r0 + r + 1 < SEG_TS ? r0 + r + 1 : SEG_TS - 1;
            row(sw, nxt, wn);
            const uint64_t k = Agg::key(w);
            int64_t v[V];
            Agg::values(w, v, prm);
            const bool in_run = (k == tail_key);
#pragma unroll
            for (int i = 0; i < V; i++)
                run[i] += in_run ? v[i] : 0;
            const bool internal = (r0 + r + 1 < SEG_TS);
            tails += (internal & (k != Agg::key(wn)) & Agg::valid(w)) ? 1u : 0u;
        }
        const uint32_t t_all = block_sum_u32(tails, tmp);
        // reduce the run sums: warp shuffles, then one value per warp
#pragma unroll
        for (int i = 0; i < V; i++) {
            const int64_t s = warp_sum_i64(run[i]);
            if ((threadIdx.x & 31) == 0)
                red[i * 8 + (threadIdx.x >> 5)] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint64_t w0[W];
            row(sw, 0, w0);
            SegTileAgg a;
            a.head_key = Agg::key(w0);
            a.tail_key = tail_key;
            a.uniform = (a.head_key == tail_key) ? 1u : 0u;
            a.tails = t_all;
            a.tail_valid = Agg::valid(wl) ? 1u : 0u;
            a.pad_ = 0;
            VELO_TRACE_AT(TS_SEG_META, aggs + tile);
            aggs[tile] = a;
#pragma unroll
            for (int i = 0; i < V; i++) {
                int64_t s = 0;
                for (int w = 0; w < SEG_THREADS / 32; w++)
                    s += red[i * 8 + w];
                tail_runs[(size_t)tile * V + i] = s;
            }
        }
    }

    // pass B: one CTA of 1024 threads
    __device__ static void carries(const SegTileAgg* aggs, const int64_t* tail_runs, int ntiles, int64_t* carry_in,
                                   uint32_t* tail_prefix, uint64_t* n_groups, char* smem)
    {
        // Rounds of blockDim.x consecutive tiles (coalesced loads, all issued
        // at once), each a block-wide segmented scan chained to the previous
        // round through (run_prev, cnt_prev).  Per tile t:
        //   run_out(t) = tail_runs[t] + (t continues t-1's run and is one run
        //                ? run_out(t-1) : 0)       (the run crossing t's end)
        //   carry_in[t] = t's first run continues t-1's last ? run_out(t-1) : 0
        //   tail_prefix[t] = groups ending in tiles before t
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        int64_t* wv = reinterpret_cast<int64_t*>(smem);                 // [V][32] warp prefixes
        uint32_t* wc = reinterpret_cast<uint32_t*>(smem + (size_t)V * 32 * 8);  // [32]
        int64_t* rv = reinterpret_cast<int64_t*>(smem + (size_t)V * 32 * 8 + 32 * 4);  // [V] round carry
        uint32_t* rc = reinterpret_cast<uint32_t*>(rv + V);              // [1]
        int64_t run_prev[V];
#pragma unroll
        for (int i = 0; i < V; i++)
            run_prev[i] = 0;
        uint32_t cnt_prev = 0;
        for (int base = 0; base < ntiles; base += blockDim.x) {
            const int t = base + (int)threadIdx.x;
            const bool in = t < ntiles;
            SegTileAgg a {};
            uint64_t prev_tail = 0, next_head = 0;
            int64_t x[V];
            if (in) {
                VELO_TRACE_AT(TS_SEG_META, aggs + t);
                a = aggs[t];
                prev_tail = t > 0 ? aggs[t - 1].tail_key : 0;
                next_head = t + 1 < ntiles ? aggs[t + 1].head_key : 0;
            }
#pragma unroll
            for (int i = 0; i < V; i++)
                x[i] = in ? tail_runs[(size_t)t * V + i] : 0;
            const bool joins = in && t > 0 && prev_tail == a.head_key;
            bool f = !(joins && a.uniform != 0); // a new run starts in this tile
            const bool last_tail = (t + 1 < ntiles) ? (a.tail_key != next_head) : true;
            const uint32_t cnt = in ? a.tails + ((last_tail && a.tail_valid != 0) ? 1u : 0u) : 0u;
            uint32_t c = cnt;
            // warp-inclusive segmented scan of x (resetting at f) and scan of c
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                int64_t y[V];
#pragma unroll
                for (int i = 0; i < V; i++)
                    y[i] = __shfl_up_sync(0xFFFFFFFFu, x[i], off);
                const int fy = __shfl_up_sync(0xFFFFFFFFu, f ? 1 : 0, off);
                const uint32_t cy = __shfl_up_sync(0xFFFFFFFFu, c, off);
                if (lane >= off) {
#pragma unroll
                    for (int i = 0; i < V; i++)
                        x[i] = f ? x[i] : x[i] + y[i];
                    f = f || fy != 0;
                    c += cy;
                }
            }
            if (lane == 31) {
#pragma unroll
                for (int i = 0; i < V; i++)
                    wv[i * 32 + warp] = x[i];
                wc[warp] = (c << 1) | (f ? 1u : 0u);
            }
            __syncthreads();
            if (warp == 0) {
                // scan of the warp totals, then exclusive prefixes that start
                // from the previous rounds' carry
                int64_t z[V];
                bool g = false;
                uint32_t d = 0;
#pragma unroll
                for (int i = 0; i < V; i++)
                    z[i] = lane < nw ? wv[i * 32 + lane] : 0;
                if (lane < nw) {
                    g = (wc[lane] & 1u) != 0;
                    d = wc[lane] >> 1;
                }
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    int64_t y[V];
#pragma unroll
                    for (int i = 0; i < V; i++)
                        y[i] = __shfl_up_sync(0xFFFFFFFFu, z[i], off);
                    const int gy = __shfl_up_sync(0xFFFFFFFFu, g ? 1 : 0, off);
                    const uint32_t dy = __shfl_up_sync(0xFFFFFFFFu, d, off);
                    if (lane >= off) {
#pragma unroll
                        for (int i = 0; i < V; i++)
                            z[i] = g ? z[i] : z[i] + y[i];
                        g = g || gy != 0;
                        d += dy;
                    }
                }
                int64_t ez[V];
#pragma unroll
                for (int i = 0; i < V; i++)
                    ez[i] = __shfl_up_sync(0xFFFFFFFFu, z[i], 1);
                int eg = __shfl_up_sync(0xFFFFFFFFu, g ? 1 : 0, 1);
                uint32_t ed = __shfl_up_sync(0xFFFFFFFFu, d, 1);
                if (lane == 0) {
#pragma unroll
                    for (int i = 0; i < V; i++)
                        ez[i] = 0;
                    eg = 0;
                    ed = 0;
                }
                __syncwarp();
                if (lane < nw) {
#pragma unroll
                    for (int i = 0; i < V; i++)
                        wv[i * 32 + lane] = eg ? ez[i] : run_prev[i] + ez[i];
                    wc[lane] = cnt_prev + ed;
                }
                if (lane == nw - 1) {
#pragma unroll
                    for (int i = 0; i < V; i++)
                        rv[i] = g ? z[i] : run_prev[i] + z[i];
                    rc[0] = cnt_prev + d;
                }
            }
            __syncthreads();
            int64_t ro[V], pr[V];
#pragma unroll
            for (int i = 0; i < V; i++) {
                const int64_t wp = wv[i * 32 + warp];
                ro[i] = f ? x[i] : wp + x[i]; // run_out(t)
                pr[i] = __shfl_up_sync(0xFFFFFFFFu, ro[i], 1);
                if (lane == 0)
                    pr[i] = wp; // run_out(t - 1)
            }
            const uint32_t cin = wc[warp] + c - cnt;
            if (in) {
                VELO_TRACE_AT(TS_SEG_META, carry_in + (size_t)t * V);
#pragma unroll
                for (int i = 0; i < V; i++)
                    carry_in[(size_t)t * V + i] = joins ? pr[i] : 0;
                tail_prefix[t] = cin;
            }
#pragma unroll
            for (int i = 0; i < V; i++)
                run_prev[i] = rv[i];
            cnt_prev = rc[0];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            *n_groups = cnt_prev;
    }

    // pass C
    __device__ static void emit(uint64_t* const* words, int tile, int ntiles, const SegTileAgg* aggs,
                                const int64_t* carry_in, const uint32_t* tail_prefix, int G, int64_t* tile_out,
                                const Params& prm, char* smem)
    {
        uint64_t* sw = reinterpret_cast<uint64_t*>(smem);
        int64_t* svals = reinterpret_cast<int64_t*>(smem + (size_t)SEG_TS_PAD * W * 8);
        uint32_t* sflags = reinterpret_cast<uint32_t*>(smem + (size_t)SEG_TS_PAD * W * 8 + (size_t)V * SEG_THREADS * 8);
        const size_t base = (size_t)tile * SEG_TS;
        load_tile(words, base, sw);
        const uint64_t next_head = (tile + 1 < ntiles) ? aggs[tile + 1].head_key : ~0ull;
        const bool last_tile = (tile + 1 >= ntiles);
        const uint64_t head_key = aggs[tile].head_key;
        const int r0 = threadIdx.x * SEG_RPT;

        // thread-local inclusive segmented scan of my rows
        int64_t pref[SEG_RPT][V];
        uint64_t keys[SEG_RPT];
        bool tail[SEG_RPT];
        bool start_flag = false; // a run starts inside my rows (at row r0 or later)
        {
            uint64_t wprev[W];
            row(sw, r0 > 0 ? r0 - 1 : 0, wprev);
            uint64_t prev_key = Agg::key(wprev);
            int64_t run[V];
#pragma unroll
            for (int i = 0; i < V; i++)
                run[i] = 0;
#pragma unroll
            for (int r = 0; r < SEG_RPT; r++) {
                uint64_t w[W];
                row(sw, r0 + r, w);
                const uint64_t k = Agg::key(w);
                int64_t v[V];
                Agg::values(w, v, prm);
                const bool starts = (r0 + r == 0) ? true : (k != prev_key);
                start_flag = start_flag | starts;
#pragma unroll
                for (int i = 0; i < V; i++)
                    run[i] = (starts ? 0 : run[i]) + v[i];
#pragma unroll
                for (int i = 0; i < V; i++)
                    pref[r][i] = run[i];
                keys[r] = k;
                prev_key = k;
                uint64_t wn[W];
                const int nxt = r0 + r + 1 < SEG_TS ? r0 + r + 1 : SEG_TS - 1;
                row(sw, nxt, wn);
                const uint64_t kn = (r0 + r + 1 < SEG_TS) ? Agg::key(wn) : next_head;
                const bool ends = (r0 + r + 1 < SEG_TS || !last_tile) ? (k != kn) : true;
                tail[r] = ends & Agg::valid(w);
            }
        }
        // exclusive block segmented scan of thread aggregates: my carry-in is
        // the inclusive result of thread-1 unless a run starts at my row r0
        int64_t agg[V];
#pragma unroll
        for (int i = 0; i < V; i++)
            agg[i] = pref[SEG_RPT - 1][i];
        bool fl = start_flag;
        block_seg_scan<V>(fl, agg, svals, sflags);
#pragma unroll
        for (int i = 0; i < V; i++)
            svals[i * SEG_THREADS + threadIdx.x] = agg[i];
        __syncthreads();
        int64_t cin[V];
#pragma unroll
        for (int i = 0; i < V; i++)
            cin[i] = (threadIdx.x > 0) ? svals[i * SEG_THREADS + threadIdx.x - 1] : 0;
        // the tile-level carry applies to rows of the tile's first run
        int64_t tc[V];
#pragma unroll
        for (int i = 0; i < V; i++)
            tc[i] = carry_in[(size_t)tile * V + i];
        // rank of my first tail: tail prefix of the tile + tails of threads before me
        uint32_t my_tails = 0;
#pragma unroll
        for (int r = 0; r < SEG_RPT; r++)
            my_tails += tail[r] ? 1u : 0u;
        uint32_t tails_total;
        const uint32_t before = block_exclusive_scan(my_tails, reinterpret_cast<uint32_t*>(svals), &tails_total);
        const uint32_t rank0 = tail_prefix[tile] + before;

        // my leading rows continue the run open at the end of thread t-1
        // unless a new run starts exactly at my first row
        bool lead = (r0 > 0);
        if (r0 > 0) {
            uint64_t wp[W];
            row(sw, r0 - 1, wp);
            lead = (Agg::key(wp) == keys[0]);
        }
        // segment totals up to each row: my prefix, the in-tile carry of the
        // preceding threads, and the cross-tile carry of the tile's first run
#pragma unroll
        for (int r = 0; r < SEG_RPT; r++) {
            if (r > 0)
                lead = lead & (keys[r] == keys[r - 1]);
            const bool first_run_of_tile = (keys[r] == head_key);
#pragma unroll
            for (int i = 0; i < V; i++)
                pref[r][i] += (lead ? cin[i] : 0) + (first_run_of_tile ? tc[i] : 0);
        }
        // output slot j receives (key, totals) of the tail whose rank is j;
        // every row is folded into every slot with a mask
        __syncthreads();
        int64_t* red = reinterpret_cast<int64_t*>(smem); // reuse the tile area
        // slots in chunks of 2: every lane folds its rows into 2 x 8 values
        // (slot, value; values past 1+V stay zero), then a warp reduce-scatter
        // leaves lanes 2L and 2L + 1 with the warp sum of value L (chunks of
        // 4 slots kept 32 sums a lane live: 102 registers, two CTAs an SM)
        static_assert(1 + V <= 8, "a slot's key and values fit 8 words");
        constexpr int SLOTS = 2;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int j0 = 0; j0 < G; j0 += SLOTS) {
            int64_t acc[8 * SLOTS];
#pragma unroll
            for (int q = 0; q < 8 * SLOTS; q++)
                acc[q] = 0;
            // the ranks of a thread's tails are distinct, so each slot takes
            // at most one of its rows: a select, not an add (the block sum
            // below adds the threads' slots, all but one zero)
            uint32_t rank = rank0;
#pragma unroll
            for (int r = 0; r < SEG_RPT; r++) {
                const int64_t kv = Agg::out_key_from(keys[r]);
#pragma unroll
                for (int jj = 0; jj < SLOTS; jj++) {
                    const bool hit = tail[r] & (rank == (uint32_t)(j0 + jj));
                    acc[jj * 8] = hit ? kv : acc[jj * 8];
#pragma unroll
                    for (int i = 0; i < V; i++)
                        acc[jj * 8 + 1 + i] = hit ? pref[r][i] : acc[jj * 8 + 1 + i];
                }
                rank += tail[r] ? 1u : 0u;
            }
            warp_reduce_scatter16(acc, lane);
            if ((lane & 1) == 0)
                red[(lane >> 1) * 8 + warp] = acc[0];
            __syncthreads();
            const int gn = G - j0 < SLOTS ? G - j0 : SLOTS;
            for (int q = threadIdx.x; q < gn * (1 + V); q += SEG_THREADS) {
                const int jj = q / (1 + V), i = q - jj * (1 + V);
                const size_t o = (size_t)tile * G * (1 + V) + (size_t)(j0 + jj) * (1 + V) + i;
                VELO_TRACE_AT(TS_SEG_OUT, tile_out + o);
                int64_t sum = 0;
#pragma unroll
                for (int w = 0; w < SEG_THREADS / 32; w++)
                    sum += red[(jj * 8 + i) * 8 + w];
                tile_out[o] = sum;
            }
            __syncthreads();
        }
    }

    // pass C for a large output bound: every row writes a group record
    // (o0 = [63] not the last row of a valid group | [31:0] Agg::out_bits,
    // o1.. = the group's sums, valid only on the group's last row); an
    // ORCompact of the records then yields the groups in key order.
    __device__ static void emit_rows(uint64_t* const* words, int tile, int ntiles, const SegTileAgg* aggs,
                                     const int64_t* carry_in, uint64_t* const* out, const Params& prm, char* smem)
    {
        emit_stage(words, tile, ntiles, aggs, carry_in, prm, smem);
        const uint64_t* so = reinterpret_cast<const uint64_t*>(smem);
        const size_t base = (size_t)tile * SEG_TS;
        for (int i = threadIdx.x; i < SEG_TS; i += SEG_THREADS) {
            VELO_TRACE_AT(TS_SEG_OUT, out[0] + base + i);
#pragma unroll
            for (int x = 0; x < OW; x++)
                out[x][base + i] = so[(size_t)x * SEG_TS_PAD + seg_slot(i)];
        }
    }

    // emit_rows without the stores: leaves the tile's OW output words of
    // row i at smem word x * SEG_TS_PAD + seg_slot(i) (after a barrier)
    // REGS: the thread's SEG_RPT rows r0 .. r0 + SEG_RPT - 1 (r0 = 4t) go
    // to regs[r][0 .. OW-1] instead of shared memory (no staging, no final
    // barriers), for a consumer that only needs the thread's own rows
    template <bool REGS = false>
    __device__ static void emit_stage(uint64_t* const* words, int tile, int ntiles, const SegTileAgg* aggs,
                                      const int64_t* carry_in, const Params& prm, char* smem,
                                      uint64_t (*regs)[OW] = nullptr)
    {
        uint64_t* sw = reinterpret_cast<uint64_t*>(smem);
        int64_t* svals = reinterpret_cast<int64_t*>(smem + (size_t)SEG_TS_PAD * TW * 8);
        uint32_t* sflags = reinterpret_cast<uint32_t*>(smem + (size_t)SEG_TS_PAD * TW * 8 + (size_t)V * SEG_THREADS * 8);
        const size_t base = (size_t)tile * SEG_TS;
        load_tile(words, base, sw);
        const uint64_t next_head = (tile + 1 < ntiles) ? aggs[tile + 1].head_key : ~0ull;
        const bool last_tile = (tile + 1 >= ntiles);
        const uint64_t head_key = aggs[tile].head_key;
        const int r0 = threadIdx.x * SEG_RPT;
        int64_t pref[SEG_RPT][V];
        uint64_t keys[SEG_RPT];
        bool tail[SEG_RPT];
        bool start_flag = false;
        {
            uint64_t wprev[W];
            row(sw, r0 > 0 ? r0 - 1 : 0, wprev);
            uint64_t prev_key = Agg::key(wprev);
            int64_t run[V];
#pragma unroll
            for (int i = 0; i < V; i++)
                run[i] = 0;
#pragma unroll
            for (int r = 0; r < SEG_RPT; r++) {
                uint64_t w[W];
                row(sw, r0 + r, w);
                const uint64_t k = Agg::key(w);
                int64_t v[V];
                Agg::values(w, v, prm);
                const bool starts = (r0 + r == 0) ? true : (k != prev_key);
                start_flag = start_flag | starts;
#pragma unroll
                for (int i = 0; i < V; i++)
                    run[i] = (starts ? 0 : run[i]) + v[i];
#pragma unroll
                for (int i = 0; i < V; i++)
                    pref[r][i] = run[i];
                keys[r] = k;
                prev_key = k;
                uint64_t wn[W];
                const int nxt = r0 + r + 1 < SEG_TS ? r0 + r + 1 : SEG_TS - 1;
                row(sw, nxt, wn);
                const uint64_t kn = (r0 + r + 1 < SEG_TS) ? Agg::key(wn) : next_head;
                const bool ends = (r0 + r + 1 < SEG_TS || !last_tile) ? (k != kn) : true;
                tail[r] = ends & Agg::valid(w);
            }
        }
        int64_t agg[V];
#pragma unroll
        for (int i = 0; i < V; i++)
            agg[i] = pref[SEG_RPT - 1][i];
        bool fl = start_flag;
        block_seg_scan<V>(fl, agg, svals, sflags);
#pragma unroll
        for (int i = 0; i < V; i++)
            svals[i * SEG_THREADS + threadIdx.x] = agg[i];
        __syncthreads();
        int64_t cin[V];
#pragma unroll
        for (int i = 0; i < V; i++)
            cin[i] = (threadIdx.x > 0) ? svals[i * SEG_THREADS + threadIdx.x - 1] : 0;
        int64_t tc[V];
#pragma unroll
        for (int i = 0; i < V; i++)
            tc[i] = carry_in[(size_t)tile * V + i];
        bool lead = (r0 > 0);
        if (r0 > 0) {
            uint64_t wp[W];
            row(sw, r0 - 1, wp);
            lead = (Agg::key(wp) == keys[0]);
        }
        if constexpr (REGS) {
#pragma unroll
            for (int r = 0; r < SEG_RPT; r++) {
                if (r > 0)
                    lead = lead & (keys[r] == keys[r - 1]);
                const bool first_run_of_tile = (keys[r] == head_key);
                if constexpr (FW == 1) {
                    regs[r][0] = Agg::out_bits(keys[r]);
                    regs[r][1] = (uint64_t)(!tail[r]) << 63;
                } else {
                    regs[r][0] = ((uint64_t)(!tail[r]) << 63) | Agg::out_bits(keys[r]);
                }
#pragma unroll
                for (int i = 0; i < V; i++)
                    regs[r][1 + FW + i] = (uint64_t)(pref[r][i] + (lead ? cin[i] : 0) + (first_run_of_tile ? tc[i] : 0));
            }
            return;
        }
        __syncthreads();
        // stage the output records in smem so the global stores stay coalesced
        uint64_t* so = sw;
#pragma unroll
        for (int r = 0; r < SEG_RPT; r++) {
            if (r > 0)
                lead = lead & (keys[r] == keys[r - 1]);
            const bool first_run_of_tile = (keys[r] == head_key);
            if constexpr (FW == 1) {
                so[seg_slot(r0 + r)] = Agg::out_bits(keys[r]);
                so[(size_t)SEG_TS_PAD + seg_slot(r0 + r)] = (uint64_t)(!tail[r]) << 63;
            } else {
                so[seg_slot(r0 + r)] = ((uint64_t)(!tail[r]) << 63) | Agg::out_bits(keys[r]);
            }
#pragma unroll
            for (int i = 0; i < V; i++)
                so[(size_t)(1 + FW + i) * SEG_TS_PAD + seg_slot(r0 + r)] =
                    (uint64_t)(pref[r][i] + (lead ? cin[i] : 0) + (first_run_of_tile ? tc[i] : 0));
        }
        __syncthreads();
    }

    // pass D: out[q] = sum over tiles of tile_out[tile][q]; one CTA of
    // SEG_THREADS threads per output word q (0 .. G*(1+V)-1)
    __device__ static void finish(const int64_t* tile_out, int ntiles, int G, int64_t* out, int q)
    {
        __shared__ int64_t part[SEG_THREADS / 32];
        const int QN = G * (1 + V);
        int64_t sum = 0;
        for (int t = threadIdx.x; t < ntiles; t += SEG_THREADS) {
            VELO_TRACE_AT(TS_SEG_OUT, tile_out + (size_t)t * QN + q);
            sum += tile_out[(size_t)t * QN + q];
        }
        sum = warp_sum_i64(sum);
        if ((threadIdx.x & 31) == 0)
            part[threadIdx.x >> 5] = sum;
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t s = 0;
            for (int w = 0; w < SEG_THREADS / 32; w++)
                s += part[w];
            out[q] = s;
        }
    }
};

} // namespace velo
