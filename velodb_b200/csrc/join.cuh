// Oblivious PK-FK join + group-by + top-k: record layout, aggregate, and the
// device steps of the pipeline (pack, forward fill, top-k rounds) plus its
// scratch layout, shared by the plain pipeline (join.cu) and the persistent
// command queue (dq_kernel.cu).  The pipeline is described in join.cu.
#pragma once

#include "common.hpp"
#include "network.cuh"
#include "segagg.cuh"
#include "topk.cuh"

namespace velo {

// ties (fact rows of one key) are aggregated, their order is irrelevant; the
// union sorts on the whole of w0, whose bits below the (key, tag) pair only
// refine that order
using JRec = RowRec<2, 1, false, KEY_FULL>;
constexpr uint64_t J_KEYTAG = 0xFFFFFFFF80000000ull;
constexpr uint64_t J_JOINED = 1ull << 29;
constexpr int J_LT = 12; // 4096-row tiles (CTA shape per record width: Tile12)
// up to 8 fused global levels: 16 contiguous rows of 8-byte words fill a line
constexpr int J_LMAX = J_LT - 4 < 8 ? J_LT - 4 : 8;
constexpr int J_TOPK_MIN = 16; // candidates a group-by tile keeps at least

// group-by over the joined prefix: run key = (fk, joined), values = (sum price, count)
struct JoinAgg {
    static constexpr int W = 2;
    static constexpr int V = 2;
    struct Params {};
    __device__ __forceinline__ static uint64_t key(const uint64_t* w) { return w[0] & (0xFFFFFFFF00000000ull | J_JOINED); }
    __device__ __forceinline__ static bool valid(const uint64_t* w) { return (w[0] & J_JOINED) != 0; }
    __device__ __forceinline__ static void values(const uint64_t* w, int64_t (&v)[V], const Params&)
    {
        const bool ok = valid(w);
        v[0] = ok ? (int64_t)w[1] : 0;
        v[1] = ok ? 1 : 0;
    }
    __device__ __forceinline__ static int64_t out_key_from(uint64_t key) { return (int64_t)(key >> 32); }
    __device__ __forceinline__ static uint64_t out_bits(uint64_t key) { return key >> 32; }
};
using JSeg = SegAgg<JoinAgg>;

// pack of the union rows handled by CTA `blk` of `nblk` (grid stride)
__device__ __forceinline__ void join_pack_body(const int32_t* dk, const int32_t* dd, size_t nd, const int32_t* ff,
                                               const int64_t* fp, size_t nf, int32_t date_hi, int64_t price_hi,
                                               size_t n_rec, uint64_t* w0, uint64_t* w1, size_t blk, size_t nblk)
{
    for (size_t g = blk * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(g, n_rec); g += nblk * blockDim.x) {
        uint64_t a = ~0ull, b = ~0ull;
        if (g < nd) {
            const uint64_t key = (uint32_t)dk[g] ^ 0x80000000u;
            a = (key << 32) | ((uint64_t)(dd[g] < date_hi) << 30);
            b = 0;
        } else if (g < nd + nf) {
            const size_t j = g - nd;
            const uint64_t key = (uint32_t)ff[j] ^ 0x80000000u;
            const int64_t pr = fp[j];
            a = (key << 32) | (1ull << 31) | ((uint64_t)(pr < price_hi) << 30);
            b = (uint64_t)pr;
        }
        w0[g] = a;
        w1[g] = b;
    }
}


// ---- forward fill: last dimension row (has, key, valid) at or before each row
struct DimCarry {
    uint32_t has;
    uint32_t valid;
    uint64_t key;
};

__device__ __forceinline__ DimCarry dim_of(uint64_t w0)
{
    const bool is_dim = ((w0 >> 31) & 1ull) == 0 && w0 != ~0ull;
    return DimCarry { is_dim ? 1u : 0u, (uint32_t)((w0 >> 30) & 1ull), w0 >> 32 };
}

__device__ __forceinline__ DimCarry dim_combine(const DimCarry& left, const DimCarry& right)
{
    return right.has ? right : left;
}

constexpr int FILL_TS = 2048, FILL_THREADS = 256, FILL_RPT = FILL_TS / FILL_THREADS;

__device__ __forceinline__ DimCarry dim_shfl(const DimCarry& c, int src_delta, bool up)
{
    DimCarry r;
    const uint32_t hv = c.has | (c.valid << 1);
    const uint32_t x = up ? __shfl_up_sync(0xFFFFFFFFu, hv, src_delta) : __shfl_xor_sync(0xFFFFFFFFu, hv, src_delta);
    r.key = up ? __shfl_up_sync(0xFFFFFFFFu, c.key, src_delta) : __shfl_xor_sync(0xFFFFFFFFu, c.key, src_delta);
    r.has = x & 1u;
    r.valid = (x >> 1) & 1u;
    return r;
}

// Block-wide exclusive scan of "the last dimension row" (warp shuffles, then
// one shared-memory round over the warp totals); wsm holds 33 entries.
__device__ __forceinline__ DimCarry block_dim_scan_excl(const DimCarry& mine, DimCarry* wsm, DimCarry* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    DimCarry inc = mine;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const DimCarry y = dim_shfl(inc, off, true);
        if (lane >= off)
            inc = dim_combine(y, inc);
    }
    __syncthreads(); // wsm may still be read by a previous call
    if (lane == 31)
        wsm[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        DimCarry z = lane < nw ? wsm[lane] : DimCarry { 0, 0, 0 };
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const DimCarry y = dim_shfl(z, off, true);
            if (lane >= off)
                z = dim_combine(y, z);
        }
        DimCarry ez = dim_shfl(z, 1, true);
        if (lane == 0)
            ez = DimCarry { 0, 0, 0 };
        __syncwarp();
        if (lane < nw)
            wsm[lane] = ez;
        if (lane == nw - 1)
            wsm[32] = z; // block total
    }
    __syncthreads();
    DimCarry ex = dim_shfl(inc, 1, true);
    if (lane == 0)
        ex = DimCarry { 0, 0, 0 };
    if (total)
        *total = wsm[32];
    return dim_combine(wsm[warp], ex);
}

// the last dimension row of fill tile `blk`; sm, idx: FILL_THREADS / 32
// entries of shared memory each
__device__ __forceinline__ void fill_summary_tile(const uint64_t* w0, DimCarry* tile_last, size_t blk, DimCarry* sm,
                                                  int* idx)
{
    // the tile's last dimension row: every thread keeps the last one of its
    // stride (rows are visited in increasing order), then a max-index
    // reduction (warp shuffles, one shared-memory round) picks the overall last
    const size_t base = blk * FILL_TS;
    DimCarry c { 0, 0, 0 };
    int last = -1;
    for (int i = threadIdx.x; i < FILL_TS; i += FILL_THREADS) {
        VELO_TRACE_AT(TS_FILL, w0 + base + i);
        const DimCarry d = dim_of(w0[base + i]);
        c = dim_combine(c, d);
        last = d.has ? i : last;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const DimCarry oc = dim_shfl(c, off, false);
        const int oi = __shfl_xor_sync(0xFFFFFFFFu, last, off);
        const bool take = oi > last;
        c = take ? oc : c;
        last = take ? oi : last;
    }
    if ((threadIdx.x & 31) == 0) {
        sm[threadIdx.x >> 5] = c;
        idx[threadIdx.x >> 5] = last;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DimCarry b = sm[0];
        int bi = idx[0];
        for (int w = 1; w < FILL_THREADS / 32; w++) {
            const bool take = idx[w] > bi;
            b = take ? sm[w] : b;
            bi = take ? idx[w] : bi;
        }
        tile_last[blk] = b;
    }
}


// exclusive "last dimension row" scan over tiles; one CTA, rounds of
// blockDim.x consecutive tiles chained through the running carry
__device__ __forceinline__ void fill_carries_body(const DimCarry* tile_last, int ntiles, DimCarry* carry,
                                                  DimCarry* wsm)
{
    DimCarry run { 0, 0, 0 };
    for (int base = 0; base < ntiles; base += blockDim.x) {
        const int t = base + (int)threadIdx.x;
        DimCarry x { 0, 0, 0 };
        if (t < ntiles) {
            VELO_TRACE_AT(TS_FILL, tile_last + t);
            x = tile_last[t];
        }
        DimCarry total;
        const DimCarry ex = block_dim_scan_excl(x, wsm, &total);
        if (t < ntiles)
            carry[t] = dim_combine(run, ex);
        run = dim_combine(run, total);
    }
}


// shared-memory slot of fill-tile row i: one pad word after every 8 rows, so
// that the 8 rows of each of 16 neighbouring threads fall in different banks
constexpr int FILL_TS_PAD = FILL_TS + FILL_TS / 8;
__device__ __forceinline__ int fill_slot(int i) { return i + (i >> 3); }

// joined flags of fill tile `blk`; sw: FILL_TS_PAD words, wsm: 33 entries of
// shared memory
__device__ __forceinline__ void fill_apply_tile(uint64_t* w0, const DimCarry* carry, size_t blk, uint64_t* sw,
                                                DimCarry* wsm)
{
    static_assert(FILL_RPT == 8, "fill_slot pads after each thread's 8 rows");
    const size_t base = blk * FILL_TS;
    for (int i = threadIdx.x; i < FILL_TS; i += FILL_THREADS) {
        VELO_TRACE_AT(TS_FILL, w0 + base + i);
        sw[fill_slot(i)] = w0[base + i];
    }
    __syncthreads();
    const int r0 = threadIdx.x * (FILL_RPT + 1);
    DimCarry mine { 0, 0, 0 };
#pragma unroll
    for (int r = 0; r < FILL_RPT; r++)
        mine = dim_combine(mine, dim_of(sw[r0 + r]));
    const DimCarry ex = block_dim_scan_excl(mine, wsm, nullptr);
    DimCarry run = dim_combine(carry[blk], ex);
#pragma unroll
    for (int r = 0; r < FILL_RPT; r++) {
        const uint64_t a = sw[r0 + r];
        run = dim_combine(run, dim_of(a));
        const bool fact = ((a >> 31) & 1ull) != 0 && a != ~0ull;
        const bool joined = fact & (((a >> 30) & 1ull) != 0) & (run.has != 0) & (run.valid != 0) & (run.key == (a >> 32));
        sw[r0 + r] = (a & ~J_JOINED) | (joined ? J_JOINED : 0ull);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < FILL_TS; i += FILL_THREADS) {
        VELO_TRACE_AT(TS_FILL, w0 + base + i);
        w0[base + i] = sw[fill_slot(i)];
    }
}


// ---- top-k keys of the groups -------------------------------------------------
// k0 = [63] not a group | [62:0] ts >> 1 ; k1 = [63] ts & 1 | [62:31] fk ^ sign |
// [30:0] count, with ts = ~(sum ^ sign), so ascending (k0, k1 & TK_M1) is
// (groups first, sum descending, fk ascending).  A count is below 2^31: the
// union holds at most 2^31 rows, one of them a dimension row.
constexpr uint64_t TK_M1 = 0xFFFFFFFF80000000ull;
constexpr uint64_t SIGN64 = 0x8000000000000000ull;
constexpr int TK_RED_ROWS = 4096, TK_RED_THREADS = 1024; // candidate blocks of the later rounds

__device__ __forceinline__ void topk_key(uint64_t o0, uint64_t sum, uint64_t cnt, uint64_t& k0, uint64_t& k1)
{
    const uint64_t ts = ~(sum ^ SIGN64);
    k0 = (o0 & SIGN64) | (ts >> 1);
    k1 = (ts << 63) | ((o0 & 0xFFFFFFFFull) << 31) | (cnt & 0x7FFFFFFFull);
}

// one round: every block of `rn` candidates (runs of c, each ascending) keeps
// its best c; odd runs are loaded reversed so that neighbouring runs form
// bitonic sequences
// (block `blk`; P = TK_RED_ROWS / 2 / blockDim.x compare-exchanges a thread;
// sm: 2 x TK_RED_ROWS words)
template <int P>
__device__ __forceinline__ void topk_reduce_tile(const uint64_t* in0, const uint64_t* in1, int rn, int c,
                                                 uint64_t* out0, uint64_t* out1, size_t blk, char* sm)
{
    uint64_t* k0 = reinterpret_cast<uint64_t*>(sm);
    uint64_t* k1 = k0 + TK_RED_ROWS;
    const size_t base = blk * rn;
    for (int i = threadIdx.x; i < rn; i += blockDim.x) {
        const int q = i / c, r = i - q * c;
        const int d = (q & 1) ? q * c + (c - 1 - r) : i;
        VELO_TRACE_AT(TS_TOPK, in0 + base + i);
        k0[d] = in0[base + i];
        k1[d] = in1[base + i];
    }
    topk_net<P>(k0, k1, rn, c, TK_M1, true);
    for (int j = threadIdx.x; j < c; j += blockDim.x) {
        VELO_TRACE_AT(TS_TOPK, out0 + blk * c + j);
        out0[blk * c + j] = k0[j];
        out1[blk * c + j] = k1[j];
    }
}


// the first k rows of the final run as (fk, sum, count), and the counts; one CTA
__device__ __forceinline__ void topk_out_body(const uint64_t* t0, const uint64_t* t1, size_t k, int64_t* out,
                                              const uint64_t* n_groups, const uint64_t* n_joined, uint64_t* d_counts)
{
    for (size_t i = threadIdx.x; i < k; i += blockDim.x) {
        VELO_TRACE_AT(TS_TOPK, t0 + i);
        const uint64_t a = t0[i], b = t1[i];
        const bool ok = (a >> 63) == 0;
        const uint64_t ts = (a << 1) | (b >> 63);
        out[i * 3 + 0] = ok ? (int64_t)(int32_t)((uint32_t)(b >> 31) ^ 0x80000000u) : 0;
        out[i * 3 + 1] = ok ? (int64_t)(~ts ^ SIGN64) : 0;
        out[i * 3 + 2] = ok ? (int64_t)(b & 0x7FFFFFFFull) : 0;
    }
    if (threadIdx.x == 0) {
        d_counts[0] = *n_joined;
        d_counts[1] = *n_groups;
    }
}


// the group-by's last pass fused with the first top-k round: the tile's group
// rows become top-k keys in shared memory and only its best `cand` are stored
constexpr size_t JSEG_KEYS_OFF = (JSeg::SMEM + 15) & ~(size_t)15;
constexpr size_t JSEG_TOPK_SMEM = JSEG_KEYS_OFF + (size_t)2 * SEG_TS * 8;
// with 16 candidates a tile only 2 x 128 words of key scratch (topk16_block):
// five CTAs an SM
constexpr size_t JSEG_TOPK16_SMEM = JSEG_KEYS_OFF + (size_t)2 * 128 * 8;

// group-by tile `blk` (SEG_THREADS threads); sm: JSEG_TOPK_SMEM bytes
// (JSEG_TOPK16_SMEM when cand == 16)
__device__ __forceinline__ void jseg_emit_topk_tile(const JRec::Cols& c, int ntiles, const SegTileAgg* aggs,
                                                    const int64_t* carry_in, int cand, uint64_t* out0, uint64_t* out1,
                                                    size_t blk, char* sm)
{
    uint64_t* k0 = reinterpret_cast<uint64_t*>(sm + JSEG_KEYS_OFF);
    uint64_t* k1 = k0 + SEG_TS;
    if (cand == 16) {
        // the 16 best in registers and warp shuffles (rows 4t .. 4t + 3 of
        // thread t, handed over in registers by the group-by's last pass),
        // then through 2 x 128 words of shared memory; thread t < 16 stores
        // row tk_row16(t)
        static_assert(SEG_TS == 4 * SEG_THREADS && SEG_THREADS == 256 && SEG_RPT == 4, "4 rows a thread, 8 warps");
        static_assert(JSeg::OW == 3, "group records (flag | key, sum, count)");
        uint64_t o[SEG_RPT][JSeg::OW];
        JSeg::emit_stage<true>(c.w, (int)blk, ntiles, aggs, carry_in, JoinAgg::Params {}, sm, o);
        uint64_t x0[4], x1[4];
#pragma unroll
        for (int e = 0; e < 4; e++)
            topk_key(o[e][0], o[e][1], o[e][2], x0[e], x1[e]);
        uint64_t r0, r1;
        topk16_block(x0, x1, k0, TK_M1, r0, r1);
        if (threadIdx.x < 16) {
            const size_t o = blk * 16 + tk_row16(threadIdx.x);
            VELO_TRACE_AT(TS_TOPK, out0 + o);
            out0[o] = r0;
            out1[o] = r1;
        }
        return;
    }
    JSeg::emit_stage(c.w, (int)blk, ntiles, aggs, carry_in, JoinAgg::Params {}, sm);
    const uint64_t* so = reinterpret_cast<const uint64_t*>(sm);
    for (int i = threadIdx.x; i < SEG_TS; i += SEG_THREADS)
        topk_key(so[seg_slot(i)], so[SEG_TS_PAD + seg_slot(i)], so[2 * SEG_TS_PAD + seg_slot(i)], k0[i], k1[i]);
    topk_net<SEG_TS / 2 / SEG_THREADS>(k0, k1, SEG_TS, cand, TK_M1, false);
    for (int j = threadIdx.x; j < cand; j += SEG_THREADS) {
        VELO_TRACE_AT(TS_TOPK, out0 + blk * cand + j);
        out0[blk * cand + j] = k0[j];
        out1[blk * cand + j] = k1[j];
    }
}


struct JoinScratch {
    uint64_t* u[2];      // union records
    uint64_t* cand[2];   // top-k candidates of the group-by tiles (later rounds reuse u)
    uint32_t* counts;
    uint32_t* prefix;
    uint64_t* n_joined;
    DimCarry* tile_last;
    DimCarry* fcarry;
    SegTileAgg* aggs;
    int64_t* runs;
    int64_t* carry;
    uint32_t* tail_prefix;
    uint64_t* n_groups;
    size_t bytes, n_rec;
};

inline JoinScratch join_layout(char* base, size_t nd, size_t nf)
{
    JoinScratch s {};
    size_t n_rec = next_pow2(nd + nf);
    const size_t floor_rows = (size_t)1 << J_LT;
    n_rec = n_rec < floor_rows ? floor_rows : n_rec;
    n_rec = n_rec < (size_t)SEG_TS ? (size_t)SEG_TS : n_rec;
    s.n_rec = n_rec;
    const size_t ntc = n_rec >> J_LT, nts = n_rec / SEG_TS, ntf = n_rec / FILL_TS;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += align_up(bytes, 256);
        return p;
    };
    for (int i = 0; i < 2; i++)
        s.u[i] = reinterpret_cast<uint64_t*>(take(n_rec * 8));
    // at most SEG_TS candidates a tile (k <= 1024)
    for (int i = 0; i < 2; i++)
        s.cand[i] = reinterpret_cast<uint64_t*>(take(n_rec * 8));
    s.counts = reinterpret_cast<uint32_t*>(take(ntc * 4));
    s.prefix = reinterpret_cast<uint32_t*>(take((ntc + 1) * 4));
    s.n_joined = reinterpret_cast<uint64_t*>(take(8));
    s.tile_last = reinterpret_cast<DimCarry*>(take(ntf * sizeof(DimCarry)));
    s.fcarry = reinterpret_cast<DimCarry*>(take(ntf * sizeof(DimCarry)));
    s.aggs = reinterpret_cast<SegTileAgg*>(take(nts * sizeof(SegTileAgg)));
    s.runs = reinterpret_cast<int64_t*>(take(nts * JoinAgg::V * 8));
    s.carry = reinterpret_cast<int64_t*>(take(nts * JoinAgg::V * 8));
    s.tail_prefix = reinterpret_cast<uint32_t*>(take(nts * 4));
    s.n_groups = reinterpret_cast<uint64_t*>(take(8));
    s.bytes = off;
    return s;
}

} // namespace velo
