// Oblivious PK-FK sort-merge join + group-by + top-k.
//
// Replaces the reference's sort-merge join (include/cuda/sort_merge_join.cuh:
// 63-199, src/operator/sort_merge_join_operator.cpp:27-257: per-block
// sequential merge, atomics, output sized by the true join cardinality) with
// the oblivious union-sort formulation:
//   1. pack     dimension rows (key, tag 0, date filter) and fact rows
//               (fk, tag 1, price filter, price) into one record array,
//               padded to a power of two
//   2. sort     bitonic network on (key, tag): each dimension row heads the
//               run of fact rows that reference it
//   3. fill     forward fill of the last dimension row (segmented scan): a
//               fact row joins iff its key's dimension row exists and passes
//   4. compact  ORCompact of joined fact rows to the front (order kept)
//   5. group    segmented sums of price per fk over the joined prefix: the
//               last row of each fk run carries the group's (sum, count)
//   6. top-k    groups ordered on (sum desc, fk asc) by a bitonic top-k
//               network (topk.cuh): each 1024-row tile of the group-by keeps
//               its best c = max(16, next_pow2(k)) rows in shared memory,
//               then rounds over blocks of 4096 candidates keep their best
//               c, until one sorted run of c is left; first k
// Record layout of the union (2 u64 words):
//   w0 = [63:32] key ^ 0x80000000 | [31] tag (0 dim, 1 fact) | [30] row passes
//        its side's filter | [29] joined (set by fill) ; w1 = price (fact rows)
#include "net_impl.cuh"
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

__global__ void __launch_bounds__(256) k_join_pack(const int32_t* dk, const int32_t* dd, size_t nd, const int32_t* ff,
                                                   const int64_t* fp, size_t nf, int32_t date_hi, int64_t price_hi,
                                                   size_t n_rec, uint64_t* w0, uint64_t* w1)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_join_pack"));
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(g, n_rec); g += (size_t)gridDim.x * blockDim.x) {
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

__global__ void __launch_bounds__(FILL_THREADS) k_fill_summary(const uint64_t* w0, DimCarry* tile_last)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_summary"));
    // the tile's last dimension row: every thread keeps the last one of its
    // stride (rows are visited in increasing order), then a max-index
    // reduction (warp shuffles, one shared-memory round) picks the overall last
    __shared__ DimCarry sm[FILL_THREADS / 32];
    __shared__ int idx[FILL_THREADS / 32];
    const size_t base = (size_t)blockIdx.x * FILL_TS;
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
        tile_last[blockIdx.x] = b;
    }
}

// exclusive "last dimension row" scan over tiles; one CTA of 1024 threads,
// rounds of 1024 consecutive tiles chained through the running carry
__global__ void __launch_bounds__(1024) k_fill_carries(const DimCarry* tile_last, int ntiles, DimCarry* carry)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_carries"));
    __shared__ DimCarry wsm[33];
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

__global__ void __launch_bounds__(FILL_THREADS) k_fill_apply(uint64_t* w0, const DimCarry* carry)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_apply"));
    __shared__ uint64_t sw[FILL_TS];
    __shared__ DimCarry wsm[33];
    const size_t base = (size_t)blockIdx.x * FILL_TS;
    for (int i = threadIdx.x; i < FILL_TS; i += FILL_THREADS) {
        VELO_TRACE_AT(TS_FILL, w0 + base + i);
        sw[i] = w0[base + i];
    }
    __syncthreads();
    const int r0 = threadIdx.x * FILL_RPT;
    DimCarry mine { 0, 0, 0 };
#pragma unroll
    for (int r = 0; r < FILL_RPT; r++)
        mine = dim_combine(mine, dim_of(sw[r0 + r]));
    const DimCarry ex = block_dim_scan_excl(mine, wsm, nullptr);
    DimCarry run = dim_combine(carry[blockIdx.x], ex);
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
        w0[base + i] = sw[i];
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
__global__ void __launch_bounds__(TK_RED_THREADS) k_topk_reduce(const uint64_t* in0, const uint64_t* in1, int rn,
                                                                int c, uint64_t* out0, uint64_t* out1)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_topk_reduce"));
    extern __shared__ __align__(16) char sm[];
    uint64_t* k0 = reinterpret_cast<uint64_t*>(sm);
    uint64_t* k1 = k0 + TK_RED_ROWS;
    const size_t base = (size_t)blockIdx.x * rn;
    for (int i = threadIdx.x; i < rn; i += blockDim.x) {
        const int q = i / c, r = i - q * c;
        const int d = (q & 1) ? q * c + (c - 1 - r) : i;
        VELO_TRACE_AT(TS_TOPK, in0 + base + i);
        k0[d] = in0[base + i];
        k1[d] = in1[base + i];
    }
    topk_net<TK_RED_ROWS / 2 / TK_RED_THREADS>(k0, k1, rn, c, TK_M1, true);
    for (int j = threadIdx.x; j < c; j += blockDim.x) {
        VELO_TRACE_AT(TS_TOPK, out0 + (size_t)blockIdx.x * c + j);
        out0[(size_t)blockIdx.x * c + j] = k0[j];
        out1[(size_t)blockIdx.x * c + j] = k1[j];
    }
}

__global__ void k_topk_out(const uint64_t* t0, const uint64_t* t1, size_t k, int64_t* out, const uint64_t* n_groups,
                           const uint64_t* n_joined, uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_topk_out"));
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

__global__ void __launch_bounds__(SEG_THREADS) k_jseg_summary(JRec::Cols c, SegTileAgg* aggs, int64_t* runs)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_jseg_summary"));
    extern __shared__ __align__(16) char sm[];
    JSeg::tile_summary(c.w, blockIdx.x, aggs, runs, JoinAgg::Params {}, sm);
}

__global__ void __launch_bounds__(1024) k_jseg_carries(const SegTileAgg* aggs, const int64_t* runs, int ntiles,
                                                       int64_t* carry_in, uint32_t* tail_prefix, uint64_t* n_groups)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_jseg_carries"));
    extern __shared__ __align__(16) char sm[];
    JSeg::carries(aggs, runs, ntiles, carry_in, tail_prefix, n_groups, sm);
}

// the group-by's last pass fused with the first top-k round: the tile's group
// rows become top-k keys in shared memory and only its best `cand` are stored
constexpr size_t JSEG_KEYS_OFF = (JSeg::SMEM + 15) & ~(size_t)15;
constexpr size_t JSEG_TOPK_SMEM = JSEG_KEYS_OFF + (size_t)2 * SEG_TS * 8;

__global__ void __launch_bounds__(SEG_THREADS) k_jseg_emit_topk(JRec::Cols c, int ntiles, const SegTileAgg* aggs,
                                                                const int64_t* carry_in, int cand, uint64_t* out0,
                                                                uint64_t* out1)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_jseg_emit_topk"));
    extern __shared__ __align__(16) char sm[];
    JSeg::emit_stage(c.w, blockIdx.x, ntiles, aggs, carry_in, JoinAgg::Params {}, sm);
    const uint64_t* so = reinterpret_cast<const uint64_t*>(sm);
    uint64_t* k0 = reinterpret_cast<uint64_t*>(sm + JSEG_KEYS_OFF);
    uint64_t* k1 = k0 + SEG_TS;
    if (cand == 16) {
        // the 16 best in registers and warp shuffles (rows 4t .. 4t + 3 of
        // thread t), then through 2 x 128 words of shared memory
        static_assert(SEG_TS == 4 * SEG_THREADS && SEG_THREADS == 256, "4 rows a thread, 8 warps");
        uint64_t x0[4], x1[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int i = 4 * threadIdx.x + e;
            topk_key(so[seg_slot(i)], so[SEG_TS_PAD + seg_slot(i)], so[2 * SEG_TS_PAD + seg_slot(i)], x0[e], x1[e]);
        }
        topk16_block(x0, x1, k0, TK_M1);
        if (threadIdx.x < 4) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const size_t o = (size_t)blockIdx.x * 16 + 4 * threadIdx.x + e;
                VELO_TRACE_AT(TS_TOPK, out0 + o);
                out0[o] = x0[e];
                out1[o] = x1[e];
            }
        }
        return;
    }
    for (int i = threadIdx.x; i < SEG_TS; i += SEG_THREADS)
        topk_key(so[seg_slot(i)], so[SEG_TS_PAD + seg_slot(i)], so[2 * SEG_TS_PAD + seg_slot(i)], k0[i], k1[i]);
    topk_net<SEG_TS / 2 / SEG_THREADS>(k0, k1, SEG_TS, cand, TK_M1, false);
    for (int j = threadIdx.x; j < cand; j += SEG_THREADS) {
        VELO_TRACE_AT(TS_TOPK, out0 + (size_t)blockIdx.x * cand + j);
        out0[(size_t)blockIdx.x * cand + j] = k0[j];
        out1[(size_t)blockIdx.x * cand + j] = k1[j];
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

static JoinScratch join_layout(char* base, size_t nd, size_t nf)
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

static velo_status join_attrs()
{
    static int done[64] = {};
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 0 && dev < 64 && done[dev])
        return VELO_OK;
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_jseg_summary, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)JSeg::SMEM_IN),
                  "cudaFuncSetAttribute");
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_jseg_emit_topk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)JSEG_TOPK_SMEM),
                  "cudaFuncSetAttribute");
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_topk_reduce, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(2 * TK_RED_ROWS * 8)),
                  "cudaFuncSetAttribute");
    if (dev >= 0 && dev < 64)
        done[dev] = 1;
    return VELO_OK;
}

} // namespace velo

using namespace velo;

extern "C" size_t velo_join_groupby_topk_scratch_bytes(size_t n_dim, size_t n_fact)
{
    return join_layout(nullptr, n_dim, n_fact).bytes;
}

extern "C" velo_status velo_join_groupby_topk(const velo_join_tables* t, const velo_join_pred* pred, uint32_t k,
                                              int64_t* d_out, uint64_t* d_counts, void* d_scratch,
                                              size_t scratch_bytes, void* stream)
{
    if (!t || !pred || !d_out || !d_counts)
        return einval("velo_join_groupby_topk: null argument");
    if (!t->dim_key || !t->dim_date || !t->fact_fk || !t->fact_price || t->n_dim == 0)
        return einval("velo_join_groupby_topk: null column or empty dimension table");
    if (k == 0 || k > 1024)
        return einval("velo_join_groupby_topk: k must be 1..1024");
    if (t->n_dim + t->n_fact > ((size_t)1 << MAX_LOGN))
        return einval("velo_join_groupby_topk: tables too large");
    JoinScratch s = join_layout(static_cast<char*>(d_scratch), t->n_dim, t->n_fact);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_join_groupby_topk: scratch must hold velo_join_groupby_topk_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    cudaStream_t st = (cudaStream_t)stream;
    velo_status rc = join_attrs();
    if (rc != VELO_OK)
        return rc;
    const int logR = ilog2_floor(s.n_rec);
    const size_t n_union = t->n_dim + t->n_fact;
    const int logU = ilog2_floor(next_pow2(n_union));
    StageTimer tm(st);

    // 1. pack
    const unsigned blocks = 148 * 8;
    k_join_pack<<<blocks, 256, 0, st>>>(t->dim_key, t->dim_date, t->n_dim, t->fact_fk, t->fact_price, t->n_fact,
                                        pred->date_hi, pred->price_hi, s.n_rec, s.u[0], s.u[1]);
    VELO_CUDA_TRY(cudaGetLastError(), "join pack launch");
    tm.mark();
    JRec::Cols uc;
    uc.w[0] = s.u[0];
    uc.w[1] = s.u[1];
    uc.mask[0] = J_KEYTAG;
    uc.pad[0] = uc.pad[1] = ~0ull;
    uc.mark_bit = 29;
    uc.mark_inv = 0;
    uc.mark_word = 0;
    // 2. sort the union on (key, tag)
    rc = launch_sort_records<JRec>(uc, logU, st);
    if (rc != VELO_OK)
        return rc;
    tm.mark();
    // 3. forward fill of the dimension side -> joined flag
    const int ntf = (int)(s.n_rec / FILL_TS);
    k_fill_summary<<<ntf, FILL_THREADS, 0, st>>>(s.u[0], s.tile_last);
    k_fill_carries<<<1, 1024, 0, st>>>(s.tile_last, ntf, s.fcarry);
    k_fill_apply<<<ntf, FILL_THREADS, 0, st>>>(s.u[0], s.fcarry);
    VELO_CUDA_TRY(cudaGetLastError(), "join fill launch");
    tm.mark();
    // 4. ORCompact of the joined fact rows
    {
        const int ntc = logR > J_LT ? 1 << (logR - J_LT) : 1;
        k_count_marks<JRec><<<ntc, 256, 0, st>>>(uc, s.n_rec, J_LT, s.counts);
        k_scan_tiles<<<1, 1024, 0, st>>>(s.counts, ntc, s.prefix, s.n_joined);
        std::vector<NetPass> passes;
        plan_compact(logR, J_LT, J_LMAX, passes);
        rc = launch_net12<JRec>(uc, NetGeom { s.n_rec, logR, 0 }, passes, s.prefix, st);
        if (rc != VELO_OK)
            return rc;
    }
    tm.mark();
    // 5. group-by fk over the joined prefix (already in fk order: the
    // compaction keeps the sorted order of the joined rows), fused with the
    // first top-k round: the best `cand` groups of every tile
    const int nts = (int)(s.n_rec / SEG_TS);
    const int cand = k <= (uint32_t)J_TOPK_MIN ? J_TOPK_MIN : (int)next_pow2(k);
    k_jseg_summary<<<nts, SEG_THREADS, JSeg::SMEM_IN, st>>>(uc, s.aggs, s.runs);
    k_jseg_carries<<<1, 1024, JoinAgg::V * 1024 * 8 + 2 * 1024 * 4, st>>>(s.aggs, s.runs, nts, s.carry,
                                                                            s.tail_prefix, s.n_groups);
    k_jseg_emit_topk<<<nts, SEG_THREADS, JSEG_TOPK_SMEM, st>>>(uc, nts, s.aggs, s.carry, cand, s.cand[0],
                                                              s.cand[1]);
    VELO_CUDA_TRY(cudaGetLastError(), "join group-by launch");
    tm.mark();
    // 6. top-k rounds over blocks of candidates (the union area is free now)
    uint64_t* cur[2] = { s.cand[0], s.cand[1] };
    uint64_t* nxt[2] = { s.u[0], s.u[1] };
    size_t n_c = (size_t)nts * cand;
    while (n_c > (size_t)cand) {
        const int rn = n_c < (size_t)TK_RED_ROWS ? (int)n_c : TK_RED_ROWS;
        const size_t blocks = n_c / rn;
        k_topk_reduce<<<(unsigned)blocks, TK_RED_THREADS, 2 * TK_RED_ROWS * 8, st>>>(cur[0], cur[1], rn, cand, nxt[0],
                                                                                    nxt[1]);
        VELO_CUDA_TRY(cudaGetLastError(), "top-k round launch");
        n_c = blocks * cand;
        std::swap(cur[0], nxt[0]);
        std::swap(cur[1], nxt[1]);
    }
    k_topk_out<<<1, 256, 0, st>>>(cur[0], cur[1], k, d_out, s.n_groups, s.n_joined, d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "top-k launch");
    tm.mark();
    tm.finish();
    return VELO_OK;
}
